/*
 * nclite — a small, self-contained implementation of the subset of the
 * NetCDF C API that the Tsunami-HySEA time stepper uses for its inputs
 * (topobathymetry / initial-state GRD files) and outputs (gridded and
 * time-series files).
 *
 * Format: NetCDF classic (CDF-1 read, CDF-2 "64-bit offset" read/write,
 * CDF-5 read), written from the public NetCDF classic format
 * specification.  Names, signatures, constants and error codes follow the
 * public NetCDF C API so that code written against libnetcdf (for example
 * src/GPU/netcdfTH.cu and src/GPU/netcdfSeries.cu of the reference) links
 * against this library unchanged.
 *
 * Differences from libnetcdf, by design:
 *   - nc_create(... | NC_NETCDF4) produces a classic 64-bit-offset file
 *     (there is no HDF5 in this build);
 *   - nc_def_var_deflate() records nothing and returns NC_NOERR
 *     (classic files are not compressed);
 *   - only one file may be open per ncid slot table entry (NCL_MAX_FILES).
 */
#ifndef NCLITE_NETCDF_H
#define NCLITE_NETCDF_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int nc_type;

#define NC_NAT    0
#define NC_BYTE   1
#define NC_CHAR   2
#define NC_SHORT  3
#define NC_INT    4
#define NC_LONG   NC_INT
#define NC_FLOAT  5
#define NC_DOUBLE 6
#define NC_UBYTE  7
#define NC_USHORT 8
#define NC_UINT   9
#define NC_INT64  10
#define NC_UINT64 11

#define NC_NOWRITE        0x0000
#define NC_WRITE          0x0001
#define NC_CLOBBER        0x0000
#define NC_NOCLOBBER      0x0004
#define NC_64BIT_OFFSET   0x0200
#define NC_64BIT_DATA     0x0020
#define NC_NETCDF4        0x1000
#define NC_CLASSIC_MODEL  0x0100

#define NC_UNLIMITED 0L
#define NC_GLOBAL   (-1)
#define NC_SHUFFLE   1
#define NC_MAX_NAME  256
#define NC_MAX_VAR_DIMS 1024

#define NC_NOERR        0
#define NC_EBADID     (-33)
#define NC_EEXIST     (-35)
#define NC_EINVAL     (-36)
#define NC_EPERM      (-37)
#define NC_ENOTINDEFINE (-38)
#define NC_EINDEFINE  (-39)
#define NC_EINVALCOORDS (-40)
#define NC_ENFILE     (-34)
#define NC_EBADTYPE   (-45)
#define NC_EBADDIM    (-46)
#define NC_EUNLIMPOS  (-47)
#define NC_ENOTATT    (-43)
#define NC_ENOTVAR    (-49)
#define NC_ENAMEINUSE (-42)
#define NC_ENOTNC     (-51)
#define NC_EUNLIMIT   (-54)
#define NC_ERANGE     (-60)
#define NC_ENOMEM     (-61)
#define NC_EEDGE      (-57)
#define NC_EIO        (-68)
#define NC_ENOTNC4    (-111)

const char *nc_strerror(int ncerr);

int nc_create(const char *path, int cmode, int *ncidp);
int nc_open(const char *path, int mode, int *ncidp);
int nc_enddef(int ncid);
int nc_redef(int ncid);
int nc_sync(int ncid);
int nc_close(int ncid);

int nc_def_dim(int ncid, const char *name, size_t len, int *idp);
int nc_def_var(int ncid, const char *name, nc_type xtype, int ndims, const int *dimidsp, int *varidp);
int nc_def_var_deflate(int ncid, int varid, int shuffle, int deflate, int deflate_level);

int nc_inq_dimid(int ncid, const char *name, int *idp);
int nc_inq_dimlen(int ncid, int dimid, size_t *lenp);
int nc_inq_varid(int ncid, const char *name, int *varidp);
int nc_inq_ndims(int ncid, int *ndimsp);
int nc_inq_nvars(int ncid, int *nvarsp);
int nc_inq_unlimdim(int ncid, int *unlimdimidp);
int nc_inq_vartype(int ncid, int varid, nc_type *xtypep);
int nc_inq_varndims(int ncid, int varid, int *ndimsp);
int nc_inq_vardimid(int ncid, int varid, int *dimidsp);
int nc_inq_attlen(int ncid, int varid, const char *name, size_t *lenp);

int nc_put_att_text(int ncid, int varid, const char *name, size_t len, const char *op);
int nc_put_att_float(int ncid, int varid, const char *name, nc_type xtype, size_t len, const float *op);
int nc_put_att_double(int ncid, int varid, const char *name, nc_type xtype, size_t len, const double *op);
int nc_put_att_int(int ncid, int varid, const char *name, nc_type xtype, size_t len, const int *op);
int nc_get_att_text(int ncid, int varid, const char *name, char *ip);
int nc_get_att_double(int ncid, int varid, const char *name, double *ip);

int nc_put_var_double(int ncid, int varid, const double *op);
int nc_put_var_float(int ncid, int varid, const float *op);
int nc_put_vara_float(int ncid, int varid, const size_t *startp, const size_t *countp, const float *op);
int nc_put_vara_double(int ncid, int varid, const size_t *startp, const size_t *countp, const double *op);

int nc_get_var_double(int ncid, int varid, double *ip);
int nc_get_var_float(int ncid, int varid, float *ip);
int nc_get_vara_float(int ncid, int varid, const size_t *startp, const size_t *countp, float *ip);

#ifdef __cplusplus
}
#endif

#endif /* NCLITE_NETCDF_H */
