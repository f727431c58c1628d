/*
 * nclite — NetCDF classic-format reader/writer implementing the subset of
 * the NetCDF C API declared in netcdf.h.
 *
 * Written from the public NetCDF classic file format specification:
 *   header  = magic numrecs dim_list gatt_list var_list
 *   magic   = 'C' 'D' 'F' version   (1: classic, 2: 64-bit offset, 5: 64-bit data)
 *   all integers and values big-endian; names and attribute values padded to
 *   4-byte boundaries; fixed-size variables stored contiguously at `begin`,
 *   record variables interleaved record by record (record size = sum of the
 *   record variables' padded slab sizes).
 * Files are written as version 2 (64-bit offsets) so that large grids fit
 * and so that common readers (e.g. scipy.io.netcdf_file) open them.
 */
#define _FILE_OFFSET_BITS 64
#define _POSIX_C_SOURCE 200809L
#include "netcdf.h"

#include <sys/types.h>

#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <pthread.h>
#include <string.h>

#define NCL_MAX_FILES 64
#define NCL_MAGIC_DIM 0x0Au
#define NCL_MAGIC_VAR 0x0Bu
#define NCL_MAGIC_ATT 0x0Cu

typedef struct {
    char name[NC_MAX_NAME + 1];
    nc_type type;
    size_t nelems;
    unsigned char *data; /* native-endian values */
} ncl_att;

typedef struct {
    char name[NC_MAX_NAME + 1];
    size_t len; /* 0 = record (unlimited) dimension */
} ncl_dim;

typedef struct {
    char name[NC_MAX_NAME + 1];
    int ndims;
    int dimids[NC_MAX_VAR_DIMS];
    nc_type type;
    ncl_att *atts;
    int natts;
    uint64_t vsize;  /* padded bytes of one (record) slab */
    uint64_t begin;  /* file offset of the first element */
    int is_record;
} ncl_var;

typedef struct {
    FILE *fp;
    int in_use;
    int writable;
    int in_define;
    int version;
    ncl_dim *dims;
    int ndims;
    ncl_att *gatts;
    int ngatts;
    ncl_var *vars;
    int nvars;
    uint64_t numrecs;
    uint64_t recsize;
    int header_dirty;
} ncl_file;

static ncl_file g_files[NCL_MAX_FILES];
/* guards claiming and freeing slots of g_files: files are opened and closed
   from several threads (one writer thread per scenario); each open file is
   used by one thread at a time */
static pthread_mutex_t g_slots_lock = PTHREAD_MUTEX_INITIALIZER;

/* ------------------------------------------------------------------ */
/* helpers                                                              */
/* ------------------------------------------------------------------ */

static ncl_file *get_file(int ncid)
{
    if (ncid < 0 || ncid >= NCL_MAX_FILES || !g_files[ncid].in_use) return NULL;
    return &g_files[ncid];
}

static size_t type_size(nc_type t)
{
    switch (t) {
    case NC_BYTE: case NC_CHAR: case NC_UBYTE: return 1;
    case NC_SHORT: case NC_USHORT: return 2;
    case NC_INT: case NC_FLOAT: case NC_UINT: return 4;
    case NC_DOUBLE: case NC_INT64: case NC_UINT64: return 8;
    default: return 0;
    }
}

static uint64_t pad4(uint64_t n) { return (n + 3u) & ~(uint64_t)3u; }

static void swap_bytes(unsigned char *p, size_t elem, size_t n)
{
    size_t i, j;
    if (elem <= 1) return;
    for (i = 0; i < n; i++) {
        unsigned char *e = p + i * elem;
        for (j = 0; j < elem / 2; j++) {
            unsigned char c = e[j];
            e[j] = e[elem - 1 - j];
            e[elem - 1 - j] = c;
        }
    }
}

static int host_is_little(void)
{
    const uint16_t one = 1;
    return *(const unsigned char *)&one == 1;
}

/* growable byte buffer used to serialise / parse the header */
typedef struct { unsigned char *p; size_t n, cap, pos; } buf_t;

static int buf_put(buf_t *b, const void *src, size_t n)
{
    if (b->n + n > b->cap) {
        size_t cap = b->cap ? b->cap * 2 : 1024;
        while (cap < b->n + n) cap *= 2;
        unsigned char *q = (unsigned char *)realloc(b->p, cap);
        if (!q) return NC_ENOMEM;
        b->p = q;
        b->cap = cap;
    }
    memcpy(b->p + b->n, src, n);
    b->n += n;
    return NC_NOERR;
}

static int put_u32(buf_t *b, uint32_t v)
{
    unsigned char c[4] = {(unsigned char)(v >> 24), (unsigned char)(v >> 16), (unsigned char)(v >> 8), (unsigned char)v};
    return buf_put(b, c, 4);
}

static int put_u64(buf_t *b, uint64_t v)
{
    unsigned char c[8];
    int i;
    for (i = 0; i < 8; i++) c[i] = (unsigned char)(v >> (56 - 8 * i));
    return buf_put(b, c, 8);
}

static int put_count(buf_t *b, int version, uint64_t v)
{
    return version == 5 ? put_u64(b, v) : put_u32(b, (uint32_t)v);
}

static int put_name(buf_t *b, int version, const char *name)
{
    size_t n = strlen(name);
    static const unsigned char zeros[4] = {0, 0, 0, 0};
    int rc = put_count(b, version, n);
    if (rc) return rc;
    if ((rc = buf_put(b, name, n))) return rc;
    return buf_put(b, zeros, (size_t)(pad4(n) - n));
}

static int put_values(buf_t *b, nc_type t, size_t nelems, const unsigned char *native)
{
    size_t es = type_size(t), bytes = es * nelems;
    static const unsigned char zeros[4] = {0, 0, 0, 0};
    unsigned char *tmp;
    int rc;
    if (bytes == 0) return NC_NOERR;
    tmp = (unsigned char *)malloc(bytes);
    if (!tmp) return NC_ENOMEM;
    memcpy(tmp, native, bytes);
    if (host_is_little()) swap_bytes(tmp, es, nelems);
    rc = buf_put(b, tmp, bytes);
    free(tmp);
    if (rc) return rc;
    return buf_put(b, zeros, (size_t)(pad4(bytes) - bytes));
}

static int put_att_list(buf_t *b, int version, const ncl_att *atts, int natts)
{
    int i, rc;
    if (natts == 0) {
        if ((rc = put_u32(b, 0))) return rc;
        return put_count(b, version, 0);
    }
    if ((rc = put_u32(b, NCL_MAGIC_ATT))) return rc;
    if ((rc = put_count(b, version, (uint64_t)natts))) return rc;
    for (i = 0; i < natts; i++) {
        if ((rc = put_name(b, version, atts[i].name))) return rc;
        if ((rc = put_u32(b, (uint32_t)atts[i].type))) return rc;
        if ((rc = put_count(b, version, atts[i].nelems))) return rc;
        if ((rc = put_values(b, atts[i].type, atts[i].nelems, atts[i].data))) return rc;
    }
    return NC_NOERR;
}

static int serialise_header(ncl_file *f, buf_t *b)
{
    int i, j, rc;
    unsigned char magic[4] = {'C', 'D', 'F', (unsigned char)f->version};
    b->n = 0;
    if ((rc = buf_put(b, magic, 4))) return rc;
    if ((rc = put_count(b, f->version, f->numrecs))) return rc;
    if (f->ndims == 0) {
        if ((rc = put_u32(b, 0)) || (rc = put_count(b, f->version, 0))) return rc;
    } else {
        if ((rc = put_u32(b, NCL_MAGIC_DIM)) || (rc = put_count(b, f->version, (uint64_t)f->ndims))) return rc;
        for (i = 0; i < f->ndims; i++) {
            if ((rc = put_name(b, f->version, f->dims[i].name))) return rc;
            if ((rc = put_count(b, f->version, f->dims[i].len))) return rc;
        }
    }
    if ((rc = put_att_list(b, f->version, f->gatts, f->ngatts))) return rc;
    if (f->nvars == 0) {
        if ((rc = put_u32(b, 0)) || (rc = put_count(b, f->version, 0))) return rc;
    } else {
        if ((rc = put_u32(b, NCL_MAGIC_VAR)) || (rc = put_count(b, f->version, (uint64_t)f->nvars))) return rc;
        for (i = 0; i < f->nvars; i++) {
            ncl_var *v = &f->vars[i];
            uint64_t vs = v->vsize;
            if ((rc = put_name(b, f->version, v->name))) return rc;
            if ((rc = put_count(b, f->version, (uint64_t)v->ndims))) return rc;
            for (j = 0; j < v->ndims; j++)
                if ((rc = put_count(b, f->version, (uint64_t)v->dimids[j]))) return rc;
            if ((rc = put_att_list(b, f->version, v->atts, v->natts))) return rc;
            if ((rc = put_u32(b, (uint32_t)v->type))) return rc;
            if (f->version != 5 && vs > 0xFFFFFFFCull) vs = 0xFFFFFFFFull;
            if ((rc = put_count(b, f->version, vs))) return rc;
            if (f->version == 1) rc = put_u32(b, (uint32_t)v->begin);
            else rc = put_u64(b, v->begin);
            if (rc) return rc;
        }
    }
    return NC_NOERR;
}

static int write_numrecs(ncl_file *f)
{
    unsigned char c[8];
    int i, n = f->version == 5 ? 8 : 4;
    for (i = 0; i < n; i++) c[i] = (unsigned char)(f->numrecs >> (8 * (n - 1 - i)));
    if (fseeko(f->fp, 4, SEEK_SET) != 0) return NC_EIO;
    if (fwrite(c, 1, (size_t)n, f->fp) != (size_t)n) return NC_EIO;
    return NC_NOERR;
}

static void free_atts(ncl_att *a, int n)
{
    int i;
    for (i = 0; i < n; i++) free(a[i].data);
    free(a);
}

static void release(ncl_file *f)
{
    int i;
    if (f->fp) fclose(f->fp);
    free(f->dims);
    free_atts(f->gatts, f->ngatts);
    for (i = 0; i < f->nvars; i++) free_atts(f->vars[i].atts, f->vars[i].natts);
    free(f->vars);
    pthread_mutex_lock(&g_slots_lock);
    memset(f, 0, sizeof(*f));
    pthread_mutex_unlock(&g_slots_lock);
}

/* claims a free slot: cleared and marked in use */
static int alloc_slot(void)
{
    int i, id = -1;
    pthread_mutex_lock(&g_slots_lock);
    for (i = 0; i < NCL_MAX_FILES; i++)
        if (!g_files[i].in_use) {
            memset(&g_files[i], 0, sizeof(ncl_file));
            g_files[i].in_use = 1;
            id = i;
            break;
        }
    pthread_mutex_unlock(&g_slots_lock);
    return id;
}

/* ------------------------------------------------------------------ */
/* public API: errors                                                   */
/* ------------------------------------------------------------------ */

const char *nc_strerror(int e)
{
    switch (e) {
    case NC_NOERR: return "No error";
    case NC_EBADID: return "NetCDF: Not a valid ID";
    case NC_ENFILE: return "NetCDF: Too many files open";
    case NC_EEXIST: return "NetCDF: File exists && NC_NOCLOBBER";
    case NC_EINVAL: return "NetCDF: Invalid argument";
    case NC_EPERM: return "NetCDF: Write to read only";
    case NC_ENOTINDEFINE: return "NetCDF: Operation not allowed in data mode";
    case NC_EINDEFINE: return "NetCDF: Operation not allowed in define mode";
    case NC_EINVALCOORDS: return "NetCDF: Index exceeds dimension bound";
    case NC_ENAMEINUSE: return "NetCDF: String match to name in use";
    case NC_ENOTATT: return "NetCDF: Attribute not found";
    case NC_EBADTYPE: return "NetCDF: Not a valid data type or _FillValue type mismatch";
    case NC_EBADDIM: return "NetCDF: Invalid dimension ID or name";
    case NC_EUNLIMPOS: return "NetCDF: NC_UNLIMITED in the wrong index";
    case NC_ENOTVAR: return "NetCDF: Variable not found";
    case NC_ENOTNC: return "NetCDF: Unknown file format";
    case NC_EUNLIMIT: return "NetCDF: NC_UNLIMITED size already in use";
    case NC_EEDGE: return "NetCDF: Start+count exceeds dimension bound";
    case NC_ERANGE: return "NetCDF: Numeric conversion not representable";
    case NC_ENOMEM: return "NetCDF: Memory allocation (malloc) failure";
    case NC_EIO: return "NetCDF: I/O failure";
    case NC_ENOTNC4: return "NetCDF: Attempting netcdf-4 operation on netcdf-3 file";
    default: return "NetCDF: Unknown error";
    }
}

/* ------------------------------------------------------------------ */
/* create / define mode                                                 */
/* ------------------------------------------------------------------ */

int nc_create(const char *path, int cmode, int *ncidp)
{
    int id;
    FILE *fp;
    if (!path || !ncidp) return NC_EINVAL;
    if (cmode & NC_NOCLOBBER) {
        fp = fopen(path, "rb");
        if (fp) { fclose(fp); return NC_EEXIST; }
    }
    id = alloc_slot();
    if (id < 0) return NC_ENFILE;
    fp = fopen(path, "w+b");
    if (!fp) {
        release(&g_files[id]);
        return NC_EIO;
    }
    g_files[id].fp = fp;
    g_files[id].in_use = 1;
    g_files[id].writable = 1;
    g_files[id].in_define = 1;
    g_files[id].version = (cmode & NC_64BIT_DATA) ? 5 : 2;
    *ncidp = id;
    return NC_NOERR;
}

static int name_ok(const char *name)
{
    return name && name[0] && strlen(name) <= NC_MAX_NAME;
}

int nc_def_dim(int ncid, const char *name, size_t len, int *idp)
{
    ncl_file *f = get_file(ncid);
    int i;
    ncl_dim *d;
    if (!f) return NC_EBADID;
    if (!f->in_define) return NC_ENOTINDEFINE;
    if (!name_ok(name)) return NC_EINVAL;
    for (i = 0; i < f->ndims; i++) {
        if (strcmp(f->dims[i].name, name) == 0) return NC_ENAMEINUSE;
        if (len == NC_UNLIMITED && f->dims[i].len == NC_UNLIMITED) return NC_EUNLIMIT;
    }
    d = (ncl_dim *)realloc(f->dims, sizeof(ncl_dim) * (size_t)(f->ndims + 1));
    if (!d) return NC_ENOMEM;
    f->dims = d;
    strcpy(d[f->ndims].name, name);
    d[f->ndims].len = len;
    if (idp) *idp = f->ndims;
    f->ndims++;
    return NC_NOERR;
}

int nc_def_var(int ncid, const char *name, nc_type xtype, int ndims, const int *dimidsp, int *varidp)
{
    ncl_file *f = get_file(ncid);
    int i;
    ncl_var *v;
    if (!f) return NC_EBADID;
    if (!f->in_define) return NC_ENOTINDEFINE;
    if (!name_ok(name)) return NC_EINVAL;
    if (type_size(xtype) == 0 || xtype > NC_DOUBLE) return NC_EBADTYPE;
    if (ndims < 0 || ndims > NC_MAX_VAR_DIMS) return NC_EINVAL;
    for (i = 0; i < f->nvars; i++)
        if (strcmp(f->vars[i].name, name) == 0) return NC_ENAMEINUSE;
    for (i = 0; i < ndims; i++) {
        if (dimidsp[i] < 0 || dimidsp[i] >= f->ndims) return NC_EBADDIM;
        if (i > 0 && f->dims[dimidsp[i]].len == NC_UNLIMITED) return NC_EUNLIMPOS;
    }
    v = (ncl_var *)realloc(f->vars, sizeof(ncl_var) * (size_t)(f->nvars + 1));
    if (!v) return NC_ENOMEM;
    f->vars = v;
    v = &f->vars[f->nvars];
    memset(v, 0, sizeof(*v));
    strcpy(v->name, name);
    v->type = xtype;
    v->ndims = ndims;
    for (i = 0; i < ndims; i++) v->dimids[i] = dimidsp[i];
    v->is_record = (ndims > 0 && f->dims[dimidsp[0]].len == NC_UNLIMITED);
    if (varidp) *varidp = f->nvars;
    f->nvars++;
    return NC_NOERR;
}

int nc_def_var_deflate(int ncid, int varid, int shuffle, int deflate, int deflate_level)
{
    ncl_file *f = get_file(ncid);
    (void)shuffle; (void)deflate;
    if (!f) return NC_EBADID;
    if (varid < 0 || varid >= f->nvars) return NC_ENOTVAR;
    if (deflate_level < 0 || deflate_level > 9) return NC_EINVAL;
    return NC_NOERR; /* classic files are stored uncompressed */
}

static int put_att(int ncid, int varid, const char *name, nc_type type, size_t len, const void *op, size_t opsize, int convert_from)
{
    ncl_file *f = get_file(ncid);
    ncl_att **list;
    int *n, i, idx = -1;
    ncl_att *a;
    size_t es;
    unsigned char *data;
    if (!f) return NC_EBADID;
    if (!f->writable) return NC_EPERM;
    if (!name_ok(name)) return NC_EINVAL;
    if (type_size(type) == 0 || type > NC_DOUBLE) return NC_EBADTYPE;
    if (varid == NC_GLOBAL) {
        list = &f->gatts;
        n = &f->ngatts;
    } else {
        if (varid < 0 || varid >= f->nvars) return NC_ENOTVAR;
        list = &f->vars[varid].atts;
        n = &f->vars[varid].natts;
    }
    for (i = 0; i < *n; i++)
        if (strcmp((*list)[i].name, name) == 0) { idx = i; break; }
    if (idx < 0 && !f->in_define) return NC_ENOTINDEFINE;
    es = type_size(type);
    data = (unsigned char *)malloc(es * (len ? len : 1));
    if (!data) return NC_ENOMEM;
    /* convert the caller's values (int/float/double/char) to the stored type */
    for (i = 0; i < (int)len; i++) {
        double v;
        const unsigned char *src = (const unsigned char *)op + (size_t)i * opsize;
        switch (convert_from) {
        case NC_CHAR: v = 0; break;
        case NC_INT: v = (double)*(const int *)src; break;
        case NC_FLOAT: v = (double)*(const float *)src; break;
        default: v = *(const double *)src; break;
        }
        if (convert_from == NC_CHAR) { data[i] = *src; continue; }
        switch (type) {
        case NC_BYTE: { signed char c = (signed char)v; memcpy(data + i * es, &c, 1); } break;
        case NC_SHORT: { short s = (short)v; memcpy(data + i * es, &s, 2); } break;
        case NC_INT: { int k = (int)v; memcpy(data + i * es, &k, 4); } break;
        case NC_FLOAT: { float x = (float)v; memcpy(data + i * es, &x, 4); } break;
        case NC_DOUBLE: memcpy(data + i * es, &v, 8); break;
        default: data[i] = (unsigned char)v; break;
        }
    }
    if (idx < 0) {
        a = (ncl_att *)realloc(*list, sizeof(ncl_att) * (size_t)(*n + 1));
        if (!a) { free(data); return NC_ENOMEM; }
        *list = a;
        idx = (*n)++;
        strcpy(a[idx].name, name);
    } else {
        a = *list;
        free(a[idx].data);
    }
    a[idx].type = type;
    a[idx].nelems = len;
    a[idx].data = data;
    f->header_dirty = 1;
    return NC_NOERR;
}

int nc_put_att_text(int ncid, int varid, const char *name, size_t len, const char *op)
{
    return put_att(ncid, varid, name, NC_CHAR, len, op, 1, NC_CHAR);
}

int nc_put_att_float(int ncid, int varid, const char *name, nc_type xtype, size_t len, const float *op)
{
    return put_att(ncid, varid, name, xtype, len, op, sizeof(float), NC_FLOAT);
}

int nc_put_att_double(int ncid, int varid, const char *name, nc_type xtype, size_t len, const double *op)
{
    return put_att(ncid, varid, name, xtype, len, op, sizeof(double), NC_DOUBLE);
}

int nc_put_att_int(int ncid, int varid, const char *name, nc_type xtype, size_t len, const int *op)
{
    return put_att(ncid, varid, name, xtype, len, op, sizeof(int), NC_INT);
}

static uint64_t slab_bytes(ncl_file *f, ncl_var *v)
{
    uint64_t n = type_size(v->type);
    int i;
    for (i = v->is_record ? 1 : 0; i < v->ndims; i++) n *= f->dims[v->dimids[i]].len;
    return n;
}

int nc_enddef(int ncid)
{
    ncl_file *f = get_file(ncid);
    buf_t b = {0, 0, 0, 0};
    uint64_t off, hdr;
    int i, rc, nrec = 0;
    if (!f) return NC_EBADID;
    if (!f->in_define) return NC_ENOTINDEFINE;
    for (i = 0; i < f->nvars; i++) {
        f->vars[i].vsize = pad4(slab_bytes(f, &f->vars[i]));
        if (f->vars[i].is_record) nrec++;
    }
    /* first pass: header size with placeholder offsets */
    if ((rc = serialise_header(f, &b))) { free(b.p); return rc; }
    hdr = pad4(b.n);
    off = hdr;
    for (i = 0; i < f->nvars; i++) {
        ncl_var *v = &f->vars[i];
        if (v->is_record) continue;
        v->begin = off;
        off += v->vsize;
    }
    f->recsize = 0;
    for (i = 0; i < f->nvars; i++) {
        ncl_var *v = &f->vars[i];
        if (!v->is_record) continue;
        v->begin = off + f->recsize;
        /* a lone record variable is stored without inter-record padding */
        f->recsize += (nrec == 1) ? slab_bytes(f, v) : v->vsize;
    }
    if ((rc = serialise_header(f, &b))) { free(b.p); return rc; }
    if (fseeko(f->fp, 0, SEEK_SET) != 0 || fwrite(b.p, 1, b.n, f->fp) != b.n) { free(b.p); return NC_EIO; }
    free(b.p);
    f->in_define = 0;
    f->header_dirty = 0;
    return NC_NOERR;
}

int nc_redef(int ncid)
{
    ncl_file *f = get_file(ncid);
    if (!f) return NC_EBADID;
    return NC_EPERM; /* re-entering define mode (which moves data) is not supported */
}

/* ------------------------------------------------------------------ */
/* open / parse                                                         */
/* ------------------------------------------------------------------ */

static int get_bytes(buf_t *b, void *dst, size_t n)
{
    if (b->pos + n > b->n) return NC_ENOTNC;
    memcpy(dst, b->p + b->pos, n);
    b->pos += n;
    return NC_NOERR;
}

static int get_u32(buf_t *b, uint32_t *v)
{
    unsigned char c[4];
    int rc = get_bytes(b, c, 4);
    if (rc) return rc;
    *v = ((uint32_t)c[0] << 24) | ((uint32_t)c[1] << 16) | ((uint32_t)c[2] << 8) | c[3];
    return NC_NOERR;
}

static int get_u64(buf_t *b, uint64_t *v)
{
    unsigned char c[8];
    int i, rc = get_bytes(b, c, 8);
    if (rc) return rc;
    *v = 0;
    for (i = 0; i < 8; i++) *v = (*v << 8) | c[i];
    return NC_NOERR;
}

static int get_count(buf_t *b, int version, uint64_t *v)
{
    if (version == 5) return get_u64(b, v);
    {
        uint32_t u;
        int rc = get_u32(b, &u);
        *v = u;
        return rc;
    }
}

static int get_name(buf_t *b, int version, char *name)
{
    uint64_t n;
    int rc = get_count(b, version, &n);
    if (rc) return rc;
    if (n > NC_MAX_NAME) return NC_ENOTNC;
    if ((rc = get_bytes(b, name, (size_t)n))) return rc;
    name[n] = 0;
    b->pos += (size_t)(pad4(n) - n);
    return b->pos <= b->n ? NC_NOERR : NC_ENOTNC;
}

static int get_att_list(buf_t *b, int version, ncl_att **atts, int *natts)
{
    uint32_t tag;
    uint64_t n, i;
    int rc;
    if ((rc = get_u32(b, &tag)) || (rc = get_count(b, version, &n))) return rc;
    *atts = NULL;
    *natts = 0;
    if (tag == 0 && n == 0) return NC_NOERR;
    if (tag != NCL_MAGIC_ATT) return NC_ENOTNC;
    *atts = (ncl_att *)calloc((size_t)n, sizeof(ncl_att));
    if (!*atts) return NC_ENOMEM;
    for (i = 0; i < n; i++) {
        ncl_att *a = &(*atts)[i];
        uint32_t t;
        uint64_t ne;
        size_t es, bytes;
        if ((rc = get_name(b, version, a->name))) return rc;
        if ((rc = get_u32(b, &t)) || (rc = get_count(b, version, &ne))) return rc;
        a->type = (nc_type)t;
        a->nelems = (size_t)ne;
        es = type_size(a->type);
        if (es == 0) return NC_ENOTNC;
        bytes = es * a->nelems;
        a->data = (unsigned char *)malloc(bytes ? bytes : 1);
        if (!a->data) return NC_ENOMEM;
        if ((rc = get_bytes(b, a->data, bytes))) return rc;
        if (host_is_little()) swap_bytes(a->data, es, a->nelems);
        b->pos += (size_t)(pad4(bytes) - bytes);
        (*natts)++;
    }
    return NC_NOERR;
}

int nc_open(const char *path, int mode, int *ncidp)
{
    int id, rc;
    uint32_t tag;
    uint64_t n, i, j;
    FILE *fp;
    ncl_file *f;
    buf_t b = {0, 0, 0, 0};
    long long fsize;
    if (!path || !ncidp) return NC_EINVAL;
    id = alloc_slot();
    if (id < 0) return NC_ENFILE;
    fp = fopen(path, (mode & NC_WRITE) ? "r+b" : "rb");
    if (!fp) {
        release(&g_files[id]);
        return NC_EIO;
    }
    f = &g_files[id];
    f->fp = fp;
    f->in_use = 1;
    f->writable = (mode & NC_WRITE) != 0;
    /* read the header: grow the buffer until it parses (headers are small) */
    fseeko(fp, 0, SEEK_END);
    fsize = (long long)ftello(fp);
    {
        size_t want = (size_t)(fsize < (1 << 20) ? fsize : (1 << 20));
        for (;;) {
            b.p = (unsigned char *)realloc(b.p, want);
            if (!b.p) { release(f); return NC_ENOMEM; }
            fseeko(fp, 0, SEEK_SET);
            b.n = fread(b.p, 1, want, fp);
            b.pos = 0;
            {
                unsigned char magic[4];
                rc = get_bytes(&b, magic, 4);
                if (rc || magic[0] != 'C' || magic[1] != 'D' || magic[2] != 'F' ||
                    (magic[3] != 1 && magic[3] != 2 && magic[3] != 5)) {
                    free(b.p);
                    release(f);
                    return NC_ENOTNC;
                }
                f->version = magic[3];
            }
            rc = get_count(&b, f->version, &f->numrecs);
            if (!rc) rc = get_u32(&b, &tag);
            if (!rc) rc = get_count(&b, f->version, &n);
            if (!rc && tag == NCL_MAGIC_DIM) {
                f->dims = (ncl_dim *)calloc((size_t)n, sizeof(ncl_dim));
                for (i = 0; i < n && !rc; i++) {
                    uint64_t len = 0;
                    rc = get_name(&b, f->version, f->dims[i].name);
                    if (!rc) rc = get_count(&b, f->version, &len);
                    f->dims[i].len = (size_t)len;
                }
                f->ndims = (int)n;
            } else if (!rc && !(tag == 0 && n == 0)) rc = NC_ENOTNC;
            if (!rc) rc = get_att_list(&b, f->version, &f->gatts, &f->ngatts);
            if (!rc) rc = get_u32(&b, &tag);
            if (!rc) rc = get_count(&b, f->version, &n);
            if (!rc && tag == NCL_MAGIC_VAR) {
                f->vars = (ncl_var *)calloc((size_t)n, sizeof(ncl_var));
                for (i = 0; i < n && !rc; i++) {
                    ncl_var *v = &f->vars[i];
                    uint64_t nd = 0, d = 0, vs = 0;
                    uint32_t t = 0;
                    rc = get_name(&b, f->version, v->name);
                    if (!rc) rc = get_count(&b, f->version, &nd);
                    if (!rc && nd > NC_MAX_VAR_DIMS) rc = NC_ENOTNC;
                    v->ndims = (int)nd;
                    for (j = 0; j < nd && !rc; j++) {
                        rc = get_count(&b, f->version, &d);
                        if (!rc && d >= (uint64_t)f->ndims) rc = NC_ENOTNC;
                        v->dimids[j] = (int)d;
                    }
                    if (!rc) rc = get_att_list(&b, f->version, &v->atts, &v->natts);
                    if (!rc) rc = get_u32(&b, &t);
                    v->type = (nc_type)t;
                    if (!rc) rc = get_count(&b, f->version, &vs);
                    v->vsize = vs;
                    if (!rc) {
                        if (f->version == 1) {
                            uint32_t o;
                            rc = get_u32(&b, &o);
                            v->begin = o;
                        } else
                            rc = get_u64(&b, &v->begin);
                    }
                    if (!rc) {
                        v->is_record = (v->ndims > 0 && f->dims[v->dimids[0]].len == NC_UNLIMITED);
                        if (type_size(v->type) == 0) rc = NC_ENOTNC;
                    }
                    f->nvars++;
                }
            } else if (!rc && !(tag == 0 && n == 0)) rc = NC_ENOTNC;
            if (rc == NC_ENOTNC && b.n == want && (long long)want < fsize) {
                /* header longer than the buffer: retry with a larger one */
                int k;
                free(f->dims); f->dims = NULL; f->ndims = 0;
                free_atts(f->gatts, f->ngatts); f->gatts = NULL; f->ngatts = 0;
                for (k = 0; k < f->nvars; k++) free_atts(f->vars[k].atts, f->vars[k].natts);
                free(f->vars); f->vars = NULL; f->nvars = 0;
                want = (size_t)((long long)want * 4 < fsize ? (long long)want * 4 : fsize);
                continue;
            }
            break;
        }
    }
    free(b.p);
    if (rc) { release(f); return rc; }
    /* record size: recomputed from the variables' slab sizes */
    {
        int k, nrec = 0;
        for (k = 0; k < f->nvars; k++) if (f->vars[k].is_record) nrec++;
        f->recsize = 0;
        for (k = 0; k < f->nvars; k++) {
            ncl_var *v = &f->vars[k];
            uint64_t sb = slab_bytes(f, v);
            if (v->vsize == 0xFFFFFFFFull || v->vsize == 0) v->vsize = pad4(sb);
            if (v->is_record) f->recsize += (nrec == 1) ? sb : v->vsize;
        }
    }
    *ncidp = id;
    return NC_NOERR;
}

int nc_sync(int ncid)
{
    ncl_file *f = get_file(ncid);
    if (!f) return NC_EBADID;
    if (f->in_define) return NC_EINDEFINE;
    if (f->writable) {
        int rc = write_numrecs(f);
        if (rc) return rc;
        fflush(f->fp);
    }
    return NC_NOERR;
}

int nc_close(int ncid)
{
    ncl_file *f = get_file(ncid);
    int rc = NC_NOERR;
    if (!f) return NC_EBADID;
    if (f->writable) {
        if (f->in_define) rc = nc_enddef(ncid);
        if (!rc) rc = write_numrecs(f);
        if (!rc && f->header_dirty) {
            /* attributes changed in data mode: same sizes, rewrite in place */
            buf_t b = {0, 0, 0, 0};
            rc = serialise_header(f, &b);
            if (!rc && (fseeko(f->fp, 0, SEEK_SET) != 0 || fwrite(b.p, 1, b.n, f->fp) != b.n)) rc = NC_EIO;
            free(b.p);
        }
    }
    release(f);
    return rc;
}

/* ------------------------------------------------------------------ */
/* inquiry                                                              */
/* ------------------------------------------------------------------ */

int nc_inq_dimid(int ncid, const char *name, int *idp)
{
    ncl_file *f = get_file(ncid);
    int i;
    if (!f) return NC_EBADID;
    for (i = 0; i < f->ndims; i++)
        if (strcmp(f->dims[i].name, name) == 0) { if (idp) *idp = i; return NC_NOERR; }
    return NC_EBADDIM;
}

int nc_inq_dimlen(int ncid, int dimid, size_t *lenp)
{
    ncl_file *f = get_file(ncid);
    if (!f) return NC_EBADID;
    if (dimid < 0 || dimid >= f->ndims) return NC_EBADDIM;
    if (lenp) *lenp = f->dims[dimid].len == NC_UNLIMITED ? (size_t)f->numrecs : f->dims[dimid].len;
    return NC_NOERR;
}

int nc_inq_varid(int ncid, const char *name, int *varidp)
{
    ncl_file *f = get_file(ncid);
    int i;
    if (!f) return NC_EBADID;
    for (i = 0; i < f->nvars; i++)
        if (strcmp(f->vars[i].name, name) == 0) { if (varidp) *varidp = i; return NC_NOERR; }
    return NC_ENOTVAR;
}

int nc_inq_ndims(int ncid, int *ndimsp)
{
    ncl_file *f = get_file(ncid);
    if (!f) return NC_EBADID;
    if (ndimsp) *ndimsp = f->ndims;
    return NC_NOERR;
}

int nc_inq_nvars(int ncid, int *nvarsp)
{
    ncl_file *f = get_file(ncid);
    if (!f) return NC_EBADID;
    if (nvarsp) *nvarsp = f->nvars;
    return NC_NOERR;
}

int nc_inq_unlimdim(int ncid, int *unlimdimidp)
{
    ncl_file *f = get_file(ncid);
    int i;
    if (!f) return NC_EBADID;
    if (unlimdimidp) *unlimdimidp = -1;
    for (i = 0; i < f->ndims; i++)
        if (f->dims[i].len == NC_UNLIMITED && unlimdimidp) *unlimdimidp = i;
    return NC_NOERR;
}

int nc_inq_vartype(int ncid, int varid, nc_type *xtypep)
{
    ncl_file *f = get_file(ncid);
    if (!f) return NC_EBADID;
    if (varid < 0 || varid >= f->nvars) return NC_ENOTVAR;
    if (xtypep) *xtypep = f->vars[varid].type;
    return NC_NOERR;
}

int nc_inq_varndims(int ncid, int varid, int *ndimsp)
{
    ncl_file *f = get_file(ncid);
    if (!f) return NC_EBADID;
    if (varid < 0 || varid >= f->nvars) return NC_ENOTVAR;
    if (ndimsp) *ndimsp = f->vars[varid].ndims;
    return NC_NOERR;
}

int nc_inq_vardimid(int ncid, int varid, int *dimidsp)
{
    ncl_file *f = get_file(ncid);
    int i;
    if (!f) return NC_EBADID;
    if (varid < 0 || varid >= f->nvars) return NC_ENOTVAR;
    if (dimidsp)
        for (i = 0; i < f->vars[varid].ndims; i++) dimidsp[i] = f->vars[varid].dimids[i];
    return NC_NOERR;
}

static ncl_att *find_att(ncl_file *f, int varid, const char *name)
{
    ncl_att *list;
    int n, i;
    if (varid == NC_GLOBAL) { list = f->gatts; n = f->ngatts; }
    else if (varid >= 0 && varid < f->nvars) { list = f->vars[varid].atts; n = f->vars[varid].natts; }
    else return NULL;
    for (i = 0; i < n; i++)
        if (strcmp(list[i].name, name) == 0) return &list[i];
    return NULL;
}

int nc_inq_attlen(int ncid, int varid, const char *name, size_t *lenp)
{
    ncl_file *f = get_file(ncid);
    ncl_att *a;
    if (!f) return NC_EBADID;
    if (varid != NC_GLOBAL && (varid < 0 || varid >= f->nvars)) return NC_ENOTVAR;
    a = find_att(f, varid, name);
    if (!a) return NC_ENOTATT;
    if (lenp) *lenp = a->nelems;
    return NC_NOERR;
}

int nc_get_att_text(int ncid, int varid, const char *name, char *ip)
{
    ncl_file *f = get_file(ncid);
    ncl_att *a;
    if (!f) return NC_EBADID;
    a = find_att(f, varid, name);
    if (!a) return NC_ENOTATT;
    if (a->type != NC_CHAR) return NC_EBADTYPE;
    memcpy(ip, a->data, a->nelems);
    return NC_NOERR;
}

static double value_as_double(nc_type t, const unsigned char *p)
{
    switch (t) {
    case NC_BYTE: return (double)*(const signed char *)p;
    case NC_CHAR: case NC_UBYTE: return (double)*p;
    case NC_SHORT: { short s; memcpy(&s, p, 2); return s; }
    case NC_USHORT: { unsigned short s; memcpy(&s, p, 2); return s; }
    case NC_INT: { int k; memcpy(&k, p, 4); return k; }
    case NC_UINT: { unsigned k; memcpy(&k, p, 4); return k; }
    case NC_FLOAT: { float x; memcpy(&x, p, 4); return x; }
    case NC_DOUBLE: { double x; memcpy(&x, p, 8); return x; }
    case NC_INT64: { long long k; memcpy(&k, p, 8); return (double)k; }
    case NC_UINT64: { unsigned long long k; memcpy(&k, p, 8); return (double)k; }
    default: return 0;
    }
}

int nc_get_att_double(int ncid, int varid, const char *name, double *ip)
{
    ncl_file *f = get_file(ncid);
    ncl_att *a;
    size_t i, es;
    if (!f) return NC_EBADID;
    a = find_att(f, varid, name);
    if (!a) return NC_ENOTATT;
    if (a->type == NC_CHAR) return NC_EBADTYPE;
    es = type_size(a->type);
    for (i = 0; i < a->nelems; i++) ip[i] = value_as_double(a->type, a->data + i * es);
    return NC_NOERR;
}

/* ------------------------------------------------------------------ */
/* data access                                                          */
/* ------------------------------------------------------------------ */

/* Visits every contiguous run of a hyperslab [start, start+count) of v.
 * `fn` receives the file offset, the number of elements and the running
 * element index into the caller's buffer. */
typedef int (*run_fn)(ncl_file *f, ncl_var *v, uint64_t off, size_t nelem, size_t bufidx, void *ctx);

static int for_each_run(ncl_file *f, ncl_var *v, const size_t *start, const size_t *count, run_fn fn, void *ctx)
{
    int nd = v->ndims, i, m, rc;
    size_t es = type_size(v->type);
    uint64_t stride[NC_MAX_VAR_DIMS];
    size_t len[NC_MAX_VAR_DIMS], idx[NC_MAX_VAR_DIMS];
    size_t runlen, bufidx = 0;
    if (nd == 0) return fn(f, v, v->begin, 1, 0, ctx);
    for (i = 0; i < nd; i++) {
        len[i] = f->dims[v->dimids[i]].len;
        if (count[i] == 0) return NC_NOERR;
    }
    /* byte strides of each dimension */
    stride[nd - 1] = es;
    for (i = nd - 2; i >= 0; i--) stride[i] = stride[i + 1] * (uint64_t)len[i + 1];
    if (v->is_record) stride[0] = f->recsize;
    /* merge trailing dimensions that are read/written in full */
    m = nd - 1;
    runlen = count[nd - 1];
    while (m > 0 && start[m] == 0 && count[m] == len[m]) {
        if (m - 1 == 0 && v->is_record) break; /* records are not contiguous */
        runlen *= count[m - 1];
        m--;
    }
    /* dims [0, m) are iterated; dim m .. nd-1 form one run of runlen elements */
    for (i = 0; i < m; i++) idx[i] = 0;
    for (;;) {
        uint64_t off = v->begin;
        for (i = 0; i < m; i++) off += (uint64_t)(start[i] + idx[i]) * stride[i];
        off += (uint64_t)start[m] * stride[m];
        if ((rc = fn(f, v, off, runlen, bufidx, ctx))) return rc;
        bufidx += runlen;
        for (i = m - 1; i >= 0; i--) {
            if (++idx[i] < count[i]) break;
            idx[i] = 0;
        }
        if (i < 0) break;
    }
    return NC_NOERR;
}

typedef struct { const void *src; nc_type memtype; } put_ctx;

static int put_run(ncl_file *f, ncl_var *v, uint64_t off, size_t n, size_t bufidx, void *vctx)
{
    put_ctx *c = (put_ctx *)vctx;
    size_t es = type_size(v->type), ms = type_size(c->memtype), i, chunk = 1 << 16, done = 0;
    unsigned char *tmp = (unsigned char *)malloc(es * (n < chunk ? n : chunk));
    if (!tmp) return NC_ENOMEM;
    if (fseeko(f->fp, (off_t)off, SEEK_SET) != 0) { free(tmp); return NC_EIO; }
    while (done < n) {
        size_t k = n - done < chunk ? n - done : chunk;
        const unsigned char *src = (const unsigned char *)c->src + (bufidx + done) * ms;
        if (c->memtype == v->type) memcpy(tmp, src, k * es);
        else {
            for (i = 0; i < k; i++) {
                double x = value_as_double(c->memtype, src + i * ms);
                if (v->type == NC_FLOAT) { float y = (float)x; memcpy(tmp + i * 4, &y, 4); }
                else if (v->type == NC_DOUBLE) memcpy(tmp + i * 8, &x, 8);
                else if (v->type == NC_INT) { int y = (int)x; memcpy(tmp + i * 4, &y, 4); }
                else if (v->type == NC_SHORT) { short y = (short)x; memcpy(tmp + i * 2, &y, 2); }
                else tmp[i] = (unsigned char)(signed char)x;
            }
        }
        if (host_is_little()) swap_bytes(tmp, es, k);
        if (fwrite(tmp, es, k, f->fp) != k) { free(tmp); return NC_EIO; }
        done += k;
    }
    free(tmp);
    return NC_NOERR;
}

static int put_vara(int ncid, int varid, const size_t *startp, const size_t *countp, const void *op, nc_type memtype)
{
    ncl_file *f = get_file(ncid);
    ncl_var *v;
    put_ctx c;
    int i, rc;
    if (!f) return NC_EBADID;
    if (!f->writable) return NC_EPERM;
    if (f->in_define) return NC_EINDEFINE;
    if (varid < 0 || varid >= f->nvars) return NC_ENOTVAR;
    v = &f->vars[varid];
    if (v->type == NC_CHAR) return NC_EBADTYPE;
    for (i = 0; i < v->ndims; i++) {
        size_t len = f->dims[v->dimids[i]].len;
        if (i == 0 && v->is_record) continue;
        if (startp[i] > len) return NC_EINVALCOORDS;
        if (startp[i] + countp[i] > len) return NC_EEDGE;
    }
    c.src = op;
    c.memtype = memtype;
    rc = for_each_run(f, v, startp, countp, put_run, &c);
    if (rc) return rc;
    if (v->is_record && startp[0] + countp[0] > f->numrecs) f->numrecs = startp[0] + countp[0];
    return NC_NOERR;
}

static void full_extent(ncl_file *f, ncl_var *v, size_t *start, size_t *count)
{
    int i;
    for (i = 0; i < v->ndims; i++) {
        start[i] = 0;
        count[i] = (i == 0 && v->is_record) ? (size_t)f->numrecs : f->dims[v->dimids[i]].len;
    }
}

int nc_put_var_double(int ncid, int varid, const double *op)
{
    ncl_file *f = get_file(ncid);
    size_t s[NC_MAX_VAR_DIMS], c[NC_MAX_VAR_DIMS];
    if (!f) return NC_EBADID;
    if (varid < 0 || varid >= f->nvars) return NC_ENOTVAR;
    full_extent(f, &f->vars[varid], s, c);
    return put_vara(ncid, varid, s, c, op, NC_DOUBLE);
}

int nc_put_var_float(int ncid, int varid, const float *op)
{
    ncl_file *f = get_file(ncid);
    size_t s[NC_MAX_VAR_DIMS], c[NC_MAX_VAR_DIMS];
    if (!f) return NC_EBADID;
    if (varid < 0 || varid >= f->nvars) return NC_ENOTVAR;
    full_extent(f, &f->vars[varid], s, c);
    return put_vara(ncid, varid, s, c, op, NC_FLOAT);
}

int nc_put_vara_float(int ncid, int varid, const size_t *startp, const size_t *countp, const float *op)
{
    return put_vara(ncid, varid, startp, countp, op, NC_FLOAT);
}

int nc_put_vara_double(int ncid, int varid, const size_t *startp, const size_t *countp, const double *op)
{
    return put_vara(ncid, varid, startp, countp, op, NC_DOUBLE);
}

typedef struct { void *dst; nc_type memtype; } get_ctx;

static int get_run(ncl_file *f, ncl_var *v, uint64_t off, size_t n, size_t bufidx, void *vctx)
{
    get_ctx *c = (get_ctx *)vctx;
    size_t es = type_size(v->type), ms = type_size(c->memtype), i, chunk = 1 << 16, done = 0;
    unsigned char *tmp = (unsigned char *)malloc(es * (n < chunk ? n : chunk));
    if (!tmp) return NC_ENOMEM;
    if (fseeko(f->fp, (off_t)off, SEEK_SET) != 0) { free(tmp); return NC_EIO; }
    while (done < n) {
        size_t k = n - done < chunk ? n - done : chunk;
        unsigned char *dst = (unsigned char *)c->dst + (bufidx + done) * ms;
        if (fread(tmp, es, k, f->fp) != k) { free(tmp); return NC_EIO; }
        if (host_is_little()) swap_bytes(tmp, es, k);
        if (c->memtype == v->type) memcpy(dst, tmp, k * es);
        else {
            for (i = 0; i < k; i++) {
                double x = value_as_double(v->type, tmp + i * es);
                if (c->memtype == NC_FLOAT) { float y = (float)x; memcpy(dst + i * 4, &y, 4); }
                else memcpy(dst + i * 8, &x, 8);
            }
        }
        done += k;
    }
    free(tmp);
    return NC_NOERR;
}

static int get_vara(int ncid, int varid, const size_t *startp, const size_t *countp, void *ip, nc_type memtype)
{
    ncl_file *f = get_file(ncid);
    ncl_var *v;
    get_ctx c;
    int i;
    if (!f) return NC_EBADID;
    if (varid < 0 || varid >= f->nvars) return NC_ENOTVAR;
    v = &f->vars[varid];
    if (v->type == NC_CHAR) return NC_EBADTYPE;
    for (i = 0; i < v->ndims; i++) {
        size_t len = (i == 0 && v->is_record) ? (size_t)f->numrecs : f->dims[v->dimids[i]].len;
        if (startp[i] + countp[i] > len) return NC_EEDGE;
    }
    c.dst = ip;
    c.memtype = memtype;
    return for_each_run(f, v, startp, countp, get_run, &c);
}

int nc_get_var_double(int ncid, int varid, double *ip)
{
    ncl_file *f = get_file(ncid);
    size_t s[NC_MAX_VAR_DIMS], c[NC_MAX_VAR_DIMS];
    if (!f) return NC_EBADID;
    if (varid < 0 || varid >= f->nvars) return NC_ENOTVAR;
    full_extent(f, &f->vars[varid], s, c);
    return get_vara(ncid, varid, s, c, ip, NC_DOUBLE);
}

int nc_get_var_float(int ncid, int varid, float *ip)
{
    ncl_file *f = get_file(ncid);
    size_t s[NC_MAX_VAR_DIMS], c[NC_MAX_VAR_DIMS];
    if (!f) return NC_EBADID;
    if (varid < 0 || varid >= f->nvars) return NC_ENOTVAR;
    full_extent(f, &f->vars[varid], s, c);
    return get_vara(ncid, varid, s, c, ip, NC_FLOAT);
}

int nc_get_vara_float(int ncid, int varid, const size_t *startp, const size_t *countp, float *ip)
{
    return get_vara(ncid, varid, startp, countp, ip, NC_FLOAT);
}
