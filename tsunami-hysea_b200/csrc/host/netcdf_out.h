// NetCDF outputs of a run, with the dimensions, variables and attributes
// the reference writes (src/GPU/netcdfTH.cu:93-545 for <prefix>.nc,
// src/GPU/netcdfSeries.cu:26-373 for <prefix>_ts.nc).  Files are NetCDF
// classic (64-bit offset) written through nclite; the reference asks
// libnetcdf for NetCDF-4 with deflate level 5, which needs HDF5.
#pragma once
#include <string>
#include <vector>

#include "../../../include/thysea.h"

namespace thy {

struct RunMeta {
    std::string problem_name;
    std::string version = "1.3.0";
    const thy_problem *p = nullptr;
};

class GridWriter {
public:
    // creates <path>, defines everything and writes lon/lat and the original bathymetry
    int open(const std::string &path, const RunMeta &m, const float *bathy_m);
    int write_snapshot(int index, double time_s, const float *eta, const float *ux, const float *uy);
    int write_final(const float *deformed_bathy, const float *max_height, const float *arrival);
    int close();
    ~GridWriter() { close(); }

private:
    int ncid_ = -1, time_id_ = -1, eta_id_ = -1, ux_id_ = -1, uy_id_ = -1, emax_id_ = -1, arr_id_ = -1,
        defb_id_ = -1;
    int nx_ = 0, ny_ = 0;
    bool okada_ = false;
};

class SeriesWriter {
public:
    // creates <path> with nP gauges; lon/lat are the gauge coordinates as listed
    int open(const std::string &path, const RunMeta &m, int nP, const double *lon, const double *lat);
    int write_sample(int index, double time_s, const float *eta, const float *ux, const float *uy);
    int write_final(const float *bathy, const float *min_height, const float *max_height);
    int close();
    ~SeriesWriter() { close(); }

private:
    int ncid_ = -1, time_id_ = -1, eta_id_ = -1, ux_id_ = -1, uy_id_ = -1, min_id_ = -1, max_id_ = -1,
        bathy_id_ = -1;
    int np_ = 0;
};

}  // namespace thy
