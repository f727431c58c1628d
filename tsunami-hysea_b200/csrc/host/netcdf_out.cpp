// NetCDF writers for the gridded output (<prefix>.nc) and the gauge time
// series (<prefix>_ts.nc).  The dimensions, variable names, attribute names,
// texts and values are those of the reference (they are the output format a
// drop-in must keep): src/GPU/netcdfTH.cu:93-545 and
// src/GPU/netcdfSeries.cu:26-373.
#include "netcdf_out.h"

#include <cmath>
#include <cstdio>
#include <cstring>
#include <ctime>
#include <sys/time.h>

#include "../nclite/netcdf.h"

namespace thy {

namespace {

constexpr double kEps = 2.220446049250313e-16;

void put_text(int nc, int var, const char *name, const char *text)
{
    nc_put_att_text(nc, var, name, strlen(text), text);
}

void put_float(int nc, int var, const char *name, double v)
{
    float f = (float)v;
    nc_put_att_float(nc, var, name, NC_FLOAT, 1, &f);
}

void put_int(int nc, int var, const char *name, int v) { nc_put_att_int(nc, var, name, NC_INT, 1, &v); }

void fill_attrs(int nc, int var)
{
    float fill = -9999.0f;
    nc_put_att_float(nc, var, "missing_value", NC_FLOAT, 1, &fill);
    nc_put_att_float(nc, var, "_FillValue", NC_FLOAT, 1, &fill);
}

// global attributes shared by both files (netcdfTH.cu:319-412, netcdfSeries.cu:218-310)
void global_attrs(int nc, const RunMeta &m, const char *title, bool grid_file)
{
    const thy_problem &p = *m.p;
    char buf[512], name[64];
    put_text(nc, NC_GLOBAL, "Conventions", "CF-1.0");
    put_text(nc, NC_GLOBAL, "title", title);
    put_text(nc, NC_GLOBAL, "Tsunami-HySEA_miniapp_version", m.version.c_str());
    put_text(nc, NC_GLOBAL, "creator_name", "EDANYA Group");
    put_text(nc, NC_GLOBAL, "institution", "University of Malaga");
    put_text(nc, NC_GLOBAL, "comments", " ");
    put_text(nc, NC_GLOBAL, "references", " ");
    {
        struct timeval tv;
        char date[24];
        gettimeofday(&tv, nullptr);
        strftime(date, sizeof(date), "%Y-%m-%d %H:%M:%S", localtime(&tv.tv_sec));
        put_text(nc, NC_GLOBAL, "history", date);
    }
    put_text(nc, NC_GLOBAL, "problem_name", m.problem_name.c_str());
    put_float(nc, NC_GLOBAL, "simulation_time", p.t_end * p.T);
    if (grid_file) put_int(nc, NC_GLOBAL, "output_grid_interval", 1);
    const bool periodic = std::fabs(p.border_left - 2.0) < kEps && std::fabs(p.border_right - 2.0) < kEps;
    put_text(nc, NC_GLOBAL, "upper_border", std::fabs(p.border_up - 1.0) < kEps ? "open" : "wall");
    put_text(nc, NC_GLOBAL, "lower_border", std::fabs(p.border_low - 1.0) < kEps ? "open" : "wall");
    if (periodic) {
        put_text(nc, NC_GLOBAL, "left_border", "periodic");
        put_text(nc, NC_GLOBAL, "right_border", "periodic");
    } else {
        put_text(nc, NC_GLOBAL, "left_border", std::fabs(p.border_left - 1.0) < kEps ? "open" : "wall");
        put_text(nc, NC_GLOBAL, "right_border", std::fabs(p.border_right - 1.0) < kEps ? "open" : "wall");
    }
    put_float(nc, NC_GLOBAL, "CFL", p.cfl);
    put_float(nc, NC_GLOBAL, "epsilon_h", p.eps_h * p.H);
    put_float(nc, NC_GLOBAL, "water_bottom_friction", std::sqrt(p.mf0 * std::pow(p.H, 4.0 / 3.0) / (9.81 * p.L)));
    put_float(nc, NC_GLOBAL, "max_velocity_water", p.vmax * p.Q / p.H);
    put_float(nc, NC_GLOBAL, "threshold_2swaf", p.hpos * p.H);
    put_float(nc, NC_GLOBAL, "stability_coefficient", 1.0 - p.cvis);
    put_float(nc, NC_GLOBAL, "threshold_arrival_times", p.dif_at * p.H);
    if (!p.okada_flag) {
        put_text(nc, NC_GLOBAL, "initialization_mode", "sea_surface_from_file");
    } else {
        put_text(nc, NC_GLOBAL, "initialization_mode", "okada_standard");
        put_int(nc, NC_GLOBAL, "num_faults", p.nfaults);
        for (int i = 0; i < p.nfaults; i++) {
            const double *f = p.faults + 10 * i;
            snprintf(name, sizeof(name), "fault_%d", i + 1);
            snprintf(buf, sizeof(buf),
                     "time: %.4f, lon: %.4f, lat: %.4f, depth: %.4f, length: %.4f, width: %.4f, strike: %.4f, dip: "
                     "%.4f, rake: %.4f, slip: %.4f",
                     f[0], f[1], f[2], f[3], f[4], f[5], f[6], f[7], f[8], f[9]);
            put_text(nc, NC_GLOBAL, name, buf);
        }
        if (p.crop_flag == 1) {
            put_text(nc, NC_GLOBAL, "crop_deformations", "relative");
            put_float(nc, NC_GLOBAL, "crop_percentage_0-1", p.crop_value);
        } else if (p.crop_flag == 2) {
            put_text(nc, NC_GLOBAL, "crop_deformations", "absolute");
            put_float(nc, NC_GLOBAL, "crop_threshold", p.crop_value * p.H);
        } else {
            put_text(nc, NC_GLOBAL, "crop_deformations", "no");
        }
    }
}

}  // namespace

int GridWriter::open(const std::string &path, const RunMeta &m, const float *bathy_m)
{
    const thy_problem &p = *m.p;
    int nc, dlon, dlat, dglon, dglat, dtime, vlon, vlat, vglon, vglat, vbat;
    if (nc_create(path.c_str(), NC_CLOBBER | NC_NETCDF4, &nc) != NC_NOERR) return THY_ERR_HOST;
    ncid_ = nc;
    nx_ = p.nx;
    ny_ = p.ny;
    okada_ = p.okada_flag != 0;
    nc_def_dim(nc, "lon", p.nx, &dlon);
    nc_def_dim(nc, "lat", p.ny, &dlat);
    nc_def_dim(nc, "grid_lon", p.nx, &dglon);
    nc_def_dim(nc, "grid_lat", p.ny, &dglat);
    nc_def_dim(nc, "time", NC_UNLIMITED, &dtime);
    nc_def_var(nc, "lon", NC_DOUBLE, 1, &dlon, &vlon);
    nc_def_var(nc, "lat", NC_DOUBLE, 1, &dlat, &vlat);
    nc_def_var(nc, "grid_lon", NC_DOUBLE, 1, &dglon, &vglon);
    nc_def_var(nc, "grid_lat", NC_DOUBLE, 1, &dglat, &vglat);
    int gdims[2] = {dglat, dglon};
    if (okada_) {
        nc_def_var(nc, "original_bathy", NC_FLOAT, 2, gdims, &vbat);
        nc_def_var(nc, "deformed_bathy", NC_FLOAT, 2, gdims, &defb_id_);
    } else {
        nc_def_var(nc, "bathymetry", NC_FLOAT, 2, gdims, &vbat);
    }
    nc_def_var(nc, "time", NC_FLOAT, 1, &dtime, &time_id_);
    int dims2[2] = {dlat, dlon}, dims3[3] = {dtime, dlat, dlon};
    nc_def_var(nc, "max_height", NC_FLOAT, 2, dims2, &emax_id_);
    nc_def_var(nc, "arrival_times", NC_FLOAT, 2, dims2, &arr_id_);
    nc_def_var(nc, "eta", NC_FLOAT, 3, dims3, &eta_id_);
    put_text(nc, eta_id_, "units", "meters");
    put_text(nc, eta_id_, "long_name", "Wave amplitude");
    nc_def_var(nc, "ux", NC_FLOAT, 3, dims3, &ux_id_);
    put_text(nc, ux_id_, "units", "meters/second");
    put_text(nc, ux_id_, "long_name", "Velocity of water along longitude");
    nc_def_var(nc, "uy", NC_FLOAT, 3, dims3, &uy_id_);
    put_text(nc, uy_id_, "units", "meters/second");
    put_text(nc, uy_id_, "long_name", "Velocity of water along latitude");
    if (okada_) {
        put_text(nc, vbat, "long_name", "Grid original bathymetry");
        put_text(nc, vbat, "standard_name", "original depth");
        put_text(nc, vbat, "units", "meters");
        fill_attrs(nc, vbat);
        put_text(nc, defb_id_, "long_name", "Grid deformed bathymetry");
        put_text(nc, defb_id_, "standard_name", "deformed depth");
        put_text(nc, defb_id_, "units", "meters");
        fill_attrs(nc, defb_id_);
    } else {
        put_text(nc, vbat, "long_name", "Grid bathymetry");
        put_text(nc, vbat, "standard_name", "depth");
        put_text(nc, vbat, "units", "meters");
        fill_attrs(nc, vbat);
    }
    put_text(nc, vglon, "long_name", "Grid longitude");
    put_text(nc, vglon, "units", "degrees_east");
    put_text(nc, vglat, "long_name", "Grid latitude");
    put_text(nc, vglat, "units", "degrees_north");
    put_text(nc, emax_id_, "long_name", "Maximum wave amplitude");
    put_text(nc, emax_id_, "units", "meters");
    fill_attrs(nc, emax_id_);
    put_text(nc, vlon, "standard_name", "longitude");
    put_text(nc, vlon, "long_name", "longitude");
    put_text(nc, vlon, "units", "degrees_east");
    put_text(nc, vlat, "standard_name", "latitude");
    put_text(nc, vlat, "long_name", "latitude");
    put_text(nc, vlat, "units", "degrees_north");
    put_text(nc, time_id_, "long_name", "Time");
    put_text(nc, time_id_, "units", "seconds since 1970-01-01");
    fill_attrs(nc, eta_id_);
    fill_attrs(nc, ux_id_);
    fill_attrs(nc, uy_id_);
    global_attrs(nc, m, "TsunamiHySEA model output", true);
    if (nc_enddef(nc) != NC_NOERR) return THY_ERR_HOST;
    nc_put_var_double(nc, vlon, p.lon);
    nc_put_var_double(nc, vlat, p.lat);
    nc_put_var_double(nc, vglon, p.lon);
    nc_put_var_double(nc, vglat, p.lat);
    nc_put_var_float(nc, vbat, bathy_m);
    return THY_OK;
}

int GridWriter::write_snapshot(int index, double time_s, const float *eta, const float *ux, const float *uy)
{
    if (ncid_ < 0) return THY_ERR_HOST;
    const size_t rec = (size_t)index, one = 1;
    const float t = (float)time_s;
    const size_t start[3] = {rec, 0, 0}, count[3] = {1, (size_t)ny_, (size_t)nx_};
    int rc = nc_put_vara_float(ncid_, time_id_, &rec, &one, &t);
    rc |= nc_put_vara_float(ncid_, eta_id_, start, count, eta);
    rc |= nc_put_vara_float(ncid_, ux_id_, start, count, ux);
    rc |= nc_put_vara_float(ncid_, uy_id_, start, count, uy);
    rc |= nc_sync(ncid_);
    return rc ? THY_ERR_HOST : THY_OK;
}

int GridWriter::write_final(const float *deformed_bathy, const float *max_height, const float *arrival)
{
    if (ncid_ < 0) return THY_ERR_HOST;
    int rc = 0;
    if (okada_ && deformed_bathy) rc |= nc_put_var_float(ncid_, defb_id_, deformed_bathy);
    rc |= nc_put_var_float(ncid_, emax_id_, max_height);
    rc |= nc_put_var_float(ncid_, arr_id_, arrival);
    return rc ? THY_ERR_HOST : THY_OK;
}

int GridWriter::close()
{
    if (ncid_ < 0) return THY_OK;
    int rc = nc_close(ncid_);
    ncid_ = -1;
    return rc ? THY_ERR_HOST : THY_OK;
}

int SeriesWriter::open(const std::string &path, const RunMeta &m, int nP, const double *lon, const double *lat)
{
    const thy_problem &p = *m.p;
    int nc, dpts, dtime, vlon, vlat;
    if (nc_create(path.c_str(), NC_CLOBBER | NC_NETCDF4, &nc) != NC_NOERR) return THY_ERR_HOST;
    ncid_ = nc;
    np_ = nP;
    nc_def_dim(nc, "grid_npoints", nP, &dpts);
    nc_def_dim(nc, "time", NC_UNLIMITED, &dtime);
    double fill_d = -9999.0;
    nc_def_var(nc, p.okada_flag ? "deformed_bathy" : "bathymetry", NC_FLOAT, 1, &dpts, &bathy_id_);
    nc_def_var(nc, "time", NC_FLOAT, 1, &dtime, &time_id_);
    nc_def_var(nc, "longitude", NC_DOUBLE, 1, &dpts, &vlon);
    put_text(nc, vlon, "units", "degrees_east");
    nc_put_att_double(nc, vlon, "missing_value", NC_DOUBLE, 1, &fill_d);
    nc_put_att_double(nc, vlon, "_FillValue", NC_DOUBLE, 1, &fill_d);
    nc_def_var(nc, "latitude", NC_DOUBLE, 1, &dpts, &vlat);
    put_text(nc, vlat, "units", "degrees_north");
    nc_put_att_double(nc, vlat, "missing_value", NC_DOUBLE, 1, &fill_d);
    nc_put_att_double(nc, vlat, "_FillValue", NC_DOUBLE, 1, &fill_d);
    nc_def_var(nc, "min_height", NC_FLOAT, 1, &dpts, &min_id_);
    put_text(nc, min_id_, "long_name", "Minimum wave amplitude");
    put_text(nc, min_id_, "units", "meters");
    fill_attrs(nc, min_id_);
    nc_def_var(nc, "max_height", NC_FLOAT, 1, &dpts, &max_id_);
    put_text(nc, max_id_, "long_name", "Maximum wave amplitude");
    put_text(nc, max_id_, "units", "meters");
    fill_attrs(nc, max_id_);
    int d2[2] = {dtime, dpts};
    nc_def_var(nc, "eta", NC_FLOAT, 2, d2, &eta_id_);
    put_text(nc, eta_id_, "units", "meters");
    put_text(nc, eta_id_, "long_name", "Wave amplitude");
    fill_attrs(nc, eta_id_);
    nc_def_var(nc, "ux", NC_FLOAT, 2, d2, &ux_id_);
    put_text(nc, ux_id_, "units", "meters/second");
    put_text(nc, ux_id_, "long_name", "Velocity of water along longitude");
    fill_attrs(nc, ux_id_);
    nc_def_var(nc, "uy", NC_FLOAT, 2, d2, &uy_id_);
    put_text(nc, uy_id_, "units", "meters/second");
    put_text(nc, uy_id_, "long_name", "Velocity of water along latitude");
    fill_attrs(nc, uy_id_);
    if (p.okada_flag) {
        put_text(nc, bathy_id_, "long_name", "Grid deformed bathymetry");
        put_text(nc, bathy_id_, "standard_name", "deformed depth");
    } else {
        put_text(nc, bathy_id_, "long_name", "Grid bathymetry");
        put_text(nc, bathy_id_, "standard_name", "depth");
    }
    put_text(nc, bathy_id_, "units", "meters");
    fill_attrs(nc, bathy_id_);
    put_text(nc, time_id_, "long_name", "Time");
    put_text(nc, time_id_, "units", "seconds since 1970-01-01");
    global_attrs(nc, m, "Time series output of TsunamiHySEA model", false);
    if (nc_enddef(nc) != NC_NOERR) return THY_ERR_HOST;
    if (nP > 0) {
        nc_put_var_double(nc, vlon, lon);
        nc_put_var_double(nc, vlat, lat);
    }
    return THY_OK;
}

int SeriesWriter::write_sample(int index, double time_s, const float *eta, const float *ux, const float *uy)
{
    if (ncid_ < 0) return THY_ERR_HOST;
    const size_t rec = (size_t)index, one = 1;
    const float t = (float)time_s;
    const size_t start[2] = {rec, 0}, count[2] = {1, (size_t)np_};
    int rc = nc_put_vara_float(ncid_, time_id_, &rec, &one, &t);
    rc |= nc_put_vara_float(ncid_, eta_id_, start, count, eta);
    rc |= nc_put_vara_float(ncid_, ux_id_, start, count, ux);
    rc |= nc_put_vara_float(ncid_, uy_id_, start, count, uy);
    rc |= nc_sync(ncid_);
    return rc ? THY_ERR_HOST : THY_OK;
}

int SeriesWriter::write_final(const float *bathy, const float *min_height, const float *max_height)
{
    if (ncid_ < 0) return THY_ERR_HOST;
    int rc = nc_put_var_float(ncid_, bathy_id_, bathy);
    rc |= nc_put_var_float(ncid_, min_id_, min_height);
    rc |= nc_put_var_float(ncid_, max_id_, max_height);
    return rc ? THY_ERR_HOST : THY_OK;
}

int SeriesWriter::close()
{
    if (ncid_ < 0) return THY_OK;
    int rc = nc_close(ncid_);
    ncid_ = -1;
    return rc ? THY_ERR_HOST : THY_OK;
}

}  // namespace thy
