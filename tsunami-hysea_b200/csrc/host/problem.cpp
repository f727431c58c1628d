// Problem set-up: the problem-file loader and the nondimensionalisation that
// the reference's cargarDatosProblema() performs before calling
// shallowWater() (src/Problema.cxx:11-477), restated in C++.
//
//   thy_load_problem_file  .txt grammar (src/Problema.cxx:150-343): one value
//                          per line, lines whose first non-blank character is
//                          '#' skipped, the first token of a line is the value;
//                          GRD files read through the NetCDF API (nclite);
//   thy_prepare            scales, dimensionless parameters, bathymetry shift
//                          by Hmin, per-row metric terms, gauge cells.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <sys/stat.h>
#include <vector>

#include "../../../include/thysea.h"
#include "../nclite/netcdf.h"

namespace {

constexpr double kEps = DBL_EPSILON;
constexpr double kEarthRadius = 6378136.6;
constexpr int kMaxFaults = 5000;
constexpr int kSpongeCells = 4;

bool file_exists(const std::string &f)
{
    struct stat st;
    return stat(f.c_str(), &st) == 0;
}

// next non-comment line (src/Problema.cxx:150-170); empty at end of file
std::string next_line(std::ifstream &in)
{
    std::string line;
    while (std::getline(in, line)) {
        size_t p = line.find_first_not_of(" \t\r\n");
        if (p == std::string::npos) continue;
        line.erase(0, p);
        if (line[0] != '#') return line;
    }
    return std::string();
}

template <class T>
bool next_value(std::ifstream &in, T &v)
{
    std::istringstream iss(next_line(in));
    return static_cast<bool>(iss >> v);
}

int read_grd(const std::string &path, std::vector<double> &lon, std::vector<double> &lat, std::vector<float> &z)
{
    int nc, dx, dy, vx, vy, vz;
    size_t nx, ny;
    if (nc_open(path.c_str(), NC_NOWRITE, &nc) != NC_NOERR) return 1;
    int bad = 0;
    if (nc_inq_dimid(nc, "lon", &dx) != NC_NOERR && nc_inq_dimid(nc, "x", &dx) != NC_NOERR) bad = 1;
    if (!bad && nc_inq_dimid(nc, "lat", &dy) != NC_NOERR && nc_inq_dimid(nc, "y", &dy) != NC_NOERR) bad = 1;
    if (!bad && (nc_inq_dimlen(nc, dx, &nx) != NC_NOERR || nc_inq_dimlen(nc, dy, &ny) != NC_NOERR)) bad = 1;
    if (!bad && nc_inq_varid(nc, "lon", &vx) != NC_NOERR && nc_inq_varid(nc, "x", &vx) != NC_NOERR) bad = 1;
    if (!bad && nc_inq_varid(nc, "lat", &vy) != NC_NOERR && nc_inq_varid(nc, "y", &vy) != NC_NOERR) bad = 1;
    if (!bad && nc_inq_varid(nc, "z", &vz) != NC_NOERR) bad = 1;
    if (!bad) {
        lon.resize(nx);
        lat.resize(ny);
        z.resize(nx * ny);
        if (nc_get_var_double(nc, vx, lon.data()) != NC_NOERR || nc_get_var_double(nc, vy, lat.data()) != NC_NOERR ||
            nc_get_var_float(nc, vz, z.data()) != NC_NOERR)
            bad = 1;
    }
    nc_close(nc);
    return bad;
}

// src/Problema.cxx:54-95: nearest cell of a gauge, -1 outside the grid
int gauge_cell(const std::vector<double> &lon, const std::vector<double> &lat, double plon, double plat)
{
    const int nx = (int)lon.size(), ny = (int)lat.size();
    if (plon < lon[0]) return -1;
    int i = 0, j = 0;
    bool found = false;
    while (i < nx && !found) {
        if (lon[i] >= plon) {
            found = true;
            const int im = std::max(i - 1, 0);
            if (std::fabs(plon - lon[im]) < std::fabs(plon - lon[i])) i = im;
        } else i++;
    }
    if (!found || plat < lat[0]) return -1;
    found = false;
    while (j < ny && !found) {
        if (lat[j] >= plat) {
            found = true;
            const int jm = std::max(j - 1, 0);
            if (std::fabs(plat - lat[jm]) < std::fabs(plat - lat[j])) j = jm;
        } else j++;
    }
    return found ? j * nx + i : -1;
}

bool border_ok(double b)
{
    return !(std::fabs(b - 1.0) > kEps && std::fabs(b - 2.0) > kEps && std::fabs(b + 1.0) > kEps);
}

}  // namespace

struct thy_raw_owned {
    thy_raw raw;
    std::vector<double> lon, lat, faults, points;
    std::vector<float> z, eta;
    std::string name, bathy, prefix;
};

struct thy_problem_owned {
    thy_problem p;
    std::vector<double> h, Hs, qx, qy, area_cos, dlon, dlat, lon, lat, faults, glon, glat;
    std::vector<int> cells;
};

extern "C" int thy_load_problem_file(const char *txt_path, thy_raw_owned **out)
{
    if (!txt_path || !out) return THY_ERR_INVALID;
    std::string fich(txt_path), dir;
    size_t slash = fich.find_last_of('/');
    if (slash != std::string::npos) dir = fich.substr(0, slash) + "/";
    std::ifstream in(fich);
    if (!in) {
        std::cerr << "Error: File '" << fich << "' not found" << std::endl;
        return THY_ERR_INVALID;
    }
    auto *R = new thy_raw_owned();
    thy_raw &r = R->raw;
    std::memset(&r, 0, sizeof(r));
    std::string topo, est, pts_file;
    int init = -1, levels = 0, read_points = 0;
    auto fail = [&](const std::string &msg) {
        std::cerr << "Error: " << msg << std::endl;
        delete R;
        return THY_ERR_INVALID;
    };
    r.series_time = -1.0;
    // every value up to H is required; a file that ends early is refused
    auto need = [&](bool ok, const char *what) { return ok ? 0 : (fail(std::string("the problem file ends before ") + what), 1); };
    if (need(next_value(in, R->name), "the problem name") || need(next_value(in, topo), "the bathymetry file"))
        return THY_ERR_INVALID;
    if (!file_exists(dir + topo)) return fail("File '" + dir + topo + "' not found");
    if (need(next_value(in, init), "the initialization type")) return THY_ERR_INVALID;
    if (init != 0 && init != 1) return fail("The initialization flag should be 0 or 1");
    if (init == 0) {
        if (need(next_value(in, est), "the initial state file")) return THY_ERR_INVALID;
        if (!file_exists(dir + est)) return fail("File '" + dir + est + "' not found");
    } else {
        if (need(next_value(in, r.nfaults), "the number of faults")) return THY_ERR_INVALID;
        if (r.nfaults < 1 || r.nfaults > kMaxFaults) return fail("The number of faults should be between 1 and 5000");
        R->faults.resize(10 * (size_t)r.nfaults);
        for (int i = 0; i < r.nfaults; i++) {
            std::istringstream iss(next_line(in));
            for (int k = 0; k < 10; k++)
                if (!(iss >> R->faults[10 * i + k])) return fail("a fault line has fewer than 10 values");
        }
        if (need(next_value(in, r.crop_flag), "the cropping flag")) return THY_ERR_INVALID;
        if (r.crop_flag < 0 || r.crop_flag > 2) return fail("The cropping flag should be 0, 1 or 2");
        if ((r.crop_flag == 1 || r.crop_flag == 2) && need(next_value(in, r.crop_value), "the cropping value"))
            return THY_ERR_INVALID;
    }
    if (need(next_value(in, R->prefix), "the output prefix")) return THY_ERR_INVALID;
    if (read_grd(dir + topo, R->lon, R->lat, R->z)) return fail("cannot read the bathymetry file '" + dir + topo + "'");
    r.nx = (int)R->lon.size();
    r.ny = (int)R->lat.size();
    if (r.nx < 2 || r.ny < 2) return fail("Mesh size too small. The number of rows and columns should be >= 2");
    if (need(next_value(in, levels), "the number of levels")) return THY_ERR_INVALID;
    if (levels != 1) return fail("The number of levels should be 1");
    for (int k = 0; k < 4; k++)
        if (need(next_value(in, r.borders[k]), "the four borders")) return THY_ERR_INVALID;
    for (int k = 0; k < 4; k++)
        if (!border_ok(r.borders[k])) return fail("The boundary conditions should be -1, 1 or 2");
    if (std::fabs(r.borders[0] - 2.0) < kEps || std::fabs(r.borders[1] - 2.0) < kEps)
        return fail("Periodic boundary conditions are only supported for left and right borders");
    if ((std::fabs(r.borders[2] - 2.0) < kEps) != (std::fabs(r.borders[3] - 2.0) < kEps))
        return fail("Both left and right borders should have periodic boundary conditions");
    if (need(next_value(in, r.sim_time), "the simulation time") ||
        need(next_value(in, r.save_time), "the NetCDF saving time") ||
        need(next_value(in, read_points), "the points flag"))
        return THY_ERR_INVALID;
    if (read_points == 1) {
        if (need(next_value(in, pts_file), "the points file") ||
            need(next_value(in, r.series_time), "the time-series saving time"))
            return THY_ERR_INVALID;
        if (!file_exists(dir + pts_file)) return fail("File '" + dir + pts_file + "' not found");
    }
    if (need(next_value(in, r.cfl), "CFL") || need(next_value(in, r.eps_h), "epsilon h") ||
        need(next_value(in, r.hpos), "the 2s+WAF threshold") || need(next_value(in, r.stability), "the stability coefficient") ||
        need(next_value(in, r.manning), "Manning") || need(next_value(in, r.vmax), "the maximum velocity") ||
        need(next_value(in, r.L), "L") || need(next_value(in, r.H), "H"))
        return THY_ERR_INVALID;
    r.dif_at = r.eps_h;   // default when the line is absent (src/Problema.cxx:327)
    next_value(in, r.dif_at);
    if (init == 0) {
        std::vector<double> lo, la;
        if (read_grd(dir + est, lo, la, R->eta) || (int)lo.size() != r.nx || (int)la.size() != r.ny)
            return fail("cannot read the initial state file '" + dir + est + "'");
    }
    if (read_points == 1) {
        std::ifstream pf(dir + pts_file);
        long long n = 0;
        pf >> n;
        for (long long i = 0; i < n; i++) {
            double lo = 0, la = 0;
            pf >> lo >> la;
            R->points.push_back(lo);
            R->points.push_back(la);
        }
        r.npoints = (int)(R->points.size() / 2);
    }
    r.lon = R->lon.data();
    r.lat = R->lat.data();
    r.z = R->z.data();
    r.eta_file = R->eta.empty() ? nullptr : R->eta.data();
    r.faults = R->faults.empty() ? nullptr : R->faults.data();
    r.points = R->points.empty() ? nullptr : R->points.data();
    R->bathy = topo;
    *out = R;
    return THY_OK;
}

extern "C" const thy_raw *thy_raw_view(const thy_raw_owned *r) { return r ? &r->raw : nullptr; }
extern "C" const char *thy_raw_name(const thy_raw_owned *r) { return r ? r->name.c_str() : ""; }
extern "C" const char *thy_raw_bathy_file(const thy_raw_owned *r) { return r ? r->bathy.c_str() : ""; }
extern "C" const char *thy_raw_prefix(const thy_raw_owned *r) { return r ? r->prefix.c_str() : ""; }
extern "C" void thy_raw_free(thy_raw_owned *r) { delete r; }

extern "C" int thy_prepare(const thy_raw *r, thy_problem_owned **out)
{
    if (!r || !out || r->nx < 2 || r->ny < 2 || !r->lon || !r->lat || !r->z) return THY_ERR_INVALID;
    if (r->eta_file == nullptr && (r->nfaults < 1 || r->nfaults > kMaxFaults || !r->faults)) return THY_ERR_INVALID;
    for (int k = 0; k < 4; k++)
        if (!border_ok(r->borders[k])) return THY_ERR_INVALID;
    auto *P = new thy_problem_owned();
    thy_problem &p = P->p;
    std::memset(&p, 0, sizeof(p));
    const int nx = r->nx, ny = r->ny;
    const size_t n = (size_t)nx * ny;
    // scales and dimensionless parameters (src/Problema.cxx:319-349)
    p.L = r->L;
    p.H = r->H;
    p.Q = std::sqrt(9.81 * std::pow(p.H, 3.0));
    p.T = p.L * p.H / p.Q;
    p.t_end = r->sim_time / p.T;
    p.save_nc = r->save_time / p.T;
    p.save_ts = r->series_time / p.T;
    p.mf0 = r->manning * (9.81 * r->manning * p.L / std::pow(p.H, 4.0 / 3.0));
    p.vmax = r->vmax / (p.Q / p.H);
    p.eps_h = r->eps_h / p.H;
    p.hpos = r->hpos / p.H;
    p.cvis = 1.0 - r->stability;
    p.dif_at = r->dif_at / p.H;
    p.cfl = r->cfl;
    const double R_nd = kEarthRadius / p.L;
    p.border_up = r->borders[0];
    p.border_low = r->borders[1];
    p.border_left = r->borders[2];
    p.border_right = r->borders[3];
    p.sponge_left = (std::fabs(p.border_left - 1.0) < kEps) ? kSpongeCells : 0;
    p.sponge_right = (std::fabs(p.border_right - 1.0) < kEps) ? kSpongeCells : 0;
    p.sponge_up = (std::fabs(p.border_up - 1.0) < kEps) ? kSpongeCells : 0;
    p.sponge_low = (std::fabs(p.border_low - 1.0) < kEps) ? kSpongeCells : 0;
    p.okada_flag = r->eta_file ? 0 : 1;
    p.crop_flag = p.okada_flag ? r->crop_flag : 0;
    p.crop_value = (p.crop_flag == 2) ? r->crop_value / p.H : r->crop_value;
    p.max_steps = -1;
    P->lon.assign(r->lon, r->lon + nx);
    P->lat.assign(r->lat, r->lat + ny);
    P->h.assign(n, 0.0);
    P->Hs.assign(n, 0.0);
    P->qx.assign(n, 0.0);
    P->qy.assign(n, 0.0);
    // bathymetry and Hmin (src/Problema.cxx:383-398)
    double Hmin = 1e30;
    for (size_t c = 0; c < n; c++) {
        double v = -1.0 * (double)r->z[c];
        v /= p.H;
        P->Hs[c] = v;
        if (p.okada_flag) P->h[c] = (v > 0.0) ? v : 0.0;
        if (v < Hmin) Hmin = v;
    }
    // gauges (src/Problema.cxx:400-429): duplicates dropped, nearest cell
    if (r->npoints > 0 && r->points && r->series_time >= 0.0) {
        std::vector<double> &glon = P->glon, &glat = P->glat;
        for (int i = 0; i < r->npoints; i++) {
            const double lo = r->points[2 * i], la = r->points[2 * i + 1];
            bool dup = false;
            for (size_t j = 0; j < glon.size(); j++)
                if (std::fabs(glon[j] - lo) < 1e-6 && std::fabs(glat[j] - la) < 1e-6) { dup = true; break; }
            if (dup) continue;
            glon.push_back(lo);
            glat.push_back(la);
            P->cells.push_back(gauge_cell(P->lon, P->lat, lo, la));
        }
    }
    // metric terms (src/Problema.cxx:431-448)
    P->dlon.assign(ny + 1, 0.0);
    P->dlat.assign(ny, 0.0);
    P->area_cos.assign(2 * (size_t)ny, 0.0);
    {
        const double g2r = M_PI / 180.0, dlon = std::fabs(r->lon[1] - r->lon[0]);
        double dl = 0.0;
        int i;
        for (i = 0; i < ny - 1; i++) {
            dl = std::fabs(r->lat[i + 1] - r->lat[i]);
            P->dlon[i] = dlon;
            P->dlat[i] = dl;
            P->area_cos[2 * i] = R_nd * dlon * dl * g2r;
            P->area_cos[2 * i + 1] = std::cos(r->lat[i] * g2r);
        }
        P->dlon[i] = dlon;
        P->dlat[i] = P->dlat[i - 1];
        P->dlon[i + 1] = dlon;
        P->area_cos[2 * i] = R_nd * dlon * dl * g2r;
        P->area_cos[2 * i + 1] = std::cos(r->lat[i] * g2r);
    }
    if (Hmin < 0.0) {
        for (size_t c = 0; c < n; c++) P->Hs[c] -= Hmin;
    } else {
        Hmin = 0.0;
    }
    p.Hmin = Hmin;
    // initial surface from file (src/Problema.cxx:458-473)
    if (!p.okada_flag) {
        for (size_t c = 0; c < n; c++) {
            double v = (double)r->eta_file[c] / p.H + P->Hs[c] + Hmin;
            P->h[c] = std::max(v, 0.0);
        }
    }
    // faults sorted by time (selection sort of src/Problema.cxx:97-126)
    if (p.okada_flag) {
        const int nf = r->nfaults;
        P->faults.assign(r->faults, r->faults + 10 * (size_t)nf);
        for (int i = 0; i < nf - 1; i++) {
            int m = i;
            for (int j = i + 1; j < nf; j++)
                if (P->faults[10 * j] < P->faults[10 * m]) m = j;
            if (m != i)
                for (int k = 0; k < 10; k++) std::swap(P->faults[10 * i + k], P->faults[10 * m + k]);
        }
        p.nfaults = nf;
        p.faults = P->faults.data();
    }
    p.nx = nx;
    p.ny = ny;
    p.h = P->h.data();
    p.Hs = P->Hs.data();
    p.qx = P->qx.data();
    p.qy = P->qy.data();
    p.area_cos = P->area_cos.data();
    p.dlon = P->dlon.data();
    p.dlat = P->dlat.data();
    p.lon = P->lon.data();
    p.lat = P->lat.data();
    p.npoints = (int)P->cells.size();
    p.point_cell = P->cells.empty() ? nullptr : P->cells.data();
    p.point_lon = P->glon.empty() ? nullptr : P->glon.data();
    p.point_lat = P->glat.empty() ? nullptr : P->glat.data();
    if (p.npoints == 0) p.save_ts = -1.0;
    *out = P;
    return THY_OK;
}

extern "C" const thy_problem *thy_problem_view(const thy_problem_owned *p) { return p ? &p->p : nullptr; }
extern "C" void thy_problem_free(thy_problem_owned *p) { delete p; }
