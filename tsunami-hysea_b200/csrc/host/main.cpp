// TsunamiHySEA command-line program over libthysea.so: the same usage and
// problem file as the reference's main() (src/ShallowWater.cxx:29-166),
// calling the exported shallowWater() drop-in with the arguments the
// reference's loader would produce.
#include <cstdio>
#include <cstring>
#include <iostream>
#include <string>
#include <sys/stat.h>
#include <vector>

#include "thysea.h"
#include "thysea_dropin.h"

static void usage(const char *argv0)
{
    std::cerr << "Tsunami-HySEA time stepper for NVIDIA B200 (" << thy_version() << ")\n\n"
              << "Use:\n" << argv0 << " dataFile\n\n"
              << "dataFile format:\n"
              << "  Problem name\n  Bathymetry file\n"
              << "  Initialization of states (0: Sea surface displacement from file,\n"
              << "                            1: Standard Okada)\n"
              << "  If 0:\n    Initial state file\n  Else if 1:\n    Number of faults (>= 1)\n"
              << "    For every fault, a line containing:\n"
              << "      Time(sec) Lon_epicenter Lat_epicenter Depth_hypocenter(km) Fault_length(km) Fault_width(km) "
                 "Strike Dip Rake Slip(m)\n"
              << "    Crop deformations (0: No, 1: Relative cropping, 2: Absolute cropping)\n"
              << "    If 1:\n      Percentage [0,1]\n    Else if 2:\n      Threshold value (m)\n"
              << "  NetCDF file prefix\n  Number of levels (should be 1)\n"
              << "  Upper border condition (1: open, -1: wall)\n  Lower border condition (1: open, -1: wall)\n"
              << "  Left border condition (1: open, -1: wall, 2: periodic)\n"
              << "  Right border condition (1: open, -1: wall, 2: periodic)\n"
              << "  Simulation time (sec)\n  Saving time of NetCDF files (sec) (-1: do not save)\n"
              << "  Read points from file (0: no, 1: yes)\n  If 1:\n    File with points\n"
              << "    Saving time of time series (sec)\n"
              << "  CFL\n  Epsilon h (m)\n  Threshold for the 2s+WAF scheme (m)\n  Stability coefficient\n"
              << "  Water-bottom friction (Manning coefficient)\n  Maximum allowed velocity of water\n"
              << "  L (typical length)\n  H (typical depth)\n"
              << "  Threshold for arrival times (m) (epsilon h if not specified)\n";
}

int main(int argc, char *argv[])
{
    if (argc < 2) {
        usage(argv[0]);
        return EXIT_FAILURE;
    }
    struct stat sb;
    if (stat(argv[1], &sb) != 0) {
        std::cerr << "Error: File '" << argv[1] << "' not found" << std::endl;
        return EXIT_FAILURE;
    }
    if (thy_device_count() == 0) {
        std::cerr << "Error: There is no graphics card supporting CUDA" << std::endl;
        return EXIT_FAILURE;
    }
    thy_raw_owned *raw = nullptr;
    if (thy_load_problem_file(argv[1], &raw) != THY_OK) return EXIT_FAILURE;
    thy_problem_owned *po = nullptr;
    if (thy_prepare(thy_raw_view(raw), &po) != THY_OK) {
        std::cerr << "Error: invalid problem" << std::endl;
        thy_raw_free(raw);
        return EXIT_FAILURE;
    }
    const thy_problem &p = *thy_problem_view(po);
    const thy_raw &r = *thy_raw_view(raw);
    std::cout << "Problem data\n"
              << "Initialization: " << (p.okada_flag ? "Standard Okada" : "Sea surface displacement from file") << "\n";
    if (p.okada_flag) std::cout << "Number of faults: " << p.nfaults << "\n";
    std::cout << "CFL: " << p.cfl << "\nSimulation time: " << p.t_end * p.T << " sec\n"
              << "Saving time of NetCDF files: " << p.save_nc * p.T << " sec\n"
              << "  Volumes: " << p.nx << " x " << p.ny << " = " << (long long)p.nx * p.ny << "\n"
              << "  Longitude: [" << p.lon[0] << ", " << p.lon[p.nx - 1] << "]\n"
              << "  Latitude: [" << p.lat[0] << ", " << p.lat[p.ny - 1] << "]\n"
              << std::endl;
    // the arguments of shallowWater() in the reference's layout
    const size_t n = (size_t)p.nx * p.ny;
    std::vector<double2> d1(n), d2(n), ac(p.ny);
    for (size_t i = 0; i < n; i++) {
        d1[i].x = p.h[i];
        d1[i].y = p.Hs[i];
        d2[i].x = p.qx ? p.qx[i] : 0.0;
        d2[i].y = p.qy ? p.qy[i] : 0.0;
    }
    for (int y = 0; y < p.ny; y++) {
        ac[y].x = p.area_cos[2 * y];
        ac[y].y = p.area_cos[2 * y + 1];
    }
    tipoDatosSubmalla dn;
    dn.areaYCosPhi = ac.data();
    dn.anchoVolumenes = const_cast<double *>(p.dlon);
    dn.altoVolumenes = const_cast<double *>(p.dlat);
    dn.longitud = const_cast<double *>(p.lon);
    dn.latitud = const_cast<double *>(p.lat);
    const int nf = p.nfaults;
    std::vector<double> f[10];
    for (int k = 0; k < 10; k++) {
        f[k].resize(nf > 0 ? nf : 1);
        for (int i = 0; i < nf; i++) f[k][i] = p.faults[10 * i + k];
    }
    std::string name = thy_raw_name(raw), prefix = thy_raw_prefix(raw), version = "1.3.0";
    double runtime = 0;
    int err = shallowWater(1, p.okada_flag, nf, p.crop_flag, p.crop_value, f[1].data(), f[2].data(), f[3].data(),
                           f[4].data(), f[5].data(), f[6].data(), f[7].data(), f[8].data(), f[9].data(), f[0].data(),
                           d1.data(), d2.data(), dn, p.npoints > 0 ? 1 : 0, p.npoints, const_cast<int *>(p.point_cell),
                           const_cast<double *>(p.point_lon), const_cast<double *>(p.point_lat), p.nx, p.ny,
                           (int64_t)n, p.Hmin, const_cast<char *>(name.c_str()), prefix, p.border_up, p.border_low,
                           p.border_left, p.border_right, p.sponge_up, p.sponge_low, p.sponge_left, p.sponge_right,
                           p.t_end, p.save_nc, r.series_time / p.T, p.cfl, p.mf0, p.vmax, p.eps_h, p.hpos, p.cvis,
                           p.dif_at, p.L, p.H, p.Q, p.T, const_cast<char *>(version.c_str()), &runtime);
    thy_problem_free(po);
    thy_raw_free(raw);
    if (err > 0) {
        if (err == 1) std::cerr << "Error: Not enough GPU memory" << std::endl;
        else std::cerr << "Error: Not enough CPU memory" << std::endl;
        return EXIT_FAILURE;
    }
    std::cout << std::endl << "Runtime: " << runtime << " sec" << std::endl;
    return EXIT_SUCCESS;
}
