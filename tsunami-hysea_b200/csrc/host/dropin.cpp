// The drop-in boundary: thy_run_netcdf (C ABI) and shallowWater() with the
// reference's prototype (src/GPU/ShallowWater.cu:182-190), both running the
// GPU time loop of thy_run and writing the reference's NetCDF outputs.
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../../include/thysea.h"
#include "../../../include/thysea_dropin.h"
#include "netcdf_out.h"

namespace {

struct NcSinks {
    thy::GridWriter *grid = nullptr;
    thy::SeriesWriter *series = nullptr;
    int error = 0;
};

void on_snapshot(void *user, int index, double time_s, const float *eta, const float *ux, const float *uy)
{
    auto *s = static_cast<NcSinks *>(user);
    if (s->grid && s->grid->write_snapshot(index, time_s, eta, ux, uy)) s->error = THY_ERR_HOST;
}

void on_series(void *user, int index, double time_s, const float *eta, const float *ux, const float *uy)
{
    auto *s = static_cast<NcSinks *>(user);
    if (s->series && s->series->write_sample(index, time_s, eta, ux, uy)) s->error = THY_ERR_HOST;
}

int run_with_files(const thy_problem *p, const char *problem_name, const std::string &prefix, const char *version,
                   thy_stats *stats)
{
    thy::RunMeta meta;
    meta.problem_name = problem_name ? problem_name : "";
    if (version) meta.version = version;
    meta.p = p;
    const size_t n = (size_t)p->nx * p->ny;
    thy::GridWriter grid;
    thy::SeriesWriter series;
    NcSinks sinks;
    std::vector<float> bathy, defb, emax, arr, smin, smax, sbat;
    const bool want_grid = p->save_nc >= 0.0;
    const bool want_series = p->npoints > 0 && p->save_ts >= 0.0;
    try {
        if (want_grid) {
            bathy.resize(n);
            for (size_t i = 0; i < n; i++) bathy[i] = (float)((p->Hs[i] + p->Hmin) * p->H);
            if (grid.open(prefix + ".nc", meta, bathy.data())) return THY_ERR_HOST;
            sinks.grid = &grid;
            defb.resize(n);
            emax.resize(n);
            arr.resize(n);
        }
        if (want_series) {
            if (series.open(prefix + "_ts.nc", meta, p->npoints, p->point_lon, p->point_lat)) return THY_ERR_HOST;
            sinks.series = &series;
            smin.resize(p->npoints);
            smax.resize(p->npoints);
            sbat.resize(p->npoints);
        }
    } catch (...) {
        return THY_ERR_HOST;
    }
    thy_outputs o;
    std::memset(&o, 0, sizeof(o));
    o.max_height = want_grid ? emax.data() : nullptr;
    o.arrival = want_grid ? arr.data() : nullptr;
    o.deformed_bathy = (want_grid && p->okada_flag) ? defb.data() : nullptr;
    o.series_min = want_series ? smin.data() : nullptr;
    o.series_max = want_series ? smax.data() : nullptr;
    o.series_bathy = want_series ? sbat.data() : nullptr;
    o.on_snapshot = on_snapshot;
    o.on_series = on_series;
    o.user = &sinks;
    int rc = thy_run(p, &o, stats);
    if (rc) return rc;
    if (want_grid) {
        if (grid.write_final(p->okada_flag ? defb.data() : nullptr, emax.data(), arr.data())) rc = THY_ERR_HOST;
        if (grid.close()) rc = THY_ERR_HOST;
    }
    if (want_series) {
        if (series.write_final(sbat.data(), smin.data(), smax.data())) rc = THY_ERR_HOST;
        if (series.close()) rc = THY_ERR_HOST;
    }
    return rc ? rc : sinks.error;
}

}  // namespace

extern "C" int thy_run_netcdf(const thy_problem *p, const char *problem_name, const char *prefix, thy_stats *stats)
{
    if (!p || !prefix) return THY_ERR_INVALID;
    return run_with_files(p, problem_name, prefix, "1.3.0", stats);
}

extern "C" int shallowWater(int numNiveles, int okada_flag, int numFaults, int crop_flag, double crop_value,
                            double *LON_C, double *LAT_C, double *DEPTH_C, double *FAULT_L, double *FAULT_W,
                            double *STRIKE, double *DIP, double *RAKE, double *SLIP, double *defTime,
                            double2 *datosVolumenesNivel_1, double2 *datosVolumenesNivel_2,
                            tipoDatosSubmalla datosNivel, int leer_fichero_puntos, int numPuntosGuardar,
                            int *posicionesVolumenesGuardado, double *lonPuntos, double *latPuntos,
                            int numVolxNivel0, int numVolyNivel0, int64_t numVolumenesNivel, double Hmin,
                            char *nombre_bati, std::string prefijo, double borde_sup, double borde_inf,
                            double borde_izq, double borde_der, int tam_spongeSup, int tam_spongeInf,
                            int tam_spongeIzq, int tam_spongeDer, double tiempo_tot, double tiempoGuardarNetCDF,
                            double tiempoGuardarSeries, double CFL, double mf0, double vmax, double epsilon_h,
                            double hpos, double cvis, double dif_at, double L, double H, double Q, double T,
                            char *version, double *tiempo)
{
    if (numNiveles != 1) return THY_ERR_HOST;
    const size_t n = (size_t)numVolumenesNivel;
    std::vector<double> h, Hs, qx, qy, faults;
    try {
        h.resize(n);
        Hs.resize(n);
        qx.resize(n);
        qy.resize(n);
        faults.resize(10 * (size_t)(numFaults > 0 ? numFaults : 0));
    } catch (...) {
        return THY_ERR_HOST;
    }
    // the reference's interleaved double2 state (h, H) and (qx, qy)
    for (size_t i = 0; i < n; i++) {
        h[i] = datosVolumenesNivel_1[i].x;
        Hs[i] = datosVolumenesNivel_1[i].y;
        qx[i] = datosVolumenesNivel_2[i].x;
        qy[i] = datosVolumenesNivel_2[i].y;
    }
    for (int i = 0; i < numFaults; i++) {
        const double row[10] = {defTime[i], LON_C[i], LAT_C[i], DEPTH_C[i], FAULT_L[i],
                                FAULT_W[i], STRIKE[i], DIP[i], RAKE[i], SLIP[i]};
        std::memcpy(&faults[10 * (size_t)i], row, sizeof(row));
    }
    thy_problem p;
    std::memset(&p, 0, sizeof(p));
    p.nx = numVolxNivel0;
    p.ny = numVolyNivel0;
    p.h = h.data();
    p.Hs = Hs.data();
    p.qx = qx.data();
    p.qy = qy.data();
    p.area_cos = reinterpret_cast<const double *>(datosNivel.areaYCosPhi);
    p.dlon = datosNivel.anchoVolumenes;
    p.dlat = datosNivel.altoVolumenes;
    p.lon = datosNivel.longitud;
    p.lat = datosNivel.latitud;
    p.Hmin = Hmin;
    p.border_up = borde_sup;
    p.border_low = borde_inf;
    p.border_left = borde_izq;
    p.border_right = borde_der;
    p.sponge_up = tam_spongeSup;
    p.sponge_low = tam_spongeInf;
    p.sponge_left = tam_spongeIzq;
    p.sponge_right = tam_spongeDer;
    p.t_end = tiempo_tot;
    p.save_nc = tiempoGuardarNetCDF;
    p.save_ts = (leer_fichero_puntos == 1) ? tiempoGuardarSeries : -1.0;
    p.cfl = CFL;
    p.mf0 = mf0;
    p.vmax = vmax;
    p.eps_h = epsilon_h;
    p.hpos = hpos;
    p.cvis = cvis;
    p.dif_at = dif_at;
    p.L = L;
    p.H = H;
    p.Q = Q;
    p.T = T;
    p.okada_flag = okada_flag;
    p.nfaults = numFaults;
    p.faults = numFaults > 0 ? faults.data() : nullptr;
    p.crop_flag = crop_flag;
    p.crop_value = crop_value;
    p.npoints = (leer_fichero_puntos == 1) ? numPuntosGuardar : 0;
    p.point_cell = posicionesVolumenesGuardado;
    p.point_lon = lonPuntos;
    p.point_lat = latPuntos;
    p.max_steps = -1;
    thy_stats st;
    std::memset(&st, 0, sizeof(st));
    int rc = run_with_files(&p, nombre_bati, prefijo, version, &st);
    if (tiempo) *tiempo = st.loop_seconds;
    if (rc == THY_OK) {
        fprintf(stdout, "Initial deltaT = %e sec\n", st.first_dt_s);
        fprintf(stdout, "Iterations: %lld, final time = %g sec\n", st.steps, st.final_time_s);
        return 0;
    }
    if (rc == THY_ERR_GPU_MEMORY) return 1;
    fprintf(stderr, "Error: %s\n", thy_strerror(rc));
    return 2;
}
