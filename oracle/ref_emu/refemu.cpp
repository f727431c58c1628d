// ref-emu: the reference's own time stepper, compiled for the host CPU.
//
// TEST INFRASTRUCTURE ONLY (an oracle).  Nothing in the product links,
// loads or calls this file.  It is built by oracle/Makefile into
// oracle/_ref/librefemu.so from the reference sources where they lie
// (REF_SRC, the reference's src directory, set by oracle/Makefile); no
// reference source is copied into this repository.
//
// What is the reference's and what is this harness's:
//   - every __global__/__device__ function (edge fluxes, cell updates,
//     metrics, output extraction, prtoxy_, dc3d_) is the reference's own
//     code, #included from REF_SRC/GPU/*.cu and compiled as host C++;
//   - the problem loader cargarDatosProblema() (src/Problema.cxx) and the
//     NetCDF writers (src/GPU/netcdfTH.cu, src/GPU/netcdfSeries.cu) are the
//     reference's own, compiled against nclite (a NetCDF-classic subset);
//   - the launch sequencing, which nvcc-only `<<<>>>` syntax prevents g++
//     from compiling, is restated here line by line from
//     src/GPU/ShallowWater.cu:182-500 (shallowWater), src/GPU/Timestep.cu:11-120
//     (obtenerDeltaTInicialNivel0, siguientePasoNivel0, the two Δt truncations)
//     and src/GPU/Deformacion.cu:55-143 (aplicarOkada);
//   - a "launch" runs every (block, thread) of the CUDA grid as a host loop,
//     blocks spread over OpenMP threads.  Each reference launch writes
//     disjoint cells (even/odd edge colouring, src/GPU/Arista_kernel.cu:484-486),
//     so this is race-free and deterministic;
//   - obtenerMinimoReduccion (src/GPU/Reduccion_kernel.cu:141-173) is taken as
//     the exact minimum.  For grids of >= 65536 cells the reference's two-pass
//     tree reduction computes exactly that.
// Numerical differences to the reference CUDA build: host libm instead of
// CUDA's math library, and no FMA contraction (-ffp-contract=off).
// DC3D's unqualified abs() is made to resolve to the double overload with
// `using std::abs` (g++ would otherwise pick int abs).

#include <cuda_runtime.h>
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <omp.h>

using std::abs;
using std::max;
using std::min;

#undef __global__
#undef __device__
#define __global__
#define __device__

static thread_local uint3 emu_threadIdx;
static thread_local uint3 emu_blockIdx;
#define threadIdx emu_threadIdx
#define blockIdx emu_blockIdx

#include "Constantes.hxx"
#include "GPU/Arista_kernel.cu"
#include "GPU/Volumen_kernel.cu"
#include "GPU/Metrics.cu"
#include "GPU/netcdf_kernel.cu"
#include "GPU/prtoxy.cu"
#include "GPU/DC3D.cu"
#include "Problema.cxx"

#undef threadIdx
#undef blockIdx

namespace {

int g_quiet = 1;
long long g_iterations = 0;
double g_final_time = 0.0;   // seconds
double g_loop_seconds = 0.0;
double g_first_dt = 0.0;     // seconds

template <class K>
void emu_launch(dim3 grid, dim3 block, K kernel)
{
    const long long nb = (long long)grid.x * grid.y;
#pragma omp parallel for schedule(static)
    for (long long b = 0; b < nb; b++) {
        emu_blockIdx.x = (unsigned)(b % grid.x);
        emu_blockIdx.y = (unsigned)(b / grid.x);
        emu_blockIdx.z = 0;
        for (unsigned ty = 0; ty < block.y; ty++)
            for (unsigned tx = 0; tx < block.x; tx++) {
                emu_threadIdx.x = tx;
                emu_threadIdx.y = ty;
                emu_threadIdx.z = 0;
                kernel();
            }
    }
}

template <class T>
T emu_min(const T *v, long long n)
{
    T m = v[0];
#pragma omp parallel for reduction(min : m)
    for (long long i = 0; i < n; i++) m = std::min(m, v[i]);
    return m;
}

// ---- src/GPU/Timestep.cu:11-33 ----------------------------------------
double emuDeltaTInicial(double2 *d1, double2 *d2, tipoDatosSubmalla *dn, double *dT, double2 *a1, int nx, int ny,
                        double bi, double bd, double bs, double binf, bool per, double CFL, double eps,
                        dim3 gV1, dim3 gV2, dim3 gH1, dim3 gH2, dim3 tA, dim3 gE, dim3 tE)
{
    emu_launch(gV1, tA, [&] { procesarAristasVerDeltaTInicialNivel0GPU(d1, d2, dn->areaYCosPhi, nx, ny, bi, bd, per, dn->altoVolumenes, a1, eps, 1); });
    emu_launch(gV2, tA, [&] { procesarAristasVerDeltaTInicialNivel0GPU(d1, d2, dn->areaYCosPhi, nx, ny, bi, bd, per, dn->altoVolumenes, a1, eps, 2); });
    emu_launch(gH1, tA, [&] { procesarAristasHorDeltaTInicialNivel0GPU(d1, d2, nx, ny, bs, binf, dn->anchoVolumenes, a1, eps, 1); });
    emu_launch(gH2, tA, [&] { procesarAristasHorDeltaTInicialNivel0GPU(d1, d2, nx, ny, bs, binf, dn->anchoVolumenes, a1, eps, 2); });
    emu_launch(gE, tE, [&] { obtenerDeltaTVolumenesGPU(dn->areaYCosPhi, a1, dT, nx, ny, (float)CFL); });
    return emu_min<double>(dT, (long long)nx * ny);
}

// ---- src/GPU/Timestep.cu:35-68 ----------------------------------------
void emuTruncar(int nf, int f, double t, double *defTime, double T, double *dt, bool *saltar)
{
    if (f < nf) {
        if ((t + (*dt)) * T > defTime[f]) {
            *dt = defTime[f] / T - t;
            *saltar = true;
        }
    }
}

void emuTruncarSaltando(int nf, int f, double t, double *defTime, double T, double *dt, bool *saltar)
{
    *saltar = false;
    if (f < nf) {
        int i = f + 1;
        bool found = false;
        while ((i < nf) && !found) {
            if (fabs(defTime[i] - defTime[f]) > EPSILON) found = true;
            else i++;
        }
        if (found) {
            if ((t + (*dt)) * T > defTime[i]) {
                *dt = defTime[i] / T - t;
                *saltar = true;
            }
        }
    }
}

// ---- src/GPU/Timestep.cu:70-120 ---------------------------------------
double emuSiguientePaso(double2 *d1, double2 *d2, tipoDatosSubmalla *dn, double2 *a1, double2 *a2, int nx, int ny,
                        double *dT, double bs, double binf, double bi, double bd, bool per, double Hmin, int sS, int sI,
                        int sIz, int sD, double sea, double *t, double CFL, double dt, double mf0, double vmax,
                        double eps, double hpos, double cvis, long long nbytes2, dim3 gV1, dim3 gV2, dim3 gH1,
                        dim3 gH2, dim3 tA, dim3 gE, dim3 tE)
{
    emu_launch(gV1, tA, [&] { procesarAristasVerNivel0Paso1GPU(d1, d2, dn->areaYCosPhi, dn->altoVolumenes, nx, ny, bi, bd, per, dt, a1, CFL, eps, hpos, cvis, 1); });
    emu_launch(gV2, tA, [&] { procesarAristasVerNivel0Paso1GPU(d1, d2, dn->areaYCosPhi, dn->altoVolumenes, nx, ny, bi, bd, per, dt, a1, CFL, eps, hpos, cvis, 2); });
    emu_launch(gH1, tA, [&] { procesarAristasHorNivel0Paso1GPU(d1, d2, dn->areaYCosPhi, dn->anchoVolumenes, nx, ny, bs, binf, dt, a1, CFL, eps, hpos, cvis, 1); });
    emu_launch(gH2, tA, [&] { procesarAristasHorNivel0Paso1GPU(d1, d2, dn->areaYCosPhi, dn->anchoVolumenes, nx, ny, bs, binf, dt, a1, CFL, eps, hpos, cvis, 2); });
    emu_launch(gE, tE, [&] { obtenerEstadosPaso1Nivel0GPU(d1, dn->areaYCosPhi, dn->anchoVolumenes, dn->altoVolumenes, a1, nx, ny, dt, Hmin, sS, sI, sIz, sD, sea); });
    memset(a1, 0, (size_t)nbytes2);
    emu_launch(gV1, tA, [&] { procesarAristasVerNivel0Paso2GPU(d1, d2, dn->areaYCosPhi, dn->altoVolumenes, nx, ny, bi, bd, per, dt, a1, a2, CFL, eps, hpos, cvis, 1); });
    emu_launch(gV2, tA, [&] { procesarAristasVerNivel0Paso2GPU(d1, d2, dn->areaYCosPhi, dn->altoVolumenes, nx, ny, bi, bd, per, dt, a1, a2, CFL, eps, hpos, cvis, 2); });
    emu_launch(gH1, tA, [&] { procesarAristasHorNivel0Paso2GPU(d1, d2, dn->areaYCosPhi, dn->anchoVolumenes, nx, ny, bs, binf, dt, a1, a2, CFL, eps, hpos, cvis, 1); });
    emu_launch(gH2, tA, [&] { procesarAristasHorNivel0Paso2GPU(d1, d2, dn->areaYCosPhi, dn->anchoVolumenes, nx, ny, bs, binf, dt, a1, a2, CFL, eps, hpos, cvis, 2); });
    emu_launch(gE, tE, [&] { obtenerEstadoYDeltaTVolumenesNivel0GPU(d1, d2, dn->areaYCosPhi, dn->anchoVolumenes, dn->altoVolumenes, a1, a2, dT, nx, ny, CFL, dt, mf0, vmax, hpos, eps, Hmin, sS, sI, sIz, sD, sea); });
    *t += dt;
    return emu_min<double>(dT, (long long)nx * ny);
}

// ---- src/GPU/ShallowWater.cu:96-119 -----------------------------------
void emuTamBloques(int nx, int ny, dim3 *gV1, dim3 *gV2, dim3 *gH1, dim3 *gH2, dim3 *gE)
{
    int v1 = (nx / 2 + 1) * ny;
    int v2 = ((nx & 1) == 0) ? nx * ny / 2 : v1;
    int h1 = (ny / 2 + 1) * nx;
    int h2 = ((ny & 1) == 0) ? nx * ny / 2 : h1;
    gV1->x = iDivUp(v1 / ny, NUM_HEBRASX_ARI); gV1->y = iDivUp(ny, NUM_HEBRASY_ARI);
    gV2->x = iDivUp(v2 / ny, NUM_HEBRASX_ARI); gV2->y = iDivUp(ny, NUM_HEBRASY_ARI);
    gH1->x = iDivUp(nx, NUM_HEBRASX_ARI); gH1->y = iDivUp(h1 / nx, NUM_HEBRASY_ARI);
    gH2->x = iDivUp(nx, NUM_HEBRASX_ARI); gH2->y = iDivUp(h2 / nx, NUM_HEBRASY_ARI);
    gE->x = iDivUp(nx, NUM_HEBRASX_EST); gE->y = iDivUp(ny, NUM_HEBRASY_EST);
    gV1->z = gV2->z = gH1->z = gH2->z = gE->z = 1;
}

// ---- src/GPU/Deformacion.cu:55-116 (per-cell body) and :118-143 -----
void emuAplicarOkada(double2 *d1, double *eta1Ini, int crop_flag, double crop_value, double *def, float *vec, int nx,
                     int ny, double lon_ini, double incx, double lat_ini, double incy, double LON_C_ent,
                     double LAT_C_ent, double DEPTH_C_ent, double FAULT_L, double FAULT_W, double STRIKE,
                     double DIP_ent, double RAKE, double SLIP, dim3 gE, dim3 tE, double H)
{
    emu_launch(gE, tE, [&] {
        int px = emu_blockIdx.x * NUM_HEBRASX_EST + emu_threadIdx.x;
        int py = emu_blockIdx.y * NUM_HEBRASY_EST + emu_threadIdx.y;
        if ((px < nx) && (py < ny)) {
            int pos = py * nx + px;
            double LON_C = LON_C_ent, LAT_C = LAT_C_ent, DEPTH_C = DEPTH_C_ent, DIP = DIP_ent;
            double RAD = M_PI / 180.0, alfa = 2.0 / 3.0;
            int i0 = 0, IRET;
            double LON_P = lon_ini + px * incx;
            double LAT_P = lat_ini + py * incy;
            double S_RAKE = sin(RAD * RAKE), C_RAKE = cos(RAD * RAKE);
            double S_STRIKE = sin(RAD * STRIKE), C_STRIKE = cos(RAD * STRIKE);
            double DISL2 = SLIP * S_RAKE, DISL1 = SLIP * C_RAKE, DISL3 = 0.0, Z = 0.0;
            double AL1 = -0.5 * FAULT_L, AL2 = 0.5 * FAULT_L, AW1 = -0.5 * FAULT_W, AW2 = 0.5 * FAULT_W;
            double XP, YP, U_X, U_Y, U_Z, UXX, UYX, UZX, UXY, UYY, UZY, UXZ, UYZ, UZZ;
            prtoxy_(&LAT_P, &LON_P, &LAT_C, &LON_C, &XP, &YP, &i0);
            double X_OKA = XP * S_STRIKE + YP * C_STRIKE;
            double Y_OKA = -XP * C_STRIKE + YP * S_STRIKE;
            dc3d_(&alfa, &X_OKA, &Y_OKA, &Z, &DEPTH_C, &DIP, &AL1, &AL2, &AW1, &AW2, &DISL1, &DISL2, &DISL3, &U_X, &U_Y,
                  &U_Z, &UXX, &UYX, &UZX, &UXY, &UYY, &UZY, &UXZ, &UYZ, &UZZ, &IRET);
            U_Z /= H;
            def[pos] = U_Z;
        }
    });
    long long n = (long long)nx * ny;
    if (crop_flag == CROP_RELATIVE) {
        for (long long i = 0; i < n; i++) vec[i] = static_cast<float>(-fabs(def[i]));
        float def_max = -emu_min<float>(vec, n);
        double crop_final = crop_value * (static_cast<double>(def_max));
        for (long long i = 0; i < n; i++) if (fabs(def[i]) < crop_final) def[i] = 0.0;
    } else if (crop_flag == CROP_ABSOLUTE) {
        for (long long i = 0; i < n; i++) if (fabs(def[i]) < crop_value) def[i] = 0.0;
    }
    for (long long i = 0; i < n; i++) {
        d1[i].y -= def[i];
        eta1Ini[i] += def[i];
    }
}

}  // namespace

// ---- src/GPU/ShallowWater.cu:182-500 ----------------------------------
extern "C" int shallowWater(int numNiveles, int okada_flag, int numFaults, int crop_flag, double crop_value, double *LON_C,
        double *LAT_C, double *DEPTH_C, double *FAULT_L, double *FAULT_W, double *STRIKE, double *DIP, double *RAKE,
        double *SLIP, double *defTime, double2 *datosVolumenesNivel_1, double2 *datosVolumenesNivel_2, tipoDatosSubmalla datosNivel,
        int leer_fichero_puntos, int numPuntosGuardar, int *posicionesVolumenesGuardado, double *lonPuntos, double *latPuntos,
        int numVolxNivel0, int numVolyNivel0, int64_t numVolumenesNivel, double Hmin, char *nombre_bati, std::string prefijo,
        double borde_sup, double borde_inf, double borde_izq, double borde_der, int tam_spongeSup, int tam_spongeInf,
        int tam_spongeIzq, int tam_spongeDer, double tiempo_tot, double tiempoGuardarNetCDF, double tiempoGuardarSeries,
        double CFL, double mf0, double vmax, double epsilon_h, double hpos, double cvis, double dif_at, double L, double H,
        double Q, double T, char *version, double *tiempo)
{
    (void)numNiveles; (void)lonPuntos; (void)latPuntos; (void)L;
    const int nx = numVolxNivel0, ny = numVolyNivel0;
    const long long N = (long long)numVolumenesNivel;
    int num = 0, fallaOkada = 0, num_ts = 0;
    bool saltar = false;
    double sea_level = SEA_LEVEL / H;
    dim3 gV1, gV2, gH1, gH2, gE;
    dim3 tA(NUM_HEBRASX_ARI, NUM_HEBRASY_ARI), tE(NUM_HEBRASX_EST, NUM_HEBRASY_EST);
    double lon_ini = datosNivel.longitud[0], lat_ini = datosNivel.latitud[0];
    double incx = (datosNivel.longitud[nx - 1] - datosNivel.longitud[0]) / (nx - 1);
    double incy = (datosNivel.latitud[ny - 1] - datosNivel.latitud[0]) / (ny - 1);
    bool per = (((fabs(borde_izq - 2.0) < EPSILON) && (fabs(borde_der - 2.0) < EPSILON)) ? true : false);
    emuTamBloques(nx, ny, &gV1, &gV2, &gH1, &gH2, &gE);

    // device buffers become host buffers
    tipoDatosSubmalla dn;
    dn.areaYCosPhi = datosNivel.areaYCosPhi;
    dn.anchoVolumenes = datosNivel.anchoVolumenes;
    dn.altoVolumenes = datosNivel.altoVolumenes;
    double2 *d1 = (double2 *)malloc(N * sizeof(double2));
    double2 *d2 = (double2 *)malloc(N * sizeof(double2));
    double *etaMax = (double *)malloc(N * sizeof(double));
    double *tLleg = (double *)malloc(N * sizeof(double));
    double *etaIni = (double *)malloc(N * sizeof(double));
    float *d_vec = (float *)malloc(N * sizeof(float));
    double *dT = (double *)malloc(N * sizeof(double));
    double2 *a1 = (double2 *)malloc(N * sizeof(double2));
    double2 *a2 = (double2 *)malloc(N * sizeof(double2));
    double2 *g1 = nullptr, *g2 = nullptr;
    if (!d1 || !d2 || !etaMax || !tLleg || !etaIni || !d_vec || !dT || !a1 || !a2) return 1;
    memcpy(d1, datosVolumenesNivel_1, N * sizeof(double2));
    memcpy(d2, datosVolumenesNivel_2, N * sizeof(double2));
    if (leer_fichero_puntos == 1) {
        g1 = (double2 *)malloc((size_t)numPuntosGuardar * sizeof(double2) + 16);
        g2 = (double2 *)malloc((size_t)numPuntosGuardar * sizeof(double2) + 16);
    }
    emu_launch(gE, tE, [&] { inicializarEta1MaximaNivel0GPU(d1, etaMax, nx, ny, epsilon_h); });
    emu_launch(gE, tE, [&] { inicializarEta1MaximaNivel0GPU(d1, etaIni, nx, ny, epsilon_h); });
    emu_launch(gE, tE, [&] { inicializarTiemposLlegadaNivel0GPU(tLleg, nx, ny); });

    float *vec = nullptr;
    float *etaP = nullptr, *uP = nullptr, *vP = nullptr, *etaMinP = nullptr, *etaMaxP = nullptr;
    double mf0_ini = sqrt(mf0 * pow(H, 4.0 / 3.0) / (9.81 * L));
    if (tiempoGuardarNetCDF >= 0.0) {
        vec = (float *)malloc(N * sizeof(float));
        for (long long i = 0; i < N; i++) vec[i] = static_cast<float>((datosVolumenesNivel_1[i].y + Hmin) * H);
        netcdfTH::crearFicherosNC(nombre_bati, okada_flag, const_cast<char *>((prefijo + ".nc").c_str()), nx, ny,
            datosNivel.longitud, datosNivel.latitud, tiempo_tot * T, CFL, epsilon_h * H, mf0_ini, vmax * Q / H, hpos * H,
            1.0 - cvis, dif_at * H, borde_sup, borde_inf, borde_izq, borde_der, per, numFaults, defTime, LON_C, LAT_C,
            DEPTH_C, FAULT_L, FAULT_W, STRIKE, DIP, RAKE, SLIP, crop_flag, crop_value, H, vec, version);
    }
    if (leer_fichero_puntos == 1) {
        etaP = (float *)malloc(numPuntosGuardar * sizeof(float) + 16);
        uP = (float *)malloc(numPuntosGuardar * sizeof(float) + 16);
        vP = (float *)malloc(numPuntosGuardar * sizeof(float) + 16);
        etaMinP = (float *)malloc(numPuntosGuardar * sizeof(float) + 16);
        etaMaxP = (float *)malloc(numPuntosGuardar * sizeof(float) + 16);
        netcdfSeries::initTimeSeriesNC(nombre_bati, const_cast<char *>((prefijo + "_ts.nc").c_str()), numPuntosGuardar,
            lonPuntos, latPuntos, tiempo_tot * T, CFL, epsilon_h * H, mf0_ini, vmax * Q / H, hpos * H, 1.0 - cvis,
            dif_at * H, borde_sup, borde_inf, borde_izq, borde_der, per, numFaults, defTime, LON_C, LAT_C, DEPTH_C,
            FAULT_L, FAULT_W, STRIKE, DIP, RAKE, SLIP, okada_flag, crop_flag, crop_value, H, version);
        for (int i = 0; i < numPuntosGuardar; i++) {
            if (posicionesVolumenesGuardado[i] == -1) {
                etaP[i] = uP[i] = vP[i] = etaMinP[i] = etaMaxP[i] = -9999.0f;
            } else {
                etaMinP[i] = 1e30f;
                etaMaxP[i] = -1e30f;
            }
        }
    }
    long long nb2 = N * (long long)sizeof(double2);
    memset(a1, 0, nb2);
    memset(a2, 0, nb2);

    auto t0 = std::chrono::high_resolution_clock::now();
    double t = 0.0;
    double dt = emuDeltaTInicial(d1, d2, &dn, dT, a1, nx, ny, borde_izq, borde_der, borde_sup, borde_inf, per, CFL,
                                 epsilon_h, gV1, gV2, gH1, gH2, tA, gE, tE);
    if (numFaults > 0) {
        if (defTime[0] < EPSILON) emuTruncarSaltando(numFaults, fallaOkada, t, defTime, T, &dt, &saltar);
        else emuTruncar(numFaults, fallaOkada, t, defTime, T, &dt, &saltar);
    }
    g_first_dt = dt * T;
    if (!g_quiet) fprintf(stdout, "Initial deltaT = %e sec\n", dt * T);
    memset(a1, 0, nb2);

    double nextNC = 0.0, nextTS = 0.0;
    long long iter = 1;
    const long long max_iter = g_iterations;  // < 0: unlimited
    g_iterations = 0;
    while (t < tiempo_tot && (max_iter < 0 || iter <= max_iter)) {
        // comprobarYAplicarDeformaciones (src/GPU/ShallowWater.cu:125-147)
        while (fallaOkada < numFaults && t * T >= defTime[fallaOkada]) {
            if (!g_quiet) fprintf(stdout, "Applying Okada with fault %d\n", fallaOkada + 1);
            emuAplicarOkada(d1, etaIni, crop_flag, crop_value, dT, d_vec, nx, ny, lon_ini, incx, lat_ini, incy,
                            LON_C[fallaOkada], LAT_C[fallaOkada], DEPTH_C[fallaOkada], FAULT_L[fallaOkada],
                            FAULT_W[fallaOkada], STRIKE[fallaOkada], DIP[fallaOkada], RAKE[fallaOkada],
                            SLIP[fallaOkada], gE, tE, H);
            fallaOkada++;
        }
        if ((tiempoGuardarNetCDF >= 0.0) && (t >= nextNC)) {
            nextNC += tiempoGuardarNetCDF;
            netcdfTH::escribirTiempoNC(num, t * T);
            emu_launch(gE, tE, [&] { obtenerEtaNetCDF(d1, d_vec, nx, ny, epsilon_h, Hmin, H); });
            netcdfTH::escribirEtaNC(nx, ny, num, d_vec);
            emu_launch(gE, tE, [&] { obtenerUxNetCDF(d1, d2, d_vec, nx, ny, epsilon_h, Hmin, H, Q); });
            netcdfTH::escribirUxNC(nx, ny, num, d_vec);
            emu_launch(gE, tE, [&] { obtenerUyNetCDF(d1, d2, d_vec, nx, ny, epsilon_h, Hmin, H, Q); });
            netcdfTH::escribirUyNC(nx, ny, num, d_vec);
            num++;
        }
        if ((tiempoGuardarSeries >= 0.0) && (t >= nextTS)) {
            nextTS += tiempoGuardarSeries;
            dim3 gP(iDivUp(numPuntosGuardar, NUM_HEBRAS_PUNTOS), 1), tP(NUM_HEBRAS_PUNTOS, 1);
            emu_launch(gP, tP, [&] { escribirVolumenesGuardadoGPU(d1, d2, g1, g2, posicionesVolumenesGuardado, numPuntosGuardar, epsilon_h); });
            memcpy(datosVolumenesNivel_1, g1, numPuntosGuardar * sizeof(double2));
            memcpy(datosVolumenesNivel_2, g2, numPuntosGuardar * sizeof(double2));
            // guardarSerieTiemposNivel0 (src/GPU/ShallowWater.cu:69-90)
            for (int i = 0; i < numPuntosGuardar; i++) {
                if (posicionesVolumenesGuardado[i] != -1) {
                    double h = datosVolumenesNivel_1[i].x;
                    etaP[i] = static_cast<float>((h - datosVolumenesNivel_1[i].y - Hmin) * H);
                    uP[i] = static_cast<float>(datosVolumenesNivel_2[i].x * Q / H);
                    vP[i] = static_cast<float>(datosVolumenesNivel_2[i].y * Q / H);
                    etaMinP[i] = min(etaP[i], etaMinP[i]);
                    etaMaxP[i] = max(etaP[i], etaMaxP[i]);
                }
            }
            netcdfSeries::writeStateTimeSeriesNC(num_ts, t * T, numPuntosGuardar, etaP, uP, vP);
            num_ts++;
        }
        emu_launch(gE, tE, [&] { actualizarEta1MaximaNivel0GPU(d1, etaMax, nx, ny, t, epsilon_h); });
        emu_launch(gE, tE, [&] { actualizarTiemposLlegadaNivel0GPU(d1, tLleg, etaIni, nx, ny, t, dif_at); });
        dt = emuSiguientePaso(d1, d2, &dn, a1, a2, nx, ny, dT, borde_sup, borde_inf, borde_izq, borde_der, per, Hmin,
                              tam_spongeSup, tam_spongeInf, tam_spongeIzq, tam_spongeDer, sea_level, &t, CFL, dt, mf0,
                              vmax, epsilon_h, hpos, cvis, nb2, gV1, gV2, gH1, gH2, tA, gE, tE);
        if (!saltar) emuTruncar(numFaults, fallaOkada, t, defTime, T, &dt, &saltar);
        else emuTruncarSaltando(numFaults, fallaOkada, t, defTime, T, &dt, &saltar);
        memset(a1, 0, nb2);
        memset(a2, 0, nb2);
        if (!g_quiet) {
            fprintf(stdout, "Iteration %3lld, deltaT = %e sec, ", iter, dt * T);
            fprintf(stdout, "Time = %g sec\n", t * T);
        }
        iter++;
    }
    auto t1 = std::chrono::high_resolution_clock::now();
    *tiempo = std::chrono::duration_cast<std::chrono::microseconds>(t1 - t0).count() * 1e-6;
    g_loop_seconds = *tiempo;
    g_iterations = iter - 1;
    g_final_time = t * T;

    if (tiempoGuardarNetCDF >= 0.0) {
        if (okada_flag == OKADA_STANDARD) {
            emu_launch(gE, tE, [&] { obtenerBatimetriaModificadaNetCDF(d1, d_vec, nx, ny, Hmin, H); });
            netcdfTH::guardarBatimetriaModificadaNC(d_vec);
        }
        emu_launch(gE, tE, [&] { obtenerEta1MaximaNetCDF(etaMax, d_vec, nx, ny, Hmin, H); });
        netcdfTH::guardarEta1MaximaNC(d_vec);
        emu_launch(gE, tE, [&] { obtenerTiemposLlegadaNetCDF(tLleg, d_vec, nx, ny, T); });
        netcdfTH::guardarTiemposLlegadaNC(d_vec);
        netcdfTH::cerrarFicheroNC();
        free(vec);
    }
    if (leer_fichero_puntos == 1) {
        dim3 gP(iDivUp(numPuntosGuardar, NUM_HEBRAS_PUNTOS), 1), tP(NUM_HEBRAS_PUNTOS, 1);
        emu_launch(gP, tP, [&] { escribirVolumenesGuardadoGPU(d1, d2, g1, g2, posicionesVolumenesGuardado, numPuntosGuardar, epsilon_h); });
        memcpy(datosVolumenesNivel_1, g1, numPuntosGuardar * sizeof(double2));
        // obtenerBatimetriaParaSerieTiempos (src/GPU/ShallowWater.cu:58-67)
        for (int i = 0; i < numPuntosGuardar; i++)
            if (posicionesVolumenesGuardado[i] != -1)
                etaP[i] = static_cast<float>((datosVolumenesNivel_1[i].y + Hmin) * H);
        netcdfSeries::guardarBatimetriaModificadaTimeSeriesNC(etaP);
        netcdfSeries::guardarAmplitudesTimeSeriesNC(etaMinP, etaMaxP);
        netcdfSeries::closeTimeSeriesNC();
        free(etaP); free(uP); free(vP); free(etaMinP); free(etaMaxP);
        free(g1); free(g2);
    }
    free(d1); free(d2); free(etaMax); free(tLleg); free(etaIni); free(d_vec); free(dT); free(a1); free(a2);
    return 0;
}

// ---- C-ABI used by the tests and by bench.py's reference arm ----------
//
// refemu_run(txt, max_iterations, threads, info):
//   loads the problem file with the reference's own loader (src/Problema.cxx)
//   and runs the time loop, writing the reference's NetCDF outputs.
//   max_iterations < 0 runs to the simulation time.  threads <= 0 keeps the
//   OpenMP default.  info receives {iterations, final time (s), loop seconds,
//   first dt (s)}.  Returns 0 on success, the reference's error codes else.
extern "C" int refemu_run(const char *txt, long long max_iterations, int threads, int quiet, double *info)
{
    if (threads > 0) omp_set_num_threads(threads);
    g_quiet = quiet;
    std::string version = "1.3.0";
    double2 *d1 = nullptr, *d2 = nullptr;
    tipoDatosSubmalla dn;
    memset(&dn, 0, sizeof(dn));
    int *pos = nullptr;
    double *lonP = nullptr, *latP = nullptr;
    int leer, nP, nx, ny, nNiv, okada, nF, crop;
    int64_t N;
    double bs, bi, bl, br, tt, tnc, tts, Hmin, eps, difat, mf0, vmax, CFL, hpos, cvis, L, H, Q, T, crop_v, tgpu;
    int sS, sI, sL, sR;
    std::string nombre, prefijo;
    static double LON_C[MAX_FAULTS], LAT_C[MAX_FAULTS], DEPTH_C[MAX_FAULTS], FL[MAX_FAULTS], FW[MAX_FAULTS];
    static double STR[MAX_FAULTS], DIP[MAX_FAULTS], RAKE[MAX_FAULTS], SLIP[MAX_FAULTS], defT[MAX_FAULTS];
    int err = cargarDatosProblema(txt, nombre, prefijo, &nNiv, &okada, &nF, &crop, &crop_v, LON_C, LAT_C, DEPTH_C, FL,
                                  FW, STR, DIP, RAKE, SLIP, defT, &d1, &d2, &dn, &nx, &ny, &N, &leer, &nP, &pos, &lonP,
                                  &latP, &Hmin, &bs, &bi, &bl, &br, &sS, &sI, &sL, &sR, &tt, &tnc, &tts, &CFL, &mf0,
                                  &vmax, &eps, &hpos, &cvis, &difat, &L, &H, &Q, &T);
    if (err > 0) return 100 + err;
    g_iterations = max_iterations;
    err = shallowWater(nNiv, okada, nF, crop, crop_v, LON_C, LAT_C, DEPTH_C, FL, FW, STR, DIP, RAKE, SLIP, defT, d1, d2,
                       dn, leer, nP, pos, lonP, latP, nx, ny, N, Hmin, const_cast<char *>(nombre.c_str()), prefijo, bs, bi,
                       bl, br, sS, sI, sL, sR, tt, tnc, tts, CFL, mf0, vmax, eps, hpos, cvis, difat, L, H, Q, T,
                       const_cast<char *>(version.c_str()), &tgpu);
    liberarMemoria(d1, d2, dn, pos, lonP, latP);
    if (info) {
        info[0] = (double)g_iterations;
        info[1] = g_final_time;
        info[2] = g_loop_seconds;
        info[3] = g_first_dt;
    }
    return err;
}

// ---- step-level session (bench.py's reference arm / CPU baseline) -----
// Loads a problem file with the reference's loader, allocates the state,
// computes the initial dt and applies the faults due at t = 0 (the first
// actions of the reference's loop); refemu_steps then times whole loop
// iterations (metrics update + siguientePasoNivel0 + dt truncation), without
// NetCDF output.
struct RefemuSession {
    int nx = 0, ny = 0, nF = 0, crop = 0, fault = 0;
    bool per = false, saltar = false;
    double bs, bi, bl, br, Hmin, eps, difat, mf0, vmax, CFL, hpos, cvis, L, H, Q, T, crop_v, tt, t = 0, dt = 0;
    int sS, sI, sL, sR;
    double LON_C[MAX_FAULTS], LAT_C[MAX_FAULTS], DEPTH_C[MAX_FAULTS], FL[MAX_FAULTS], FW[MAX_FAULTS];
    double STR[MAX_FAULTS], DIPA[MAX_FAULTS], RAKE[MAX_FAULTS], SLIP[MAX_FAULTS], defT[MAX_FAULTS];
    double2 *h1 = nullptr, *h2 = nullptr, *a1 = nullptr, *a2 = nullptr;
    double *etaMax = nullptr, *tLleg = nullptr, *etaIni = nullptr, *dT = nullptr;
    float *vec = nullptr;
    tipoDatosSubmalla dn;
    dim3 gV1, gV2, gH1, gH2, gE, tA, tE;
    long long steps = 0;
};

extern "C" void *refemu_open(const char *txt, int threads)
{
    if (threads > 0) omp_set_num_threads(threads);
    auto *S = new RefemuSession();
    std::memset(&S->dn, 0, sizeof(S->dn));
    int *pos = nullptr, leer, nP, nNiv, okada;
    double *lonP = nullptr, *latP = nullptr, tnc, tts;
    int64_t N;
    std::string nombre, prefijo;
    int err = cargarDatosProblema(txt, nombre, prefijo, &nNiv, &okada, &S->nF, &S->crop, &S->crop_v, S->LON_C, S->LAT_C,
                                  S->DEPTH_C, S->FL, S->FW, S->STR, S->DIPA, S->RAKE, S->SLIP, S->defT, &S->h1, &S->h2,
                                  &S->dn, &S->nx, &S->ny, &N, &leer, &nP, &pos, &lonP, &latP, &S->Hmin, &S->bs, &S->bi,
                                  &S->bl, &S->br, &S->sS, &S->sI, &S->sL, &S->sR, &S->tt, &tnc, &tts, &S->CFL, &S->mf0,
                                  &S->vmax, &S->eps, &S->hpos, &S->cvis, &S->difat, &S->L, &S->H, &S->Q, &S->T);
    if (err > 0) {
        delete S;
        return nullptr;
    }
    free(pos); free(lonP); free(latP);
    const long long n = (long long)S->nx * S->ny;
    S->per = (fabs(S->bl - 2.0) < EPSILON) && (fabs(S->br - 2.0) < EPSILON);
    emuTamBloques(S->nx, S->ny, &S->gV1, &S->gV2, &S->gH1, &S->gH2, &S->gE);
    S->tA = dim3(NUM_HEBRASX_ARI, NUM_HEBRASY_ARI);
    S->tE = dim3(NUM_HEBRASX_EST, NUM_HEBRASY_EST);
    S->a1 = (double2 *)calloc(n, sizeof(double2));
    S->a2 = (double2 *)calloc(n, sizeof(double2));
    S->etaMax = (double *)malloc(n * sizeof(double));
    S->tLleg = (double *)malloc(n * sizeof(double));
    S->etaIni = (double *)malloc(n * sizeof(double));
    S->dT = (double *)malloc(n * sizeof(double));
    S->vec = (float *)malloc(n * sizeof(float));
    int nx = S->nx, ny = S->ny;
    emu_launch(S->gE, S->tE, [&] { inicializarEta1MaximaNivel0GPU(S->h1, S->etaMax, nx, ny, S->eps); });
    emu_launch(S->gE, S->tE, [&] { inicializarEta1MaximaNivel0GPU(S->h1, S->etaIni, nx, ny, S->eps); });
    emu_launch(S->gE, S->tE, [&] { inicializarTiemposLlegadaNivel0GPU(S->tLleg, nx, ny); });
    S->dt = emuDeltaTInicial(S->h1, S->h2, &S->dn, S->dT, S->a1, nx, ny, S->bl, S->br, S->bs, S->bi, S->per, S->CFL,
                             S->eps, S->gV1, S->gV2, S->gH1, S->gH2, S->tA, S->gE, S->tE);
    if (S->nF > 0) {
        if (S->defT[0] < EPSILON) emuTruncarSaltando(S->nF, S->fault, S->t, S->defT, S->T, &S->dt, &S->saltar);
        else emuTruncar(S->nF, S->fault, S->t, S->defT, S->T, &S->dt, &S->saltar);
    }
    memset(S->a1, 0, n * sizeof(double2));
    double lon_ini = S->dn.longitud[0], lat_ini = S->dn.latitud[0];
    double incx = (S->dn.longitud[nx - 1] - lon_ini) / (nx - 1), incy = (S->dn.latitud[ny - 1] - lat_ini) / (ny - 1);
    while (S->fault < S->nF && S->t * S->T >= S->defT[S->fault]) {
        int f = S->fault;
        emuAplicarOkada(S->h1, S->etaIni, S->crop, S->crop_v, S->dT, S->vec, nx, ny, lon_ini, incx, lat_ini, incy,
                        S->LON_C[f], S->LAT_C[f], S->DEPTH_C[f], S->FL[f], S->FW[f], S->STR[f], S->DIPA[f], S->RAKE[f],
                        S->SLIP[f], S->gE, S->tE, S->H);
        S->fault++;
    }
    return S;
}

// Runs k loop iterations; returns their wall seconds (negative on error).
extern "C" double refemu_steps(void *handle, long long k)
{
    auto *S = (RefemuSession *)handle;
    if (!S) return -1.0;
    const int nx = S->nx, ny = S->ny;
    const long long nb2 = (long long)nx * ny * (long long)sizeof(double2);
    auto t0 = std::chrono::high_resolution_clock::now();
    for (long long i = 0; i < k; i++) {
        double t = S->t;
        emu_launch(S->gE, S->tE, [&] { actualizarEta1MaximaNivel0GPU(S->h1, S->etaMax, nx, ny, t, S->eps); });
        emu_launch(S->gE, S->tE, [&] { actualizarTiemposLlegadaNivel0GPU(S->h1, S->tLleg, S->etaIni, nx, ny, t, S->difat); });
        S->dt = emuSiguientePaso(S->h1, S->h2, &S->dn, S->a1, S->a2, nx, ny, S->dT, S->bs, S->bi, S->bl, S->br, S->per,
                                 S->Hmin, S->sS, S->sI, S->sL, S->sR, SEA_LEVEL / S->H, &S->t, S->CFL, S->dt, S->mf0,
                                 S->vmax, S->eps, S->hpos, S->cvis, nb2, S->gV1, S->gV2, S->gH1, S->gH2, S->tA, S->gE,
                                 S->tE);
        if (!S->saltar) emuTruncar(S->nF, S->fault, S->t, S->defT, S->T, &S->dt, &S->saltar);
        else emuTruncarSaltando(S->nF, S->fault, S->t, S->defT, S->T, &S->dt, &S->saltar);
        memset(S->a1, 0, nb2);
        memset(S->a2, 0, nb2);
        S->steps++;
    }
    auto t1 = std::chrono::high_resolution_clock::now();
    return std::chrono::duration<double>(t1 - t0).count();
}

extern "C" long long refemu_cells(void *handle)
{
    auto *S = (RefemuSession *)handle;
    return S ? (long long)S->nx * S->ny : 0;
}

extern "C" void refemu_close(void *handle)
{
    auto *S = (RefemuSession *)handle;
    if (!S) return;
    liberarMemoria(S->h1, S->h2, S->dn, nullptr, nullptr, nullptr);
    free(S->a1); free(S->a2); free(S->etaMax); free(S->tLleg); free(S->etaIni); free(S->dT); free(S->vec);
    delete S;
}

// Okada vertical displacement (meters) at arbitrary points, via the
// reference's prtoxy_ + dc3d_ exactly as aplicarOkadaStandardGPU calls them.
extern "C" void refemu_okada_points(int n, const double *lon, const double *lat, const double *fault, double *uz)
{
    for (int i = 0; i < n; i++) {
        double LON_P = lon[i], LAT_P = lat[i];
        double LON_C = fault[1], LAT_C = fault[2], DEPTH_C = fault[3], FL = fault[4], FW = fault[5];
        double STRIKE = fault[6], DIP = fault[7], RAKE = fault[8], SLIP = fault[9];
        double RAD = M_PI / 180.0, alfa = 2.0 / 3.0;
        int i0 = 0, IRET;
        double DISL2 = SLIP * sin(RAD * RAKE), DISL1 = SLIP * cos(RAD * RAKE), DISL3 = 0.0, Z = 0.0;
        double AL1 = -0.5 * FL, AL2 = 0.5 * FL, AW1 = -0.5 * FW, AW2 = 0.5 * FW;
        double XP, YP, U_X, U_Y, U_Z, UXX, UYX, UZX, UXY, UYY, UZY, UXZ, UYZ, UZZ;
        prtoxy_(&LAT_P, &LON_P, &LAT_C, &LON_C, &XP, &YP, &i0);
        double X_OKA = XP * sin(RAD * STRIKE) + YP * cos(RAD * STRIKE);
        double Y_OKA = -XP * cos(RAD * STRIKE) + YP * sin(RAD * STRIKE);
        dc3d_(&alfa, &X_OKA, &Y_OKA, &Z, &DEPTH_C, &DIP, &AL1, &AL2, &AW1, &AW2, &DISL1, &DISL2, &DISL3, &U_X, &U_Y,
              &U_Z, &UXX, &UYX, &UZX, &UXY, &UYY, &UZY, &UXZ, &UYZ, &UZZ, &IRET);
        uz[i] = U_Z;
    }
}
