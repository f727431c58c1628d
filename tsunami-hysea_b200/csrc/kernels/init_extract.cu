// State initialisation and output extraction kernels.
//
// init:    the reference's dimensionless double state (h, H shifted by Hmin,
//          qx, qy; src/Problema.cxx:383-473) -> FP32 (eta, dep, qx, qy), and
//          the max-height / arrival metrics of src/GPU/Metrics.cu:6-21,44-55.
// extract: dimensional float fields as src/GPU/netcdf_kernel.cu:6-126 and
//          the gauge samples of src/GPU/Volumen_kernel.cu:223-254 +
//          src/GPU/ShallowWater.cu:69-90 (computed in FP64 from the FP32 state).
#include "device.cuh"
#include "kernels.h"

namespace thy {

__global__ void init_state_kernel(ScenarioDev s, const double *__restrict__ h, const double *__restrict__ Hs,
                                  const double *__restrict__ qx, const double *__restrict__ qy, double Hmin, double eps_h)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    if (y >= s.ny || x >= s.pitch) return;
    const size_t idx = (size_t)y * s.pitch + x;
    if (x >= s.nx) {
        // row padding: never read by the stencils, kept finite
        for (int k = 0; k < 2; k++) { s.eta[k][idx] = 0.f; s.qx[k][idx] = 0.f; s.qy[k][idx] = 0.f; }
        s.dep[idx] = 0.f; s.eta_max[idx] = -1e30f; s.arr[idx] = -1.f; s.eta_ini[idx] = -1e30f;
        return;
    }
    const size_t i = (size_t)y * s.nx + x;
    const double hd = h[i];
    const double D = Hs[i] + Hmin;          // true still-water depth (m / H)
    const float dep = (float)D;
    const float eta = (hd == 0.0) ? -dep : (float)(hd - D);
    const float fx = qx ? (float)qx[i] : 0.f, fy = qy ? (float)qy[i] : 0.f;
    for (int k = 0; k < 2; k++) { s.eta[k][idx] = eta; s.qx[k][idx] = fx; s.qy[k][idx] = fy; }
    s.dep[idx] = dep;
    const float em = (hd < eps_h) ? -1e30f : eta;
    s.eta_max[idx] = em;
    s.eta_ini[idx] = em;
    s.arr[idx] = -1.f;
}

void launch_init_state(const ScenarioDev *s_host, const ScenarioDev *s_dev, const double *h, const double *Hs,
                       const double *qx, const double *qy, double Hmin, cudaStream_t st)
{
    (void)s_dev;
    dim3 grid((s_host->pitch + 255) / 256, s_host->ny);
    init_state_kernel<<<grid, 256, 0, st>>>(*s_host, h, Hs, qx, qy, Hmin, s_host->eps_h64);
}

__global__ void extract_kernel(ScenarioDev s, int field, int parity, float *__restrict__ out, double Hs, double Qs,
                               double eps_h)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    if (x >= s.nx || y >= s.ny) return;
    const size_t idx = (size_t)y * s.pitch + x;
    const size_t o = (size_t)y * s.nx + x;
    switch (field) {
    case kFieldEta: {
        const double h = (double)s.eta[parity][idx] + (double)s.dep[idx];
        out[o] = (h < eps_h) ? -9999.0f : (float)((double)s.eta[parity][idx] * Hs);
    } break;
    case kFieldUx:
    case kFieldUy: {
        const double h = (double)s.eta[parity][idx] + (double)s.dep[idx];
        double f;
        if (h < eps_h) {
            const double e4 = eps_h * eps_h * eps_h * eps_h;
            f = 1.41421356237309505 * h / sqrt(h * h * h * h + e4) * (Qs / Hs);
        } else {
            f = Qs / (h * Hs);
        }
        const float q = (field == kFieldUx) ? s.qx[parity][idx] : s.qy[parity][idx];
        out[o] = (float)((double)q * f);
    } break;
    case kFieldMaxHeight: {
        const float em = s.eta_max[idx];
        out[o] = (em < -1e20f) ? -9999.0f : (float)((double)em * Hs);
    } break;
    case kFieldArrival: {
        const float a = s.arr[idx];
        out[o] = (a < 0.f) ? -1.0f : a;
    } break;
    default:
        out[o] = (float)((double)s.dep[idx] * Hs);
    }
}

void launch_extract(const ScenarioDev *s_host, int field, int parity, float *out, double Hs, double Qs, double Hmin,
                    cudaStream_t st)
{
    (void)Hmin;
    dim3 grid((s_host->nx + 255) / 256, s_host->ny);
    extract_kernel<<<grid, 256, 0, st>>>(*s_host, field, parity, out, Hs, Qs, s_host->eps_h64);
}

__global__ void gauges_kernel(ScenarioDev s, int parity, const int *__restrict__ cells, int nP, float *__restrict__ out4,
                              double Hs, double Qs, double eps_h)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nP) return;
    const int c = cells[k];
    if (c < 0) {
        out4[4 * k + 0] = out4[4 * k + 1] = out4[4 * k + 2] = out4[4 * k + 3] = -9999.0f;
        return;
    }
    const int x = c % s.nx, y = c / s.nx;
    const size_t idx = (size_t)y * s.pitch + x;
    const double eta = (double)s.eta[parity][idx], D = (double)s.dep[idx];
    const double h = eta + D;
    double f;
    if (h < eps_h) {
        const double e4 = eps_h * eps_h * eps_h * eps_h;
        f = 1.41421356237309505 * h / sqrt(h * h * h * h + e4);
    } else {
        f = 1.0 / h;
    }
    out4[4 * k + 0] = (float)(eta * Hs);
    out4[4 * k + 1] = (float)(f * (double)s.qx[parity][idx] * Qs / Hs);
    out4[4 * k + 2] = (float)(f * (double)s.qy[parity][idx] * Qs / Hs);
    out4[4 * k + 3] = (float)(D * Hs);
}

void launch_gauges(const ScenarioDev *s_host, int parity, const int *cells, int nP, float *out4, double Hs, double Qs,
                   double Hmin, cudaStream_t st)
{
    (void)Hmin;
    if (nP <= 0) return;
    gauges_kernel<<<(nP + 127) / 128, 128, 0, st>>>(*s_host, parity, cells, nP, out4, Hs, Qs, s_host->eps_h64);
}

}  // namespace thy
