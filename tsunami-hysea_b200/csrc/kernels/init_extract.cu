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
                              float2 *__restrict__ minmax)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nP) return;
    gauge_values(s, parity, cells[k], out4 + 4 * k, minmax ? minmax + k : nullptr);
}

void launch_gauges(const ScenarioDev *s_host, int parity, const int *cells, int nP, float *out4, bool fold_minmax,
                   cudaStream_t st)
{
    if (nP <= 0) return;
    gauges_kernel<<<(nP + 127) / 128, 128, 0, st>>>(*s_host, parity, cells, nP, out4,
                                                    fold_minmax ? s_host->gauge_minmax : nullptr);
}

// ---------------------------------------------------------------------------
// Step controller (the last launch of every step), one block per scenario
// slot (src/GPU/ShallowWater.cu:397-450 loop body after the step;
// src/GPU/Timestep.cu:35-68 dt truncation to fault times).  Thread 0 reads
// the control block once (plain loads see the step's atomics), advances time
// and dt in registers and writes the changed fields back.  At a gauge time
// the block samples the gauges of the state the step produced into the
// scenario's ring (the reference copies them to the host at every gauge
// time, src/GPU/ShallowWater.cu:410-421), so that a gauge time does not stop
// the scenario; only a gauge time that coincides with a fault pauses it (the
// reference applies the fault first), like snapshots and faults do.  Compiled
// without fast math, as the other output kernels, so that a gauge sample is
// the same whether the device or the host takes it.
// ---------------------------------------------------------------------------
constexpr int kControllerThreads = 128;

__global__ void __launch_bounds__(kControllerThreads) controller_kernel(const ScenarioDev *__restrict__ scen, int nslots)
{
    const ScenarioDev &s = scen[blockIdx.x];
    __shared__ int s_sample;   // ring slot of a gauge sample taken at this step, or -1
    __shared__ int s_parity;
    if (threadIdx.x == 0) {
        s_sample = -1;
        ScenarioCtl *cp = s.ctl;
        if (cp && cp->status == kRunning) {
            ScenarioCtl c = *cp;
            const float dmin = __uint_as_float(c.dt_bits);
            const unsigned errs = c.errors;
            c.t += c.dt;
            double dt = (double)dmin;
            // truncation so that t lands on the next fault time
            const int nf = c.nfaults;
            const int f = c.fault_next;
            const double *tf = c.fault_times;
            if (!c.jumping) {
                if (f < nf && (c.t + dt) * c.T > tf[f]) {
                    dt = tf[f] / c.T - c.t;
                    c.jumping = 1;
                }
            } else {
                c.jumping = 0;
                if (f < nf) {
                    int i = f + 1;
                    while (i < nf && !(fabs(tf[i] - tf[f]) > 2.220446049250313e-16)) i++;
                    if (i < nf && (c.t + dt) * c.T > tf[i]) {
                        dt = tf[i] / c.T - c.t;
                        c.jumping = 1;
                    }
                }
            }
            c.dt = dt;
            c.step += 1;
            c.parity ^= 1;
            c.dt_bits = 0x7f7fffffu;
            c.tiles_done = 0u;
            int ev = 0;
            if (errs || !(dmin > 0.f) || isnan(dmin)) {
                c.status = kFailed;
            } else if (!(c.t < c.t_end)) {
                c.status = kDone;
            } else if (c.max_steps >= 0 && c.step >= c.max_steps) {
                c.events = kEvStepBudget;
                c.status = kDone;
            } else {
                if (f < nf && c.t * c.T >= tf[f]) ev |= kEvFault;
                if (c.save_nc >= 0.0 && c.t >= c.next_nc) ev |= kEvSnapshot;
                if (c.save_ts >= 0.0 && c.t >= c.next_ts) {
                    if (s.ngauges > 0 && !(ev & kEvFault)) {
                        // the loop's gauge event on the device: same time test
                        // and interval update as the host's
                        s_sample = (int)(c.gauge_count % kGaugeRing);
                        s.gauge_ring_t[s_sample] = c.t * c.T;
                        c.next_ts += c.save_ts;
                        c.gauge_count += 1;
                    } else {
                        ev |= kEvSeries;
                    }
                }
                if (ev) {
                    c.events = ev;
                    c.status = kPaused;
                }
            }
            cp->t = c.t;
            cp->dt = c.dt;
            cp->step = c.step;
            cp->parity = c.parity;
            cp->jumping = c.jumping;
            cp->dt_bits = c.dt_bits;
            cp->tiles_done = c.tiles_done;
            cp->events = c.events;
            cp->status = c.status;
            cp->next_ts = c.next_ts;
            cp->gauge_count = c.gauge_count;
            s_parity = c.parity;
        }
    }
    __syncthreads();
    const int slot = s_sample;
    if (slot < 0) return;
    float *dst = s.gauge_ring + (size_t)slot * 4 * s.ngauges;
    for (int k = threadIdx.x; k < s.ngauges; k += blockDim.x)
        gauge_values(s, s_parity, s.gauge_cells[k], dst + 4 * k, s.gauge_minmax + k);
    (void)nslots;
}

// Per unit: the largest still-water depth step |dep1 - dep0| over the edges
// of its cells (ScenarioDev::unit_gmax), one block per unit.
constexpr int kGmaxThreads = 128;
__global__ void __launch_bounds__(kGmaxThreads) unit_gmax_kernel(ScenarioDev s, int nunits)
{
    const int u = blockIdx.x;
    if (u >= nunits) return;
    const int uy = u / s.tiles_x, tx = u - uy * s.tiles_x;
    const int x0 = s.x_org + tx * kTileX, yb = uy * kHalfRows;
    const size_t pitch = (size_t)s.pitch;
    float m = 0.f;
    // x edges between columns x-1 and x, x = x0 .. x0 + kTileX, of the unit's rows
    for (int k = threadIdx.x; k < (kTileX + 1) * kHalfRows; k += blockDim.x) {
        const int y = yb + k / (kTileX + 1), x = x0 + k % (kTileX + 1);
        if (x >= 1 && x < s.nx && y < s.ny) m = fmaxf(m, fabsf(s.dep[y * pitch + x] - s.dep[y * pitch + x - 1]));
    }
    // y edges between rows y-1 and y, y = yb .. yb + kHalfRows, of the unit's columns
    for (int k = threadIdx.x; k < (kHalfRows + 1) * kTileX; k += blockDim.x) {
        const int y = yb + k / kTileX, x = x0 + k % kTileX;
        if (x >= 0 && x < s.nx && y >= 1 && y < s.ny) m = fmaxf(m, fabsf(s.dep[y * pitch + x] - s.dep[(y - 1) * pitch + x]));
    }
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    __shared__ float w[kGmaxThreads / 32];
    if ((threadIdx.x & 31) == 0) w[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 1; k < kGmaxThreads / 32; k++) m = fmaxf(m, w[k]);
        s.unit_gmax[u] = fmaxf(m, w[0]);
    }
}

void launch_unit_gmax(const ScenarioDev *s_host, cudaStream_t st)
{
    const int nunits = s_host->tiles_x * ((s_host->ny + kHalfRows - 1) / kHalfRows);
    if (nunits > 0) unit_gmax_kernel<<<nunits, kGmaxThreads, 0, st>>>(*s_host, nunits);
}

cudaError_t preload_output_kernels()
{
    cudaFuncAttributes a;
    cudaError_t e;
    if ((e = cudaFuncGetAttributes(&a, controller_kernel)) || (e = cudaFuncGetAttributes(&a, init_state_kernel)) ||
        (e = cudaFuncGetAttributes(&a, extract_kernel)) || (e = cudaFuncGetAttributes(&a, gauges_kernel)) ||
        (e = cudaFuncGetAttributes(&a, unit_gmax_kernel)))
        return e;
    return cudaSuccess;
}

void launch_controller(const StepLaunch &L, cudaStream_t st)
{
    controller_kernel<<<L.nslots, kControllerThreads, 0, st>>>(L.scen, L.nslots);
}

}  // namespace thy
