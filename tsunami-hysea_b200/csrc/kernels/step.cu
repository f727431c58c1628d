// Time-step kernels of the B200 stepper.
//
// One time step = two launches over a work list of (scenario, tile) items:
//   phase 1  mass fluxes of every edge of the tile -> new surface elevation;
//            fused with the max-height / arrival-time diagnostics of the
//            state the step starts from (src/GPU/Metrics.cu:23-77);
//   phase 2  momentum fluxes with the phase-1 depths -> new discharges,
//            sponge, shallow-water filter, Manning friction, local CFL dt,
//            tile min -> one atomicMin per tile; the last tile of a
//            scenario runs the step controller (time, next dt, events).
// Each tile stages its stencil (tile + 2-cell halo) in shared memory, each
// edge flux is computed once into shared memory and gathered by the two
// cells it separates: no accumulator arrays, no edge colouring, no atomics
// on cells.  The same template computes the initial dt (phase 0).
//
// Reference: src/GPU/Timestep.cu:11-120 (launch sequence),
// src/GPU/Arista_kernel.cu (edge fluxes), src/GPU/Volumen_kernel.cu (cell
// updates), src/GPU/Reduccion_kernel.cu (dt min).
#include "device.cuh"
#include "kernels.h"

#include <cfloat>

namespace thy {

constexpr int TX = kTileX;
constexpr int TY = kTileY;
constexpr int NT = kStepThreads;
constexpr int SW = TX + 4;   // staged columns (2-cell halo each side)
constexpr int SH = TY + 4;   // staged rows

struct StageTile {
    float eta[SH][SW];
    float dep[SH][SW];
    float h[SH][SW];
    float qx[SH][SW];
    float qy[SH][SW];
};

// per-edge contributions to the cell on the low side (L) and high side (R):
// {d(mass or qx), d(qy), lambda}
struct EdgeTile {
    float xl[TY][TX + 1][3];
    float xr[TY][TX + 1][3];
    float yl[TY + 1][TX][3];
    float yr[TY + 1][TX][3];
};

struct __align__(16) StepSmem {
    StageTile st;
    EdgeTile ed;
    float red[NT / 32];
    int last;
};

// Column of a staged cell: periodic wrap or clamp (src/GPU/Arista_kernel.cu:6-21).
// Staged columns reach up to TX+1 past the grid on partial tiles; those are
// never used by an edge, the modulo only keeps the load in bounds.
__device__ __forceinline__ int map_col(int gx, int nx, int periodic)
{
    if (gx >= 0 && gx < nx) return gx;
    if (periodic) {
        const int m = gx % nx;
        return m < 0 ? m + nx : m;
    }
    return gx < 0 ? 0 : nx - 1;
}

__device__ __forceinline__ int clamp_row(int gy, int ny) { return gy < 0 ? 0 : (gy >= ny ? ny - 1 : gy); }

template <int PHASE>
__device__ void stage(StepSmem &sm, const ScenarioDev &s, int x0, int y0, int p)
{
    // phase 1 reads eta[p]; phase 2 reads the phase-1 output eta[p^1] and q[p];
    // phase 0 (initial dt) reads eta[p], q[p]
    const float *eta = (PHASE == 2) ? s.eta[p ^ 1] : s.eta[p];
    const float *qx = s.qx[p];
    const float *qy = s.qy[p];
    for (int i = threadIdx.x; i < SW * SH; i += NT) {
        const int r = i / SW, c = i - r * SW;
        const int gx = map_col(x0 - 2 + c, s.nx, s.periodic);
        const int gy = clamp_row(y0 - 2 + r, s.ny);
        const size_t idx = (size_t)gy * s.pitch + gx;
        const float e = eta[idx], d = s.dep[idx];
        sm.st.eta[r][c] = e;
        sm.st.dep[r][c] = d;
        sm.st.h[r][c] = e + d;
        sm.st.qx[r][c] = qx[idx];
        sm.st.qy[r][c] = qy[idx];
    }
}

// x edge at global column gx (between cells gx-1 and gx) of tile row r
__device__ __forceinline__ void gather_x(Edge &e, const StepSmem &sm, const ScenarioDev &s, int r, int ex, int gx, int gy,
                                         bool &ghost_lo, bool &ghost_hi)
{
    const int sr = r + 2;
    const int cm = ex, c0 = ex + 1, c1 = ex + 2, cp = ex + 3;   // cells gx-2 .. gx+1
    e.h0m = sm.st.h[sr][cm]; e.h0 = sm.st.h[sr][c0]; e.h1 = sm.st.h[sr][c1]; e.h1p = sm.st.h[sr][cp];
    e.e0m = sm.st.eta[sr][cm]; e.e0 = sm.st.eta[sr][c0]; e.e1 = sm.st.eta[sr][c1]; e.e1p = sm.st.eta[sr][cp];
    e.D0 = sm.st.dep[sr][c0]; e.D1 = sm.st.dep[sr][c1];
    e.u0m = sm.st.qx[sr][cm]; e.u0 = sm.st.qx[sr][c0]; e.u1 = sm.st.qx[sr][c1]; e.u1p = sm.st.qx[sr][cp];
    e.v0m = sm.st.qy[sr][cm]; e.v0 = sm.st.qy[sr][c0]; e.v1 = sm.st.qy[sr][c1]; e.v1p = sm.st.qy[sr][cp];
    e.area0 = e.area1 = s.row.area[gy];
    e.cos0 = e.cos1 = s.row.cosphi[gy];
    e.len = s.row.ilcos[gy];
    e.normal = 1.f;
    e.front = false;
    ghost_lo = ghost_hi = false;
    if (!s.periodic) {
        if (gx == 0) {
            e.u0 *= s.b_left;
            e.normal = -1.f;
            e.front = true;
            ghost_lo = true;
        }
        if (gx == s.nx) {
            e.u1 *= s.b_right;
            ghost_hi = true;
        }
    }
    e.no_lim = (gx < 2) || (gx > s.nx - 2);
}

// y edge at global row gy (between rows gy-1 and gy) of tile column c
__device__ __forceinline__ void gather_y(Edge &e, const StepSmem &sm, const ScenarioDev &s, int ey, int c, int gy,
                                         bool &ghost_lo, bool &ghost_hi)
{
    const int sc = c + 2;
    const int rm = ey, r0 = ey + 1, r1 = ey + 2, rp = ey + 3;   // rows gy-2 .. gy+1
    e.h0m = sm.st.h[rm][sc]; e.h0 = sm.st.h[r0][sc]; e.h1 = sm.st.h[r1][sc]; e.h1p = sm.st.h[rp][sc];
    e.e0m = sm.st.eta[rm][sc]; e.e0 = sm.st.eta[r0][sc]; e.e1 = sm.st.eta[r1][sc]; e.e1p = sm.st.eta[rp][sc];
    e.D0 = sm.st.dep[r0][sc]; e.D1 = sm.st.dep[r1][sc];
    e.u0m = sm.st.qy[rm][sc]; e.u0 = sm.st.qy[r0][sc]; e.u1 = sm.st.qy[r1][sc]; e.u1p = sm.st.qy[rp][sc];
    e.v0m = sm.st.qx[rm][sc]; e.v0 = sm.st.qx[r0][sc]; e.v1 = sm.st.qx[r1][sc]; e.v1p = sm.st.qx[rp][sc];
    const int ra = clamp_row(gy - 1, s.ny), rb = clamp_row(gy, s.ny);
    e.area0 = s.row.area[ra]; e.cos0 = s.row.cosphi[ra];
    e.area1 = s.row.area[rb]; e.cos1 = s.row.cosphi[rb];
    e.len = s.row.dlon[gy];
    e.normal = 1.f;
    e.front = false;
    ghost_lo = ghost_hi = false;
    if (gy == 0) {
        e.u0 *= s.b_up;
        e.normal = -1.f;
        e.front = true;
        ghost_lo = true;
    }
    if (gy == s.ny) {
        e.u1 *= s.b_low;
        ghost_hi = true;
    }
    e.no_lim = (gy < 2) || (gy > s.ny - 2);
}

__device__ __forceinline__ void put3(float (&dst)[3], float a, float b, float c)
{
    dst[0] = a; dst[1] = b; dst[2] = c;
}

// Wave-speed sum of one edge for the initial dt (src/GPU/Arista_kernel.cu:1237-1280).
__device__ __forceinline__ float initial_speed(Edge &e, const ScenarioDev &s, bool lat)
{
    if (e.front) {
        swapf(e.h0, e.h1); swapf(e.u0, e.u1);
        swapf(e.cos0, e.cos1);
    }
    const float w0 = e.u0 * e.normal, w1 = e.u1 * e.normal;
    const float h0 = e.h0, h1 = e.h1, hij = 0.5f * (h0 + h1);
    const float u0n = inv_depth(h0, s.eps_h) * w0, u1n = inv_depth(h1, s.eps_h) * w1;
    const float s0 = sqrtf(h0), s1 = sqrtf(h1);
    const float uij = (s0 * u0n + s1 * u1n) / (s0 + s1 + kEps);
    float maxa = fabsf(uij) + sqrtf(hij);
    if (maxa < s.eps_h) maxa += s.eps_h;
    // x edges: e.len is already len / cos(lat)
    (void)lat;
    return e.len * maxa;
}

// Step controller, run by the last phase-2 tile of a scenario
// (src/GPU/ShallowWater.cu:397-450 loop body after the step;
//  src/GPU/Timestep.cu:35-68 dt truncation to fault times).
__device__ void controller(const ScenarioDev &s)
{
    ScenarioCtl *c = s.ctl;
    const float dmin = __uint_as_float(atomicOr(&c->dt_bits, 0u));
    const unsigned errs = atomicOr(&c->errors, 0u);
    c->t += c->dt;
    double dt = (double)dmin;
    // truncation so that t lands on the next fault time
    const int nf = c->nfaults;
    const int f = c->fault_next;
    const double *tf = c->fault_times;
    if (!c->jumping) {
        if (f < nf && (c->t + dt) * c->T > tf[f]) {
            dt = tf[f] / c->T - c->t;
            c->jumping = 1;
        }
    } else {
        c->jumping = 0;
        if (f < nf) {
            int i = f + 1;
            while (i < nf && !(fabs(tf[i] - tf[f]) > 2.220446049250313e-16)) i++;
            if (i < nf && (c->t + dt) * c->T > tf[i]) {
                dt = tf[i] / c->T - c->t;
                c->jumping = 1;
            }
        }
    }
    c->dt = dt;
    c->step += 1;
    c->parity ^= 1;
    c->dt_bits = 0x7f7fffffu;
    c->tiles_done = 0u;
    int ev = 0;
    if (errs || !(dmin > 0.f) || isnan(dmin)) {
        c->status = kFailed;
        return;
    }
    if (!(c->t < c->t_end)) {
        c->status = kDone;
        return;
    }
    if (c->max_steps >= 0 && c->step >= c->max_steps) {
        c->events = kEvStepBudget;
        c->status = kDone;
        return;
    }
    if (f < nf && c->t * c->T >= tf[f]) ev |= kEvFault;
    if (c->save_nc >= 0.0 && c->t >= c->next_nc) ev |= kEvSnapshot;
    if (c->save_ts >= 0.0 && c->t >= c->next_ts) ev |= kEvSeries;
    if (ev) {
        c->events = ev;
        c->status = kPaused;
    }
}

template <int PHASE>
__global__ void __launch_bounds__(NT) step_kernel(const ScenarioDev *__restrict__ scen, const int2 *__restrict__ work,
                                                  const int *__restrict__ nwork_ptr)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    StepSmem &sm = *reinterpret_cast<StepSmem *>(smem_raw);
    const int nwork = *nwork_ptr;
    for (int w = blockIdx.x; w < nwork; w += gridDim.x) {
        const int2 item = work[w];
        const ScenarioDev &s = scen[item.x];
        ScenarioCtl *ctl = s.ctl;
        const int status = *((volatile int *)&ctl->status);
        if (PHASE != 0 && status != kRunning) continue;
        const int ty = item.y / s.tiles_x, tx = item.y - ty * s.tiles_x;
        const int x0 = tx * TX, y0 = ty * TY;
        const int p = ctl->parity;
        const float dt = (float)ctl->dt;
        __syncthreads();   // previous item's smem use is complete
        stage<PHASE>(sm, s, x0, y0, p);
        __syncthreads();

        // ---- x edges: TY rows x (TX+1) edges ----
        for (int i = threadIdx.x; i < TY * (TX + 1); i += NT) {
            const int r = i / (TX + 1), ex = i - r * (TX + 1);
            const int gx = x0 + ex, gy = y0 + r;
            if (gy >= s.ny || gx > s.nx) continue;
            Edge e;
            bool glo, ghi;
            gather_x(e, sm, s, r, ex, gx, gy, glo, ghi);
            if (PHASE == 1) {
                const float F = mass_flux<false>(e, s, dt);
                if (glo) put3(sm.ed.xr[r][ex], -F, 0.f, 0.f);
                else put3(sm.ed.xr[r][ex], F, 0.f, 0.f);
                put3(sm.ed.xl[r][ex], -F, 0.f, 0.f);
            } else if (PHASE == 2) {
                MomFlux m = momentum_flux_x(e, s, dt);
                if (!m.active) { m.m_x = m.m_y = m.p_x = m.p_y = m.lam = 0.f; }
                put3(sm.ed.xl[r][ex], -m.m_x, -m.m_y, m.lam);
                if (glo) put3(sm.ed.xr[r][ex], -m.m_x, -m.m_y, m.lam);
                else put3(sm.ed.xr[r][ex], -m.p_x, -m.p_y, m.lam);
            } else {
                const float lam = initial_speed(e, s, false);
                put3(sm.ed.xl[r][ex], 0.f, 0.f, lam);
                put3(sm.ed.xr[r][ex], 0.f, 0.f, lam);
            }
            (void)ghi;
        }
        // ---- y edges: (TY+1) edge rows x TX columns ----
        for (int i = threadIdx.x; i < (TY + 1) * TX; i += NT) {
            const int ey = i / TX, c = i - ey * TX;
            const int gx = x0 + c, gy = y0 + ey;
            if (gx >= s.nx || gy > s.ny) continue;
            Edge e;
            bool glo, ghi;
            gather_y(e, sm, s, ey, c, gy, glo, ghi);
            if (PHASE == 1) {
                const float F = mass_flux<true>(e, s, dt);
                // after a ghost swap cos0 is the boundary cell's own row
                put3(sm.ed.yl[ey][c], -F / e.cos0, 0.f, 0.f);
                if (glo) put3(sm.ed.yr[ey][c], -F / e.cos0, 0.f, 0.f);
                else put3(sm.ed.yr[ey][c], F / e.cos1, 0.f, 0.f);
            } else if (PHASE == 2) {
                MomFlux m = momentum_flux_y(e, s, dt);
                if (!m.active) { m.m_x = m.m_y = m.p_x = m.p_y = m.lam = 0.f; }
                put3(sm.ed.yl[ey][c], -m.m_x, -m.m_y, m.lam);
                if (glo) put3(sm.ed.yr[ey][c], -m.m_x, -m.m_y, m.lam);
                else put3(sm.ed.yr[ey][c], -m.p_x, -m.p_y, m.lam);
            } else {
                const float lam = initial_speed(e, s, true);
                put3(sm.ed.yl[ey][c], 0.f, 0.f, lam);
                put3(sm.ed.yr[ey][c], 0.f, 0.f, lam);
            }
            (void)ghi;
        }
        __syncthreads();

        // ---- cells ----
        float local_min = FLT_MAX;
        bool bad = false;
        const double t_now = ctl->t;
        for (int i = threadIdx.x; i < TX * TY; i += NT) {
            const int r = i / TX, c = i - r * TX;
            const int gx = x0 + c, gy = y0 + r;
            if (gx >= s.nx || gy >= s.ny) continue;
            const size_t idx = (size_t)gy * s.pitch + gx;
            const float *a = sm.ed.xr[r][c], *b = sm.ed.xl[r][c + 1], *u = sm.ed.yr[r][c], *d = sm.ed.yl[r + 1][c];
            const float area = s.row.area[gy];
            const int sr = r + 2, sc = c + 2;
            if (PHASE == 0) {
                const float lam = ((a[2] + b[2]) + u[2]) + d[2];
                const float step = (lam < kEps) ? 1e30f : (2.f * s.cfl * area) / lam;
                local_min = fminf(local_min, step);
                continue;
            }
            const float dtf = dt;
            const float val = dtf / area;
            if (PHASE == 1) {
                // diagnostics of the state the step starts from
                const float e_old = sm.st.eta[sr][sc], h_old = sm.st.h[sr][sc];
                const float em = s.eta_max[idx];
                if (e_old > em && h_old > s.eps_h) s.eta_max[idx] = e_old;
                if (s.arr[idx] < 0.f && fabsf(e_old - s.eta_ini[idx]) > s.dif_at) s.arr[idx] = (float)(t_now * ctl->T);
                // mass update (src/GPU/Volumen_kernel.cu:111-157)
                const float acc = ((a[0] + b[0]) + u[0]) + d[0];
                const float D = sm.st.dep[sr][sc];
                float eta = e_old + val * acc;
                float h = eta + D;
                if (!(h > 0.f)) { eta = -D; h = 0.f; }
                if ((s.sp_left | s.sp_right | s.sp_up | s.sp_low) &&
                    ((gx < s.sp_left) || (gx >= s.nx - s.sp_right) || (gy < s.sp_up) || (gy >= s.ny - s.sp_low))) {
                    const float dx = s.row.dlon[gy], dy = s.row.dlat[gy];
                    float dl = (s.sp_left - gx - 0.5f) * dx, dr = (gx - (s.nx - 1 - s.sp_right) - 0.5f) * dx;
                    float du = (s.sp_up - gy - 0.5f) * dy, dd = (gy - (s.ny - 1 - s.sp_low) - 0.5f) * dy;
                    if (dl <= 0.f) dl = 1e30f;
                    if (dr <= 0.f) dr = 1e30f;
                    if (du <= 0.f) du = 1e30f;
                    if (dd <= 0.f) dd = 1e30f;
                    float dist, ls;
                    if ((dl <= dr) && (dl <= du) && (dl <= dd)) { dist = dl; ls = dx * s.sp_left; }
                    else if ((dr <= dl) && (dr <= du) && (dr <= dd)) { dist = dr; ls = dx * s.sp_right; }
                    else if ((du <= dl) && (du <= dr) && (du <= dd)) { dist = du; ls = dy * s.sp_up; }
                    else { dist = dd; ls = dy * s.sp_low; }
                    const float rr = dist / ls, co = 0.9f * rr * rr;
                    // relax h towards max(D + sea level, 0), expressed on eta
                    const float eta_rest = (D + s.sea > 0.f) ? s.sea : -D;
                    eta -= co * (eta - eta_rest);
                    if (!(eta + D >= 0.f)) eta = -D;
                }
                if (!isfinite(eta)) bad = true;
                s.eta[p ^ 1][idx] = eta;
            } else {
                // momentum update (src/GPU/Volumen_kernel.cu:175-219)
                const float lam = ((a[2] + b[2]) + u[2]) + d[2];
                const float step = (lam < kEps) ? 1e30f : (2.f * s.cfl * area) / lam;
                local_min = fminf(local_min, step);
                const float qx_old = sm.st.qx[sr][sc], qy_old = sm.st.qy[sr][sc];
                float qx = qx_old + val * (((a[0] + b[0]) + u[0]) + d[0]);
                float qy = qy_old + val * (((a[1] + b[1]) + u[1]) + d[1]);
                const float h = sm.st.h[sr][sc];
                if (s.sp_left | s.sp_right | s.sp_up | s.sp_low) {
                    const float dx = s.row.dlon[gy], dy = s.row.dlat[gy];
                    if (gx < s.sp_left) {
                        const float rr = ((s.sp_left - gx - 0.5f) * dx) / (dx * s.sp_left);
                        qx -= 0.9f * rr * rr * qx;
                    }
                    if (gx >= s.nx - s.sp_right) {
                        const float rr = ((gx - (s.nx - 1 - s.sp_right) - 0.5f) * dx) / (dx * s.sp_right);
                        qx -= 0.9f * rr * rr * qx;
                    }
                    if (gy < s.sp_up) {
                        const float rr = ((s.sp_up - gy - 0.5f) * dy) / (dy * s.sp_up);
                        qy -= 0.9f * rr * rr * qy;
                    }
                    if (gy >= s.ny - s.sp_low) {
                        const float rr = ((gy - (s.ny - 1 - s.sp_low) - 0.5f) * dy) / (dy * s.sp_low);
                        qy -= 0.9f * rr * rr * qy;
                    }
                }
                if (h <= s.hpos) {
                    // damping of almost-dry cells and velocity cap (filtroEstado)
                    const float f = h / s.eps_h;
                    const float damp = __expf(-dtf * (1.f / (pow4f(f) + kEps)));
                    qx *= damp;
                    qy *= damp;
                    const float fac = inv_depth(h, s.eps_h);
                    if (s.vmax > 0.f) {
                        float ux = fac * qx, uy = fac * qy;
                        const float uu = sqrtf(ux * ux + uy * uy);
                        if (uu > s.vmax) { ux *= s.vmax / uu; uy *= s.vmax / uu; }
                        qx = ux * h;
                        qy = uy * h;
                    }
                    // semi-implicit Manning friction with the pre-update speed (disImplicita)
                    const float u1x = fac * qx, u1y = fac * qy;
                    const float u1 = sqrtf(qx_old * qx_old + qy_old * qy_old) * fac;
                    if (h > 0.f) {
                        const float c1 = dtf * s.mf0 * fabsf(u1) / (exp2f(log2f(h) * (4.f / 3.f)) + kEps);
                        const float fr = h / (1.f + c1);
                        qx = fr * u1x;
                        qy = fr * u1y;
                    }
                }
                if (!isfinite(qx) || !isfinite(qy)) bad = true;
                s.qx[p ^ 1][idx] = qx;
                s.qy[p ^ 1][idx] = qy;
            }
        }
        if (bad) atomicOr(&ctl->errors, 1u);
        if (PHASE == 1) continue;

        // ---- tile min of the local dt -> scenario min; last tile runs the controller ----
        for (int o = 16; o > 0; o >>= 1) local_min = fminf(local_min, __shfl_xor_sync(0xffffffffu, local_min, o));
        if ((threadIdx.x & 31) == 0) sm.red[threadIdx.x >> 5] = local_min;
        __syncthreads();
        if (threadIdx.x == 0) {
            float m = sm.red[0];
            for (int k = 1; k < NT / 32; k++) m = fminf(m, sm.red[k]);
            atomicMin(&ctl->dt_bits, __float_as_uint(m));
            __threadfence();
            const unsigned prev = atomicAdd(&ctl->tiles_done, 1u);
            sm.last = (prev == (unsigned)(s.ntiles - 1));
            if (sm.last) {
                __threadfence();
                if (PHASE == 2) {
                    controller(s);
                } else {
                    // initial dt: store the min and reset the counters
                    ctl->dt = (double)__uint_as_float(atomicOr(&ctl->dt_bits, 0u));
                    ctl->dt_bits = 0x7f7fffffu;
                    ctl->tiles_done = 0u;
                }
            }
        }
    }
}

size_t step_smem_bytes() { return sizeof(StepSmem); }

void launch_step_phase(int phase, const ScenarioDev *scen, const int2 *work, const int *nwork, int grid, cudaStream_t st)
{
    const size_t smem = sizeof(StepSmem);
    switch (phase) {
    case 0: step_kernel<0><<<grid, NT, smem, st>>>(scen, work, nwork); break;
    case 1: step_kernel<1><<<grid, NT, smem, st>>>(scen, work, nwork); break;
    default: step_kernel<2><<<grid, NT, smem, st>>>(scen, work, nwork); break;
    }
}

cudaError_t configure_step_kernels()
{
    const int smem = (int)sizeof(StepSmem);
    cudaError_t e;
    if ((e = cudaFuncSetAttribute(step_kernel<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem))) return e;
    if ((e = cudaFuncSetAttribute(step_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem))) return e;
    return cudaFuncSetAttribute(step_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
}

int step_blocks_per_sm()
{
    int n = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, step_kernel<2>, NT, sizeof(StepSmem));
    return n;
}

}  // namespace thy
