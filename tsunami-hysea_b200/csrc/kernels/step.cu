// Time-step kernels of the B200 stepper.
//
// One time step = two launches over a work list of (scenario, tile) items:
//   phase 1  mass fluxes -> new surface elevation, fused with the
//            max-height / arrival-time diagnostics of the state the step
//            starts from (src/GPU/Metrics.cu:23-77);
//   phase 2  momentum fluxes with the phase-1 depths -> new discharges,
//            sponge, shallow-water filter, Manning friction, local CFL dt,
//            tile min -> one atomicMin per tile; the last tile of a
//            scenario runs the step controller (time, next dt, events).
// Phase 0 (same template) computes the initial dt.
//
// Row marching: a tile is kWarps column strips side by side; in a strip each
// lane owns one column and the warp marches down the tile's rows keeping a
// five-row window of its column in registers.  The y edge below the current
// row needs nothing but that window; x edges take their left/right
// neighbours from warp shuffles.  The 32 lanes cover 28 output columns plus
// a two-column halo on each side (the x stencil reaches two cells), so the
// loads of a strip are whole rows and need no shared memory.  Rows are
// loaded two ahead of the one being computed.  Each edge flux is evaluated once
// per strip: the lane right of an x edge computes it and hands the left
// cell's share to its neighbour with one shuffle; the y edge below row y is
// carried to row y+1 in registers.  No accumulator arrays, no edge
// colouring, no atomics on cells.
//
// Reference: src/GPU/Timestep.cu:11-120 (launch sequence),
// src/GPU/Arista_kernel.cu (edge fluxes), src/GPU/Volumen_kernel.cu (cell
// updates), src/GPU/Reduccion_kernel.cu (dt min).
#include "device.cuh"
#include "kernels.h"

#include <cfloat>

namespace thy {

constexpr int NT = kStepThreads;
constexpr int WARPS = NT / 32;
constexpr int OUTW = 28;              // output columns per warp
constexpr int TY = kTileY;            // output rows per tile
static_assert(kTileX == WARPS * OUTW, "tile width = warps x 28 columns");

// one cell of a lane's column: depth, surface elevation, still-water depth, discharges
struct Cell {
    float h, e, D, qx, qy;
};

// Column of a loaded cell: periodic wrap or clamp (src/GPU/Arista_kernel.cu:6-21).
// Halo lanes beyond the grid load a valid column (modulo / clamp); only the
// columns the reference would read are used by an edge.
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

__device__ __forceinline__ Cell load_cell(const float *__restrict__ eta, const float *__restrict__ dep,
                                          const float *__restrict__ qx, const float *__restrict__ qy, size_t idx)
{
    Cell c;
    c.e = __ldg(eta + idx);
    c.D = __ldg(dep + idx);
    c.qx = __ldg(qx + idx);
    c.qy = __ldg(qy + idx);
    c.h = c.e + c.D;
    return c;
}

// raw loads of a row that is still in flight (prefetch two rows ahead)
struct RawCell {
    float e, D, qx, qy;
};

__device__ __forceinline__ RawCell load_raw(const float *__restrict__ eta, const float *__restrict__ dep,
                                            const float *__restrict__ qx, const float *__restrict__ qy, size_t idx)
{
    RawCell r;
    r.e = __ldg(eta + idx);
    r.D = __ldg(dep + idx);
    r.qx = __ldg(qx + idx);
    r.qy = __ldg(qy + idx);
    return r;
}

__device__ __forceinline__ Cell finish(const RawCell &r)
{
    Cell c;
    c.e = r.e;
    c.D = r.D;
    c.qx = r.qx;
    c.qy = r.qy;
    c.h = r.e + r.D;
    return c;
}

__device__ __forceinline__ float shup(float v, int d) { return __shfl_up_sync(0xffffffffu, v, d); }
__device__ __forceinline__ float shdn(float v, int d) { return __shfl_down_sync(0xffffffffu, v, d); }

// Wave-speed term of one edge for the initial dt (src/GPU/Arista_kernel.cu:1237-1280);
// x edges carry len/cos in e.len.
__device__ __forceinline__ float initial_speed(Edge &e, const ScenarioDev &s)
{
    if (e.front) {
        swapf(e.h0, e.h1);
        swapf(e.u0, e.u1);
    }
    const float w0 = e.u0 * e.normal, w1 = e.u1 * e.normal;
    const float h0 = e.h0, h1 = e.h1, hij = 0.5f * (h0 + h1);
    const float u0n = inv_depth(h0, s.eps_h) * w0, u1n = inv_depth(h1, s.eps_h) * w1;
    const float s0 = sqrtf(h0), s1 = sqrtf(h1);
    const float uij = (s0 * u0n + s1 * u1n) / (s0 + s1 + kEps);
    float maxa = fabsf(uij) + sqrtf(hij);
    if (maxa < s.eps_h) maxa += s.eps_h;
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

// Edge between rows gy-1 (a) and gy (b) of this lane's column, stencil rows
// gy-2 .. gy+1 = (m, a, b, p).  "u" is qy (normal), "v" qx (tangential).
__device__ __forceinline__ void gather_y(Edge &e, const ScenarioDev &s, const Cell &m, const Cell &a, const Cell &b,
                                         const Cell &p, int gy)
{
    e.h0m = m.h; e.h0 = a.h; e.h1 = b.h; e.h1p = p.h;
    e.e0m = m.e; e.e0 = a.e; e.e1 = b.e; e.e1p = p.e;
    e.D0 = a.D; e.D1 = b.D;
    e.u0m = m.qy; e.u0 = a.qy; e.u1 = b.qy; e.u1p = p.qy;
    e.v0m = m.qx; e.v0 = a.qx; e.v1 = b.qx; e.v1p = p.qx;
    const int ra = clamp_row(gy - 1, s.ny), rb = clamp_row(gy, s.ny);
    e.area0 = __ldg(s.row.area + ra); e.cos0 = __ldg(s.row.cosphi + ra);
    e.area1 = __ldg(s.row.area + rb); e.cos1 = __ldg(s.row.cosphi + rb);
    e.len = __ldg(s.row.dlon + gy);
    e.normal = 1.f;
    e.front = false;
    if (gy == 0) {
        e.u0 *= s.b_up;
        e.normal = -1.f;
        e.front = true;
    }
    if (gy == s.ny) e.u1 *= s.b_low;
    e.no_lim = (gy < 2) || (gy > s.ny - 2);
}

// contributions of an edge to the cell on its low side (lo) and high side (hi):
// {mass or qx, qy, lambda}
struct Contrib {
    float a, b, lam;
};

template <int PHASE>
__device__ __forceinline__ void y_edge(const ScenarioDev &s, const Cell &m, const Cell &a, const Cell &b, const Cell &p,
                                       int gy, float dt, Contrib &lo, Contrib &hi)
{
    Edge e;
    gather_y(e, s, m, a, b, p, gy);
    const bool ghost_lo = (gy == 0);
    if (PHASE == 1) {
        const float F = mass_flux<true>(e, s, dt);
        lo = {-F / e.cos0, 0.f, 0.f};
        // top ghost: the boundary cell is the low side of the mirrored edge
        hi = ghost_lo ? Contrib{-F / e.cos0, 0.f, 0.f} : Contrib{F / e.cos1, 0.f, 0.f};
    } else if (PHASE == 2) {
        MomFlux f = momentum_flux_y(e, s, dt);
        if (!f.active) { f.m_x = f.m_y = f.p_x = f.p_y = f.lam = 0.f; }
        lo = {-f.m_x, -f.m_y, f.lam};
        hi = ghost_lo ? lo : Contrib{-f.p_x, -f.p_y, f.lam};
    } else {
        const float lam = initial_speed(e, s);
        lo = {0.f, 0.f, lam};
        hi = lo;
    }
}

template <int PHASE>
__global__ void __launch_bounds__(NT) step_kernel(const ScenarioDev *__restrict__ scen, const int2 *__restrict__ work,
                                                  const int *__restrict__ nwork_ptr)
{
    __shared__ float red[WARPS];
    __shared__ int is_last;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nwork = *nwork_ptr;
    for (int w = blockIdx.x; w < nwork; w += gridDim.x) {
        const int2 item = work[w];
        const ScenarioDev &s = scen[item.x];
        ScenarioCtl *ctl = s.ctl;
        const int status = *((volatile int *)&ctl->status);
        if (PHASE != 0 && status != kRunning) continue;
        const int nx = s.nx, ny = s.ny;
        const int ty = item.y / s.tiles_x, tx = item.y - ty * s.tiles_x;
        const int x0 = tx * kTileX + warp * OUTW, y0 = ty * TY;
        const int p = ctl->parity;
        const float dt = (float)ctl->dt;
        const float t_sec = (float)(ctl->t * ctl->T);
        const int gx = x0 - 2 + lane;
        const int col = map_col(gx, nx, s.periodic);
        const bool has_edge = (lane >= 2) && (lane <= 30) && (gx <= nx);
        const bool has_cell = (lane >= 2) && (lane <= 29) && (gx < nx);
        const int y_end = min(y0 + TY, ny);
        const float *eta_in = (PHASE == 2) ? s.eta[p ^ 1] : s.eta[p];
        const float *qx_in = s.qx[p], *qy_in = s.qy[p];
        const size_t pitch = (size_t)s.pitch;
        const bool x_ghost_lo = !s.periodic && gx == 0, x_ghost_hi = !s.periodic && gx == nx;
        const bool x_nolim = (gx < 2) || (gx > nx - 2);
        const bool sponge = (s.sp_left | s.sp_right | s.sp_up | s.sp_low) != 0;
        float local_min = FLT_MAX;
        bool bad = false;

        if (x0 < nx) {
            Cell c0 = load_cell(eta_in, s.dep, qx_in, qy_in, clamp_row(y0 - 2, ny) * pitch + col);
            Cell c1 = load_cell(eta_in, s.dep, qx_in, qy_in, clamp_row(y0 - 1, ny) * pitch + col);
            Cell c2 = load_cell(eta_in, s.dep, qx_in, qy_in, clamp_row(y0, ny) * pitch + col);
            Cell c3 = load_cell(eta_in, s.dep, qx_in, qy_in, clamp_row(y0 + 1, ny) * pitch + col);
            Cell c4 = load_cell(eta_in, s.dep, qx_in, qy_in, clamp_row(y0 + 2, ny) * pitch + col);
            RawCell n1 = load_raw(eta_in, s.dep, qx_in, qy_in, clamp_row(y0 + 3, ny) * pitch + col);
            // y edge at the top of the first row (stencil rows y0-2 .. y0+1)
            Contrib top, dummy;
            y_edge<PHASE>(s, c0, c1, c2, c3, y0, dt, dummy, top);

            for (int yo = y0; yo < y_end; yo++) {
                // rows yo+3 (loaded an iteration ago) and yo+4 (now) are in flight
                const RawCell n2 = load_raw(eta_in, s.dep, qx_in, qy_in, clamp_row(yo + 4, ny) * pitch + col);
                const size_t idx = (size_t)yo * pitch + col;
                float em = 0.f, ar = 0.f, ei = 0.f;
                if (PHASE == 1 && has_cell) {
                    em = s.eta_max[idx];
                    ar = s.arr[idx];
                    ei = s.eta_ini[idx];
                }
                // ---- y edge below this row (between yo and yo+1) ----
                Contrib below, next_top;
                y_edge<PHASE>(s, c1, c2, c3, c4, yo + 1, dt, below, next_top);

                // ---- x edge left of this lane's cell (row yo) ----
                Edge e;
                e.h0m = shup(c2.h, 2);
                e.e0m = shup(c2.e, 2);
                e.h0 = shup(c2.h, 1);
                e.u0 = shup(c2.qx, 1);
                e.h1 = c2.h;
                e.u1 = c2.qx;
                if (PHASE != 0) {
                    e.e0 = shup(c2.e, 1);
                    e.D0 = shup(c2.D, 1);
                    e.h1p = shdn(c2.h, 1);
                    e.e1p = shdn(c2.e, 1);
                    e.e1 = c2.e;
                    e.D1 = c2.D;
                }
                if (PHASE == 2) {
                    // the tangential discharge only enters the momentum flux
                    e.v0m = shup(c2.qy, 2);
                    e.v0 = shup(c2.qy, 1);
                    e.v1p = shdn(c2.qy, 1);
                    e.v1 = c2.qy;
                } else {
                    e.v0m = e.v0 = e.v1p = e.v1 = 0.f;
                }
                e.u0m = e.u1p = 0.f;
                const float area = __ldg(s.row.area + yo);
                e.area0 = e.area1 = area;
                e.cos0 = e.cos1 = __ldg(s.row.cosphi + yo);
                e.len = __ldg(s.row.ilcos + yo);
                e.normal = 1.f;
                e.front = false;
                if (x_ghost_lo) {
                    e.u0 *= s.b_left;
                    e.normal = -1.f;
                    e.front = true;
                }
                if (x_ghost_hi) e.u1 *= s.b_right;
                e.no_lim = x_nolim;
                Contrib xl = {0.f, 0.f, 0.f}, xr = {0.f, 0.f, 0.f};
                if (has_edge) {
                    if (PHASE == 1) {
                        const float F = mass_flux<false>(e, s, dt);
                        xl = {-F, 0.f, 0.f};
                        xr = x_ghost_lo ? Contrib{-F, 0.f, 0.f} : Contrib{F, 0.f, 0.f};
                    } else if (PHASE == 2) {
                        MomFlux f = momentum_flux_x(e, s, dt);
                        if (!f.active) { f.m_x = f.m_y = f.p_x = f.p_y = f.lam = 0.f; }
                        xl = {-f.m_x, -f.m_y, f.lam};
                        xr = x_ghost_lo ? xl : Contrib{-f.p_x, -f.p_y, f.lam};
                    } else {
                        const float lam = initial_speed(e, s);
                        xl = {0.f, 0.f, lam};
                        xr = xl;
                    }
                }
                // the right edge of this cell is the left edge of lane+1
                Contrib xrr;
                xrr.a = shdn(xl.a, 1);
                if (PHASE == 2) xrr.b = shdn(xl.b, 1);
                if (PHASE != 1) xrr.lam = shdn(xl.lam, 1);

                // ---- cell (gx, yo) ----
                if (has_cell) {
                    if (PHASE == 0) {
                        const float lam = ((xr.lam + xrr.lam) + top.lam) + below.lam;
                        const float step = (lam < kEps) ? 1e30f : __fdividef(2.f * s.cfl * area, lam);
                        local_min = fminf(local_min, step);
                    } else if (PHASE == 1) {
                        // diagnostics of the state the step starts from
                        const float e_old = c2.e, h_old = c2.h;
                        if (e_old > em && h_old > s.eps_h) s.eta_max[idx] = e_old;
                        if (ar < 0.f && fabsf(e_old - ei) > s.dif_at) s.arr[idx] = t_sec;
                        // mass update (src/GPU/Volumen_kernel.cu:111-157)
                        const float acc = ((xr.a + xrr.a) + top.a) + below.a;
                        const float D = c2.D;
                        float eta = e_old + __fdividef(dt, area) * acc;
                        if (!(eta + D > 0.f)) eta = -D;
                        if (sponge && ((gx < s.sp_left) || (gx >= nx - s.sp_right) || (yo < s.sp_up) ||
                                       (yo >= ny - s.sp_low))) {
                            const float dx = __ldg(s.row.dlon + yo), dy = __ldg(s.row.dlat + yo);
                            float dl = (s.sp_left - gx - 0.5f) * dx, dr = (gx - (nx - 1 - s.sp_right) - 0.5f) * dx;
                            float du = (s.sp_up - yo - 0.5f) * dy, dd = (yo - (ny - 1 - s.sp_low) - 0.5f) * dy;
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
                        const float lam = ((xr.lam + xrr.lam) + top.lam) + below.lam;
                        const float step = (lam < kEps) ? 1e30f : __fdividef(2.f * s.cfl * area, lam);
                        local_min = fminf(local_min, step);
                        const float val = __fdividef(dt, area);
                        const float qx_old = c2.qx, qy_old = c2.qy;
                        float qx = qx_old + val * (((xr.a + xrr.a) + top.a) + below.a);
                        float qy = qy_old + val * (((xr.b + xrr.b) + top.b) + below.b);
                        const float h = c2.h;
                        if (sponge) {
                            const float dx = __ldg(s.row.dlon + yo), dy = __ldg(s.row.dlat + yo);
                            if (gx < s.sp_left) {
                                const float rr = ((s.sp_left - gx - 0.5f) * dx) / (dx * s.sp_left);
                                qx -= 0.9f * rr * rr * qx;
                            }
                            if (gx >= nx - s.sp_right) {
                                const float rr = ((gx - (nx - 1 - s.sp_right) - 0.5f) * dx) / (dx * s.sp_right);
                                qx -= 0.9f * rr * rr * qx;
                            }
                            if (yo < s.sp_up) {
                                const float rr = ((s.sp_up - yo - 0.5f) * dy) / (dy * s.sp_up);
                                qy -= 0.9f * rr * rr * qy;
                            }
                            if (yo >= ny - s.sp_low) {
                                const float rr = ((yo - (ny - 1 - s.sp_low) - 0.5f) * dy) / (dy * s.sp_low);
                                qy -= 0.9f * rr * rr * qy;
                            }
                        }
                        if (h <= s.hpos) {
                            // damping of almost-dry cells and velocity cap (filtroEstado)
                            const float f = h / s.eps_h;
                            const float damp = __expf(-dt * (1.f / (pow4f(f) + kEps)));
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
                                const float c1 = dt * s.mf0 * fabsf(u1) / (exp2f(log2f(h) * (4.f / 3.f)) + kEps);
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
                top = next_top;
                c0 = c1;
                c1 = c2;
                c2 = c3;
                c3 = c4;
                c4 = finish(n1);
                n1 = n2;
            }
        }
        if (bad) atomicOr(&ctl->errors, 1u);
        if (PHASE == 1) continue;

        // ---- tile min of the local dt -> scenario min; last tile runs the controller ----
        for (int o = 16; o > 0; o >>= 1) local_min = fminf(local_min, __shfl_xor_sync(0xffffffffu, local_min, o));
        if (lane == 0) red[warp] = local_min;
        __syncthreads();
        if (threadIdx.x == 0) {
            float m = red[0];
            for (int k = 1; k < WARPS; k++) m = fminf(m, red[k]);
            atomicMin(&ctl->dt_bits, __float_as_uint(m));
            __threadfence();
            const unsigned prev = atomicAdd(&ctl->tiles_done, 1u);
            is_last = (prev == (unsigned)(s.ntiles - 1));
            if (is_last) {
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
        __syncthreads();   // red[] is reused by the next item
    }
}

size_t step_smem_bytes() { return sizeof(float) * WARPS + sizeof(int); }

void launch_step_phase(int phase, const ScenarioDev *scen, const int2 *work, const int *nwork, int grid, cudaStream_t st)
{
    switch (phase) {
    case 0: step_kernel<0><<<grid, NT, 0, st>>>(scen, work, nwork); break;
    case 1: step_kernel<1><<<grid, NT, 0, st>>>(scen, work, nwork); break;
    default: step_kernel<2><<<grid, NT, 0, st>>>(scen, work, nwork); break;
    }
}

cudaError_t configure_step_kernels() { return cudaSuccess; }

int step_blocks_per_sm()
{
    int n = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, step_kernel<2>, NT, 0);
    return n;
}

}  // namespace thy
