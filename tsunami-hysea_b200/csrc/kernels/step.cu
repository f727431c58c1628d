// Time-step kernels of the B200 stepper.
//
// One time step = six launches over a work list of (scenario, tile) items:
//   phase 1  mass fluxes -> new surface elevation, fused with the
//            max-height / arrival-time diagnostics of the state the step
//            starts from (src/GPU/Metrics.cu:23-77) and with the depth
//            summary of each work unit of the new state (deep and general
//            kernels, concurrent);
//   classification of the units for the state phase 1 produced;
//   phase 2  momentum fluxes with the phase-1 depths -> new discharges,
//            sponge, shallow-water filter, Manning friction, local CFL dt,
//            one atomicMin per deep unit or general warp task (deep and
//            general kernels, concurrent);
//   control  one block per scenario: time, next dt, events, gauges.
// Phases 1 and 2 are each a deep-water kernel and a general kernel.  A tile
// is deep when every cell within two cells of it is deeper than hpos and it
// is at least two cells from the boundaries and outside the sponge layers:
// then every edge flux is the pure 2s flux and no cell is dried, damped or
// relaxed, and the deep kernel marches the tile with a two-row window and
// a fraction of the instructions and registers.  Both kernels evaluate the
// same predicate on per-tile minimum depths that no launch of the phase
// writes, so every tile is stepped by exactly one of them.
// Phase 0 (the general kernel's arithmetic, one unit per CTA) computes the
// initial dt.
//
// Row marching (general kernel): a unit is 4 column strips side by side, each
// in row groups (a tiling: 1, 2 or 8), and each (strip, row group) is a task
// of one warp, claimed independently of the others; each lane owns one
// column and the warp marches down its rows keeping a five-row window of its
// column in registers.  The y edge below the current
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

#include <algorithm>
#include <type_traits>
#include <cfloat>

namespace thy {

constexpr int STRIPS = kStepThreads / 32;   // column strips of a tile
constexpr int OUTW = 28;              // output columns per strip
constexpr int TY = kTileY;            // output rows per tile
static_assert(kTileX == STRIPS * OUTW, "tile width = strips x 28 columns");
static_assert(STRIPS == 4, "deep and general kernels: 4 column-strip warps per row group");

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

// raw loads of a row that is still in flight (prefetch two rows ahead); in
// phase 1 also the cell's max-height / arrival-time / initial-surface values
struct RawCell {
    float e, D, qx, qy;
    float em, ar, ei;
};

template <bool DIAG>
__device__ __forceinline__ RawCell load_raw(const ScenarioDev &s, const float *__restrict__ eta,
                                            const float *__restrict__ qx, const float *__restrict__ qy, size_t idx,
                                            bool diag)
{
    RawCell r;
    r.e = __ldg(eta + idx);
    r.D = __ldg(s.dep + idx);
    r.qx = __ldg(qx + idx);
    r.qy = __ldg(qy + idx);
    r.em = r.ar = r.ei = 0.f;
    if (DIAG && diag) {
        r.em = s.eta_max[idx];
        r.ar = s.arr[idx];
        r.ei = __ldg(s.eta_ini + idx);
    }
    return r;
}

// Max-height / arrival-time update of one cell from the state the step starts
// from (src/GPU/Metrics.cu:23-77).
__device__ __forceinline__ void diagnostics(const ScenarioDev &s, const RawCell &r, size_t idx, float t_sec)
{
    const float h = r.e + r.D;
    if (r.e > r.em && h > s.eps_h) s.eta_max[idx] = r.e;
    if (r.ar < 0.f && fabsf(r.e - r.ei) > s.dif_at) s.arr[idx] = t_sec;
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
    const float s0 = sqrt_ap(h0), s1 = sqrt_ap(h1);
    const float uij = (s0 * u0n + s1 * u1n) / (s0 + s1 + kEps);
    float maxa = fabsf(uij) + sqrt_ap(hij);
    if (maxa < s.eps_h) maxa += s.eps_h;
    return e.len * maxa;
}

// Edge between rows gy-1 (a) and gy (b) of this lane's column, stencil rows
// gy-2 .. gy+1 = (m, a, b, p).  "u" is qy (normal), "v" qx (tangential).
// ka, kb: row metrics {cos, ilcos, area, dlon} of rows clamp(gy-1) and
// clamp(gy); dlon: the edge row's length (rowpack[gy].w).
__device__ __forceinline__ void gather_y(Edge &e, const ScenarioDev &s, const Cell &m, const Cell &a, const Cell &b,
                                         const Cell &p, int gy, const float4 &ka, const float4 &kb, float dlon)
{
    e.h0m = m.h; e.h0 = a.h; e.h1 = b.h; e.h1p = p.h;
    e.e0m = m.e; e.e0 = a.e; e.e1 = b.e; e.e1p = p.e;
    e.D0 = a.D; e.D1 = b.D;
    e.u0m = m.qy; e.u0 = a.qy; e.u1 = b.qy; e.u1p = p.qy;
    e.v0m = m.qx; e.v0 = a.qx; e.v1 = b.qx; e.v1p = p.qx;
    e.area0 = ka.z; e.cos0 = ka.x;
    e.area1 = kb.z; e.cos1 = kb.x;
    e.len = dlon;
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
                                       int gy, float dt, Contrib &lo, Contrib &hi, const float4 &ka, const float4 &kb,
                                       float dlon)
{
    Edge e;
    gather_y(e, s, m, a, b, p, gy, ka, kb, dlon);
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

// ---------------------------------------------------------------------------
// Work units and their classes.  A unit is a half tile (kTileX x kHalfRows
// cells; tile column tx starts at grid column x_org + tx kTileX, so tile 0
// and the last tile may hold fewer columns); work-list entry w (scenario,
// tile) holds units 2w (upper half) and 2w+1 (lower half).  Phase 1 records each unit's depth summary (UnitSum);
// from the unit's own cells and the border strips and corners of its eight
// neighbours - exactly its two-cell stencil ring -
//   deep:  every cell of unit and ring deeper than hpos, and the unit at
//          least two cells from the boundaries and outside the sponge
//          layers - every edge is a pure 2s edge and no cell is dried,
//          damped or relaxed;
//   dry:   every cell of unit and ring dry (depth 0) at three consecutive
//          classifications - then both state buffers hold the scheme's
//          fixed point (eta = -dep, q = 0), which a step would write again,
//          so the unit is skipped;
//   general: the rest.
// ---------------------------------------------------------------------------
__device__ __forceinline__ int units_y(const ScenarioDev &s) { return (s.ny + kHalfRows - 1) / kHalfRows; }

// The geometric tests imply 1 <= tx <= tiles_x - 2 and 1 <= uy <= units_y - 2.
// *hmin: the smallest depth over the unit and its two-cell ring (when deep).
__device__ __forceinline__ bool unit_deep(const ScenarioDev &s, const UnitSum *__restrict__ sum, int tx, int uy,
                                          float *hmin)
{
    if (!s.tmap) return false;
    const int x0 = s.x_org + tx * kTileX, yb = uy * kHalfRows;
    if (x0 < max(2, s.sp_left) || x0 + kTileX > s.nx - max(2, s.sp_right)) return false;
    if (yb < max(2, s.sp_up) || yb + kHalfRows > s.ny - max(2, s.sp_low)) return false;
    const int W = s.tiles_x;
    const UnitSum *c = sum + (size_t)uy * W + tx;
    const float hp = s.hpos;
    // all nine loads first and no short-circuit, so that they are in flight
    // together (a NaN, an unknown summary, fails its test as before)
    const float v0 = c->all.x, v1 = c[-1].R.x, v2 = c[1].L.x, v3 = c[-W].B.x, v4 = c[W].T.x;
    const float v5 = c[-W - 1].BR.x, v6 = c[-W + 1].BL.x, v7 = c[W - 1].TR.x, v8 = c[W + 1].TL.x;
    *hmin = fminf(fminf(fminf(v0, v1), fminf(v2, v3)), fminf(fminf(v4, v5), fminf(fminf(v6, v7), v8)));
    return (v0 > hp) & (v1 > hp) & (v2 > hp) & (v3 > hp) & (v4 > hp) & (v5 > hp) & (v6 > hp) & (v7 > hp) & (v8 > hp);
}

// Deep-list entries: the unit code (2 x work-list index + half) and, in bit
// kJumpPlain, whether every surface jump of the unit's edges in the state
// the list was made for is the plain difference of the elevations (its unit
// and ring deeper than unit_gmax, with a margin for the FP32 rounding of the
// test itself).
constexpr int kJumpPlain = 30;
__device__ __forceinline__ int unit_code(int entry) { return entry & ((1 << kJumpPlain) - 1); }
__device__ __forceinline__ bool jump_plain(int entry) { return (entry >> kJumpPlain) & 1; }

// Outside the grid counts as dry (ghost cells copy the boundary cell), except
// across a periodic x boundary, where the wrapped unit counts.
__device__ __forceinline__ bool unit_dry(const ScenarioDev &s, const UnitSum *__restrict__ sum, int tx, int uy)
{
    const int ny_u = units_y(s), nx_u = s.tiles_x;
    bool dry = true;
    // every neighbour's load issued without waiting for the previous test
#pragma unroll
    for (int dy = -1; dy <= 1; dy++) {
        const int y = uy + dy;
        if (y < 0 || y >= ny_u) continue;
#pragma unroll
        for (int dx = -1; dx <= 1; dx++) {
            int x = tx + dx;
            if (x < 0 || x >= nx_u) {
                if (!s.periodic) continue;
                x = (x + nx_u) % nx_u;
            }
            const UnitSum &u = sum[(size_t)y * nx_u + x];
            // the part of neighbour (dx, dy) inside the ring
            const float2 v = (dx == 0 && dy == 0) ? u.all
                           : (dy == 0) ? (dx < 0 ? u.R : u.L)
                           : (dx == 0) ? (dy < 0 ? u.B : u.T)
                           : (dy < 0) ? (dx < 0 ? u.BR : u.BL)
                                      : (dx < 0 ? u.TR : u.TL);
            dry &= (v.y <= 0.f);
        }
    }
    return dry;
}

// Per-lane depth accumulators of a unit: every row, the unit's first two
// rows and its last two rows.
struct DepthAcc {
    float amin, amax, tmin, tmax, bmin, bmax;
    __device__ __forceinline__ void init()
    {
        amin = tmin = bmin = FLT_MAX;
        amax = tmax = bmax = -FLT_MAX;
    }
    __device__ __forceinline__ void add(float h, bool top, bool bot)
    {
        amin = fminf(amin, h);
        amax = fmaxf(amax, h);
        if (top) { tmin = fminf(tmin, h); tmax = fmaxf(tmax, h); }
        if (bot) { bmin = fminf(bmin, h); bmax = fmaxf(bmax, h); }
    }
};

// {min, max} over the lanes of a warp that are members
__device__ __forceinline__ float2 warp_minmax(float mn, float mx, bool member)
{
    if (!member) {
        mn = FLT_MAX;
        mx = -FLT_MAX;
    }
    for (int o = 16; o > 0; o >>= 1) {
        mn = fminf(mn, __shfl_xor_sync(0xffffffffu, mn, o));
        mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    }
    return make_float2(mn, mx);
}

// The nine {min, max} of one warp for the unit summary: lanes in the unit's
// first two / last two columns (is_l / is_r); every field of a warp without
// such cells is the empty value.  Written to slot[0..8] in UnitSum order.
__device__ __forceinline__ void warp_unit_summary(const DepthAcc &a, bool cell, bool is_l, bool is_r, float2 *slot)
{
    // rows / columns a warp holds no cell of are skipped (warp-uniform tests)
    const float2 none = make_float2(FLT_MAX, -FLT_MAX);
    const bool has_t = __any_sync(0xffffffffu, cell && a.tmin != FLT_MAX);
    const bool has_b = __any_sync(0xffffffffu, cell && a.bmin != FLT_MAX);
    const bool has_l = __any_sync(0xffffffffu, is_l), has_r = __any_sync(0xffffffffu, is_r);
    const float2 all = warp_minmax(a.amin, a.amax, cell);
    const float2 top = has_t ? warp_minmax(a.tmin, a.tmax, cell) : none;
    const float2 bot = has_b ? warp_minmax(a.bmin, a.bmax, cell) : none;
    const float2 L = has_l ? warp_minmax(a.amin, a.amax, is_l) : none;
    const float2 R = has_r ? warp_minmax(a.amin, a.amax, is_r) : none;
    const float2 TL = (has_l && has_t) ? warp_minmax(a.tmin, a.tmax, is_l) : none;
    const float2 TR = (has_r && has_t) ? warp_minmax(a.tmin, a.tmax, is_r) : none;
    const float2 BL = (has_l && has_b) ? warp_minmax(a.bmin, a.bmax, is_l) : none;
    const float2 BR = (has_r && has_b) ? warp_minmax(a.bmin, a.bmax, is_r) : none;
    if ((threadIdx.x & 31) == 0) {
        slot[0] = all; slot[1] = L; slot[2] = R; slot[3] = top; slot[4] = bot;
        slot[5] = TL; slot[6] = TR; slot[7] = BL; slot[8] = BR;
    }
}

// Combines the per-warp slots (nw warps, 9 float2 each, UnitSum order) into
// the unit summary: thread t < 18 reduces float t (a field's min or max).
__device__ __forceinline__ void store_unit_summary(UnitSum *dst, const float2 *slots, int nw)
{
    static_assert(sizeof(UnitSum) == 18 * sizeof(float), "UnitSum is 9 float2");
    const int t = threadIdx.x;
    if (t < 18) {
        const float *v = reinterpret_cast<const float *>(slots) + t;
        float r = v[0];
        for (int w = 1; w < nw; w++) r = (t & 1) ? fmaxf(r, v[18 * w]) : fminf(r, v[18 * w]);
        reinterpret_cast<float *>(dst)[t] = r;
    }
}

constexpr int kDryAge = 3;   // classifications a unit must stay dry before it is skipped

// ---------------------------------------------------------------------------
// TMA staging: one elected thread issues 2D tensor copies of a half tile's
// window into shared memory, completing on an mbarrier that every thread
// waits on with an iteration limit.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Waits for the phase with this parity to complete; false when it has not
// after kWaitNs of global time or 2^28 polls, whichever comes first (each
// try_wait may suspend the thread for a while), so that no wait is endless.
// A staging copy lands within microseconds; the limit is seconds so that a
// context that is time-sliced or pre-empted on a shared GPU does not take a
// healthy copy for a lost one.
constexpr unsigned long long kWaitNs = 4000000000ull;
// try_wait that may suspend the thread for up to hint_ns while the phase is
// incomplete (it resumes as soon as the phase completes), so that waiting
// warps do not take issue slots from the warps that compute
__device__ __forceinline__ bool mbar_try_wait_hint(uint64_t *bar, uint32_t parity, uint32_t hint_ns)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity), "r"(hint_ns)
        : "memory");
    return ok != 0;
}
constexpr uint32_t kSuspendNs = 1000000;   // at most 1 ms per try
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity)
{
    if (mbar_try_wait(bar, parity)) return true;
    const unsigned long long t0 = global_ns();
    for (int i = 0; i < (1 << 28); i++) {
        if (mbar_try_wait_hint(bar, parity, kSuspendNs)) return true;
        if (global_ns() - t0 > kWaitNs) return false;
    }
    return false;
}

// 2D tile load; x must be a multiple of 4 floats (16 bytes)
__device__ __forceinline__ void tma_load_2d(float *dst, const TmaMap *map, int x, int y, uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
        ::"r"(smem_addr(dst)), "l"(map), "r"(x), "r"(y), "r"(smem_addr(bar))
        : "memory");
}

// untiled bulk copy global -> shared (no multicast): both addresses 16-byte
// aligned, bytes a multiple of 16
__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes, uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
        ::"r"(smem_addr(dst)), "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

__device__ __forceinline__ void tmap_acquire(const TmaMap *map)
{
    asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(map) : "memory");
}

// Warps of a deep-kernel CTA: 4 column strips x NG row groups (the tiling's
// variant: by default phase 1, two CTAs per SM as its double-buffered staging
// is larger, uses 3 row groups so that 24 warps per SM hide the latency;
// phase 2 uses 2 at three CTAs per SM).
constexpr int SPLANE = (kStageRows * kStageW + 31) / 32 * 32;   // floats per staged plane (128-byte multiple)
constexpr int DPLANE = kHalfRows * kTileX;          // floats per staged diagnostics plane
constexpr uint32_t kStateBytes = kStageRows * kStageW * 4;
constexpr uint32_t kDiagBytes = kHalfRows * kTileX * 4;
// x0 = x_org + tx kTileX with x_org a multiple of 4 (tile_origin)
static_assert(kTileX % 4 == 0, "TMA x coordinates x0 - 4 and x0 must be 16-byte aligned");
static_assert(kTileY == 2 * kHalfRows, "two half tiles per tile");
static_assert((SPLANE * 4) % 128 == 0 && (DPLANE * 4) % 128 == 0, "staged planes 128-byte aligned");

// Shared memory of a deep kernel CTA: two staging buffers (double buffering
// across work units), then the two mbarriers, the claimed next unit (index
// and descriptor, one slot per buffer parity) and the error flag, the staged
// row metrics of the current unit and the reduction scratch (one set per
// buffer parity).
constexpr size_t kNextBytes = 16 + 2 * 112;   // s_next[2], s_err, pad, s_unit[2]
// A staging buffer also receives the unit's packed row metrics, rows
// yb-2 .. yb+16 (a deep unit lies at least two rows inside the grid), copied
// with the planes so that they arrive one unit ahead too; each phase derives
// its row constants from them in shared memory.
constexpr int kRawRows = kStageRows + 1;
constexpr uint32_t kRawRowBytes = kRawRows * 16;
__host__ __device__ constexpr size_t deep_raw_rows_offset(int phase)
{
    return (size_t)(4 * SPLANE + (phase == 1 ? 3 * DPLANE : 0)) * sizeof(float);
}
__host__ __device__ constexpr size_t deep_stage_bytes(int phase)
{
    return deep_raw_rows_offset(phase) + (kRawRowBytes + 127) / 128 * 128;   // 128-byte aligned
}
struct DeepRow {
    float4 m;      // cos, ilcos, area, dlon (edge row)
    float icos;    // 1/cos, correctly rounded
    // phase 2, for the unit's dt: dt / area, 1 / (2 cfl area), the x edges'
    // XRowK::kdes, and the YRowK of the y edge above the row (y0: len, cmid,
    // cdiff, c10; y1: c01, li0, kdes0, kdes1)
    float dtA, kcfl, kdx;
    float4 y0, y1;
};
static_assert(sizeof(DeepRow) == 64, "row metrics: four float4");
__host__ __device__ constexpr size_t deep_misc_offset(int phase) { return 2 * deep_stage_bytes(phase); }
static size_t deep_smem_bytes(int phase, int ng)
{
    return deep_misc_offset(phase) + 16 + kNextBytes + kStageRows * sizeof(DeepRow) + 2 * 2 * 4 * ng * sizeof(float);
}

// one cell of a staged row (shared memory; the depth is formed here)
__device__ __forceinline__ Cell staged_cell(const float *st, int i)
{
    Cell c;
    c.e = st[i];
    c.D = st[SPLANE + i];
    c.qx = st[2 * SPLANE + i];
    c.qy = st[3 * SPLANE + i];
    c.h = c.e + c.D;
    return c;
}

// Work lists of a step (device memory, cap entries each): lists[0] = deep
// count, lists[1] = general count, deep work-list indices at lists + 2,
// general ones at lists + 2 + cap.
__device__ __forceinline__ const int *deep_items(const int *lists) { return lists + 2; }
__device__ __forceinline__ const int *general_items(const int *lists, int cap) { return lists + 2 + cap; }

// Splits the work units into deep and general lists (dry units go to
// neither) for the state the next phase reads.  In the step (before_step = 0,
// after phase 1): for a running scenario that is the state phase 1 produced
// (summaries at parity^1), which phase 2 of this step and phase 1 of the next
// step both read, and the dry counts advance; for a scenario that is not
// running it is the state at its current parity.  From the host before a
// chunk (before_step = 1, the work list or a state changed): the state at the
// current parity for every scenario, dry counts unchanged; a state the host
// changed has unknown (NaN) summaries, so its units are general.  Units below
// the grid (the lower half of a last tile row of <= 16 rows) are not listed.
// The counts are zeroed before the launch.
constexpr int kClassifyThreads = 128, kClassifyWarps = kClassifyThreads / 32;
__global__ void __launch_bounds__(kClassifyThreads) classify_kernel(const ScenarioDev *__restrict__ scen,
                                                                   const int2 *__restrict__ work,
                                const int *__restrict__ nwork_ptr, int *__restrict__ lists, int cap, int before_step,
                                int *__restrict__ claims)
{
    const int n = 2 * *nwork_ptr;
    // the deep kernels that read these lists claim units from zero (the
    // previous ones are done: this kernel runs after phase 1)
    if (blockIdx.x == 0 && threadIdx.x < 4) claims[threadIdx.x] = 0;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __shared__ int cnt[2][kClassifyWarps];   // per warp: deep and general units of this round
    __shared__ int base2[2];                 // the block's first deep and general list slots
    for (int base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
        const int u = base + threadIdx.x;
        bool listed = false, deep = false, plain = false;
        ScenarioCtl *dry_ctl = nullptr;   // the scenario of a unit skipped as dry land this step
        if (u < n) {
            const int2 item = work[u >> 1];
            const ScenarioDev &s = scen[item.x];
            const int ty = item.y / s.tiles_x, tx = item.y - ty * s.tiles_x;
            const int uy = 2 * ty + (u & 1);
            listed = uy * kHalfRows < s.ny;
            if (listed) {
                ScenarioCtl *ctl = s.ctl;
                const bool running = !before_step && ctl->status == kRunning;
                const int par = running ? (ctl->parity ^ 1) : ctl->parity;
                const UnitSum *sum = s.usum[par];
                float hmin = 0.f;
                deep = unit_deep(s, sum, tx, uy, &hmin);
                const size_t k = (size_t)uy * s.tiles_x + tx;
                plain = deep && hmin > 1.001f * s.unit_gmax[k] + 1e-6f;
                int age = s.dry_age[k];
                if (running) {
                    age = (!deep && unit_dry(s, sum, tx, uy)) ? min(age + 1, 255) : 0;
                    s.dry_age[k] = (unsigned char)age;
                }
                if (age >= kDryAge) {
                    listed = false;
                    if (running) dry_ctl = ctl;
                } else if (!deep) {
                    // a general unit: the general kernel of the next phase 1
                    // folds its summary into the other parity's entry, from
                    // the empty value (nothing reads that entry before then)
                    float2 *e = reinterpret_cast<float2 *>(&s.usum[par ^ 1][k]);
#pragma unroll
                    for (int f = 0; f < 9; f++) e[f] = make_float2(FLT_MAX, -FLT_MAX);
                }
            }
        }
        // dry units counted with one atomic per scenario and warp (the lanes
        // of a warp can belong to different scenarios of a batch)
        {
            const unsigned peers = __match_any_sync(0xffffffffu, (unsigned long long)dry_ctl);
            if (dry_ctl && lane == __ffs(peers) - 1) atomicAdd(&dry_ctl->units_dry, (unsigned long long)__popc(peers));
        }
        // block-aggregated appends: one atomic per list and block (the
        // counters are two words that every block appends to)
        const unsigned dm = __ballot_sync(0xffffffffu, listed && deep);
        const unsigned gm = __ballot_sync(0xffffffffu, listed && !deep);
        if (lane == 0) {
            cnt[0][warp] = __popc(dm);
            cnt[1][warp] = __popc(gm);
        }
        __syncthreads();
        if (threadIdx.x < 2) {
            int tot = 0;
            for (int w = 0; w < kClassifyWarps; w++) tot += cnt[threadIdx.x][w];
            base2[threadIdx.x] = tot ? atomicAdd(&lists[threadIdx.x], tot) : 0;
        }
        __syncthreads();
        int dbase = base2[0], gbase = base2[1];
        for (int w = 0; w < warp; w++) {
            dbase += cnt[0][w];
            gbase += cnt[1][w];
        }
        const unsigned below = (1u << lane) - 1u;
        if (listed) {
            if (deep) lists[2 + dbase + __popc(dm & below)] = u | (plain ? 1 << kJumpPlain : 0);
            else lists[2 + cap + gbase + __popc(gm & below)] = u;
        }
        __syncthreads();   // cnt and base2 are reused by the next round
    }
}

// ---------------------------------------------------------------------------
// Deep phase 2 in pairs: a lane steps two adjacent columns, and the 2s
// momentum fluxes, y edges and updates of the pair run in packed FP32x2
// arithmetic (two lanes of FP32 per instruction, explicit round-to-nearest,
// so no compiler contraction changes a result between code copies).  The
// formulas are those of momentum_2s_x / momentum_2s_y.
// ---------------------------------------------------------------------------
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __fadd2_rn(a, make_float2(-b.x, -b.y)); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 bc2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 neg2(float2 a) { return make_float2(-a.x, -a.y); }
__device__ __forceinline__ float2 sel2(bool px, bool py, float2 a, float2 b)
{
    return make_float2(px ? a.x : b.x, py ? a.y : b.y);
}
// Square roots of a pair (sqrt_ap per component, with its zero test: written
// as a packed x * rsqrt(x) without it, the 16-warp deep phase 2 no longer
// rounded like the other tilings), and 1/h and sqrt(h) of a cell pair from one
// reciprocal square root per cell (deep cells: h > hpos >= 0)
__device__ __forceinline__ float2 sqrt2(float2 h) { return make_float2(sqrt_ap(h.x), sqrt_ap(h.y)); }
struct Depth2 {
    float2 rh, sh;
};
__device__ __forceinline__ Depth2 depth2(float2 h)
{
    const float2 rs = make_float2(rsqrt_ap(h.x), rsqrt_ap(h.y));
    return Depth2{mul2(rs, rs), make_float2(h.x == 0.f ? 0.f : __fmul_rn(h.x, rs.x), h.y == 0.f ? 0.f : __fmul_rn(h.y, rs.y))};
}

// two cells of a staged row (columns i, i + 1; i even)
struct Cell2 {
    float2 h, e, D, qx, qy;
};
__device__ __forceinline__ Cell2 staged_cell2(const float *st, int i)
{
    Cell2 c;
    c.e = *reinterpret_cast<const float2 *>(st + i);
    c.D = *reinterpret_cast<const float2 *>(st + SPLANE + i);
    c.qx = *reinterpret_cast<const float2 *>(st + 2 * SPLANE + i);
    c.qy = *reinterpret_cast<const float2 *>(st + 3 * SPLANE + i);
    c.h = add2(c.e, c.D);
    return c;
}

struct MomFlux2 {
    float2 m_x, m_y, p_x, p_y, lam;
};
// an edge's fluxes into one of its cells, as momentum_2s_* returns them (the
// cell's update subtracts dt/area times their sum), and its wave-speed term
struct Contrib2 {
    float2 a, b, lam;
};

// momentum_2s_x for two edges at once
__device__ __forceinline__ void momentum_2s_x2(MomFlux2 &r, float2 h0, float2 h1, float2 rh0, float2 rh1, float2 s0,
                                               float2 s1, float2 u0, float2 u1, float2 v0, float2 v1, float2 jump,
                                               const XRowK &k)
{
    const float2 hij = mul2(bc2(0.5f), add2(h0, h1));
    const float2 u0n = mul2(u0, rh0), u1n = mul2(u1, rh1);
    const float2 num = fma2(s0, u0n, mul2(s1, u1n));
    const float2 den = add2(add2(s0, s1), bc2(kEps));
    const float2 uijn = make_float2(__fdividef(num.x, den.x), __fdividef(num.y, den.y));
    const float2 maxa = add2(make_float2(fabsf(uijn.x), fabsf(uijn.y)), sqrt2(hij));
    const bool nx_ = uijn.x < 0.f, ny_ = uijn.y < 0.f;
    const float2 un = sel2(nx_, ny_, u1n, u0n), uu = sel2(nx_, ny_, u1, u0), vv = sel2(nx_, ny_, v1, v0);
    const float2 il = bc2(k.ilcos);
    const float2 mx0 = mul2(mul2(un, uu), il);
    const float2 mx = fma2(mul2(hij, jump), il, mx0);
    const float2 my = mul2(mul2(un, vv), il);
    const float2 des = mul2(mul2(bc2(k.kdes), mul2(maxa, maxa)), sub2(u1, u0));
    r.m_x = sub2(mx, des);
    r.m_y = my;
    r.p_x = sub2(des, mx0);
    r.p_y = neg2(my);
    r.lam = mul2(il, maxa);
}

// momentum_2s_y for two edges at once (one row pair: the constants are shared)
__device__ __forceinline__ void momentum_2s_y2(MomFlux2 &r, float2 h0, float2 h1, float2 rh0, float2 rh1, float2 s0,
                                               float2 s1, float2 u0, float2 u1, float2 v0, float2 v1, float2 jump,
                                               const YRowK &k)
{
    const float2 hij = mul2(bc2(0.5f), add2(h0, h1));
    const float2 u0n = mul2(u0, rh0), u1n = mul2(u1, rh1);
    const float2 num = fma2(s0, u0n, mul2(s1, u1n));
    const float2 den = add2(add2(s0, s1), bc2(kEps));
    const float2 uijn = make_float2(__fdividef(num.x, den.x), __fdividef(num.y, den.y));
    const float2 maxa = add2(make_float2(fabsf(uijn.x), fabsf(uijn.y)), sqrt2(hij));
    const float2 deta = fma2(neg2(mul2(uijn, uijn)), bc2(k.cdiff), mul2(bc2(k.cmid), jump));
    const bool nx_ = uijn.x < 0.f, ny_ = uijn.y < 0.f;
    const float2 un = sel2(nx_, ny_, u1n, u0n), uu = sel2(nx_, ny_, u1, u0), vv = sel2(nx_, ny_, v1, v0);
    const float2 len = bc2(k.len);
    const float2 fym0 = mul2(mul2(un, uu), len);
    // upwind from below: fyp = -fym0, fym = fym0 cos1/cos0; from above: fyp = -fym0 cos0/cos1, fym = fym0
    const float2 fyp = mul2(neg2(fym0), sel2(nx_, ny_, bc2(1.f), bc2(k.c01)));
    const float2 fym = fma2(mul2(hij, deta), bc2(k.li0), mul2(fym0, sel2(nx_, ny_, bc2(k.c10), bc2(1.f))));
    const float2 fxm = mul2(mul2(un, vv), len);
    const float2 m2 = mul2(mul2(maxa, maxa), fma2(u1, bc2(k.cos1), neg2(mul2(u0, bc2(k.cos0)))));
    r.m_x = fxm;
    r.m_y = fma2(bc2(-k.kdes0), m2, fym);
    r.p_x = neg2(fxm);
    r.p_y = fma2(bc2(k.kdes1), m2, fyp);
    r.lam = mul2(len, maxa);
}

// y edge between rows gy-1 (a, row metrics ra) and gy (b, rb) of a deep tile;
// phase 2 also takes 1/h and sqrt(h) of both cells, and the edge's constants
// from rb
template <int PHASE>
__device__ __forceinline__ void y_edge_deep(const ScenarioDev &s, const Cell &a, const Cell &b, float rha, float sha,
                                            float rhb, float shb, const DeepRow &ra, const DeepRow &rb, float dt,
                                            Contrib &lo, Contrib &hi)
{
    const float cos0 = ra.m.x, cos1 = rb.m.x;
    if (PHASE == 1) {
        const float F = mass_2s_y(a.qy, rb.m.w, cos0, cos1, a.h, b.h, dt, ra.m.z, rb.m.z);
        lo = {-F * ra.icos, 0.f, 0.f};
        hi = {F * rb.icos, 0.f, 0.f};
    } else {
        YRowK k;
        k.len = rb.y0.x; k.cmid = rb.y0.y; k.cdiff = rb.y0.z; k.c10 = rb.y0.w;
        k.c01 = rb.y1.x; k.li0 = rb.y1.y; k.kdes0 = rb.y1.z; k.kdes1 = rb.y1.w;
        k.cos0 = cos0; k.cos1 = cos1;
        MomFlux f;
        momentum_2s_y(f, a.h, b.h, rha, rhb, sha, shb, a.qy, b.qy, a.qx, b.qx, surface_jump(a.e, b.e, a.D, b.D), k);
        lo = {-f.m_x, -f.m_y, f.lam};
        hi = {-f.p_x, -f.p_y, f.lam};
    }
}

// surface jumps of two edges (e0 -> e1); PLAIN: the unit's depths exceed its
// depth steps, so each is the plain difference (the same value)
template <bool PLAIN>
__device__ __forceinline__ float2 jump2(float2 e0, float2 e1, float2 D0, float2 D1)
{
    if (PLAIN) return sub2(e1, e0);
    return make_float2(surface_jump(e0.x, e1.x, D0.x, D1.x), surface_jump(e0.y, e1.y, D0.y, D1.y));
}

// y edge of phase 2 between rows a (metrics ra) and b (rb) for two columns
template <bool PLAIN>
__device__ __forceinline__ void y_edge_deep2(const Cell2 &a, const Cell2 &b, float2 rha, float2 sha, float2 rhb,
                                             float2 shb, const DeepRow &ra, const DeepRow &rb, Contrib2 &lo,
                                             Contrib2 &hi)
{
    YRowK k;
    k.len = rb.y0.x; k.cmid = rb.y0.y; k.cdiff = rb.y0.z; k.c10 = rb.y0.w;
    k.c01 = rb.y1.x; k.li0 = rb.y1.y; k.kdes0 = rb.y1.z; k.kdes1 = rb.y1.w;
    k.cos0 = ra.m.x; k.cos1 = rb.m.x;
    const float2 jump = jump2<PLAIN>(a.e, b.e, a.D, b.D);
    MomFlux2 f;
    momentum_2s_y2(f, a.h, b.h, rha, rhb, sha, shb, a.qy, b.qy, a.qx, b.qx, jump, k);
    lo = {f.m_x, f.m_y, f.lam};
    hi = {f.p_x, f.p_y, f.lam};
}

// A deep work unit: unit code u = 2 * (work-list index) + half.
// A deep unit and what its compute warps read of its scenario (read by the
// producer when it claims the unit, so that the compute warps start the unit
// from shared memory): dt, time and parity are fixed during a launch.
struct DeepUnit {
    const ScenarioDev *s;
    ScenarioCtl *ctl;
    float *out0, *out1;       // phase 1: eta at the new parity; phase 2: qx, qy at the new parity
    float *eta_max, *arr;     // phase 1 diagnostics
    const float4 *rowpack;    // phase 2 row metrics
    int uidx, x0, yb, p;      // uidx: the unit's index in the scenario's unit grid
    int pitch;
    float dt, t_sec, eps_h, dif_at, cfl, cvis;
    bool run;
    bool drop;                // test hook: issue no copy for it (its wait runs out)
    bool plain;               // phase 2: every surface jump of the unit is the plain difference
};
static_assert(2 * sizeof(DeepUnit) + 16 <= kNextBytes, "claimed units' slots in shared memory");

template <int PHASE>
__device__ __forceinline__ DeepUnit deep_unit(const ScenarioDev *__restrict__ scen, const int2 *__restrict__ work,
                                              const int *__restrict__ lists, int i)
{
    DeepUnit d;
    const int entry = deep_items(lists)[i];
    const int u = unit_code(entry);
    d.plain = jump_plain(entry);
    const int2 item = work[u >> 1];
    d.s = &scen[item.x];
    const int ty = item.y / d.s->tiles_x, tx = item.y - ty * d.s->tiles_x;
    const int uy = 2 * ty + (u & 1);
    d.uidx = uy * d.s->tiles_x + tx;
    d.x0 = d.s->x_org + tx * kTileX;
    d.yb = uy * kHalfRows;
    const ScenarioDev &s = *d.s;
    ScenarioCtl *ctl = s.ctl;
    d.ctl = ctl;
    d.p = ctl->parity;
    d.run = *((volatile const int *)&ctl->status) == kRunning;
    d.drop = (ctl->inject & 1) != 0;
    d.pitch = s.pitch;
    d.dt = (float)ctl->dt;
    d.t_sec = (PHASE == 1) ? (float)(ctl->t * ctl->T) : 0.f;
    d.eps_h = s.eps_h;
    d.dif_at = s.dif_at;
    d.cfl = s.cfl;
    d.cvis = s.cvis;
    d.out0 = (PHASE == 1) ? s.eta[d.p ^ 1] : s.qx[d.p ^ 1];
    d.out1 = s.qy[d.p ^ 1];
    d.eta_max = s.eta_max;
    d.arr = s.arr;
    d.rowpack = s.rowpack;
    return d;
}

// TMA copies of a unit's window into one staging buffer (one thread).  The
// maps are written by host copies before the launch; a CTA acquires a
// scenario's maps once, when it first copies from that scenario (acq).
template <int PHASE>
__device__ __forceinline__ void deep_issue(const DeepUnit &d, float *stage, uint64_t *bar, const TmaMap *&acq)
{
    const TmaMap *m = d.s->tmap;
    const int p = d.p;
    const int me = (PHASE == 2) ? kMapEta0 + (p ^ 1) : kMapEta0 + p;
    if (m != acq) {
        for (int k = 0; k < kNumMaps; k++) tmap_acquire(m + k);
        acq = m;
    }
    mbar_expect_tx(bar, 4 * kStateBytes + kRawRowBytes + (PHASE == 1 ? 3 * kDiagBytes : 0));
    bulk_load(reinterpret_cast<unsigned char *>(stage) + deep_raw_rows_offset(PHASE), d.s->rowpack + d.yb - 2,
              kRawRowBytes, bar);
    tma_load_2d(stage, m + me, d.x0 - 4, d.yb - 1, bar);
    tma_load_2d(stage + SPLANE, m + kMapDep, d.x0 - 4, d.yb - 1, bar);
    tma_load_2d(stage + 2 * SPLANE, m + kMapQx0 + p, d.x0 - 4, d.yb - 1, bar);
    tma_load_2d(stage + 3 * SPLANE, m + kMapQy0 + p, d.x0 - 4, d.yb - 1, bar);
    if (PHASE == 1) {
        tma_load_2d(stage + 4 * SPLANE, m + kMapEtaMax, d.x0, d.yb, bar);
        tma_load_2d(stage + 4 * SPLANE + DPLANE, m + kMapArr, d.x0, d.yb, bar);
        tma_load_2d(stage + 4 * SPLANE + 2 * DPLANE, m + kMapEtaIni, d.x0, d.yb, bar);
    }
}

// Phase 1 / 2 of the deep tiles, persistent, over the units of the deep list
// (two per tile: its upper and lower half).  A unit's window - its rows plus
// one above and one below, columns x0-4 .. x0+115 of eta, dep, qx, qy, and in
// phase 1 the diagnostics of its own cells and the row metrics - is staged by
// TMA, the next unit's copy in flight while the current one is computed.
// Compute warp w marches its row group (w >> 2) of column strip w & 3 (28
// output columns, lanes 2..29) with a two-row window; one more warp is the
// producer.
template <int PHASE, int NG, int MINB>
__global__ void __launch_bounds__(128 * NG + 32, MINB) deep_kernel(const ScenarioDev *__restrict__ scen,
                                                                const int2 *__restrict__ work,
                                                                const int *__restrict__ lists, int *__restrict__ claim)
{
    extern __shared__ __align__(1024) unsigned char dsm[];
    constexpr size_t SB = deep_stage_bytes(PHASE);
    constexpr int NW = 4 * NG;      // compute warps
    constexpr int PT = NW * 32;     // the producer: lane 0 of warp NW
    // staging buffer b at dsm + b * SB
    unsigned char *misc = dsm + deep_misc_offset(PHASE);
    uint64_t *bars = reinterpret_cast<uint64_t *>(misc);
    int *s_next = reinterpret_cast<int *>(misc + 16);          // [parity]: the unit after the current one
    int &s_err = *reinterpret_cast<int *>(misc + 24);          // a copy did not land in time
    DeepUnit *s_unit = reinterpret_cast<DeepUnit *>(misc + 32);   // [parity]: its descriptor
    DeepRow *rows = reinterpret_cast<DeepRow *>(misc + 16 + kNextBytes);
    float *red0 = reinterpret_cast<float *>(rows + kStageRows);   // [parity][2 NW]: per warp dt, or depth min and max
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const bool producer = warp == NW;
    const int strip = warp & 3, group = warp >> 2;
    // a compute warp's rows of the unit: kHalfRows * group / NG .. kHalfRows * (group + 1) / NG - 1
    const int row0 = kHalfRows * group / NG, nrows = kHalfRows * (group + 1) / NG - row0;
    const int nunits = lists[0];
    if (blockIdx.x >= nunits) return;
    // TMA destinations must be 128-byte aligned: a misaligned buffer is
    // reported on every scenario of the CTA's units and nothing is copied
    if (smem_addr(dsm) & 127u) {
        if (threadIdx.x == PT)
            for (int u = blockIdx.x; u < nunits; u += gridDim.x)
                atomicOr(&scen[work[unit_code(deep_items(lists)[u]) >> 1].x].ctl->errors, 4u);
        return;
    }
    if (threadIdx.x == PT) {
        mbar_init(&bars[0]);
        mbar_init(&bars[1]);
        s_err = 0;
    }
    __syncthreads();
    uint32_t phase_bits = 0;     // bit b: parity of the next completion of bars[b]
    const TmaMap *acq = nullptr; // maps acquired by this CTA (producer)
    DeepUnit d = deep_unit<PHASE>(scen, work, lists, blockIdx.x);
    if (threadIdx.x == PT && d.run && !d.drop) deep_issue<PHASE>(d, reinterpret_cast<float *>(dsm), &bars[0], acq);
    int buf = 0;
    // The first two waves take units blockIdx.x and blockIdx.x + gridDim.x;
    // after that each CTA claims its units from the counter (2 gridDim.x,
    // 2 gridDim.x + 1, ...), so a CTA that started late, or whose units took
    // longer, takes fewer.  A producer warp claims the units, reads their
    // descriptors, issues their copies one unit ahead and reduces each unit's
    // results, while the compute warps step the current unit; they meet once
    // per unit, and the producer publishes the next unit there.
    int pending = blockIdx.x + gridDim.x;   // producer: the unit after the next one
    for (int u = blockIdx.x; u < nunits; buf ^= 1) {
        float *red = red0 + buf * 2 * NW;
        if (producer) {
            // the next unit's copy goes to the other buffer, free since the
            // compute warps passed the end of the previous unit
            if (lane == 0) {
                const int un = pending;
                s_next[buf ^ 1] = un;
                if (un < nunits) {
                    const DeepUnit dn = deep_unit<PHASE>(scen, work, lists, un);
                    s_unit[buf ^ 1] = dn;
                    if (dn.run && !dn.drop)
                        deep_issue<PHASE>(dn, reinterpret_cast<float *>(dsm + (buf ^ 1) * SB), &bars[buf ^ 1], acq);
                    pending = 2 * (int)gridDim.x + atomicAdd(claim, 1);
                }
            }
        } else if (d.run) {
            const ScenarioDev &s = *d.s;
            ScenarioCtl *ctl = d.ctl;
            const int x0 = d.x0, yb = d.yb;
            const float dt = d.dt;
            if (!mbar_wait_bounded(&bars[buf], (phase_bits >> buf) & 1u)) s_err = 1;
            const float4 *raw = reinterpret_cast<const float4 *>(dsm + buf * SB + deep_raw_rows_offset(PHASE));
            if (PHASE == 2 && threadIdx.x < kStageRows) {
                // row constants of the window with the unit's dt folded in, from
                // the staged row metrics (row t of the window at t + 1; staged
                // row t is grid row yb - 1 + t)
                DeepRow r;
                r.m = raw[threadIdx.x + 1];
                const float4 a = raw[threadIdx.x];   // the row above
                r.icos = __frcp_rn(r.m.x);
                r.dtA = __fdividef(dt, r.m.z);
                r.kcfl = 1.f / (2.f * d.cfl * r.m.z);
                r.kdx = make_xrow(r.m.y, r.m.z + r.m.z, dt, d.cvis).kdes;
                const YRowK k = make_yrow(a.x, r.m.x, __frcp_rn(a.x), r.icos, r.m.w, a.z + r.m.z, dt, d.cvis);
                r.y0 = make_float4(k.len, k.cmid, k.cdiff, k.c10);
                r.y1 = make_float4(k.c01, k.li0, k.kdes0, k.kdes1);
                rows[threadIdx.x] = r;
            }
            if (PHASE == 1 && threadIdx.x < kStageRows) {
                // phase 1 row constants from the staged row metrics: 1/cos for
                // the y edges, dt/area
                DeepRow r;
                r.m = raw[threadIdx.x + 1];
                r.icos = __frcp_rn(r.m.x);
                r.dtA = __fdividef(dt, r.m.z);
                rows[threadIdx.x] = r;
            }
            // the compute warps only: the row constants are written, every copy checked
            asm volatile("bar.sync 1, %0;" ::"r"(PT) : "memory");
            if (!s_err) {
              if constexpr (PHASE == 1) {
                auto row = [&](int t) { return rows[t]; };
                const float *stage = reinterpret_cast<const float *>(dsm + buf * SB);
                const float t_sec = d.t_sec;
                const int pitch = d.pitch;
                const int r_first = row0 + 1;                           // staged row of this warp's first output row
                const int sc = strip * 28 + 2 + lane;                   // staged column of this lane
                const int gx = x0 - 4 + sc;                             // grid column
                const bool has_cell = (lane >= 2) && (lane <= 29);
                const int dcol = strip * 28 - 2 + lane;                 // diagnostics column (cells only)
                float local_min = FLT_MAX;    // phase 1: depth minimum
                float local_max = -FLT_MAX;   // phase 1: depth maximum; phase 2: max of lam / (2 cfl area)
                bool bad = false;
                int i = r_first * kStageW + sc;
                Cell c = staged_cell(stage, i);
                float rh_c = 0.f, sh_c = 0.f;
                if (PHASE == 2) {
                    rh_c = rcp_depth(c.h);
                    sh_c = sqrt_ap(c.h);
                }
                DeepRow rc = row(r_first);
                Contrib top;
                {
                    const Cell a = staged_cell(stage, i - kStageW);
                    float rh_a = 0.f, sh_a = 0.f;
                    if (PHASE == 2) {
                        rh_a = rcp_depth(a.h);
                        sh_a = sqrt_ap(a.h);
                    }
                    Contrib dummy;
                    y_edge_deep<PHASE>(s, a, c, rh_a, sh_a, rh_c, sh_c, row(r_first - 1), rc, dt, dummy, top);
                }
                float *out0 = d.out0;
                float *out1 = d.out1;
                int off = (yb + r_first - 1) * pitch + gx;
                // running sum of the cells' new values: non-finite iff one of them is
                float fin = 0.f;
                for (int k = 0; k < nrows; k++, i += kStageW, off += pitch) {
                    const DeepRow rn = row(r_first + k + 1);
                    const Cell n = staged_cell(stage, i + kStageW);
                    const float area = rc.m.z;
                    float rh_n = 0.f, sh_n = 0.f;
                    if (PHASE == 2) {
                        rh_n = rcp_depth(n.h);
                        sh_n = sqrt_ap(n.h);
                    }
                    // y edge below this row
                    Contrib below, next_top;
                    y_edge_deep<PHASE>(s, c, n, rh_c, sh_c, rh_n, sh_n, rc, rn, dt, below, next_top);
                    // x edge left of this lane's cell
                    Contrib xl, xr;
                    if (PHASE == 1) {
                        const float F = mass_2s_x(stage[2 * SPLANE + i - 1], rc.m.y, stage[i - 1] + stage[SPLANE + i - 1],
                                                  c.h, dt, area, area);
                        xl = {-F, 0.f, 0.f};
                        xr = {F, 0.f, 0.f};
                    } else {
                        const float e0 = stage[i - 1], D0 = stage[SPLANE + i - 1];
                        MomFlux f;
                        momentum_2s_x(f, e0 + D0, c.h, shup(rh_c, 1), rh_c, shup(sh_c, 1), sh_c, stage[2 * SPLANE + i - 1],
                                      c.qx, stage[3 * SPLANE + i - 1], c.qy, surface_jump(e0, c.e, D0, c.D),
                                      XRowK{rc.m.y, rc.kdx});
                        xl = {-f.m_x, -f.m_y, f.lam};
                        xr = {-f.p_x, -f.p_y, f.lam};
                    }
                    // the right edge of this cell is the left edge of lane+1
                    Contrib xrr;
                    xrr.a = shdn(xl.a, 1);
                    if (PHASE == 2) {
                        xrr.b = shdn(xl.b, 1);
                        xrr.lam = shdn(xl.lam, 1);
                    }
                    if (PHASE == 1 && has_cell) {
                        // diagnostics of the state the step starts from (src/GPU/Metrics.cu:23-77)
                        const float *dg = stage + 4 * SPLANE + (r_first - 1 + k) * kTileX + dcol;
                        const float em = dg[0], ar = dg[DPLANE], ei = dg[2 * DPLANE];
                        if (c.e > em && c.h > d.eps_h) d.eta_max[off] = c.e;
                        if (ar < 0.f && fabsf(c.e - ei) > d.dif_at) d.arr[off] = t_sec;
                        // mass update (src/GPU/Volumen_kernel.cu:111-157)
                        const float acc = ((xr.a + xrr.a) + top.a) + below.a;
                        float eta = c.e + rc.dtA * acc;
                        if (!(eta + c.D > 0.f)) eta = -c.D;
                        fin += eta;
                        out0[off] = eta;
                        local_min = fminf(local_min, eta + c.D);
                        local_max = fmaxf(local_max, eta + c.D);
                    } else if (PHASE == 2 && has_cell) {
                        // momentum update; no sponge, filter or friction in a deep
                        // tile.  The cell's dt bound 2 cfl area / lam (1e30 for
                        // lam < eps) is taken as the unit's largest lam / (2 cfl
                        // area), inverted once per unit.
                        const float lam = ((xr.lam + xrr.lam) + top.lam) + below.lam;
                        local_max = fmaxf(local_max, (lam < kEps) ? 0.f : lam * rc.kcfl);
                        const float val = rc.dtA;
                        const float qx = c.qx + val * (((xr.a + xrr.a) + top.a) + below.a);
                        const float qy = c.qy + val * (((xr.b + xrr.b) + top.b) + below.b);
                        fin += qx + qy;
                        out0[off] = qx;
                        out1[off] = qy;
                    }
                    top = next_top;
                    rc = rn;
                    c = n;
                    rh_c = rh_n;
                    sh_c = sh_n;
                }
                if (!isfinite(fin)) bad = true;
                if (bad) atomicOr(&ctl->errors, 1u);
                for (int o = 16; o > 0; o >>= 1) {
                    if (PHASE == 1) local_min = fminf(local_min, __shfl_xor_sync(0xffffffffu, local_min, o));
                    local_max = fmaxf(local_max, __shfl_xor_sync(0xffffffffu, local_max, o));
                }
                if (lane == 0) {
                    red[warp] = (PHASE == 1) ? local_min : local_max;
                    if (PHASE == 1) red[NW + warp] = local_max;
                }
              } else {
                // phase 2 in pairs: two column strips of 56 cells; lane l
                // steps staged columns sc0 and sc0 + 1 (lanes 1..28 are cells,
                // lanes 0 and 29 the halo, lanes 30 and 31 repeat lane 29)
                constexpr int NG2 = 2 * NG, PROWS = kHalfRows / NG2;   // row groups, rows per warp
                static_assert(kHalfRows % NG2 == 0, "phase-2 row groups of equal height");
                const int strip2 = warp & 1, group2 = warp >> 1;
                const int prow0 = PROWS * group2;
                const int sc0 = strip2 * 56 + 2 + 2 * min(lane, 29);
                const bool out_lane = (lane >= 1) && (lane <= 28);
                float local_max = -FLT_MAX;                        // max of lam / (2 cfl area)
                float2 fin = make_float2(0.f, 0.f);   // running sum: non-finite iff a new value is
                // the row loop in two copies: surface jumps with their wet/dry
                // tests, or as plain differences (a unit the classification
                // found deeper than its depth steps); a uniform branch per unit
                auto pair_rows = [&](auto plain_tag) {
                    constexpr bool PLAIN = decltype(plain_tag)::value;
                    const float *stage = reinterpret_cast<const float *>(dsm + buf * SB);
                    const int pitch = d.pitch;
                    const int r_first = prow0 + 1;                    // staged row of this warp's first output row
                    int i = r_first * kStageW + sc0;
                    Cell2 c = staged_cell2(stage, i);
                    const Depth2 fc = depth2(c.h);
                    float2 rh_c = fc.rh, sh_c = fc.sh;
                    DeepRow rc = rows[r_first];
                    Contrib2 top;
                    {
                        const Cell2 a = staged_cell2(stage, i - kStageW);
                        Contrib2 dummy;
                        const Depth2 fa = depth2(a.h);
                        y_edge_deep2<PLAIN>(a, c, fa.rh, fa.sh, rh_c, sh_c, rows[r_first - 1], rc, dummy, top);
                    }
                    float *out0 = d.out0, *out1 = d.out1;
                    int off = (yb + r_first - 1) * pitch + x0 - 4 + sc0;
                    // two rows an iteration, so that the row window is renamed
                    // rather than copied (every operation here is explicitly
                    // rounded: the copies compute alike)
    #pragma unroll 2
                    for (int k = 0; k < PROWS; k++, i += kStageW, off += pitch) {
                        const DeepRow rn = rows[r_first + k + 1];
                        const Cell2 n = staged_cell2(stage, i + kStageW);
                        const Depth2 fn = depth2(n.h);
                        const float2 rh_n = fn.rh, sh_n = fn.sh;
                        // y edges below this row
                        Contrib2 below, next_top;
                        y_edge_deep2<PLAIN>(c, n, rh_c, sh_c, rh_n, sh_n, rc, rn, below, next_top);
                        // x edges left of column sc0 (its left neighbour, with its 1/h
                        // and sqrt h, is lane l-1's second column) and between sc0 and
                        // sc0 + 1 (lane 0 is halo: its left edge is not used)
                        const float le = shup(c.e.y, 1), lh = shup(c.h.y, 1);
                        const float lqx = shup(c.qx.y, 1), lqy = shup(c.qy.y, 1);
                        const float rhL = shup(rh_c.y, 1), shL = shup(sh_c.y, 1);
                        // (the left depth D only for the wet/dry tests of the jump)
                        const float2 jump = PLAIN ? sub2(c.e, make_float2(le, c.e.x))
                                                  : jump2<false>(make_float2(le, c.e.x), c.e,
                                                                 make_float2(shup(c.D.y, 1), c.D.x), c.D);
                        MomFlux2 f;
                        momentum_2s_x2(f, make_float2(lh, c.h.x), c.h, make_float2(rhL, rh_c.x), rh_c,
                                       make_float2(shL, sh_c.x), sh_c, make_float2(lqx, c.qx.x), c.qx,
                                       make_float2(lqy, c.qy.x), c.qy, jump, XRowK{rc.m.y, rc.kdx});
                        // column sc0: right cell of the left edge, left cell of the
                        // middle edge; column sc0 + 1: right cell of the middle edge,
                        // left cell of lane l+1's left edge
                        const Contrib2 xr = {f.p_x, f.p_y, f.lam};
                        const Contrib2 xrr = {make_float2(f.m_x.y, shdn(f.m_x.x, 1)),
                                              make_float2(f.m_y.y, shdn(f.m_y.x, 1)),
                                              make_float2(f.lam.y, shdn(f.lam.x, 1))};
                        // momentum update; the dt bound as in the scalar path
                        const float2 lam = add2(add2(add2(xr.lam, xrr.lam), top.lam), below.lam);
                        const float2 w = mul2(lam, bc2(rc.kcfl));
                        const float wm = fmaxf(lam.x < kEps ? 0.f : w.x, lam.y < kEps ? 0.f : w.y);
                        if (out_lane) local_max = fmaxf(local_max, wm);
                        // q - dtA * (sum of the fluxes), bitwise the sum of the
                        // negated fluxes times dtA (negation is exact)
                        const float2 val = bc2(-rc.dtA);
                        const float2 qx = fma2(val, add2(add2(add2(xr.a, xrr.a), top.a), below.a), c.qx);
                        const float2 qy = fma2(val, add2(add2(add2(xr.b, xrr.b), top.b), below.b), c.qy);
                        if (out_lane) {
                            fin = add2(fin, add2(qx, qy));
                            *reinterpret_cast<float2 *>(out0 + off) = qx;
                            *reinterpret_cast<float2 *>(out1 + off) = qy;
                        }
                        top = next_top;
                        rc = rn;
                        c = n;
                        rh_c = rh_n;
                        sh_c = sh_n;
                    }
                };
                if (d.plain) pair_rows(std::true_type{});
                else pair_rows(std::false_type{});
                if (!isfinite(fin.x) || !isfinite(fin.y)) atomicOr(&ctl->errors, 1u);
                for (int o = 16; o > 0; o >>= 1) local_max = fmaxf(local_max, __shfl_xor_sync(0xffffffffu, local_max, o));
                if (lane == 0) red[warp] = local_max;
              }
            }
        }
        if (d.run) phase_bits ^= 1u << buf;
        // every compute warp is done with the staged window, the row metrics
        // and its results; the next unit and the error flag are published
        __syncthreads();
        if (s_err) {
            // a copy did not land in time: report; the producer gives both
            // buffers' copies one more bounded wait so none is still writing; stop
            if (threadIdx.x == PT) {
                atomicOr(&d.s->ctl->errors, 2u);
                if (!d.drop) mbar_wait_bounded(&bars[buf], ((phase_bits >> buf) & 1u) ^ 1u);
                if (s_next[buf ^ 1] < nunits && s_unit[buf ^ 1].run && !s_unit[buf ^ 1].drop)
                    mbar_wait_bounded(&bars[buf ^ 1], (phase_bits >> (buf ^ 1)) & 1u);
            }
            return;
        }
        const int un = s_next[buf ^ 1];
        const DeepUnit dn = s_unit[buf ^ 1];   // valid when un < nunits
        if (d.run && threadIdx.x == PT) {
            const ScenarioDev &s = *d.s;
            ScenarioCtl *ctl = d.ctl;
            float m = red[0];
            for (int k = 1; k < NW; k++) m = (PHASE == 1) ? fminf(m, red[k]) : fmaxf(m, red[k]);
            // phase 2: the unit's dt bound from its largest lam / (2 cfl area),
            // inverted once per unit so that it does not depend on the warps' rows
            if (PHASE == 2) m = (m > 0.f) ? 1.f / m : 1e30f;
            if (PHASE == 1) {
                // a deep unit reports its whole-unit {min, max} for its strips
                // and corners too: conservative for a neighbour's deep test,
                // and a wet unit fails a neighbour's dry test either way
                float mx = red[NW];
                for (int k = 1; k < NW; k++) mx = fmaxf(mx, red[NW + k]);
                const float2 v = make_float2(m, mx);
                s.usum[d.p ^ 1][d.uidx] = UnitSum{v, v, v, v, v, v, v, v, v};
            } else {
                atomicMin(&ctl->dt_bits, __float_as_uint(m));
                atomicAdd(&ctl->units_deep, 1ull);
            }
        }
        u = un;
        d = dn;
    }
}

// General kernel: units that are not deep water (boundaries, sponge layers,
// coasts, wet/dry fronts).  A unit's work is split into tasks of one warp
// each: column strip `strip` (28 output columns and a two-column halo on
// each side) and row group `group` (kHalfRows / NG rows).  general_part runs
// one task: it marches the group's rows and returns the lane's dt bound
// (phases 0 / 2), depth summary (phase 1) and error flag; cell: the lane
// holds one of the strip's output cells, gx_out its grid column.
template <int PHASE, int NG>
__device__ __forceinline__ void general_part(const ScenarioDev &s, const ScenarioCtl *ctl, int tx, int uy, int strip,
                                             int group, float &local_min, DepthAcc &hacc, bool &bad, bool &cell,
                                             int &gx_out)
{
    constexpr int GROWS = kHalfRows / NG;
    static_assert(kHalfRows % NG == 0, "row groups of equal height");
    const int lane = threadIdx.x & 31;
    const int nx = s.nx, ny = s.ny;
    const int uy0 = uy * kHalfRows;
    const int unit_end = min(uy0 + kHalfRows, ny);
    // this warp: column strip `strip`, rows y0 .. y_end-1 of the unit
    const int x0 = s.x_org + tx * kTileX + strip * OUTW, y0 = uy0 + group * GROWS;
    const int p = ctl->parity;
    const float dt = (float)ctl->dt;
    const float t_sec = (float)(ctl->t * ctl->T);
    const int gx = x0 - 2 + lane;
    const int col = map_col(gx, nx, s.periodic);
    const bool has_edge = (lane >= 2) && (lane <= 30) && (gx >= 0) && (gx <= nx);
    const bool has_cell = (lane >= 2) && (lane <= 29) && (gx >= 0) && (gx < nx);
    const int y_end = min(y0 + GROWS, unit_end);
    const float *eta_in = (PHASE == 2) ? s.eta[p ^ 1] : s.eta[p];
    const float *qx_in = s.qx[p], *qy_in = s.qy[p];
    const size_t pitch = (size_t)s.pitch;
    const bool x_ghost_lo = !s.periodic && gx == 0, x_ghost_hi = !s.periodic && gx == nx;
    const bool x_nolim = (gx < 2) || (gx > nx - 2);
    const bool sponge = (s.sp_left | s.sp_right | s.sp_up | s.sp_low) != 0;
    local_min = FLT_MAX;
    hacc.init();
    bad = false;
    gx_out = gx;
    cell = has_cell && x0 < nx && x0 + OUTW > 0;

    if (x0 < nx && x0 + OUTW > 0 && y0 < y_end) {
        constexpr bool DIAG = (PHASE == 1);
        Cell c0 = load_cell(eta_in, s.dep, qx_in, qy_in, clamp_row(y0 - 2, ny) * pitch + col);
        Cell c1 = load_cell(eta_in, s.dep, qx_in, qy_in, clamp_row(y0 - 1, ny) * pitch + col);
        Cell c2, c3, c4;
        {
            // rows y0 .. y0+2 with their diagnostics (rows below the grid are clamped and skipped)
            const RawCell r0 = load_raw<DIAG>(s, eta_in, qx_in, qy_in, clamp_row(y0, ny) * pitch + col, has_cell);
            const RawCell r1 = load_raw<DIAG>(s, eta_in, qx_in, qy_in, clamp_row(y0 + 1, ny) * pitch + col,
                                              has_cell && y0 + 1 < y_end);
            const RawCell r2 = load_raw<DIAG>(s, eta_in, qx_in, qy_in, clamp_row(y0 + 2, ny) * pitch + col,
                                              has_cell && y0 + 2 < y_end);
            if (DIAG && has_cell) {
                diagnostics(s, r0, (size_t)y0 * pitch + col, t_sec);
                if (y0 + 1 < y_end) diagnostics(s, r1, (size_t)(y0 + 1) * pitch + col, t_sec);
                if (y0 + 2 < y_end) diagnostics(s, r2, (size_t)(y0 + 2) * pitch + col, t_sec);
            }
            c2 = finish(r0);
            c3 = finish(r1);
            c4 = finish(r2);
        }
        RawCell n1 = load_raw<DIAG>(s, eta_in, qx_in, qy_in, clamp_row(y0 + 3, ny) * pitch + col,
                                    has_cell && y0 + 3 < y_end);
        // y edge at the top of the first row (stencil rows y0-2 .. y0+1)
        // row metrics {cos, ilcos, area, dlon} (rowpack), loaded a row
        // ahead: kc of row yo, kn of row yo+1 (entry ny: dlon only)
        const float4 *__restrict__ rp = s.rowpack;
        float4 kc = __ldg(rp + y0);
        float4 kn = __ldg(rp + y0 + 1);
        Contrib top, dummy;
        y_edge<PHASE>(s, c0, c1, c2, c3, y0, dt, dummy, top, __ldg(rp + clamp_row(y0 - 1, ny)), kc, kc.w);

        for (int yo = y0; yo < y_end; yo++) {
            const float4 knn = __ldg(rp + min(yo + 2, ny));
            // rows yo+3 (loaded an iteration ago) and yo+4 (now) are in flight
            const RawCell n2 = load_raw<DIAG>(s, eta_in, qx_in, qy_in, clamp_row(yo + 4, ny) * pitch + col,
                                              has_cell && yo + 4 < y_end);
            const size_t idx = (size_t)yo * pitch + col;
            // ---- y edge below this row (between yo and yo+1) ----
            Contrib below, next_top;
            y_edge<PHASE>(s, c1, c2, c3, c4, yo + 1, dt, below, next_top, kc, (yo + 1 < ny) ? kn : kc, kn.w);

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
            const float area = kc.z;
            e.area0 = e.area1 = area;
            e.cos0 = e.cos1 = kc.x;
            e.len = kc.y;
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
                    // mass update (src/GPU/Volumen_kernel.cu:111-157); the
                    // diagnostics run when a row's loads complete
                    const float acc = ((xr.a + xrr.a) + top.a) + below.a;
                    const float D = c2.D;
                    float eta = c2.e + __fdividef(dt, area) * acc;
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
                    hacc.add(eta + D, yo - uy0 < 2, unit_end - yo <= 2);
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
                            const float uu = sqrt_ap(ux * ux + uy * uy);
                            if (uu > s.vmax) { ux *= s.vmax / uu; uy *= s.vmax / uu; }
                            qx = ux * h;
                            qy = uy * h;
                        }
                        // semi-implicit Manning friction with the pre-update speed (disImplicita)
                        const float u1x = fac * qx, u1y = fac * qy;
                        const float u1 = sqrt_ap(qx_old * qx_old + qy_old * qy_old) * fac;
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
            kc = kn;
            kn = knn;
            c0 = c1;
            c1 = c2;
            c2 = c3;
            c3 = c4;
            if (DIAG && has_cell && yo + 3 < y_end) diagnostics(s, n1, idx + 3 * pitch, t_sec);
            c4 = finish(n1);
            n1 = n2;
        }
    }
}

// Phase 0 (the initial dt) over every unit of the work list, one unit per CTA
// iteration, 4 x NG warps; the last unit of a scenario stores its dt.
template <int NG>
__global__ void __launch_bounds__(128 * NG) initial_dt_kernel(const ScenarioDev *__restrict__ scen,
                                                              const int2 *__restrict__ work,
                                                              const int *__restrict__ nwork_ptr)
{
    constexpr int GWARPS = 4 * NG;
    __shared__ float red[GWARPS];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int strip = warp % STRIPS, group = warp / STRIPS;
    const int nitems = 2 * *nwork_ptr;
    for (int u = blockIdx.x; u < nitems; u += gridDim.x) {
        const int2 item = work[u >> 1];
        const ScenarioDev &s = scen[item.x];
        ScenarioCtl *ctl = s.ctl;
        const int ty = item.y / s.tiles_x, tx = item.y - ty * s.tiles_x;
        const int uy = 2 * ty + (u & 1);
        if (uy * kHalfRows >= s.ny) continue;   // a unit below the grid (CTA-uniform)
        float local_min;
        DepthAcc hacc;
        bool bad, cell;
        int gx;
        general_part<0, NG>(s, ctl, tx, uy, strip, group, local_min, hacc, bad, cell, gx);
        if (bad) atomicOr(&ctl->errors, 1u);
        for (int o = 16; o > 0; o >>= 1) local_min = fminf(local_min, __shfl_xor_sync(0xffffffffu, local_min, o));
        if (lane == 0) red[warp] = local_min;
        __syncthreads();
        if (threadIdx.x == 0) {
            float m = red[0];
            for (int k = 1; k < GWARPS; k++) m = fminf(m, red[k]);
            atomicMin(&ctl->dt_bits, __float_as_uint(m));
            // the last unit stores the min and resets the counters
            __threadfence();
            const unsigned prev = atomicAdd(&ctl->tiles_done, 1u);
            if (prev == (unsigned)(s.tiles_x * units_y(s) - 1)) {
                __threadfence();
                ctl->dt = (double)__uint_as_float(atomicOr(&ctl->dt_bits, 0u));
                ctl->dt_bits = 0x7f7fffffu;
                ctl->tiles_done = 0u;
            }
        }
        __syncthreads();   // red[] is reused by the next unit
    }
}

// Folds one warp's share of a unit's depth summary (nine {min, max}, UnitSum
// order; a field the warp holds no cell of is left alone) into the unit's
// summary with integer atomics on the float bits: depths are >= 0, where the
// bit patterns order as the values do (a -0 counts as +0), and min and max are
// exact in any order, so the summary does not depend on which warp came
// first.  The classification resets the summaries of the general units it
// lists to the empty value (FLT_MAX, -FLT_MAX) before this phase runs.
__device__ __forceinline__ void fold_unit_summary(const DepthAcc &a, bool cell, bool is_l, bool is_r, UnitSum *dst)
{
    const float2 none = make_float2(FLT_MAX, -FLT_MAX);
    const bool has_t = __any_sync(0xffffffffu, cell && a.tmin != FLT_MAX);
    const bool has_b = __any_sync(0xffffffffu, cell && a.bmin != FLT_MAX);
    const bool has_l = __any_sync(0xffffffffu, is_l), has_r = __any_sync(0xffffffffu, is_r);
    float2 f[9];
    f[0] = warp_minmax(a.amin, a.amax, cell);
    f[1] = has_l ? warp_minmax(a.amin, a.amax, is_l) : none;
    f[2] = has_r ? warp_minmax(a.amin, a.amax, is_r) : none;
    f[3] = has_t ? warp_minmax(a.tmin, a.tmax, cell) : none;
    f[4] = has_b ? warp_minmax(a.bmin, a.bmax, cell) : none;
    f[5] = (has_l && has_t) ? warp_minmax(a.tmin, a.tmax, is_l) : none;
    f[6] = (has_r && has_t) ? warp_minmax(a.tmin, a.tmax, is_r) : none;
    f[7] = (has_l && has_b) ? warp_minmax(a.bmin, a.bmax, is_l) : none;
    f[8] = (has_r && has_b) ? warp_minmax(a.bmin, a.bmax, is_r) : none;
    if ((threadIdx.x & 31) == 0) {
        int *d = reinterpret_cast<int *>(dst);
#pragma unroll
        for (int k = 0; k < 9; k++) {
            if (f[k].x == FLT_MAX) continue;   // no cell of this field in the task
            const int lo = __float_as_int(f[k].x), hi = __float_as_int(f[k].y);
            atomicMin(d + 2 * k, lo == (int)0x80000000 ? 0 : lo);
            atomicMax(d + 2 * k + 1, hi == (int)0x80000000 ? 0 : hi);
        }
    }
}

// Phases 1 and 2 over the general list of the step.  Every warp runs tasks on
// its own: the first wave takes tasks by warp index, then each warp claims
// its next task from *claim (zeroed by the classification), so no warp waits
// for another and a unit's strips outside the grid (in the first and last
// tile columns) cost nothing.  The tasks of a unit are consecutive, so that
// its strips and row groups run side by side and share their halo rows in L2.
constexpr int kGeneralThreads = 128;
template <int PHASE, int NG>
__global__ void __launch_bounds__(kGeneralThreads, 4) general_kernel(const ScenarioDev *__restrict__ scen,
                                                                    const int2 *__restrict__ work,
                                                                    const int *__restrict__ lists, int cap,
                                                                    int *__restrict__ claim)
{
    constexpr int TASKS = STRIPS * NG;   // tasks per unit
    constexpr int WPB = kGeneralThreads / 32;
    const int lane = threadIdx.x & 31;
    const int ntasks = lists[1] * TASKS;
    const int first_wave = (int)gridDim.x * WPB;
    int t = blockIdx.x * WPB + (threadIdx.x >> 5);
    while (t < ntasks) {
        const int g = t / TASKS, r = t - g * TASKS;
        const int group = r / STRIPS, strip = r - group * STRIPS;
        const int u = general_items(lists, cap)[g];
        const int2 item = work[u >> 1];
        const ScenarioDev &s = scen[item.x];
        ScenarioCtl *ctl = s.ctl;
        if (*((volatile int *)&ctl->status) == kRunning) {
            const int ty = item.y / s.tiles_x, tx = item.y - ty * s.tiles_x;
            const int uy = 2 * ty + (u & 1);
            float local_min;
            DepthAcc hacc;
            bool bad, cell;
            int gx;
            general_part<PHASE, NG>(s, ctl, tx, uy, strip, group, local_min, hacc, bad, cell, gx);
            if (bad) atomicOr(&ctl->errors, 1u);
            if (PHASE == 1) {
                // the unit's first two and last two columns inside the grid
                const int tx0 = s.x_org + tx * kTileX, ux0 = max(tx0, 0), ux1 = min(tx0 + kTileX, s.nx);
                fold_unit_summary(hacc, cell, cell && gx < ux0 + 2, cell && gx >= ux1 - 2,
                                  &s.usum[ctl->parity ^ 1][(size_t)uy * s.tiles_x + tx]);
            } else {
                // the minimum is exact in any order
                for (int o = 16; o > 0; o >>= 1)
                    local_min = fminf(local_min, __shfl_xor_sync(0xffffffffu, local_min, o));
                if (lane == 0) atomicMin(&ctl->dt_bits, __float_as_uint(local_min));
            }
        }
        int next = 0;
        if (lane == 0) next = first_wave + atomicAdd(claim, 1);
        t = __shfl_sync(0xffffffffu, next, 0);
    }
}

// One launch of deep phase PHASE / the general kernel in variant V.
template <int PHASE, int V>
static void launch_deep(const StepLaunch &L, cudaStream_t st)
{
    constexpr int NG = deep_ng(PHASE, V);
    deep_kernel<PHASE, NG, deep_minb(PHASE, V)>
        <<<L.deep_grid[PHASE - 1], 128 * NG + 32, deep_smem_bytes(PHASE, NG), st>>>(L.scen, L.work, L.lists,
                                                                            L.claims + (PHASE - 1));
}
template <int PHASE>
static void launch_deep_any(const StepLaunch &L, cudaStream_t st)
{
    switch (PHASE == 1 ? L.tiling.deep1 : L.tiling.deep2) {
    case 1: launch_deep<PHASE, 1>(L, st); break;
    case 2: launch_deep<PHASE, 2>(L, st); break;
    default: launch_deep<PHASE, 0>(L, st); break;
    }
}
template <int PHASE, int V>
static void launch_general_v(const StepLaunch &L, cudaStream_t st)
{
    general_kernel<PHASE, general_ng(V)><<<L.grid, kGeneralThreads, 0, st>>>(L.scen, L.work, L.lists, L.cap,
                                                                            L.claims + 2 + (PHASE - 1));
}
template <int PHASE>
static void launch_general(const StepLaunch &L, cudaStream_t st)
{
    switch (L.tiling.general) {
    case 1: launch_general_v<PHASE, 1>(L, st); break;
    case 2: launch_general_v<PHASE, 2>(L, st); break;
    default: launch_general_v<PHASE, 0>(L, st); break;
    }
}

void launch_step_kernel(int k, const StepLaunch &L, cudaStream_t st)
{
    switch (k) {
    case 0: launch_deep_any<1>(L, st); break;
    case 1: launch_general<1>(L, st); break;
    case 2:
        cudaMemsetAsync(L.lists, 0, 2 * sizeof(int), st);
        classify_kernel<<<L.classify_grid, kClassifyThreads, 0, st>>>(L.scen, L.work, L.nwork, L.lists, L.cap, 0, L.claims);
        break;
    case 3: launch_deep_any<2>(L, st); break;
    case 4: launch_general<2>(L, st); break;
    default: launch_controller(L, st); break;
    }
}

// phase 0 (initial dt) runs once per scenario: default tiling, the grid of L
void launch_initial_dt(const StepLaunch &L, cudaStream_t st)
{
    initial_dt_kernel<general_ng(0)><<<L.grid, 128 * general_ng(0), 0, st>>>(L.scen, L.work, L.nwork);
}

void launch_lists_current(const StepLaunch &L, cudaStream_t st)
{
    cudaMemsetAsync(L.lists, 0, 2 * sizeof(int), st);
    classify_kernel<<<L.classify_grid, kClassifyThreads, 0, st>>>(L.scen, L.work, L.nwork, L.lists, L.cap, 1, L.claims);
}

template <int PHASE, int V>
static cudaError_t configure_deep()
{
    constexpr int NG = deep_ng(PHASE, V);
    auto *f = deep_kernel<PHASE, NG, deep_minb(PHASE, V)>;
    cudaError_t e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)deep_smem_bytes(PHASE, NG));
    if (e) return e;
    return cudaFuncSetAttribute(f, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
}

// Loads every step kernel now (module loading is otherwise lazy, at a
// kernel's first launch or graph instantiation: inside the first run's loop).
template <typename F>
static cudaError_t preload(F *f)
{
    cudaFuncAttributes a;
    return cudaFuncGetAttributes(&a, f);
}

cudaError_t configure_step_kernels()
{
    cudaError_t e;
    if ((e = preload(initial_dt_kernel<general_ng(0)>)) || (e = preload(general_kernel<1, general_ng(0)>)) ||
        (e = preload(general_kernel<1, general_ng(1)>)) || (e = preload(general_kernel<1, general_ng(2)>)) ||
        (e = preload(general_kernel<2, general_ng(0)>)) || (e = preload(general_kernel<2, general_ng(1)>)) ||
        (e = preload(general_kernel<2, general_ng(2)>)) || (e = preload(classify_kernel)))
        return e;
    if ((e = configure_deep<1, 0>()) || (e = configure_deep<1, 1>()) || (e = configure_deep<1, 2>()) ||
        (e = configure_deep<2, 0>()) || (e = configure_deep<2, 1>()) || (e = configure_deep<2, 2>()))
        return e;
    return cudaSuccess;
}

// Resident CTAs per SM of the phase-2 general kernel / a deep kernel in a variant.
int step_blocks_per_sm(int v)
{
    int n = 0;
    switch (v) {
    case 1: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, general_kernel<2, general_ng(1)>, kGeneralThreads, 0); break;
    case 2: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, general_kernel<2, general_ng(2)>, kGeneralThreads, 0); break;
    default: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, general_kernel<2, general_ng(0)>, kGeneralThreads, 0); break;
    }
    return n;
}

template <int PHASE, int V>
static int deep_occupancy()
{
    constexpr int NG = deep_ng(PHASE, V);
    int n = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, deep_kernel<PHASE, NG, deep_minb(PHASE, V)>, 128 * NG + 32,
                                                  deep_smem_bytes(PHASE, NG));
    return n;
}

int deep_blocks_per_sm(int phase, int v)
{
    if (phase == 1) return v == 1 ? deep_occupancy<1, 1>() : v == 2 ? deep_occupancy<1, 2>() : deep_occupancy<1, 0>();
    return v == 1 ? deep_occupancy<2, 1>() : v == 2 ? deep_occupancy<2, 2>() : deep_occupancy<2, 0>();
}

}  // namespace thy
