// Device-side data structures and FP32 edge-flux arithmetic of the B200
// time stepper.
//
// State of one scenario in HBM (all FP32, row-major with a padded pitch):
//   eta[2]  free-surface elevation above the undisturbed sea level (m / H)
//   dep     still-water depth, positive down, Okada-deformed (m / H);
//           water depth h = eta + dep (h = 0 exactly on dry cells: eta = -dep)
//   qx[2], qy[2]  discharges (x: along longitude, y: along latitude)
//   eta_max, arr, eta_ini   max-height / arrival-time diagnostics
// eta and q are double-buffered: phase 1 reads eta[p] and writes eta[p^1],
// phase 2 reads eta[p^1], q[p] and writes q[p^1]; the controller flips p.
//
// Storing eta instead of h keeps ~1e-10 resolution on the wave itself
// (h ~ 4 in units of H would quantise the surface to ~0.5 mm); every place
// where the reference forms a surface difference from h - H uses eta.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace thy {

constexpr float kEps = 2.220446049250313e-16f;  // the reference's EPSILON (DBL_EPSILON)
constexpr float kSqrt2 = 1.41421356237309505f;
constexpr int kSponge = 4;

// scenario status (ScenarioCtl::status)
enum : int {
    kRunning = 0,
    kPaused = 1,   // an event (fault, snapshot, gauge sample) is due at time t
    kDone = 2,     // t >= t_end or the step budget is used
    kFailed = 3,   // non-finite state or time step
    kIdle = 4,     // slot not in use / not started
};

// pause reasons (bit mask, ScenarioCtl::events)
enum : int { kEvFault = 1, kEvSnapshot = 2, kEvSeries = 4, kEvStepBudget = 8 };

struct RowMetrics {
    // per row y (ny entries unless noted), FP64 on the host, rounded once
    const float *cosphi;     // cos(lat)
    const float *ilcos;      // x-edge length / cos(lat)  (dlat / cos)
    const float *area;       // cell area
    const float *dlon;       // y-edge length at edge row y (ny+1 entries); sponge dx
    const float *dlat;       // sponge dy
};

// Mutable per-scenario control block; written by the host between graph
// launches and by the controller launch that ends each step.
struct ScenarioCtl {
    double t;            // simulated time (dimensionless)
    double dt;           // time step of the next step
    double t_end;
    double save_nc, next_nc;   // snapshot interval / next snapshot time (< 0: off)
    double save_ts, next_ts;   // gauge interval / next gauge time
    double T;                  // time scale (s)
    long long step;            // completed steps
    long long max_steps;       // < 0: unlimited
    int status;
    int events;
    int parity;
    int fault_next;            // index of the next fault to apply
    int jumping;               // the reference's saltar_deformacion
    int nfaults;
    unsigned int dt_bits;      // atomicMin target (positive float bits)
    unsigned int tiles_done;   // phase-0 tiles finished (initial dt)
    unsigned int errors;       // bit 0 non-finite values, bit 1 a staging copy did not land, bit 2 misaligned staging
    int inject;                // test hook: bit 0 = the deep kernels issue none of this scenario's copies
    const double *fault_times; // nfaults fault times (s), sorted, device memory
    unsigned long long units_deep;   // work units stepped by the deep-water kernels (phase 2)
    unsigned long long units_dry;    // work units skipped as dry land (classifications)
    unsigned int gauge_count;  // gauge samples the controller took (ring slot = count % kGaugeRing)
};

// Gauge samples taken on the device between two reads by the host: at most
// one per step, and the host reads them after every chunk of at most
// kGaugeRing steps.
constexpr int kGaugeRing = 32;

// Opaque 128-byte TMA tensor map (CUtensorMap), 64-byte aligned in device memory.
struct alignas(64) TmaMap {
    unsigned long long opaque[16];
};

// tensor maps of a scenario: state planes boxed kStageW x kStageRows (the
// staged window of a half tile), diagnostics boxed kTileX x kHalfRows
enum : int {
    kMapEta0 = 0, kMapEta1, kMapQx0, kMapQx1, kMapQy0, kMapQy1, kMapDep, kMapEtaMax, kMapArr, kMapEtaIni, kNumMaps
};
constexpr int kHalfRows = 16;                 // rows of a half tile
constexpr int kStageW = 120;                  // staged columns: x0-4 .. x0+115 (16-byte aligned start)
constexpr int kStageRows = kHalfRows + 2;     // staged rows: one above and one below the half tile

// Depth summary of a work unit for one state: {min, max} of eta + dep over
// the unit, over its two-cell border strips (left, right, top, bottom: the
// unit's first / last two columns or rows inside the grid) and over its four
// 2 x 2 corners - exactly the cells the two-cell stencil ring of a
// neighbouring unit reaches into.
struct UnitSum {
    float2 all, L, R, T, B, TL, TR, BL, BR;
};

struct ScenarioDev {
    int nx, ny, pitch;
    int tiles_x, tiles_y, ntiles;
    int x_org;   // grid column of tile 0's first column (tile_origin: 0 or -4 .. -108)
    int periodic;
    float b_up, b_low, b_left, b_right;
    int sp_up, sp_low, sp_left, sp_right;
    float cfl, eps_h, hpos, cvis, mf0, vmax, dif_at, sea;
    double eps_h64;   // eps_h in double for the FP64 set-up / output thresholds
    float *eta[2];
    float *qx[2];
    float *qy[2];
    float *dep;
    float *eta_max;
    float *arr;
    float *eta_ini;
    // per work unit (half tile of kTileX x kHalfRows cells from column
    // x_org + tx kTileX; unit (tx, uy) at uy * tiles_x + tx): depth summary of the state phase 1 produces (index
    // parity^1); NaN = unknown
    UnitSum *usum[2];
    // per unit: consecutive classifications that found its 3 x 3 unit
    // neighbourhood dry (saturating)
    unsigned char *dry_age;
    // per unit: the largest |dep1 - dep0| between the two cells of an edge of
    // the unit's cells (x edges x0 .. x0+112 of its rows, y edges yb .. yb+16
    // of its columns, inside the grid); fixed between faults.  A deep unit
    // whose unit and two-cell ring are all deeper than this steps its
    // surface jumps as the plain difference (see surface_jump)
    float *unit_gmax;
    // TMA tensor maps of the field planes (kMap* order), null when the grid
    // is too small to have deep tiles
    const struct TmaMap *tmap;
    // per row y (ny+1 entries): {cos, ilcos, area, dlon} (dlon of edge row y;
    // the other three unused in entry ny)
    const float4 *rowpack;
    RowMetrics row;
    ScenarioCtl *ctl;
    // gauges (time-series points), sampled by the step controller at each
    // gauge time that does not coincide with a fault
    const int *gauge_cells;   // ngauges cell indices (y nx + x; -1: outside the grid)
    int ngauges;
    float *gauge_ring;        // kGaugeRing samples of ngauges x {eta, ux, uy, depth} (m, m/s)
    double *gauge_ring_t;     // their times (s)
    float2 *gauge_minmax;     // per gauge {min, max} of eta over every sample (-9999 outside the grid)
    double Hs, Qs;            // depth and discharge scales (dimensional outputs)
};

// One gauge of the state at `parity` in dimensional units (eta, ux, uy,
// depth: src/GPU/Volumen_kernel.cu:223-254 with the output scaling of
// src/GPU/netcdfSeries.cu), -9999 for a point outside the grid; folds eta into
// the gauge's {min, max} when minmax is not null (the running extremes of
// src/GPU/netcdfSeries.cu:125,138).
__device__ __forceinline__ void gauge_values(const ScenarioDev &s, int parity, int cell, float *out4, float2 *minmax)
{
    if (cell < 0) {
        out4[0] = out4[1] = out4[2] = out4[3] = -9999.0f;
        return;
    }
    const int x = cell % s.nx, y = cell / s.nx;
    const size_t idx = (size_t)y * s.pitch + x;
    const double eta = (double)s.eta[parity][idx], D = (double)s.dep[idx];
    const double h = eta + D, eps_h = s.eps_h64;
    double f;
    if (h < eps_h) {
        const double e4 = eps_h * eps_h * eps_h * eps_h;
        f = 1.41421356237309505 * h / sqrt(h * h * h * h + e4);
    } else {
        f = 1.0 / h;
    }
    const float e = (float)(eta * s.Hs);
    out4[0] = e;
    out4[1] = (float)(f * (double)s.qx[parity][idx] * s.Qs / s.Hs);
    out4[2] = (float)(f * (double)s.qy[parity][idx] * s.Qs / s.Hs);
    out4[3] = (float)(D * s.Hs);
    if (minmax) {
        float2 m = *minmax;
        m.x = (m.x < e) ? m.x : e;
        m.y = (e < m.y) ? m.y : e;
        *minmax = m;
    }
}

__host__ __device__ inline float fmax_(float a, float b) { return (a < b) ? b : a; }
__host__ __device__ inline float fmin_(float a, float b) { return (b < a) ? b : a; }

__device__ __forceinline__ float sgnf(float a) { return (a > 0.f) ? 1.f : ((a < 0.f) ? -1.f : 0.f); }
__device__ __forceinline__ float pow4f(float a) { float b = a * a; return b * b; }

// Approximate reciprocal square root and square root of the stepping
// kernels.  The square root is x * rsqrt(x), an approximate reciprocal square
// root and one multiply, written out so that every call site computes it
// with the same two instructions: an approximate sqrtf is not lowered alike
// at every site, and then two warp tilings of the same cells, which reach the
// same formula through different code, differ in the last bit.
// sqrt_ap(0) = 0; a negative or NaN argument gives NaN.
__device__ __forceinline__ float rsqrt_ap(float x)
{
    float r;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ float sqrt_ap(float x)
{
    return x == 0.f ? 0.f : __fmul_rn(x, rsqrt_ap(x));
}

// Desingularised 1/h (src/GPU/Arista_kernel.cu:164): sqrt2 h / sqrt(h^4 + max(h,eps)^4),
// which is exactly 1/h for h >= eps.
__device__ __forceinline__ float inv_depth(float h, float eps)
{
    if (h >= eps) return __frcp_rn(h);
    return kSqrt2 * h * rsqrt_ap(pow4f(h) + pow4f(eps));
}

// Monotone limiter of the WAF correction (src/GPU/Arista_kernel.cu:45-68).
__device__ __forceinline__ float monotone_limiter(float pm, float p0, float p1, float pp, float wave)
{
    float d_mid = p1 - p0;
    float d_up = (wave < 0.f) ? (pp - p1) : ((wave > 0.f) ? (p0 - pm) : 0.5f * (pp - pm));
    float same = (d_mid * d_up >= 0.f) ? 1.f : 0.f;
    d_mid = fabsf(d_mid);
    d_up = fabsf(d_up);
    if (d_mid < kEps) return 1.f;
    float a = fabsf(__fdividef(d_up - d_mid, d_up + d_mid));
    d_up = 0.5f * (d_up + d_mid) * (1.f - a * a * a);
    float r = (d_mid > d_up) ? __fdividef(d_up, d_mid + kEps) : __fdividef(d_mid, d_up + kEps);
    return same * r * __fdividef(1.f + r, 1.f + r * r);
}

// Limits a mass flux so that neither side loses more than 1/4 of its water in
// one step (src/GPU/Arista_kernel.cu:79-114; c0/c1 = cos(lat) for y edges).
// dt > dt0 = cap / (|F| + eps) is tested as dt (|F| + eps) > cap, so the
// divisions only run when the limit applies.
__device__ __forceinline__ float limit_outflow(float F, float h0, float h1, float c0, float c1, float dt, float a0, float a1)
{
    const float cap = (F > 0.f) ? 0.25f * h0 * c0 * a0 : 0.25f * h1 * c1 * a1;
    const float aF = fabsf(F) + kEps;
    if (dt * aF > cap) F *= (cap / aF) / (dt + kEps);
    return F;
}

// Blend weight of the 2s flux against the WAF flux (src/GPU/Arista_kernel.cu:208).
__device__ __forceinline__ float blend_2s(float hij, float hpos, bool no_lim)
{
    if (no_lim) return 0.f;
    if (hij < hpos) return __frcp_rn(1.f + __expf(-15.f * (1.f - 0.5f * hpos / (hij + kEps))));
    return 1.f;
}

// Surface-gradient term max(eta1+Hm,0) - max(eta0+Hm,0) with Hm = min(D0,D1),
// evaluated as eta1 - eta0 whenever both sides are wet at the lower bed so that
// FP32 does not lose the wave to the depth's magnitude.  With h0, h1 > |D1 - D0|
// both sides are (eta1 + Hm >= h1 - |D1 - D0| and eta0 + Hm >= h0 - |D1 - D0|),
// and the term is eta1 - eta0 without the tests.
__device__ __forceinline__ float surface_jump(float e0, float e1, float D0, float D1)
{
    float Hm = fmin_(D0, D1);
    float a = e1 + Hm, b = e0 + Hm;
    if (a > 0.f && b > 0.f) return e1 - e0;
    return fmax_(a, 0.f) - fmax_(b, 0.f);
}

// One edge: four stencil cells along the edge normal.  "u" is the momentum
// component normal to the edge, "v" the tangential one.
struct Edge {
    float h0m, h0, h1, h1p;
    float e0m, e0, e1, e1p;
    float D0, D1;
    float u0m, u0, u1, u1p;
    float v0m, v0, v1, v1p;
    float area0, area1, cos0, cos1;
    float len;      // x edges: len/cos (ilcos); y edges: len
    float normal;
    bool front;     // ghost on the low side: sides swapped, flux computed mirrored
    bool no_lim;    // within two cells of a boundary: first order, no 2s blend
};

__device__ __forceinline__ void swapf(float &a, float &b) { float t = a; a = b; b = t; }

__device__ __forceinline__ void swap_sides(Edge &e)
{
    swapf(e.h0m, e.h1p); swapf(e.h0, e.h1);
    swapf(e.e0m, e.e1p); swapf(e.e0, e.e1);
    swapf(e.D0, e.D1);
    swapf(e.u0m, e.u1p); swapf(e.u0, e.u1);
    swapf(e.v0m, e.v1p); swapf(e.v0, e.v1);
    swapf(e.area0, e.area1); swapf(e.cos0, e.cos1);
}

__device__ __forceinline__ bool all_deep(const Edge &e, float hpos)
{
    return (e.h0 > hpos) && (e.h1 > hpos) && (e.h0m > hpos) && (e.h1p > hpos) && !e.no_lim;
}

// ---------------------------------------------------------------------------
// Edges whose four stencil cells are all deeper than hpos and which lie at
// least two cells from a boundary: the 2s blend weight is exactly 1, so the
// flux is the 2s flux alone (the WAF part, the wet/dry tests and the limiter
// drop out).  The general functions below and deep phase 1 call these; deep
// phase 2 evaluates the same formulas two edges at a time in packed FP32x2
// arithmetic (step.cu), which can round its last bit differently.
// ---------------------------------------------------------------------------

// x edge: F = q0 len, outflow-limited (src/GPU/Arista_kernel.cu:118-219, alfa = 1)
__device__ __forceinline__ float mass_2s_x(float q0, float len, float h0, float h1, float dt, float a0, float a1)
{
    return limit_outflow(q0 * len, h0, h1, 1.f, 1.f, dt, a0, a1);
}

// y edge: F = len q0 cos0 (src/GPU/Arista_kernel.cu:674-778, alfa = 1)
__device__ __forceinline__ float mass_2s_y(float q0, float len, float cos0, float cos1, float h0, float h1, float dt,
                                           float a0, float a1)
{
    return limit_outflow(len * q0 * cos0, h0, h1, cos0, cos1, dt, a0, a1);
}

// Result of a momentum flux: contributions to the two cells (already with
// the "acc -= F" sign applied) and the wave-speed term for the time step.
struct MomFlux {
    float m_x, m_y;   // to cell0: subtract
    float p_x, p_y;   // to cell1: subtract
    float lam;        // edge length * max wave speed (added to both)
    bool active;
};

// Per-cell factors of the 2s fluxes, computed once per cell and shared by
// its four edges: 1/h (approximate reciprocal) and sqrt(h).
__device__ __forceinline__ float rcp_depth(float h) { return __fdividef(1.f, h); }

// Constants of the 2s momentum flux that depend only on the edge's row (its
// metrics), the step's dt and the scenario's viscosity: the deep-water kernels
// form them once per row of a unit, the general kernel per edge, with the same
// expressions.
struct XRowK {
    float ilcos;   // len / cos of the row
    float kdes;    // cd * val * ilcos, val = 2 ilcos dt / (area0 + area1), cd = (1 - cvis) / 2
};
__device__ __forceinline__ XRowK make_xrow(float ilcos, float asum, float dt, float cvis)
{
    XRowK k;
    const float val = (2.f * ilcos * dt) / asum;
    k.ilcos = ilcos;
    k.kdes = (0.5f * (1.f - cvis)) * val * ilcos;
    return k;
}
struct YRowK {
    float len, cmid, cdiff, c10;   // len; (cos0 + cos1) / 2; cos1 - cos0; cos1 / cos0
    float c01, li0, kdes0, kdes1;  // cos0 / cos1; len / cos0; cd val len / cos0; cd val len / cos1
    float cos0, cos1;
};
__device__ __forceinline__ YRowK make_yrow(float cos0, float cos1, float icos0, float icos1, float len, float asum,
                                           float dt, float cvis)
{
    YRowK k;
    const float val = (2.f * len * dt) / asum;
    const float kd = (0.5f * (1.f - cvis)) * val * len;
    k.len = len;
    k.cmid = 0.5f * (cos0 + cos1);
    k.cdiff = cos1 - cos0;
    k.c10 = cos1 * icos0;
    k.c01 = cos0 * icos1;
    k.li0 = len * icos0;
    k.kdes0 = kd * icos0;
    k.kdes1 = kd * icos1;
    k.cos0 = cos0;
    k.cos1 = cos1;
    return k;
}

// x edge, components (qx, qy); u = qx normal, v = qy tangential, rh = 1/h,
// sh = sqrt(h) of each side, jump = the surface jump, k = the row's constants
// (src/GPU/Arista_kernel.cu:221-464, alfa = 1)
__device__ __forceinline__ void momentum_2s_x(MomFlux &r, float h0, float h1, float rh0, float rh1, float s0, float s1,
                                              float u0, float u1, float v0, float v1, float jump, const XRowK &k)
{
    const float ilcos = k.ilcos;
    const float hij = 0.5f * (h0 + h1);
    const float u0n = u0 * rh0, u1n = u1 * rh1;
    const float uijn = __fdividef(s0 * u0n + s1 * u1n, s0 + s1 + kEps);
    const float maxa = fabsf(uijn) + sqrt_ap(hij);
    float mx, my, px, py;
    if (uijn < 0.f) {
        mx = u1n * u1 * ilcos; px = -mx; mx += hij * jump * ilcos;
        my = u1n * v1 * ilcos; py = -my;
    } else {
        mx = u0n * u0 * ilcos; px = -mx; mx += hij * jump * ilcos;
        my = u0n * v0 * ilcos; py = -my;
    }
    const float des = k.kdes * (maxa * maxa) * (u1 - u0);
    r.m_x = mx - des; r.m_y = my;
    r.p_x = px + des; r.p_y = py;
    r.lam = ilcos * maxa;
    r.active = true;
}

// y edge, components (qx, qy); u = qy normal, v = qx tangential; k = the
// constants of the edge's row pair (src/GPU/Arista_kernel.cu:780-1026, alfa = 1)
__device__ __forceinline__ void momentum_2s_y(MomFlux &r, float h0, float h1, float rh0, float rh1, float s0, float s1,
                                              float u0, float u1, float v0, float v1, float jump, const YRowK &k)
{
    const float hij = 0.5f * (h0 + h1);
    const float u0n = u0 * rh0, u1n = u1 * rh1;
    const float uijn = __fdividef(s0 * u0n + s1 * u1n, s0 + s1 + kEps);
    const float maxa = fabsf(uijn) + sqrt_ap(hij);
    const float deta = k.cmid * jump - uijn * uijn * k.cdiff;
    float fym, fyp, fxm, fxp;
    if (uijn < 0.f) {
        fym = u1n * u1 * k.len; fyp = -fym; fym *= k.c10; fym += hij * deta * k.li0;
        fxm = u1n * v1 * k.len; fxp = -fxm;
    } else {
        fym = u0n * u0 * k.len; fyp = -fym * k.c01; fym += hij * deta * k.li0;
        fxm = u0n * v0 * k.len; fxp = -fxm;
    }
    const float m2 = (maxa * maxa) * (u1 * k.cos1 - u0 * k.cos0);
    r.m_x = fxm; r.m_y = fym - k.kdes0 * m2;
    r.p_x = fxp; r.p_y = fyp + k.kdes1 * m2;
    r.lam = k.len * maxa;
    r.active = true;
}

// ---------------------------------------------------------------------------
// phase 1: mass flux through one edge (src/GPU/Arista_kernel.cu:118-219 for
// x edges, 674-778 for y edges).  Returns F; the caller applies it as
// cell0 -= F (/cos0 for y), cell1 += F (/cos1).
// ---------------------------------------------------------------------------
template <bool LAT>
__device__ __forceinline__ float mass_flux(Edge &e, const ScenarioDev &s, float dt)
{
    if (all_deep(e, s.hpos)) {
        if (!LAT) return mass_2s_x(e.u0, e.len, e.h0, e.h1, dt, e.area0, e.area1);
        return mass_2s_y(e.u0, e.len, e.cos0, e.cos1, e.h0, e.h1, dt, e.area0, e.area1);
    }
    if (e.front) swap_sides(e);
    const float h0 = e.h0, h1 = e.h1;
    if (!((h0 > kEps) || (h1 > kEps))) return 0.f;
    float q0n = e.u0 * e.normal, q1n = e.u1 * e.normal;
    const float hij = 0.5f * (h0 + h1);
    const float c0 = sqrt_ap(hij);
    if ((h0 < s.eps_h) && (-e.e1 > e.D0)) q1n = 0.f;
    if ((h1 < s.eps_h) && (-e.e0 > e.D1)) q0n = 0.f;
    const float u0n = inv_depth(h0, s.eps_h) * q0n;
    const float u1n = inv_depth(h1, s.eps_h) * q1n;
    q0n = u0n * h0;
    q1n = u1n * h1;
    const float F2s = LAT ? e.len * q0n * e.cos0 * e.normal : e.len * q0n * e.normal;
    const float s0 = sqrt_ap(h0), s1 = sqrt_ap(h1);
    const float uijn = (s0 * u0n + s1 * u1n) / (s0 + s1 + kEps);
    const float val = (2.f * e.len * dt) / (e.area0 + e.area1);
    const float aut1 = fmin_(uijn - c0, u0n - s0);
    const float aut2 = fmax_(uijn + c0, u1n + s1);
    const float maxa = fmax_(fabsf(aut2), fabsf(aut1));
    float xiL = 0.f, xiR = 0.f;
    if (!e.no_lim) {
        xiL = monotone_limiter(e.e0m, e.e0, e.e1, e.e1p, aut1);
        xiR = monotone_limiter(e.e0m, e.e0, e.e1, e.e1p, aut2);
    }
    float a0;
    if (fabsf(aut1 - aut2) >= kEps) {
        const float alr = sgnf(aut1) * (1.f - xiL) + val * aut1 * xiL;
        const float blr = sgnf(aut2) * (1.f - xiR) + val * aut2 * xiR;
        a0 = (alr - blr) * (aut1 * aut2) / (aut2 - aut1);
    } else {
        a0 = maxa;
    }
    const float jump = surface_jump(e.e0, e.e1, e.D0, e.D1);
    float Fwaf;
    if (!LAT) {
        Fwaf = 0.5f * (q1n + q0n - a0 * jump) * e.len;
    } else {
        const float deta = 0.5f * (e.cos0 + e.cos1) * jump - uijn * uijn * (e.cos1 - e.cos0);
        Fwaf = 0.5f * (q0n * e.cos0 + q1n * e.cos1 - a0 * deta) * e.len;
    }
    const float alfa = blend_2s(hij, s.hpos, e.no_lim);
    const float F = alfa * F2s + (1.f - alfa) * Fwaf;
    if (!LAT) return limit_outflow(F, h0, h1, 1.f, 1.f, dt, e.area0, e.area1);
    return limit_outflow(F, h0, h1, e.cos0, e.cos1, dt, e.area0, e.area1);
}

// ---------------------------------------------------------------------------
// phase 2: momentum flux of an x edge (src/GPU/Arista_kernel.cu:221-464).
// Components are (qx, qy).
// ---------------------------------------------------------------------------
__device__ __forceinline__ MomFlux momentum_flux_x(Edge &e, const ScenarioDev &s, float dt)
{
    MomFlux r;
    r.active = true;
    const float ilcos = e.len;
    if (all_deep(e, s.hpos)) {
        momentum_2s_x(r, e.h0, e.h1, rcp_depth(e.h0), rcp_depth(e.h1), sqrt_ap(e.h0), sqrt_ap(e.h1), e.u0, e.u1, e.v0,
                      e.v1, surface_jump(e.e0, e.e1, e.D0, e.D1), make_xrow(ilcos, e.area0 + e.area1, dt, s.cvis));
        return r;
    }
    if (e.front) swap_sides(e);
    const float h0 = e.h0, h1 = e.h1;
    if (!((h0 > kEps) || (h1 > kEps))) { r.active = false; return r; }
    float w0 = e.u0 * e.normal, w1 = e.u1 * e.normal;
    const float hij = 0.5f * (h0 + h1);
    if ((h0 < s.eps_h) && (-e.e1 > e.D0)) w1 = 0.f;
    if ((h1 < s.eps_h) && (-e.e0 > e.D1)) w0 = 0.f;
    const float h0rg = inv_depth(h0, s.eps_h), h1rg = inv_depth(h1, s.eps_h);
    float u0n = h0rg * w0, u1n = h1rg * w1;
    w0 = u0n * h0;
    w1 = u1n * h1;
    const float s0 = sqrt_ap(h0), s1 = sqrt_ap(h1);
    float uijn = (s0 * u0n + s1 * u1n) / (s0 + s1 + kEps);
    const float val = (2.f * ilcos * dt) / (e.area0 + e.area1);
    const float c0 = sqrt_ap(hij);
    const float aut1 = fmin_(uijn - c0, u0n - s0);
    const float aut2 = fmax_(uijn + c0, u1n + s1);
    float maxa = fmax_(fabsf(aut2), fabsf(aut1));
    const float fl1x = w1, fl1y = u1n * w1, fl0x = w0, fl0y = u0n * w0;
    const float dq = fl1x - fl0x;
    const float deta = surface_jump(e.e0, e.e1, e.D0, e.D1);
    float s_my, s_py, s_mz, s_pz;
    if (uijn < 0.f) {
        s_my = u1n * w1 * ilcos * e.normal; s_py = -s_my; s_my += hij * deta * ilcos;
        s_mz = u1n * e.v1 * ilcos; s_pz = -s_mz;
    } else {
        s_my = u0n * w0 * ilcos * e.normal; s_py = -s_my; s_my += hij * deta * ilcos;
        s_mz = u0n * e.v0 * ilcos; s_pz = -s_mz;
    }
    const float cd = 0.5f * (1.f - s.cvis / (1.f + __expf(-20.f * (1.f - s.hpos / hij))));
    const float des = cd * val * maxa * maxa * dq * ilcos * e.normal;
    s_my -= des;
    s_py += des;
    float xiL = 0.f, xiR = 0.f;
    if (!e.no_lim) {
        xiL = monotone_limiter(e.e0m, e.e0, e.e1, e.e1p, aut1);
        xiR = monotone_limiter(e.e0m, e.e0, e.e1, e.e1p, aut2);
    }
    float a0, a1;
    if (fabsf(aut1 - aut2) >= kEps) {
        const float alr = sgnf(aut1) * (1.f - xiL) + val * aut1 * xiL;
        const float blr = sgnf(aut2) * (1.f - xiR) + val * aut2 * xiR;
        const float aux = 1.f / (aut2 - aut1);
        a0 = (alr - blr) * (aut1 * aut2) * aux;
        a1 = (blr * aut2 - alr * aut1) * aux;
    } else {
        a0 = maxa;
        a1 = 0.f;
    }
    float mx = 0.5f * dq, px = mx;
    float my = 0.5f * (fl1y - fl0y + hij * deta), py = my;
    const float desx = 0.5f * a0 * deta, desy = 0.5f * a0 * dq + a1 * my;
    mx += fl0x - desx; my += fl0y - desy;
    px += desx - fl1x; py += desy - fl1y;
    mx *= ilcos; my *= ilcos; px *= ilcos; py *= ilcos;
    // transverse momentum carried with a limited tangential velocity
    const float q0mt = e.v0m * e.normal, q0t = e.v0 * e.normal, q1t = e.v1 * e.normal, q1pt = e.v1p * e.normal;
    const float p0m = inv_depth(e.h0m, s.eps_h) * q0mt;
    const float p1p = inv_depth(e.h1p, s.eps_h) * q1pt;
    u0n = h0rg * q0t;
    u1n = h1rg * q1t;
    const float sg = -1.f * (mx < 0.f) + 1.f * (mx > 0.f);
    uijn = fabsf(uijn) * sg;
    const float xit = e.no_lim ? 0.f : monotone_limiter(p0m, u0n, u1n, p1p, uijn);
    const float uijt = 0.5f * (u0n + u1n) - 0.5f * ((1.f - xit) * sg + xit * uijn * val) * (u1n - u0n);
    const float aux = mx * uijt;
    const float t_py = py * e.normal, t_pz = -aux * e.normal, t_my = my * e.normal, t_mz = aux * e.normal;
    const float alfa = blend_2s(hij, s.hpos, e.no_lim);
    r.m_x = alfa * s_my + (1.f - alfa) * t_my;
    r.m_y = alfa * s_mz + (1.f - alfa) * t_mz;
    r.p_x = alfa * s_py + (1.f - alfa) * t_py;
    r.p_y = alfa * s_pz + (1.f - alfa) * t_pz;
    if (maxa < s.eps_h) maxa += s.eps_h;
    r.lam = ilcos * maxa;
    return r;
}

// ---------------------------------------------------------------------------
// phase 2: momentum flux of a y edge (src/GPU/Arista_kernel.cu:780-1026).
// Edge "u" is qy, "v" is qx; components returned as (qx, qy).
// ---------------------------------------------------------------------------
__device__ __forceinline__ MomFlux momentum_flux_y(Edge &e, const ScenarioDev &s, float dt)
{
    MomFlux r;
    r.active = true;
    const float len = e.len;
    if (all_deep(e, s.hpos)) {
        momentum_2s_y(r, e.h0, e.h1, rcp_depth(e.h0), rcp_depth(e.h1), sqrt_ap(e.h0), sqrt_ap(e.h1), e.u0, e.u1, e.v0,
                      e.v1, surface_jump(e.e0, e.e1, e.D0, e.D1),
                      make_yrow(e.cos0, e.cos1, __frcp_rn(e.cos0), __frcp_rn(e.cos1), len, e.area0 + e.area1, dt,
                                s.cvis));
        return r;
    }
    if (e.front) swap_sides(e);
    const float h0 = e.h0, h1 = e.h1;
    if (!((h0 > kEps) || (h1 > kEps))) { r.active = false; return r; }
    const float icos0 = __frcp_rn(e.cos0), icos1 = __frcp_rn(e.cos1);
    float w0 = e.u0 * e.normal, w1 = e.u1 * e.normal;
    const float hij = 0.5f * (h0 + h1);
    const float c0 = sqrt_ap(hij);
    if ((h0 < s.eps_h) && (-e.e1 > e.D0)) w1 = 0.f;
    if ((h1 < s.eps_h) && (-e.e0 > e.D1)) w0 = 0.f;
    const float h0rg = inv_depth(h0, s.eps_h), h1rg = inv_depth(h1, s.eps_h);
    float u0n = h0rg * w0, u1n = h1rg * w1;
    const float s0 = sqrt_ap(h0), s1 = sqrt_ap(h1);
    float uijn = (s0 * u0n + s1 * u1n) / (s0 + s1 + kEps);
    const float val = (2.f * len * dt) / (e.area0 + e.area1);
    const float aut1 = fmin_(uijn - c0, u0n - s0);
    const float aut2 = fmax_(uijn + c0, u1n + s1);
    float maxa = fmax_(fabsf(aut2), fabsf(aut1));
    const float deta = 0.5f * (e.cos0 + e.cos1) * surface_jump(e.e0, e.e1, e.D0, e.D1) - uijn * uijn * (e.cos1 - e.cos0);
    float s_mz, s_pz, s_my, s_py;
    if (uijn < 0.f) {
        s_mz = u1n * w1 * len * e.normal; s_pz = -s_mz; s_mz *= e.cos1 * icos0; s_mz += hij * deta * len * icos0;
        s_my = u1n * e.v1 * len; s_py = -s_my;
    } else {
        s_mz = u0n * w0 * len * e.normal; s_pz = -s_mz * e.cos0 * icos1; s_mz += hij * deta * len * icos0;
        s_my = u0n * e.v0 * len; s_py = -s_my;
    }
    const float cd = 0.5f * (1.f - s.cvis / (1.f + __expf(-20.f * (1.f - s.hpos / hij))));
    const float fl1x = w1 * e.cos1, fl1y = u1n * fl1x, fl0x = w0 * e.cos0, fl0y = u0n * fl0x;
    const float dq = fl1x - fl0x;
    const float des = cd * val * maxa * maxa * dq * len;
    s_mz -= des * icos0;
    s_pz += des * icos1;
    float xiL = 0.f, xiR = 0.f;
    if (!e.no_lim) {
        xiL = monotone_limiter(e.e0m, e.e0, e.e1, e.e1p, aut1);
        xiR = monotone_limiter(e.e0m, e.e0, e.e1, e.e1p, aut2);
    }
    float a0, a1;
    if (fabsf(aut1 - aut2) >= kEps) {
        const float alr = sgnf(aut1) * (1.f - xiL) + val * aut1 * xiL;
        const float blr = sgnf(aut2) * (1.f - xiR) + val * aut2 * xiR;
        const float aux = 1.f / (aut2 - aut1);
        a0 = (alr - blr) * (aut1 * aut2) * aux;
        a1 = (blr * aut2 - alr * aut1) * aux;
    } else {
        a0 = maxa;
        a1 = 0.f;
    }
    float mx = 0.5f * dq, px = mx;
    float my = 0.5f * (fl1y - fl0y + hij * deta), py = my;
    const float desx = 0.5f * a0 * deta, desy = 0.5f * a0 * dq + a1 * my;
    mx += fl0x - desx; my += fl0y - desy;
    px += desx - fl1x; py += desy - fl1y;
    mx *= len; my *= len; px *= len; py *= len;
    const float q0mt = -e.v0m * e.normal, q0t = -e.v0 * e.normal, q1t = -e.v1 * e.normal, q1pt = -e.v1p * e.normal;
    const float p0m = inv_depth(e.h0m, s.eps_h) * q0mt;
    const float p1p = inv_depth(e.h1p, s.eps_h) * q1pt;
    u0n = h0rg * q0t;
    u1n = h1rg * q1t;
    const float sg = -1.f * (mx < 0.f) + 1.f * (mx > 0.f);
    uijn = fabsf(uijn) * sg;
    const float xit = e.no_lim ? 0.f : monotone_limiter(p0m, u0n, u1n, p1p, uijn);
    const float uijt = 0.5f * (u0n * icos0 + u1n * icos1) -
                       0.5f * ((1.f - xit) * sg + xit * uijn * val) * (u1n * icos1 - u0n * icos0);
    const float aux = mx * uijt;
    const float t_py = aux * e.normal, t_pz = py * e.normal * icos1;
    const float t_my = -aux * e.normal, t_mz = my * e.normal * icos0;
    if (maxa < s.eps_h) maxa += s.eps_h;
    const float alfa = blend_2s(hij, s.hpos, e.no_lim);
    r.m_x = alfa * s_my + (1.f - alfa) * t_my;
    r.m_y = alfa * s_mz + (1.f - alfa) * t_mz;
    r.p_x = alfa * s_py + (1.f - alfa) * t_py;
    r.p_y = alfa * s_pz + (1.f - alfa) * t_pz;
    r.lam = len * maxa;
    return r;
}

}  // namespace thy
