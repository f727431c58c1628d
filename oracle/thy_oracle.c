/*
 * thy_oracle.c — FP64 CPU restatement of the Tsunami-HySEA explicit
 * finite-volume time stepper (2s / 2s+WAF path-conservative fluxes with
 * wet/dry treatment, sponge layers, Manning friction, CFL time step) and
 * of its Okada seafloor-deformation initialisation.
 *
 * TEST INFRASTRUCTURE ONLY: the oracle the CUDA path is checked against and
 * the CPU baseline bench.py times.  The product never links or calls it.
 *
 * Each function names the reference code it restates (paths relative to the
 * reference project).  Expressions keep the reference's evaluation order so
 * that, compiled with -ffp-contract=off against the same libm, results agree
 * with the reference's own kernels compiled for the host (oracle/_ref) to the
 * last few ulps; the Okada displacement uses Okada's (1985) closed-form
 * surface solution, which the reference's DC3D (Okada 1992) equals at z = 0.
 */
#define _GNU_SOURCE
#include "thy_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define EPS DBL_EPSILON
#define SQRT2 1.41421356237309504880
#define EARTH_RADIUS_M 6378136.6
#define SPONGE_CELLS 4
#define SEA_LEVEL_M 0.0

static inline double dmax(double a, double b) { return (a < b) ? b : a; }
static inline double dmin(double a, double b) { return (b < a) ? b : a; }
static inline double sgn(double a) { return (a > 0.0) ? 1.0 : ((a < 0.0) ? -1.0 : 0.0); }
static inline double pow4(double a) { return a * a * a * a; }

/* ---------------------------------------------------------------------- */
/* grid state                                                              */
/* ---------------------------------------------------------------------- */

typedef struct {
    int nx, ny;
    long long n;
    int periodic;
    double b_up, b_low, b_left, b_right;      /* border flags */
    int sp_up, sp_low, sp_left, sp_right;     /* sponge widths */
    double cfl, eps_h, hpos, cvis, mf0, vmax, dif_at, Hmin, sea;
    double Ls, Hs, Qs, Ts;                    /* scales */
    double *h, *dep, *qx, *qy;                /* state: water depth, shifted depth, momenta */
    double *area, *cosphi, *dlat, *dlon;      /* metric: per row (dlon has ny+1) */
    double *acc_m, *acc_l, *acc_qx, *acc_qy;  /* accumulators: mass, lambda*len, momenta */
    double *dtc;                              /* per-cell dt */
    double *eta_max, *t_arr, *eta_ini;
    int row_lo, row_hi;                       /* rows this process updates: [row_lo, row_hi) (all of them in
                                                 a single-process run; a row slab in a decomposed run, whose
                                                 two rows above and below are halos kept current by the caller) */
} grid_t;

/* src/GPU/Arista_kernel.cu:6-21 — x index with periodic wrap or clamp */
static inline int col_index(int c, int periodic, int nx)
{
    if (c >= 0 && c < nx) return c;
    if (c < 0) return periodic ? nx + c : 0;
    return periodic ? c - nx : nx - 1;
}

/* src/GPU/Arista_kernel.cu:45-68 — monotone limiter of the WAF correction */
static double monotone_limiter(double pm, double p0, double p1, double pp, double wave)
{
    double d_mid = p1 - p0;
    double d_up = (wave < 0.0) ? (pp - p1) : ((wave > 0.0) ? (p0 - pm) : 0.5 * (pp - pm));
    double same_sign = (d_mid * d_up >= 0.0) ? 1.0 : 0.0;
    double a, r;
    d_mid = fabs(d_mid);
    d_up = fabs(d_up);
    if (d_mid < EPS) return 1.0;
    a = fabs((d_up - d_mid) / (d_up + d_mid));
    d_up = 0.5 * (d_up + d_mid) * (1.0 - a * a * a);
    r = (d_mid > d_up) ? (d_up / (d_mid + EPS)) : (d_mid / (d_up + EPS));
    return same_sign * r * (1.0 + r) / (1.0 + r * r);
}

/* src/GPU/Arista_kernel.cu:70-77 — no momentum into a dry cell lying above the wet neighbour's surface */
static inline void dry_wet(double h0, double h1, double e0, double e1, double H0, double H1, double eps,
                           double *q0n, double *q1n)
{
    if ((h0 < eps) && (-e1 > H0)) *q1n = 0.0;
    if ((h1 < eps) && (-e0 > H1)) *q0n = 0.0;
}

/* src/GPU/Arista_kernel.cu:79-114 — limit a mass flux so neither cell loses more than 1/4 of its water */
static inline void limit_outflow(double h0, double h1, double c0, double c1, double dt, double a0, double a1, double *F)
{
    double dt0;
    if (*F > 0.0) dt0 = 0.25 * h0 * c0 * a0 / ((*F) + EPS);
    else dt0 = 0.25 * h1 * c1 * a1 / (-(*F) + EPS);
    if (dt > dt0) *F *= dt0 / (dt + EPS);
}

/* desingularised 1/h factor sqrt(2) h / sqrt(h^4 + max(h,eps)^4) */
static inline double inv_depth(double h, double eps)
{
    double m = dmax(h, eps);
    return SQRT2 * h / sqrt(pow4(h) + pow4(m));
}

/* src/GPU/Arista_kernel.cu:208,437,1002 — blend weight between the 2s and WAF fluxes */
static inline double blend_2s(double hij, double hpos, int no_limiter)
{
    if (no_limiter) return 0.0;
    if (hij < hpos) return 1.0 / (1.0 + exp(-15.0 * (1.0 - 0.5 * hpos / (hij + EPS))));
    return 1.0;
}

/* WAF coefficients from the two wave speeds (src/GPU/Arista_kernel.cu:190-199,381-393);
 * the mass flux divides by (aut2 - aut1), the momentum flux multiplies by its reciprocal. */
static inline void waf_coefficients(double aut1, double aut2, double xiL, double xiR, double val, double maxa,
                                    double *a0, double *a1)
{
    if (fabs(aut1 - aut2) >= EPS) {
        double alr = sgn(aut1) * (1.0 - xiL) + val * aut1 * xiL;
        double blr = sgn(aut2) * (1.0 - xiR) + val * aut2 * xiR;
        double aux = 1.0 / (aut2 - aut1);
        if (!a1) {
            *a0 = (alr - blr) * (aut1 * aut2) / (aut2 - aut1);
            return;
        }
        *a0 = (alr - blr) * (aut1 * aut2) * aux;
        *a1 = (blr * aut2 - alr * aut1) * aux;
    } else {
        *a0 = maxa;
        if (a1) *a1 = 0.0;
    }
}

/* ---------------------------------------------------------------------- */
/* stencil of one edge                                                     */
/* ---------------------------------------------------------------------- */

typedef struct {
    double h0m, h0, h1, h1p;     /* water depth at the 4 stencil cells */
    double H0m, H0, H1, H1p;     /* shifted bathymetry depth */
    double u0m, u0, u1, u1p;     /* normal momentum (x-momentum for x edges, y for y edges) */
    double v0m, v0, v1, v1p;     /* tangential momentum */
    double area0, area1, cos0, cos1;
    double len, normal;
    int cell0, cell1;            /* receiving cells, -1 = none */
    int front;                   /* ghost on the low side: roles of the two sides swapped */
    int no_limiter;              /* within two cells of a boundary */
} edge_t;

static void swap_d(double *a, double *b) { double t = *a; *a = *b; *b = t; }

static void edge_swap_sides(edge_t *e)
{
    swap_d(&e->h0m, &e->h1p); swap_d(&e->h0, &e->h1);
    swap_d(&e->H0m, &e->H1p); swap_d(&e->H0, &e->H1);
    swap_d(&e->u0m, &e->u1p); swap_d(&e->u0, &e->u1);
    swap_d(&e->v0m, &e->v1p); swap_d(&e->v0, &e->v1);
    swap_d(&e->area0, &e->area1); swap_d(&e->cos0, &e->cos1);
}

/* Gathers the x-edge at column x (between cells x-1 and x) of row y:
 * src/GPU/Arista_kernel.cu:484-544 (phase 1) / 582-652 (phase 2). */
static void gather_x_edge(const grid_t *g, int x, int y, edge_t *e)
{
    const int nx = g->nx;
    long long row = (long long)y * nx;
    int c;
    e->cell0 = (int)(row + x - 1);
    e->cell1 = e->cell0 + 1;
    e->len = g->dlat[y];
    e->area0 = e->area1 = g->area[y];
    e->cos0 = e->cos1 = g->cosphi[y];
    e->normal = 1.0;
    e->front = 0;
    c = col_index(x - 1, g->periodic, nx);
    e->h0 = g->h[row + c]; e->H0 = g->dep[row + c]; e->u0 = g->qx[row + c]; e->v0 = g->qy[row + c];
    if ((x - 1 < 0) && !g->periodic) {
        e->u0 *= g->b_left;
        e->cell0 = (int)row;
        e->cell1 = -1;
        e->normal = -1.0;
        e->front = 1;
    }
    c = col_index(x, g->periodic, nx);
    e->h1 = g->h[row + c]; e->H1 = g->dep[row + c]; e->u1 = g->qx[row + c]; e->v1 = g->qy[row + c];
    if ((x >= nx) && !g->periodic) {
        e->u1 *= g->b_right;
        e->cell0 = (int)(row + nx - 1);
        e->cell1 = -1;
    }
    c = col_index(x - 2, g->periodic, nx);
    e->h0m = g->h[row + c]; e->H0m = g->dep[row + c]; e->u0m = g->qx[row + c]; e->v0m = g->qy[row + c];
    c = col_index(x + 1, g->periodic, nx);
    e->h1p = g->h[row + c]; e->H1p = g->dep[row + c]; e->u1p = g->qx[row + c]; e->v1p = g->qy[row + c];
    if (g->periodic && x == 0) e->cell0 = -1;
    if (g->periodic && x == nx) e->cell1 = -1;
    e->no_limiter = (x < 2) || (x > nx - 2);
}

/* Gathers the y-edge at row y (between rows y-1 and y) of column x:
 * src/GPU/Arista_kernel.cu:1046-1104 (phase 1) / 1144-1213 (phase 2).
 * For y edges the "normal" momentum is qy and the tangential one qx. */
static void gather_y_edge(const grid_t *g, int x, int y, edge_t *e)
{
    const int nx = g->nx, ny = g->ny;
    int r;
    e->cell0 = (y - 1) * nx + x;
    e->cell1 = e->cell0 + nx;
    e->len = g->dlon[y];
    e->normal = 1.0;
    e->front = 0;
    r = (y - 1 >= 0) ? y - 1 : 0;
    e->h0 = g->h[(long long)r * nx + x]; e->H0 = g->dep[(long long)r * nx + x];
    e->u0 = g->qy[(long long)r * nx + x]; e->v0 = g->qx[(long long)r * nx + x];
    e->area0 = g->area[r]; e->cos0 = g->cosphi[r];
    if (y - 1 < 0) {
        e->u0 *= g->b_up;
        e->cell0 = x;
        e->cell1 = -1;
        e->front = 1;
        e->normal = -1.0;
    }
    r = (y < ny) ? y : ny - 1;
    e->h1 = g->h[(long long)r * nx + x]; e->H1 = g->dep[(long long)r * nx + x];
    e->u1 = g->qy[(long long)r * nx + x]; e->v1 = g->qx[(long long)r * nx + x];
    e->area1 = g->area[r]; e->cos1 = g->cosphi[r];
    if (y >= ny) {
        e->u1 *= g->b_low;
        e->cell0 = (y - 1) * nx + x;
        e->cell1 = -1;
    }
    r = (y - 2 >= 0) ? y - 2 : 0;
    e->h0m = g->h[(long long)r * nx + x]; e->H0m = g->dep[(long long)r * nx + x];
    e->u0m = g->qy[(long long)r * nx + x]; e->v0m = g->qx[(long long)r * nx + x];
    r = (y + 1 < ny) ? y + 1 : ny - 1;
    e->h1p = g->h[(long long)r * nx + x]; e->H1p = g->dep[(long long)r * nx + x];
    e->u1p = g->qy[(long long)r * nx + x]; e->v1p = g->qx[(long long)r * nx + x];
    e->no_limiter = (y < 2) || (y > ny - 2);
}

static inline int all_deep(const edge_t *e, double hpos)
{
    return (e->h0 > hpos) && (e->h1 > hpos) && (e->h0m > hpos) && (e->h1p > hpos) && !e->no_limiter;
}

/* ---------------------------------------------------------------------- */
/* phase 1: mass fluxes                                                    */
/* ---------------------------------------------------------------------- */

/* src/GPU/Arista_kernel.cu:118-219 (x) and 674-778 (y; lat=1 adds the
 * cos(phi) weighting and the spherical term of the surface gradient). */
static void mass_flux(grid_t *g, edge_t *e, int lat, double dt)
{
    double F;
    if (all_deep(e, g->hpos)) {
        if (!lat) {
            F = e->u0 * e->len / e->cos0;
            limit_outflow(e->h0, e->h1, 1.0, 1.0, dt, e->area0, e->area1, &F);
        } else {
            F = e->len * e->u0 * e->cos0;
            limit_outflow(e->h0, e->h1, e->cos0, e->cos1, dt, e->area0, e->area1, &F);
        }
    } else {
        double h0 = e->h0, h1 = e->h1, q0n, q1n, hij, e0m, e0, e1, e1p, u0n, u1n, s0, s1, uijn, val, c0;
        double aut1, aut2, maxa, xiL, xiR, a0, Hm, deta, F2s, Fwaf, alfa, ilcos;
        if (e->front) edge_swap_sides(e);
        h0 = e->h0; h1 = e->h1;
        if (!((h0 > EPS) || (h1 > EPS))) return;
        q0n = e->u0 * e->normal;
        q1n = e->u1 * e->normal;
        hij = 0.5 * (h0 + h1);
        c0 = sqrt(hij);
        e0m = e->h0m - e->H0m; e0 = h0 - e->H0; e1 = h1 - e->H1; e1p = e->h1p - e->H1p;
        dry_wet(h0, h1, e0, e1, e->H0, e->H1, g->eps_h, &q0n, &q1n);
        u0n = inv_depth(h0, g->eps_h) * q0n;
        u1n = inv_depth(h1, g->eps_h) * q1n;
        q0n = u0n * h0;
        q1n = u1n * h1;
        ilcos = lat ? e->len : e->len / e->cos0;
        F2s = lat ? e->len * q0n * e->cos0 * e->normal : ilcos * q0n * e->normal;
        s0 = sqrt(h0);
        s1 = sqrt(h1);
        uijn = (s0 * u0n + s1 * u1n) / (s0 + s1 + EPS);
        val = (2.0 * ilcos * dt) / (e->area0 + e->area1);
        aut1 = dmin(uijn - c0, u0n - s0);
        aut2 = dmax(uijn + c0, u1n + s1);
        maxa = dmax(fabs(aut2), fabs(aut1));
        if (e->no_limiter) xiL = xiR = 0.0;
        else {
            xiL = monotone_limiter(e0m, e0, e1, e1p, aut1);
            xiR = monotone_limiter(e0m, e0, e1, e1p, aut2);
        }
        waf_coefficients(aut1, aut2, xiL, xiR, val, maxa, &a0, NULL);
        Hm = dmin(e->H0, e->H1);
        if (!lat) {
            deta = dmax(e1 + Hm, 0.0) - dmax(e0 + Hm, 0.0);
            Fwaf = 0.5 * (q1n + q0n - a0 * deta) * ilcos;
        } else {
            double fl1 = q1n * e->cos1, fl0 = q0n * e->cos0;
            deta = 0.5 * (e->cos0 + e->cos1) * (dmax(e1 + Hm, 0.0) - dmax(e0 + Hm, 0.0)) - uijn * uijn * (e->cos1 - e->cos0);
            Fwaf = 0.5 * (fl0 + fl1 - a0 * deta) * e->len;
        }
        alfa = blend_2s(hij, g->hpos, e->no_limiter);
        F = alfa * F2s + (1.0 - alfa) * Fwaf;
        if (!lat) limit_outflow(h0, h1, 1.0, 1.0, dt, e->area0, e->area1, &F);
        else limit_outflow(h0, h1, e->cos0, e->cos1, dt, e->area0, e->area1, &F);
    }
    if (!lat) {
        if (e->cell0 != -1) g->acc_m[e->cell0] -= F;
        if (e->cell1 != -1) g->acc_m[e->cell1] += F;
    } else {
        if (e->cell0 >= 0) g->acc_m[e->cell0] -= F / e->cos0;
        if (e->cell1 != -1) g->acc_m[e->cell1] += F / e->cos1;
    }
}

/* ---------------------------------------------------------------------- */
/* phase 2: momentum fluxes                                                */
/* ---------------------------------------------------------------------- */

static inline void add_momentum(grid_t *g, int cell, double lam, double fx, double fy)
{
    g->acc_l[cell] += lam;
    g->acc_qx[cell] -= fx;
    g->acc_qy[cell] -= fy;
}

/* x edges: deep 2s src/GPU/Arista_kernel.cu:221-280, WAF 282-464.
 * Flux pairs are (x-momentum, y-momentum); `m` goes to cell0, `p` to cell1. */
static void momentum_flux_x(grid_t *g, edge_t *e, double dt)
{
    double mx, my, px, py, lam;
    if (all_deep(e, g->hpos)) {
        double h0 = e->h0, h1 = e->h1, hij = 0.5 * (h0 + h1), Hm = dmin(e->H0, e->H1);
        double u0n = e->u0 / h0, u1n = e->u1 / h1, s0 = sqrt(h0), s1 = sqrt(h1);
        double uijn = (s0 * u0n + s1 * u1n) / (s0 + s1 + EPS), c0 = sqrt(hij), maxa = fabs(uijn) + c0;
        double deta = dmax(h1 - e->H1 + Hm, 0.0) - dmax(h0 - e->H0 + Hm, 0.0);
        double ilcos = e->len / e->cos0, cd, val, des;
        if (uijn < 0.0) {
            mx = u1n * e->u1 * ilcos; px = -mx; mx += hij * deta * ilcos;
            my = u1n * e->v1 * ilcos; py = -my;
        } else {
            mx = u0n * e->u0 * ilcos; px = -mx; mx += hij * deta * ilcos;
            my = u0n * e->v0 * ilcos; py = -my;
        }
        cd = 0.5 * (1.0 - g->cvis);
        val = (2.0 * ilcos * dt) / (e->area0 + e->area1);
        des = cd * val * maxa * maxa * (e->u1 - e->u0) * ilcos;
        mx -= des;
        px += des;
        lam = ilcos * maxa;
    } else {
        double h0, h1, hij, e0m, e0, e1, e1p, w0, w1, h0rg, h1rg, u0n, u1n, s0, s1, uijn, val, c0;
        double aut1, aut2, maxa, fl1x, fl1y, fl0x, fl0y, dq, Hm, deta, cd, des, xiL, xiR, a0, a1;
        double s_my, s_mz, s_py, s_pz, desx, desy, q0mt, q0t, q1t, q1pt, p0m, p0, p1, p1p, uijt, aux, alfa;
        double t_my, t_mz, t_py, t_pz, ilcos = e->len / e->cos0;
        if (e->front) edge_swap_sides(e);
        if (!((e->h0 > EPS) || (e->h1 > EPS))) return;
        h0 = e->h0; h1 = e->h1;
        w0 = e->u0 * e->normal;
        w1 = e->u1 * e->normal;
        hij = 0.5 * (h0 + h1);
        e0m = e->h0m - e->H0m; e0 = h0 - e->H0; e1 = h1 - e->H1; e1p = e->h1p - e->H1p;
        dry_wet(h0, h1, e0, e1, e->H0, e->H1, g->eps_h, &w0, &w1);
        h0rg = inv_depth(h0, g->eps_h);
        u0n = h0rg * w0;
        h1rg = inv_depth(h1, g->eps_h);
        u1n = h1rg * w1;
        w0 = u0n * h0;
        w1 = u1n * h1;
        s0 = sqrt(h0);
        s1 = sqrt(h1);
        uijn = (s0 * u0n + s1 * u1n) / (s0 + s1 + EPS);
        val = (2.0 * ilcos * dt) / (e->area0 + e->area1);
        c0 = sqrt(hij);
        aut1 = dmin(uijn - c0, u0n - s0);
        aut2 = dmax(uijn + c0, u1n + s1);
        maxa = dmax(fabs(aut2), fabs(aut1));
        fl1x = w1; fl1y = u1n * w1;
        fl0x = w0; fl0y = u0n * w0;
        dq = fl1x - fl0x;
        Hm = dmin(e->H0, e->H1);
        deta = dmax(e1 + Hm, 0.0) - dmax(e0 + Hm, 0.0);
        if (uijn < 0.0) {
            s_my = u1n * w1 * ilcos * e->normal; s_py = -s_my; s_my += hij * deta * ilcos;
            s_mz = u1n * e->v1 * ilcos; s_pz = -s_mz;
        } else {
            s_my = u0n * w0 * ilcos * e->normal; s_py = -s_my; s_my += hij * deta * ilcos;
            s_mz = u0n * e->v0 * ilcos; s_pz = -s_mz;
        }
        cd = 0.5 * (1.0 - g->cvis / (1.0 + exp(-20.0 * (1.0 - g->hpos / hij))));
        des = cd * val * maxa * maxa * dq * ilcos * e->normal;
        s_my -= des;
        s_py += des;
        if (e->no_limiter) xiL = xiR = 0.0;
        else {
            xiL = monotone_limiter(e0m, e0, e1, e1p, aut1);
            xiR = monotone_limiter(e0m, e0, e1, e1p, aut2);
        }
        waf_coefficients(aut1, aut2, xiL, xiR, val, maxa, &a0, &a1);
        mx = px = 0.5 * dq;
        my = py = 0.5 * (fl1y - fl0y + hij * deta);
        desx = 0.5 * a0 * deta;
        desy = 0.5 * a0 * dq + a1 * my;
        mx += fl0x - desx; my += fl0y - desy;
        px += desx - fl1x; py += desy - fl1y;
        mx *= ilcos; my *= ilcos; px *= ilcos; py *= ilcos;
        /* transverse momentum carried with the limited tangential velocity */
        q0mt = e->v0m * e->normal; q0t = e->v0 * e->normal; q1t = e->v1 * e->normal; q1pt = e->v1p * e->normal;
        {
            double m = dmax(e->h0m, g->eps_h);
            p0m = SQRT2 * e->h0m * q0mt / sqrt(pow4(e->h0m) + pow4(m));
        }
        p0 = u0n = h0rg * q0t;
        p1 = u1n = h1rg * q1t;
        {
            double m = dmax(e->h1p, g->eps_h);
            p1p = SQRT2 * e->h1p * q1pt / sqrt(pow4(e->h1p) + pow4(m));
        }
        a0 = -1.0 * (mx < 0.0) + 1.0 * (mx > 0.0);
        uijn = fabs(uijn) * a0;
        xiL = e->no_limiter ? 0.0 : monotone_limiter(p0m, p0, p1, p1p, uijn);
        uijt = 0.5 * (u0n + u1n) - 0.5 * ((1.0 - xiL) * a0 + xiL * uijn * val) * (u1n - u0n);
        aux = mx * uijt;
        t_py = py * e->normal;
        t_pz = -aux * e->normal;
        t_my = my * e->normal;
        t_mz = aux * e->normal;
        alfa = blend_2s(hij, g->hpos, e->no_limiter);
        mx = alfa * s_my + (1.0 - alfa) * t_my;
        my = alfa * s_mz + (1.0 - alfa) * t_mz;
        px = alfa * s_py + (1.0 - alfa) * t_py;
        py = alfa * s_pz + (1.0 - alfa) * t_pz;
        if (maxa < g->eps_h) maxa += g->eps_h;
        lam = ilcos * maxa;
    }
    if (e->cell0 != -1) add_momentum(g, e->cell0, lam, mx, my);
    if (e->cell1 != -1) add_momentum(g, e->cell1, lam, px, py);
}

/* y edges: deep 2s src/GPU/Arista_kernel.cu:780-843, WAF 845-1026.
 * Flux pairs are returned as (x-momentum, y-momentum). */
static void momentum_flux_y(grid_t *g, edge_t *e, double dt)
{
    double fx_m, fy_m, fx_p, fy_p, lam;
    if (all_deep(e, g->hpos)) {
        double icos0 = 1.0 / e->cos0, icos1 = 1.0 / e->cos1;
        double h0 = e->h0, h1 = e->h1, hij = 0.5 * (h0 + h1), Hm = dmin(e->H0, e->H1);
        double u0n = e->u0 / h0, u1n = e->u1 / h1, s0 = sqrt(h0), s1 = sqrt(h1);
        double uijn = (s0 * u0n + s1 * u1n) / (s0 + s1 + EPS), c0 = sqrt(hij), maxa = fabs(uijn) + c0;
        double deta = 0.5 * (e->cos0 + e->cos1) * (dmax(h1 - e->H1 + Hm, 0.0) - dmax(h0 - e->H0 + Hm, 0.0)) -
                      uijn * uijn * (e->cos1 - e->cos0);
        double val, cd, des;
        if (uijn < 0.0) {
            fy_m = u1n * e->u1 * e->len;
            fy_p = -fy_m;
            fy_m *= e->cos1 * icos0;
            fy_m += hij * deta * e->len * icos0;
            fx_m = u1n * e->v1 * e->len;
            fx_p = -fx_m;
        } else {
            fy_m = u0n * e->u0 * e->len;
            fy_p = -fy_m * e->cos0 * icos1;
            fy_m += hij * deta * e->len * icos0;
            fx_m = u0n * e->v0 * e->len;
            fx_p = -fx_m;
        }
        val = (2.0 * e->len * dt) / (e->area0 + e->area1);
        cd = 0.5 * (1.0 - g->cvis);
        des = cd * val * maxa * maxa * (e->u1 * e->cos1 - e->u0 * e->cos0) * e->len;
        fy_m -= des * icos0;
        fy_p += des * icos1;
        lam = e->len * maxa;
    } else {
        double icos0, icos1, h0, h1, hij, c0, p0m, p0, p1, p1p, w0, w1, h0rg, h1rg, u0n, u1n, s0, s1, uijn, val;
        double aut1, aut2, maxa, Hm, deta, s_mz, s_pz, s_my, s_py, cd, fl1x, fl1y, fl0x, fl0y, dq, des;
        double xiL, xiR, a0, a1, desx, desy, mx, my, px, py, q0mt, q0t, q1t, q1pt, uijt, aux, alfa;
        double t_my, t_mz, t_py, t_pz;
        if (e->front) edge_swap_sides(e);
        if (!((e->h0 > EPS) || (e->h1 > EPS))) return;
        icos0 = 1.0 / e->cos0;
        icos1 = 1.0 / e->cos1;
        h0 = e->h0; h1 = e->h1;
        w0 = e->u0 * e->normal;
        w1 = e->u1 * e->normal;
        hij = 0.5 * (h0 + h1);
        c0 = sqrt(hij);
        p0m = e->h0m - e->H0m; p0 = h0 - e->H0; p1 = h1 - e->H1; p1p = e->h1p - e->H1p;
        dry_wet(h0, h1, p0, p1, e->H0, e->H1, g->eps_h, &w0, &w1);
        h0rg = inv_depth(h0, g->eps_h);
        u0n = h0rg * w0;
        h1rg = inv_depth(h1, g->eps_h);
        u1n = h1rg * w1;
        s0 = sqrt(h0);
        s1 = sqrt(h1);
        uijn = (s0 * u0n + s1 * u1n) / (s0 + s1 + EPS);
        val = (2.0 * e->len * dt) / (e->area0 + e->area1);
        aut1 = dmin(uijn - c0, u0n - s0);
        aut2 = dmax(uijn + c0, u1n + s1);
        maxa = dmax(fabs(aut2), fabs(aut1));
        Hm = dmin(e->H0, e->H1);
        deta = 0.5 * (e->cos0 + e->cos1) * (dmax(p1 + Hm, 0.0) - dmax(p0 + Hm, 0.0)) - uijn * uijn * (e->cos1 - e->cos0);
        if (uijn < 0.0) {
            s_mz = u1n * w1 * e->len * e->normal;
            s_pz = -s_mz;
            s_mz *= e->cos1 * icos0;
            s_mz += hij * deta * e->len * icos0;
            s_my = u1n * e->v1 * e->len;
            s_py = -s_my;
        } else {
            s_mz = u0n * w0 * e->len * e->normal;
            s_pz = -s_mz * e->cos0 * icos1;
            s_mz += hij * deta * e->len * icos0;
            s_my = u0n * e->v0 * e->len;
            s_py = -s_my;
        }
        cd = 0.5 * (1.0 - g->cvis / (1.0 + exp(-20.0 * (1.0 - g->hpos / hij))));
        fl1x = w1 * e->cos1; fl1y = u1n * fl1x;
        fl0x = w0 * e->cos0; fl0y = u0n * fl0x;
        dq = fl1x - fl0x;
        des = cd * val * maxa * maxa * dq * e->len;
        s_mz -= des * icos0;
        s_pz += des * icos1;
        if (e->no_limiter) xiL = xiR = 0.0;
        else {
            xiL = monotone_limiter(p0m, p0, p1, p1p, aut1);
            xiR = monotone_limiter(p0m, p0, p1, p1p, aut2);
        }
        waf_coefficients(aut1, aut2, xiL, xiR, val, maxa, &a0, &a1);
        mx = px = 0.5 * dq;
        my = py = 0.5 * (fl1y - fl0y + hij * deta);
        desx = 0.5 * a0 * deta;
        desy = 0.5 * a0 * dq + a1 * my;
        mx += fl0x - desx; my += fl0y - desy;
        px += desx - fl1x; py += desy - fl1y;
        mx *= e->len; my *= e->len; px *= e->len; py *= e->len;
        q0mt = -e->v0m * e->normal; q0t = -e->v0 * e->normal; q1t = -e->v1 * e->normal; q1pt = -e->v1p * e->normal;
        {
            double m = dmax(e->h0m, g->eps_h);
            p0m = SQRT2 * e->h0m * q0mt / sqrt(pow4(e->h0m) + pow4(m));
        }
        p0 = u0n = h0rg * q0t;
        p1 = u1n = h1rg * q1t;
        {
            double m = dmax(e->h1p, g->eps_h);
            p1p = SQRT2 * e->h1p * q1pt / sqrt(pow4(e->h1p) + pow4(m));
        }
        a0 = -1.0 * (mx < 0.0) + 1.0 * (mx > 0.0);
        uijn = fabs(uijn) * a0;
        xiL = e->no_limiter ? 0.0 : monotone_limiter(p0m, p0, p1, p1p, uijn);
        uijt = 0.5 * (u0n * icos0 + u1n * icos1) - 0.5 * ((1.0 - xiL) * a0 + xiL * uijn * val) * (u1n * icos1 - u0n * icos0);
        aux = mx * uijt;
        t_py = aux * e->normal;
        t_pz = py * e->normal * icos1;
        t_my = -aux * e->normal;
        t_mz = my * e->normal * icos0;
        if (maxa < g->eps_h) maxa += g->eps_h;
        alfa = blend_2s(hij, g->hpos, e->no_limiter);
        fx_m = alfa * s_my + (1.0 - alfa) * t_my;
        fy_m = alfa * s_mz + (1.0 - alfa) * t_mz;
        fx_p = alfa * s_py + (1.0 - alfa) * t_py;
        fy_p = alfa * s_pz + (1.0 - alfa) * t_pz;
        lam = e->len * maxa;
    }
    if (e->cell0 >= 0) add_momentum(g, e->cell0, lam, fx_m, fy_m);
    if (e->cell1 != -1) add_momentum(g, e->cell1, lam, fx_p, fy_p);
}

/* src/GPU/Arista_kernel.cu:1237-1428 — wave-speed sums for the initial dt */
static void initial_speed_edge(grid_t *g, edge_t *e, int lat)
{
    double h0, h1, hij, w0, w1, u0n, u1n, s0, s1, uij, maxa, v;
    if (e->front) {
        swap_d(&e->H0, &e->H1); swap_d(&e->h0, &e->h1); swap_d(&e->u0, &e->u1); swap_d(&e->v0, &e->v1);
    }
    /* rotated normal momentum: x edges use (normal, 0), y edges (0, normal) on (qx, qy) */
    if (!lat) {
        w0 = e->u0 * e->normal + e->v0 * 0.0;
        w1 = e->u1 * e->normal + e->v1 * 0.0;
    } else {
        w0 = e->v0 * 0.0 + e->u0 * e->normal;
        w1 = e->v1 * 0.0 + e->u1 * e->normal;
    }
    h0 = e->h0;
    h1 = e->h1;
    hij = 0.5 * (h0 + h1);
    {
        double m = dmax(h0, g->eps_h);
        u0n = SQRT2 * h0 * w0 / sqrt(pow4(h0) + pow4(m));
        m = dmax(h1, g->eps_h);
        u1n = SQRT2 * h1 * w1 / sqrt(pow4(h1) + pow4(m));
    }
    s0 = sqrt(h0);
    s1 = sqrt(h1);
    uij = (s0 * u0n + s1 * u1n) / (s0 + s1 + EPS);
    maxa = fabs(uij) + sqrt(hij);
    if (maxa < g->eps_h) maxa += g->eps_h;
    v = e->len * maxa / (lat ? 1.0 : e->cos0);
    if (e->cell0 >= 0) g->acc_l[e->cell0] += v;
    if (e->cell1 != -1) g->acc_l[e->cell1] += v;
}

/* ---------------------------------------------------------------------- */
/* passes over the edges (even then odd, as the reference's launches)      */
/* ---------------------------------------------------------------------- */

typedef enum { PASS_MASS, PASS_MOMENTUM, PASS_INITIAL } pass_t;

static void x_edge_pass(grid_t *g, int parity, pass_t kind, double dt)
{
    int y;
#pragma omp parallel for schedule(static)
    for (y = g->row_lo; y < g->row_hi; y++) {
        int x;
        for (x = parity; x <= g->nx; x += 2) {
            edge_t e;
            gather_x_edge(g, x, y, &e);
            if (kind == PASS_MASS) mass_flux(g, &e, 0, dt);
            else if (kind == PASS_MOMENTUM) momentum_flux_x(g, &e, dt);
            else initial_speed_edge(g, &e, 0);
        }
    }
}

static void y_edge_pass(grid_t *g, int parity, pass_t kind, double dt)
{
    int y;
    /* rows of edges of one parity touch disjoint cells: parallel over them */
#pragma omp parallel for schedule(static)
    for (y = parity; y <= g->ny; y += 2) {
        int x;
        if (y < g->row_lo || y > g->row_hi) continue;   /* touches no row this process updates */
        for (x = 0; x < g->nx; x++) {
            edge_t e;
            gather_y_edge(g, x, y, &e);
            if (kind == PASS_MASS) mass_flux(g, &e, 1, dt);
            else if (kind == PASS_MOMENTUM) momentum_flux_y(g, &e, dt);
            else initial_speed_edge(g, &e, 1);
        }
    }
}

static void all_edges(grid_t *g, pass_t kind, double dt)
{
    x_edge_pass(g, 0, kind, dt);
    x_edge_pass(g, 1, kind, dt);
    y_edge_pass(g, 0, kind, dt);
    y_edge_pass(g, 1, kind, dt);
}

/* ---------------------------------------------------------------------- */
/* cell updates                                                            */
/* ---------------------------------------------------------------------- */

/* src/GPU/Volumen_kernel.cu:96-158 (+ spongeLayerPaso1 6-14) */
static void update_mass(grid_t *g, double dt)
{
    int y;
    const int any_sponge = g->sp_left > 0 || g->sp_right > 0 || g->sp_up > 0 || g->sp_low > 0;
#pragma omp parallel for schedule(static)
    for (y = g->row_lo; y < g->row_hi; y++) {
        int x;
        double val = dt / g->area[y];
        for (x = 0; x < g->nx; x++) {
            long long i = (long long)y * g->nx + x;
            double h = g->h[i] + val * g->acc_m[i];
            h *= (h > 0.0);
            if (any_sponge && ((x < g->sp_left) || (x >= g->nx - g->sp_right) || (y < g->sp_up) || (y >= g->ny - g->sp_low))) {
                double dx = g->dlon[y], dy = g->dlat[y], dist, ls, co, r;
                double h_rest = dmax(g->dep[i] + g->Hmin + g->sea, 0.0);
                double d_l = (g->sp_left - x - 0.5) * dx, d_r = (x - (g->nx - 1 - g->sp_right) - 0.5) * dx;
                double d_u = (g->sp_up - y - 0.5) * dy, d_d = (y - (g->ny - 1 - g->sp_low) - 0.5) * dy;
                if (d_l <= 0.0) d_l = 1e30;
                if (d_r <= 0.0) d_r = 1e30;
                if (d_u <= 0.0) d_u = 1e30;
                if (d_d <= 0.0) d_d = 1e30;
                if ((d_l <= d_r) && (d_l <= d_u) && (d_l <= d_d)) { dist = d_l; ls = dx * g->sp_left; }
                else if ((d_r <= d_l) && (d_r <= d_u) && (d_r <= d_d)) { dist = d_r; ls = dx * g->sp_right; }
                else if ((d_u <= d_l) && (d_u <= d_r) && (d_u <= d_d)) { dist = d_u; ls = dy * g->sp_up; }
                else { dist = d_d; ls = dy * g->sp_low; }
                r = dist / ls;
                co = 0.9 * r * r;
                h -= co * (h - h_rest);
                h *= (h >= 0);
            }
            g->h[i] = h;
        }
    }
}

/* src/GPU/Volumen_kernel.cu:160-221 (+ spongeLayerPaso2 16-23, filtroEstado
 * 49-76, disImplicita 25-47): momenta, sponge, shallow-water filter and
 * semi-implicit Manning friction, next local dt.  Returns min dt. */
static double update_momentum(grid_t *g, double dt)
{
    int y;
    double dtmin = 1e300;
    const int any_sponge = g->sp_left > 0 || g->sp_right > 0 || g->sp_up > 0 || g->sp_low > 0;
#pragma omp parallel for schedule(static) reduction(min : dtmin)
    for (y = g->row_lo; y < g->row_hi; y++) {
        int x;
        double area = g->area[y], val = dt / area;
        for (x = 0; x < g->nx; x++) {
            long long i = (long long)y * g->nx + x;
            double lam = g->acc_l[i];
            double step = (lam < EPS) ? 1e30 : (2.0 * g->cfl * area) / lam;
            double qx_old = g->qx[i], qy_old = g->qy[i], h = g->h[i];
            double qx = qx_old + val * g->acc_qx[i];
            double qy = qy_old + val * g->acc_qy[i];
            g->dtc[i] = step;
            if (step < dtmin) dtmin = step;
            if (any_sponge) {
                double dx = g->dlon[y], dy = g->dlat[y], r, co, dist;
                double h_rest = dmax(g->dep[i] + g->Hmin + g->sea, 0.0), v_rest = 0.0;
                if (x < g->sp_left) {
                    dist = (g->sp_left - x - 0.5) * dx; r = dist / (dx * g->sp_left); co = 0.9 * r * r;
                    qx -= co * (qx - h_rest * v_rest);
                }
                if (x >= g->nx - g->sp_right) {
                    dist = (x - (g->nx - 1 - g->sp_right) - 0.5) * dx; r = dist / (dx * g->sp_right); co = 0.9 * r * r;
                    qx -= co * (qx - h_rest * v_rest);
                }
                if (y < g->sp_up) {
                    dist = (g->sp_up - y - 0.5) * dy; r = dist / (dy * g->sp_up); co = 0.9 * r * r;
                    qy -= co * (qy - h_rest * v_rest);
                }
                if (y >= g->ny - g->sp_low) {
                    dist = (y - (g->ny - 1 - g->sp_low) - 0.5) * dy; r = dist / (dy * g->sp_low); co = 0.9 * r * r;
                    qy -= co * (qy - h_rest * v_rest);
                }
            }
            if (h <= g->hpos) {
                /* exponential damping in almost-dry cells and velocity cap */
                double f = h / g->eps_h, damp = exp(-dt * (1.0 / (pow4(f) + EPS)));
                qx *= damp;
                qy *= damp;
                if (g->vmax > 0.0) {
                    double m = dmax(h, g->eps_h), fac = SQRT2 * h / sqrt(pow4(h) + pow4(m));
                    double ux = fac * qx, uy = fac * qy, u = sqrt(ux * ux + uy * uy);
                    if (u > g->vmax) {
                        ux *= g->vmax / u;
                        uy *= g->vmax / u;
                    }
                    qx = ux * h;
                    qy = uy * h;
                }
                /* semi-implicit Manning friction with the pre-update speed */
                {
                    double m = dmax(h, g->eps_h), fac = SQRT2 * h / sqrt(pow4(h) + pow4(m));
                    double u1x = fac * qx, u1y = fac * qy, u1;
                    m = dmax(h, g->eps_h);
                    u1 = SQRT2 * sqrt(qx_old * qx_old + qy_old * qy_old) * h / sqrt(pow4(h) + pow4(m));
                    if (h > 0.0) {
                        double c1 = dt * g->mf0 * fabs(u1) / (pow(h, 4.0 / 3.0) + EPS);
                        double fr = h / (1.0 + c1);
                        qx = fr * u1x;
                        qy = fr * u1y;
                    }
                }
            }
            g->qx[i] = qx;
            g->qy[i] = qy;
        }
    }
    return dtmin;
}

static void zero_acc(grid_t *g)
{
    memset(g->acc_m, 0, sizeof(double) * g->n);
    memset(g->acc_l, 0, sizeof(double) * g->n);
    memset(g->acc_qx, 0, sizeof(double) * g->n);
    memset(g->acc_qy, 0, sizeof(double) * g->n);
}

/* src/GPU/Timestep.cu:11-33 (+ obtenerDeltaTVolumenesGPU, CFL passed as float) */
static double initial_dt(grid_t *g)
{
    long long i;
    double m = 1e300;
    float cfl_f = (float)g->cfl;
    memset(g->acc_l, 0, sizeof(double) * g->n);
    all_edges(g, PASS_INITIAL, 0.0);
    for (i = (long long)g->row_lo * g->nx; i < (long long)g->row_hi * g->nx; i++) {
        int y = (int)(i / g->nx);
        double area = g->area[y];
        double s = (g->acc_l[i] < EPS) ? 1e30 : (2.0 * cfl_f * area) / g->acc_l[i];
        g->dtc[i] = s;
        if (s < m) m = s;
    }
    return m;
}

/* src/GPU/Timestep.cu:70-120 — one full step; returns the next dt */
static double full_step(grid_t *g, double dt)
{
    double next;
    memset(g->acc_m, 0, sizeof(double) * g->n);
    all_edges(g, PASS_MASS, dt);
    update_mass(g, dt);
    memset(g->acc_l, 0, sizeof(double) * g->n);
    memset(g->acc_qx, 0, sizeof(double) * g->n);
    memset(g->acc_qy, 0, sizeof(double) * g->n);
    all_edges(g, PASS_MOMENTUM, dt);
    next = update_momentum(g, dt);
    return next;
}

/* ---------------------------------------------------------------------- */
/* Okada                                                                   */
/* ---------------------------------------------------------------------- */

/* Gauss-Krueger projection of (lat, lon) about (lat0, lon0), kilometres
 * east / north (src/GPU/prtoxy.cu:33-54).  The constants are those of the
 * reference: a = 6378.16 km, e^2 = 0.0066946053, e'^2 = 0.0067397251,
 * a(1 - e^2) = 6335.4607362597517 km, 57.29578 deg/rad, 6 (57.29578)^2 and
 * pi/180 rounded to single precision. */
static void gauss_krueger(double lat, double lon, double lat0, double lon0, double *x, double *y)
{
    const double deg = 0.017453292371619689;
    double rlat = lat * deg, slat = sin(rlat), clat = cos(rlat);
    double v2 = clat * 0.0067397251 * clat + 1.0;
    double dl = lon - lon0;
    double ph1 = lat + v2 * 0.5 * dl * dl * slat * clat * deg;
    double rph1 = ph1 * deg, rph2 = (ph1 + lat0) * 0.5 * deg;
    double s1 = sin(rph1), s2 = sin(rph2);
    double d = sqrt(1.0 - s2 * 0.0066946053 * s2);
    double rm = 6335.4607362597517 / (d * (d * d));
    double rn = 6378.16 / sqrt(1.0 - s1 * 0.0066946053 * s1);
    double c1 = 57.29578 / rm, c2 = 57.29578 / rn;
    *y = (ph1 - lat0) / c1;
    *x = dl * clat / c2 * (dl * dl * cos(rlat * 2.0) / 19696.838434850401 + 1.0);
}

/* Vertical surface displacement of a rectangular dislocation (Okada 1985,
 * BSSA 75(4), eqs. 25-30, the u_z components for strike-slip U1 and dip-slip
 * U2; Poisson solid alpha = 2/3, i.e. mu/(lambda+mu) = 1/2).
 * x along strike, y across; the fault centroid is at depth d; the fault spans
 * xi in [x-L/2, x+L/2] and eta in [p-W/2, p+W/2] (Chinnery notation).
 * Singular stations follow DC3D's conventions (snap |.| < 1e-6 to 0, theta = 0
 * for q = 0, log/1/(R+.) terms switched when R+xi or R+eta vanishes). */
static double okada_uz(double x, double y, double d, double dip_deg, double L, double W, double U1, double U2)
{
    const double two_pi = 6.283185307179586, eps = 1e-6, mu_lm = 0.5;
    double sd = sin(dip_deg * (two_pi / 360.0)), cd = cos(dip_deg * (two_pi / 360.0));
    double xi[2], et[2], p, q, uz = 0.0;
    int kxi[2] = {0, 0}, ket[2] = {0, 0}, j, k;
    if (fabs(cd) < eps) {
        cd = 0.0;
        sd = (sd > 0.0) ? 1.0 : -1.0;
    }
    xi[0] = x + 0.5 * L;
    xi[1] = x - 0.5 * L;
    if (fabs(xi[0]) < eps) xi[0] = 0.0;
    if (fabs(xi[1]) < eps) xi[1] = 0.0;
    p = y * cd + d * sd;
    q = y * sd - d * cd;
    et[0] = p + 0.5 * W;
    et[1] = p - 0.5 * W;
    if (fabs(q) < eps) q = 0.0;
    if (fabs(et[0]) < eps) et[0] = 0.0;
    if (fabs(et[1]) < eps) et[1] = 0.0;
    if ((q == 0.0) && ((xi[0] * xi[1] <= 0.0 && et[0] * et[1] == 0.0) || (et[0] * et[1] <= 0.0 && xi[0] * xi[1] == 0.0)))
        return 0.0; /* station on a fault edge */
    {
        double r12 = sqrt(xi[0] * xi[0] + et[1] * et[1] + q * q);
        double r21 = sqrt(xi[1] * xi[1] + et[0] * et[0] + q * q);
        double r22 = sqrt(xi[1] * xi[1] + et[1] * et[1] + q * q);
        if (xi[0] < 0.0 && r21 + xi[1] < eps) kxi[0] = 1;
        if (xi[0] < 0.0 && r22 + xi[1] < eps) kxi[1] = 1;
        if (et[0] < 0.0 && r12 + et[1] < eps) ket[0] = 1;
        if (et[0] < 0.0 && r22 + et[1] < eps) ket[1] = 1;
    }
    for (k = 0; k < 2; k++) {
        for (j = 0; j < 2; j++) {
            double s = (j + k == 1) ? -1.0 : 1.0;
            double X = xi[j], E = et[k];
            double R = sqrt(X * X + E * E + q * q);
            double yt = E * cd + q * sd, dt = E * sd - q * cd;
            double theta = (q == 0.0) ? 0.0 : atan(X * E / (q * R));
            double inv_re, ln_re, inv_rx, I4, I5, fss, fds;
            (void)yt;
            if (R == 0.0) continue;
            /* 1/(R+eta), log(R+eta) and 1/(R+xi) with DC3D's switches (index as in DC3D) */
            if (kxi[k]) inv_rx = 0.0;
            else inv_rx = 1.0 / (R + X);
            if (ket[j]) { inv_re = 0.0; ln_re = -log(R - E); }
            else { inv_re = 1.0 / (R + E); ln_re = log(R + E); }
            if (cd != 0.0) {
                double Xs = sqrt(X * X + q * q);
                I4 = mu_lm / cd * (log(R + dt) - sd * ln_re);
                if (X == 0.0) I5 = 0.0;
                else I5 = mu_lm * 2.0 / cd * atan((E * (Xs + q * cd) + Xs * (R + Xs) * sd) / (X * (R + Xs) * cd));
            } else {
                I4 = -mu_lm * q / (R + dt);
                I5 = -mu_lm * X * sd / (R + dt);
            }
            fss = dt * q / R * inv_re + q * sd * inv_re + I4 * sd;
            fds = dt * q / R * inv_rx + sd * theta - I5 * sd * cd;
            uz += s * (-U1 / two_pi * fss - U2 / two_pi * fds);
        }
    }
    return uz;
}

/* Displacement (m) at one station for one fault, as aplicarOkadaStandardGPU
 * sets it up (src/GPU/Deformacion.cu:83-111). */
static double fault_uz_at(double lon, double lat, const double *f)
{
    const double rad = M_PI / 180.0;
    double xp, yp, ss = sin(rad * f[6]), cs = cos(rad * f[6]);
    double u_dip = f[9] * sin(rad * f[8]), u_str = f[9] * cos(rad * f[8]);
    gauss_krueger(lat, lon, f[2], f[1], &xp, &yp);
    return okada_uz(xp * ss + yp * cs, -xp * cs + yp * ss, f[3], f[7], f[4], f[5], u_str, u_dip);
}

void thy_oracle_okada_points(int n, const double *lon, const double *lat, const double *fault, double *uz)
{
    int i;
    for (i = 0; i < n; i++) uz[i] = fault_uz_at(lon[i], lat[i], fault);
}

/* src/GPU/Deformacion.cu:118-143 — deformation of one fault, crop, apply */
static void apply_fault(grid_t *g, const double *f, const double *lon, const double *lat, int crop_flag,
                        double crop_value, double *def)
{
    long long i;
    int y;
    double lon0 = lon[0], lat0 = lat[0];
    double dlon = (lon[g->nx - 1] - lon[0]) / (g->nx - 1), dlat = (lat[g->ny - 1] - lat[0]) / (g->ny - 1);
#pragma omp parallel for schedule(dynamic, 4)
    for (y = 0; y < g->ny; y++) {
        int x;
        for (x = 0; x < g->nx; x++)
            def[(long long)y * g->nx + x] = fault_uz_at(lon0 + x * dlon, lat0 + y * dlat, f) / g->Hs;
    }
    if (crop_flag == 1) {
        float mx = 0.0f;
        double thr;
        for (i = 0; i < g->n; i++) {
            float a = (float)fabs(def[i]);
            if (a > mx) mx = a;
        }
        thr = crop_value * (double)mx;
        for (i = 0; i < g->n; i++) if (fabs(def[i]) < thr) def[i] = 0.0;
    } else if (crop_flag == 2) {
        for (i = 0; i < g->n; i++) if (fabs(def[i]) < crop_value) def[i] = 0.0;
    }
    for (i = 0; i < g->n; i++) {
        g->dep[i] -= def[i];
        g->eta_ini[i] += def[i];
    }
}

/* ---------------------------------------------------------------------- */
/* output extraction (src/GPU/netcdf_kernel.cu:6-126)                      */
/* ---------------------------------------------------------------------- */

static void extract_state(const grid_t *g, float *eta, float *ux, float *uy)
{
    long long i;
    double QH = g->Qs / g->Hs;
    for (i = 0; i < g->n; i++) {
        double h = g->h[i], f;
        if (eta) eta[i] = (float)((h < g->eps_h) ? -9999.0f : (h - g->dep[i] - g->Hmin) * g->Hs);
        if (h < g->eps_h) f = SQRT2 * h / sqrt(pow4(h) + pow4(g->eps_h)) * QH;
        else f = g->Qs / (h * g->Hs);
        if (ux) ux[i] = (float)(g->qx[i] * f);
        if (uy) uy[i] = (float)(g->qy[i] * f);
    }
}

/* ---------------------------------------------------------------------- */
/* problem set-up (src/Problema.cxx:176-477) and the time loop             */
/* (src/GPU/ShallowWater.cu:182-500)                                       */
/* ---------------------------------------------------------------------- */

/* src/Problema.cxx:54-95 — nearest cell of a gauge, -1 outside the grid */
static int gauge_cell(const double *lon, const double *lat, int nx, int ny, double plon, double plat)
{
    int i = 0, j = 0, found = 0;
    if (plon < lon[0]) return -1;
    while (i < nx && !found) {
        if (lon[i] >= plon) {
            int im = (i - 1 > 0) ? i - 1 : 0;
            found = 1;
            if (fabs(plon - lon[im]) < fabs(plon - lon[i])) i = im;
        } else i++;
    }
    if (!found || plat < lat[0]) return -1;
    found = 0;
    while (j < ny && !found) {
        if (lat[j] >= plat) {
            int jm = (j - 1 > 0) ? j - 1 : 0;
            found = 1;
            if (fabs(plat - lat[jm]) < fabs(plat - lat[j])) j = jm;
        } else j++;
    }
    return found ? j * nx + i : -1;
}

/* src/GPU/Timestep.cu:76-109 */
static void clip_to_fault(int nf, int f, double t, const double *tf, double T, double *dt, int *jumping)
{
    if (f < nf && (t + *dt) * T > tf[f]) {
        *dt = tf[f] / T - t;
        *jumping = 1;
    }
}

static void clip_to_next_distinct_fault(int nf, int f, double t, const double *tf, double T, double *dt, int *jumping)
{
    *jumping = 0;
    if (f < nf) {
        int i = f + 1;
        while (i < nf && !(fabs(tf[i] - tf[f]) > EPS)) i++;
        if (i < nf && (t + *dt) * T > tf[i]) {
            *dt = tf[i] / T - t;
            *jumping = 1;
        }
    }
}

static void free_grid(grid_t *g)
{
    free(g->h); free(g->dep); free(g->qx); free(g->qy);
    free(g->area); free(g->cosphi); free(g->dlat); free(g->dlon);
    free(g->acc_m); free(g->acc_l); free(g->acc_qx); free(g->acc_qy); free(g->dtc);
    free(g->eta_max); free(g->t_arr); free(g->eta_ini);
}

/* The problem loader's set-up (src/Problema.cxx:319-448): scales,
 * dimensionless parameters, arrays, bathymetry with the Hmin shift, metric
 * terms and the initial state (Okada-style or from the initial-state file).
 * Returns 0, 1 (bad size) or 2 (no memory). */
static int grid_setup(grid_t *gp, const thy_oracle_problem *p)
{
#define g (*gp)
    int nx = p->nx, ny = p->ny, i;
    long long n = (long long)nx * ny, c;
    double R_nd;
    const double g2r = M_PI / 180.0;
    if (nx < 2 || ny < 2) return 1;
#ifdef _OPENMP
    if (p->threads > 0) omp_set_num_threads(p->threads);
#endif
    memset(&g, 0, sizeof(g));
    g.nx = nx; g.ny = ny; g.n = n;
    g.row_lo = 0; g.row_hi = ny;
    /* scales and dimensionless parameters (src/Problema.cxx:319-349) */
    g.Ls = p->L; g.Hs = p->H;
    g.Qs = sqrt(9.81 * pow(g.Hs, 3.0));
    g.Ts = g.Ls * g.Hs / g.Qs;
    g.mf0 = p->manning * (9.81 * p->manning * g.Ls / pow(g.Hs, 4.0 / 3.0));
    g.vmax = p->vmax / (g.Qs / g.Hs);
    g.eps_h = p->eps_h / g.Hs;
    g.hpos = p->hpos / g.Hs;
    g.cvis = 1.0 - p->stability;
    g.dif_at = p->dif_at / g.Hs;
    g.cfl = p->cfl;
    R_nd = EARTH_RADIUS_M / g.Ls;
    g.b_up = p->borders[0]; g.b_low = p->borders[1]; g.b_left = p->borders[2]; g.b_right = p->borders[3];
    g.periodic = (fabs(g.b_left - 2.0) < EPS) && (fabs(g.b_right - 2.0) < EPS);
    g.sp_left = (fabs(g.b_left - 1.0) < EPS) ? SPONGE_CELLS : 0;
    g.sp_right = (fabs(g.b_right - 1.0) < EPS) ? SPONGE_CELLS : 0;
    g.sp_up = (fabs(g.b_up - 1.0) < EPS) ? SPONGE_CELLS : 0;
    g.sp_low = (fabs(g.b_low - 1.0) < EPS) ? SPONGE_CELLS : 0;
    g.sea = SEA_LEVEL_M / g.Hs;

    g.h = malloc(sizeof(double) * n); g.dep = malloc(sizeof(double) * n);
    g.qx = calloc((size_t)n, sizeof(double)); g.qy = calloc((size_t)n, sizeof(double));
    g.area = malloc(sizeof(double) * ny); g.cosphi = malloc(sizeof(double) * ny);
    g.dlat = malloc(sizeof(double) * ny); g.dlon = malloc(sizeof(double) * (ny + 1));
    g.acc_m = calloc((size_t)n, sizeof(double)); g.acc_l = calloc((size_t)n, sizeof(double));
    g.acc_qx = calloc((size_t)n, sizeof(double)); g.acc_qy = calloc((size_t)n, sizeof(double));
    g.dtc = malloc(sizeof(double) * n);
    g.eta_max = malloc(sizeof(double) * n); g.t_arr = malloc(sizeof(double) * n); g.eta_ini = malloc(sizeof(double) * n);
    if (!g.h || !g.dep || !g.qx || !g.qy || !g.area || !g.cosphi || !g.dlat || !g.dlon || !g.acc_m || !g.acc_l ||
        !g.acc_qx || !g.acc_qy || !g.dtc || !g.eta_max || !g.t_arr || !g.eta_ini) {
        free_grid(&g);
        return 2;
    }
    /* bathymetry, Hmin, Okada-style initial state (src/Problema.cxx:383-398) */
    g.Hmin = 1e30;
    for (c = 0; c < n; c++) {
        double v = -1.0 * (double)p->z[c];
        v /= g.Hs;
        g.dep[c] = v;
        if (!p->eta_file) g.h[c] = (v > 0.0) ? v : 0.0;
        if (v < g.Hmin) g.Hmin = v;
    }
    /* metric terms (src/Problema.cxx:431-448) */
    {
        double dlon = fabs(p->lon[1] - p->lon[0]), dl = 0.0;
        for (i = 0; i < ny - 1; i++) {
            dl = fabs(p->lat[i + 1] - p->lat[i]);
            g.dlon[i] = dlon;
            g.dlat[i] = dl;
            g.area[i] = R_nd * dlon * dl * g2r;
            g.cosphi[i] = cos(p->lat[i] * g2r);
        }
        g.dlon[ny - 1] = dlon;
        g.dlat[ny - 1] = g.dlat[ny - 2];
        g.dlon[ny] = dlon;
        g.area[ny - 1] = R_nd * dlon * dl * g2r;
        g.cosphi[ny - 1] = cos(p->lat[ny - 1] * g2r);
    }
    if (g.Hmin < 0.0) for (c = 0; c < n; c++) g.dep[c] -= g.Hmin;
    else g.Hmin = 0.0;
    if (p->eta_file) {
        for (c = 0; c < n; c++) {
            double v = (double)p->eta_file[c] / g.Hs + g.dep[c] + g.Hmin;
            g.h[c] = dmax(v, 0.0);
        }
    }
    return 0;
#undef g
}

int thy_oracle_run(const thy_oracle_problem *p, thy_oracle_result *r)
{
    grid_t g;
    int nx = p->nx, ny = p->ny, i, nf = p->nfaults, fidx = 0, jumping = 0, snaps = 0, series = 0, rc;
    long long n = (long long)nx * ny, c, iter;
    double *faults = NULL, *tfault = NULL, tend, save_nc, save_ts, t = 0.0, dt, next_nc = 0.0, next_ts = 0.0;
    int *gpos = NULL, ngauge = 0;
    double *glon = NULL, *glat = NULL;
    struct timespec ts0, ts1;

    if ((rc = grid_setup(&g, p))) return rc;
    tend = p->sim_time / g.Ts;
    save_nc = p->save_time / g.Ts;
    save_ts = p->series_time / g.Ts;
    /* faults sorted by time (src/Problema.cxx:97-126, selection sort) */
    if (nf > 0) {
        faults = malloc(sizeof(double) * 10 * nf);
        tfault = malloc(sizeof(double) * nf);
        memcpy(faults, p->faults, sizeof(double) * 10 * nf);
        for (i = 0; i < nf - 1; i++) {
            int j, m = i;
            for (j = i + 1; j < nf; j++) if (faults[10 * j] < faults[10 * m]) m = j;
            if (m != i) {
                double tmp[10];
                memcpy(tmp, faults + 10 * i, sizeof(tmp));
                memcpy(faults + 10 * i, faults + 10 * m, sizeof(tmp));
                memcpy(faults + 10 * m, tmp, sizeof(tmp));
            }
        }
        for (i = 0; i < nf; i++) tfault[i] = faults[10 * i];
    }
    /* gauges: duplicates dropped, nearest cell (src/Problema.cxx:400-429) */
    if (p->npoints > 0 && p->series_time >= 0.0) {
        gpos = malloc(sizeof(int) * p->npoints);
        glon = malloc(sizeof(double) * p->npoints);
        glat = malloc(sizeof(double) * p->npoints);
        for (i = 0; i < p->npoints; i++) {
            double plon = p->points[2 * i], plat = p->points[2 * i + 1];
            int j, dup = 0;
            for (j = 0; j < ngauge; j++)
                if (fabs(glon[j] - plon) < 1e-6 && fabs(glat[j] - plat) < 1e-6) { dup = 1; break; }
            if (dup) continue;
            glon[ngauge] = plon;
            glat[ngauge] = plat;
            gpos[ngauge] = gauge_cell(p->lon, p->lat, nx, ny, plon, plat);
            ngauge++;
        }
        for (i = 0; i < ngauge; i++) {
            if (r->ts_min) r->ts_min[i] = (gpos[i] == -1) ? -9999.0f : 1e30f;
            if (r->ts_max) r->ts_max[i] = (gpos[i] == -1) ? -9999.0f : -1e30f;
        }
    }
    r->npoints_unique = ngauge;
    /* metrics initialised on the pre-deformation state (src/GPU/ShallowWater.cu:305-309) */
    for (c = 0; c < n; c++) {
        g.eta_max[c] = (g.h[c] < g.eps_h) ? -1e30 : g.h[c] - g.dep[c];
        g.eta_ini[c] = g.eta_max[c];
        g.t_arr[c] = -1.0;
    }

    clock_gettime(CLOCK_MONOTONIC, &ts0);
    dt = initial_dt(&g);
    if (nf > 0) {
        if (tfault[0] < EPS) clip_to_next_distinct_fault(nf, fidx, t, tfault, g.Ts, &dt, &jumping);
        else clip_to_fault(nf, fidx, t, tfault, g.Ts, &dt, &jumping);
    }
    r->first_dt = dt * g.Ts;
    iter = 0;
    {
        double *def = malloc(sizeof(double) * n);
        float *seta = NULL, *sux = NULL, *suy = NULL;
        if (ngauge > 0) { seta = malloc(sizeof(float) * ngauge); sux = malloc(sizeof(float) * ngauge); suy = malloc(sizeof(float) * ngauge); }
        while (t < tend && (p->max_iterations < 0 || iter < p->max_iterations)) {
            while (fidx < nf && t * g.Ts >= tfault[fidx]) {
                apply_fault(&g, faults + 10 * fidx, p->lon, p->lat, p->crop_flag,
                            p->crop_flag == 2 ? p->crop_value / g.Hs : p->crop_value, def);
                fidx++;
            }
            if (save_nc >= 0.0 && t >= next_nc) {
                next_nc += save_nc;
                if (snaps < r->max_snaps) {
                    size_t off = (size_t)snaps * (size_t)n;
                    extract_state(&g, r->snap_eta ? r->snap_eta + off : NULL, r->snap_ux ? r->snap_ux + off : NULL,
                                  r->snap_uy ? r->snap_uy + off : NULL);
                    if (r->snap_time) r->snap_time[snaps] = (float)(t * g.Ts);
                }
                snaps++;
            }
            if (save_ts >= 0.0 && ngauge > 0 && t >= next_ts) {
                next_ts += save_ts;
                for (i = 0; i < ngauge; i++) {
                    int cell = gpos[i];
                    if (cell >= 0) {
                        double h = g.h[cell], f;
                        if (h < g.eps_h) f = SQRT2 * h / sqrt(pow4(h) + pow4(g.eps_h));
                        else f = 1.0 / h;
                        seta[i] = (float)((h - g.dep[cell] - g.Hmin) * g.Hs);
                        sux[i] = (float)(f * g.qx[cell] * g.Qs / g.Hs);
                        suy[i] = (float)(f * g.qy[cell] * g.Qs / g.Hs);
                        if (r->ts_min) r->ts_min[i] = (seta[i] < r->ts_min[i]) ? seta[i] : r->ts_min[i];
                        if (r->ts_max) r->ts_max[i] = (r->ts_max[i] < seta[i]) ? seta[i] : r->ts_max[i];
                    } else seta[i] = sux[i] = suy[i] = -9999.0f;
                }
                if (series < r->max_series) {
                    size_t off = (size_t)series * ngauge;
                    if (r->ts_eta) memcpy(r->ts_eta + off, seta, sizeof(float) * ngauge);
                    if (r->ts_ux) memcpy(r->ts_ux + off, sux, sizeof(float) * ngauge);
                    if (r->ts_uy) memcpy(r->ts_uy + off, suy, sizeof(float) * ngauge);
                    if (r->ts_time) r->ts_time[series] = (float)(t * g.Ts);
                }
                series++;
            }
            /* metrics (src/GPU/Metrics.cu:23-77) */
#pragma omp parallel for schedule(static)
            for (c = 0; c < n; c++) {
                double e = g.h[c] - g.dep[c];
                if (e > g.eta_max[c] && g.h[c] > g.eps_h) g.eta_max[c] = e;
                if (g.t_arr[c] < 0.0 && fabs(e - g.eta_ini[c]) > g.dif_at) g.t_arr[c] = t;
            }
            {
                double next = full_step(&g, dt);
                t += dt;
                dt = next;
            }
            if (!jumping) clip_to_fault(nf, fidx, t, tfault, g.Ts, &dt, &jumping);
            else clip_to_next_distinct_fault(nf, fidx, t, tfault, g.Ts, &dt, &jumping);
            iter++;
        }
        free(def); free(seta); free(sux); free(suy);
    }
    clock_gettime(CLOCK_MONOTONIC, &ts1);
    r->loop_seconds = (ts1.tv_sec - ts0.tv_sec) + 1e-9 * (ts1.tv_nsec - ts0.tv_nsec);
    r->iterations = iter;
    r->final_time = t * g.Ts;
    r->nsnaps = snaps;
    r->nseries = series;
    for (c = 0; c < n; c++) {
        if (r->max_height) r->max_height[c] = (float)((g.eta_max[c] < -1e20) ? -9999.0f : (g.eta_max[c] - g.Hmin) * g.Hs);
        if (r->arrival) r->arrival[c] = (float)((g.t_arr[c] < 0.0) ? -1.0f : g.t_arr[c] * g.Ts);
        if (r->deformed_bathy) r->deformed_bathy[c] = (float)((g.dep[c] + g.Hmin) * g.Hs);
    }
    extract_state(&g, r->eta, r->ux, r->uy);
    if (ngauge > 0 && r->ts_bathy)
        for (i = 0; i < ngauge; i++)
            r->ts_bathy[i] = (gpos[i] >= 0) ? (float)((g.dep[gpos[i]] + g.Hmin) * g.Hs) : -9999.0f;
    free(faults); free(tfault); free(gpos); free(glon); free(glat);
    free_grid(&g);
    (void)zero_acc;
    return 0;
}

/* ---------------------------------------------------------------------- */
/* Row slabs: the same stepper on a process that updates only rows         */
/* [row_lo, row_hi) of the grid.  The caller keeps the two rows above and   */
/* below the slab current (halo exchange) after each phase, and takes the   */
/* minimum of every process's next dt; then each updated cell sees exactly  */
/* the values it would see in a single-process run (the stencil reaches two */
/* rows), so the decomposed run gives bitwise the same state.               */
/* ---------------------------------------------------------------------- */

struct thy_oracle_slab {
    grid_t g;
    const thy_oracle_problem *p;
    double *def;
};

thy_oracle_slab *thy_oracle_slab_open(const thy_oracle_problem *p, int row_lo, int row_hi)
{
    long long c;
    thy_oracle_slab *s;
    if (row_lo < 0 || row_hi > p->ny || row_lo >= row_hi) return NULL;
    s = calloc(1, sizeof(*s));
    if (!s) return NULL;
    if (grid_setup(&s->g, p)) {
        free(s);
        return NULL;
    }
    s->p = p;
    s->g.row_lo = row_lo;
    s->g.row_hi = row_hi;
    /* metrics initialised on the pre-deformation state (src/GPU/ShallowWater.cu:305-309) */
    for (c = 0; c < s->g.n; c++) {
        s->g.eta_max[c] = (s->g.h[c] < s->g.eps_h) ? -1e30 : s->g.h[c] - s->g.dep[c];
        s->g.eta_ini[c] = s->g.eta_max[c];
        s->g.t_arr[c] = -1.0;
    }
    s->def = malloc(sizeof(double) * s->g.n);
    if (!s->def) {
        thy_oracle_slab_close(s);
        return NULL;
    }
    return s;
}

double thy_oracle_slab_initial_dt(thy_oracle_slab *s) { return initial_dt(&s->g); }

void thy_oracle_slab_apply_fault(thy_oracle_slab *s, int k)
{
    const thy_oracle_problem *p = s->p;
    apply_fault(&s->g, p->faults + 10 * k, p->lon, p->lat, p->crop_flag,
                p->crop_flag == 2 ? p->crop_value / s->g.Hs : p->crop_value, s->def);
}

void thy_oracle_slab_phase1(thy_oracle_slab *s, double t, double dt)
{
    grid_t *g = &s->g;
    long long c;
    /* metrics of the state the step starts from (src/GPU/Metrics.cu:23-77) */
    for (c = (long long)g->row_lo * g->nx; c < (long long)g->row_hi * g->nx; c++) {
        double e = g->h[c] - g->dep[c];
        if (e > g->eta_max[c] && g->h[c] > g->eps_h) g->eta_max[c] = e;
        if (g->t_arr[c] < 0.0 && fabs(e - g->eta_ini[c]) > g->dif_at) g->t_arr[c] = t;
    }
    memset(g->acc_m, 0, sizeof(double) * g->n);
    all_edges(g, PASS_MASS, dt);
    update_mass(g, dt);
}

double thy_oracle_slab_phase2(thy_oracle_slab *s, double dt)
{
    grid_t *g = &s->g;
    memset(g->acc_l, 0, sizeof(double) * g->n);
    memset(g->acc_qx, 0, sizeof(double) * g->n);
    memset(g->acc_qy, 0, sizeof(double) * g->n);
    all_edges(g, PASS_MOMENTUM, dt);
    return update_momentum(g, dt);
}

double *thy_oracle_slab_field(thy_oracle_slab *s, int which)
{
    switch (which) {
    case 0: return s->g.h;
    case 1: return s->g.qx;
    case 2: return s->g.qy;
    case 3: return s->g.eta_max;
    case 4: return s->g.t_arr;
    case 5: return s->g.dep;
    default: return NULL;
    }
}

void thy_oracle_slab_scales(const thy_oracle_slab *s, double *ts_hs_hmin)
{
    ts_hs_hmin[0] = s->g.Ts;
    ts_hs_hmin[1] = s->g.Hs;
    ts_hs_hmin[2] = s->g.Hmin;
}

void thy_oracle_slab_close(thy_oracle_slab *s)
{
    if (!s) return;
    free(s->def);
    free_grid(&s->g);
    free(s);
}
