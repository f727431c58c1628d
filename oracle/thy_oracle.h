/*
 * thy_oracle — FP64 CPU restatement of the Tsunami-HySEA time stepper.
 *
 * TEST INFRASTRUCTURE.  Only tests/, __graft_entry__.smoke() and bench.py's
 * CPU-baseline leg load this library, and only as the checker / CPU
 * baseline.  The product (tsunami-hysea_b200/) never links or calls it.
 *
 * Inputs are exactly what the reference's problem file and its GRD /
 * points files carry (dimensional: degrees, metres, seconds); the oracle
 * performs the reference loader's nondimensionalisation itself.
 */
#ifndef THY_ORACLE_H
#define THY_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int nx, ny;
    const double *lon;        /* nx, degrees */
    const double *lat;        /* ny, degrees */
    const float *z;           /* ny*nx topobathymetry, metres, positive up */
    const float *eta_file;    /* ny*nx initial sea surface (m); NULL = Okada initialisation */
    int nfaults;
    const double *faults;     /* nfaults*10: time lon lat depth_km length_km width_km strike dip rake slip_m */
    int crop_flag;            /* 0 none, 1 relative, 2 absolute */
    double crop_value;
    double borders[4];        /* upper, lower, left, right: 1 open, -1 wall, 2 periodic (left/right) */
    double sim_time, save_time, series_time; /* seconds; < 0 disables saving */
    int npoints;
    const double *points;     /* npoints*2 (lon, lat) as listed in the points file */
    double cfl, eps_h, hpos, stability, manning, vmax, L, H, dif_at;
    long long max_iterations; /* < 0: run to sim_time */
    int threads;              /* <= 0: OpenMP default */
} thy_oracle_problem;

typedef struct {
    /* fields, ny*nx each, may be NULL */
    float *max_height;        /* m, -9999 where never wet */
    float *arrival;           /* s, -1 where never reached */
    float *deformed_bathy;    /* m, positive down */
    float *eta, *ux, *uy;     /* final state, extracted like a snapshot */
    /* snapshots (max_snaps*ny*nx each, may be NULL) */
    int max_snaps;
    float *snap_eta, *snap_ux, *snap_uy;
    double *snap_time;        /* max_snaps */
    int nsnaps;
    /* time series (max_series*npoints each) */
    int max_series;
    float *ts_eta, *ts_ux, *ts_uy;
    double *ts_time;
    float *ts_min, *ts_max, *ts_bathy; /* npoints */
    int nseries, npoints_unique;
    /* run summary */
    long long iterations;
    double final_time, first_dt, loop_seconds;
} thy_oracle_result;

int thy_oracle_run(const thy_oracle_problem *p, thy_oracle_result *r);

/* Okada vertical seafloor displacement (m) at n (lon, lat) points for one
 * fault (10 values as in thy_oracle_problem.faults). */
void thy_oracle_okada_points(int n, const double *lon, const double *lat, const double *fault, double *uz);

/* Row slabs, for the test of a row-slab decomposition of one grid: the
 * process updates only rows [row_lo, row_hi) of its copy of the whole grid;
 * the caller keeps the two rows above and below the slab current after each
 * phase (h after phase 1; qx, qy after phase 2) and steps every process
 * with the minimum of their next dt.  Faults are applied when the caller
 * says so (thy_oracle_slab_apply_fault, fault k of the problem's list). */
typedef struct thy_oracle_slab thy_oracle_slab;
thy_oracle_slab *thy_oracle_slab_open(const thy_oracle_problem *p, int row_lo, int row_hi);
double thy_oracle_slab_initial_dt(thy_oracle_slab *s);        /* minimum over the slab's rows */
void thy_oracle_slab_apply_fault(thy_oracle_slab *s, int k);
void thy_oracle_slab_phase1(thy_oracle_slab *s, double t, double dt);   /* metrics at t, mass update */
double thy_oracle_slab_phase2(thy_oracle_slab *s, double dt);  /* momentum update; next dt over the slab */
/* the whole-grid arrays (ny*nx doubles, dimensionless): 0 h, 1 qx, 2 qy,
 * 3 eta_max, 4 arrival time, 5 shifted depth */
double *thy_oracle_slab_field(thy_oracle_slab *s, int which);
void thy_oracle_slab_scales(const thy_oracle_slab *s, double *ts_hs_hmin);   /* time scale, depth scale, Hmin */
void thy_oracle_slab_close(thy_oracle_slab *s);

#ifdef __cplusplus
}
#endif

#endif
