/*
 * thysea.h — C ABI of the B200 Tsunami-HySEA time stepper (libthysea.so).
 *
 * The boundary this library replaces is the reference's single plug point
 *   extern "C" int shallowWater(...)          src/GPU/ShallowWater.cu:182-190
 * called once by main() (src/ShallowWater.cxx:146-151) with the
 * dimensionless problem produced by cargarDatosProblema()
 * (src/Problema.cxx:176-477).  That symbol is exported unchanged (see
 * thysea_dropin.h); this header is the same contract over plain C types:
 *
 *   thy_problem   the arguments of shallowWater() (dimensionless arrays in
 *                 the reference's layout) gathered in one struct;
 *   thy_outputs   where the results go (host buffers and callbacks, instead
 *                 of the NetCDF files shallowWater() writes itself);
 *   thy_run       the time loop of shallowWater() on the GPU.
 *
 * Plus the pieces around it that a caller of the reference gets from its
 * main(): the problem-file loader (thy_load_problem_file), the
 * nondimensionalisation (thy_prepare), and the NetCDF writers
 * (thy_write_netcdf), and the batched / serving entry points that run many
 * scenarios in one persistent launch (thy_batch_*, thy_server_*).
 *
 * Return codes 1 and 2 keep the meaning shallowWater() gives them
 * (src/GPU/ShallowWater.cu:262-353).
 */
#ifndef THYSEA_H
#define THYSEA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define THY_OK 0
#define THY_ERR_GPU_MEMORY 1   /* not enough GPU memory (shallowWater() returns 1) */
#define THY_ERR_HOST 2         /* host memory or output file (shallowWater() returns 2) */
#define THY_ERR_INVALID 3      /* invalid argument or problem file */
#define THY_ERR_CUDA 4         /* CUDA runtime error */
#define THY_ERR_NO_DEVICE 5    /* no CUDA device (main() prints "There is no graphics card") */
#define THY_ERR_NONFINITE 6    /* the state or the time step became non-finite */
#define THY_ERR_BUDGET 7       /* a scenario does not fit the server's HBM budget */
#define THY_ERR_CANCELLED 8    /* a served request was cancelled */
#define THY_ERR_TOO_LARGE 9    /* grid larger than an allocation-free entry point's fixed scratch */
#define THY_ERR_TIMEOUT 10     /* a bounded wait on the device ran out (a staging copy did not land) */

/* ------------------------------------------------------------------------
 * Raw problem: the contents of the problem .txt file and of its GRD and
 * points files, in their own units (degrees, metres, seconds).
 * Grammar: src/Problema.cxx:219-343; formats: README.md "File formats".
 * ---------------------------------------------------------------------- */
typedef struct thy_raw {
    int nx, ny;
    const double *lon;        /* nx */
    const double *lat;        /* ny */
    const float *z;           /* ny*nx topobathymetry, metres, positive up */
    const float *eta_file;    /* ny*nx initial surface (m); NULL selects Okada initialisation */
    int nfaults;
    const double *faults;     /* nfaults*10: time(s) lon lat depth(km) length(km) width(km) strike dip rake slip(m) */
    int crop_flag;            /* 0 none, 1 relative, 2 absolute */
    double crop_value;
    double borders[4];        /* upper, lower, left, right: 1 open, -1 wall, 2 periodic (left/right) */
    double sim_time, save_time, series_time;   /* seconds; < 0 disables */
    int npoints;
    const double *points;     /* npoints*2 lon lat, duplicates allowed (dropped as the reference does) */
    double cfl, eps_h, hpos, stability, manning, vmax, L, H, dif_at;
} thy_raw;

/* ------------------------------------------------------------------------
 * Dimensionless problem: the arguments of shallowWater().
 * ---------------------------------------------------------------------- */
typedef struct thy_problem {
    int nx, ny;
    const double *h;          /* nx*ny water depth           (datosVolumenesNivel_1[i].x) */
    const double *Hs;         /* nx*ny depth shifted by Hmin (datosVolumenesNivel_1[i].y) */
    const double *qx;         /* nx*ny discharges (datosVolumenesNivel_2[i].x), NULL = 0 */
    const double *qy;         /*                  (datosVolumenesNivel_2[i].y), NULL = 0 */
    const double *area_cos;   /* ny*2: cell area, cos(lat)   (datosNivel.areaYCosPhi) */
    const double *dlon;       /* ny+1                         (datosNivel.anchoVolumenes) */
    const double *dlat;       /* ny                           (datosNivel.altoVolumenes) */
    const double *lon;        /* nx degrees                   (datosNivel.longitud) */
    const double *lat;        /* ny degrees                   (datosNivel.latitud) */
    double Hmin;
    double border_up, border_low, border_left, border_right;
    int sponge_up, sponge_low, sponge_left, sponge_right;
    double t_end, save_nc, save_ts;   /* dimensionless; save_* < 0 disables */
    double cfl, mf0, vmax, eps_h, hpos, cvis, dif_at;
    double L, H, Q, T;                /* scales */
    int okada_flag;                   /* 1: faults below; 0: initial state from file (already in h) */
    int nfaults;
    const double *faults;             /* nfaults*10, sorted by time, as in thy_raw */
    int crop_flag;
    double crop_value;                /* dimensionless for absolute cropping */
    int npoints;
    const int *point_cell;            /* npoints cell indices (-1: outside the grid) */
    const double *point_lon;          /* npoints gauge longitudes (lonPuntos) */
    const double *point_lat;          /* npoints gauge latitudes  (latPuntos) */
    long long max_steps;              /* < 0: run to t_end */
} thy_problem;

/* Snapshot / gauge callbacks: fields are dimensional float arrays laid out
 * like the reference's NetCDF variables (eta, ux, uy: ny*nx; gauges:
 * npoints each).  `index` counts from 0, time is in seconds. */
typedef void (*thy_field_fn)(void *user, int index, double time_s, const float *eta, const float *ux, const float *uy);

typedef struct thy_outputs {
    float *max_height;        /* ny*nx, m, -9999 never wet         (may be NULL) */
    float *arrival;           /* ny*nx, s, -1 never reached         (may be NULL) */
    float *deformed_bathy;    /* ny*nx, m, positive down            (may be NULL) */
    float *eta, *ux, *uy;     /* ny*nx final state like a snapshot  (may be NULL) */
    float *series_min, *series_max, *series_bathy;   /* npoints      (may be NULL) */
    thy_field_fn on_snapshot; /* called at every snapshot time     (may be NULL) */
    thy_field_fn on_series;   /* called at every gauge time        (may be NULL) */
    void *user;
} thy_outputs;

/* Warp tiling of the stepping kernels: a variant index 0..2 per kernel
   (row groups of warps per work unit: deep phase 1 {3, 2, 4} of 4 column
   strips, deep phase 2 {4, 2, 8} of 2 strips of column pairs, general
   {2, 1, 8} of 4 strips; 0 is the default).  No result
   depends on the tiling; the autotuner picks one per device and work size. */
typedef struct thy_tiling {
    int deep1, deep2, general;
} thy_tiling;

typedef struct thy_stats {
    long long steps;          /* time steps taken */
    double final_time_s;      /* simulated time reached */
    double first_dt_s;        /* initial dt after fault-time truncation */
    double loop_seconds;      /* wall time of the time loop (the reference's "Runtime") */
    double device_loop_ms;    /* device time of the stepping kernels (CUDA events) */
    long long kernel_launches;/* kernels launched by the time loop */
    int snapshots, series_samples;
    long long tiles;          /* work units (112 x 16-cell half tiles) x steps */
    long long deep_tiles;     /* ... stepped by the deep-water kernels (phase 2) */
    long long dry_tiles;      /* ... skipped as settled dry land */
    double setup_seconds;     /* device set-up before the loop: upload, metrics, graph capture */
    double output_seconds;    /* extraction and download of the output fields after the loop */
    double total_seconds;     /* the whole call, release of the device buffers included */
    thy_tiling tiling;        /* the warp tiling of the loop's last chunk */
    long long tune_samples;   /* chunks of the loop timed for the autotuner */
    double release_seconds;   /* release of the device buffers, graphs and streams after the outputs */
    long long chunks;         /* graph launches of the time loop */
    long long graph_captures; /* step graphs captured (per tiling and chunk length) */
    double capture_seconds;   /* host time spent capturing and instantiating them */
    double event_seconds;     /* host time spent on the loop's events (faults, snapshots, gauges) */
    double initial_seconds;   /* initial dt and the t = 0 faults, before the first chunk */
} thy_stats;

/* Library / device. */
const char *thy_version(void);
const char *thy_strerror(int code);
int thy_device_count(void);                       /* 0 when no CUDA device is usable */
int thy_set_device(int device);
/* Page-lock / release caller-owned host memory (inputs of thy_problem, output
   fields) so that thy_run's host<->device copies run at full speed. */
int thy_host_register(void *p, size_t bytes);
int thy_host_unregister(void *p);

/* Problem set-up: file loader (problem .txt + GRD + points, the grammar of
 * src/Problema.cxx:176-343) into a raw problem owned by the library, and the
 * nondimensionalisation of src/Problema.cxx:319-477 into an owned problem. */
typedef struct thy_raw_owned thy_raw_owned;
int thy_load_problem_file(const char *txt_path, thy_raw_owned **out);
const thy_raw *thy_raw_view(const thy_raw_owned *r);
const char *thy_raw_name(const thy_raw_owned *r);     /* problem name (first line) */
const char *thy_raw_bathy_file(const thy_raw_owned *r);
const char *thy_raw_prefix(const thy_raw_owned *r);   /* NetCDF output prefix */
void thy_raw_free(thy_raw_owned *r);

typedef struct thy_problem_owned thy_problem_owned;
int thy_prepare(const thy_raw *raw, thy_problem_owned **out);
const thy_problem *thy_problem_view(const thy_problem_owned *p);
void thy_problem_free(thy_problem_owned *p);

/* The time loop of shallowWater() on the GPU (device 0 or thy_set_device). */
int thy_run(const thy_problem *p, const thy_outputs *o, thy_stats *stats);

/* Same problem through the reference's NetCDF outputs: <prefix>.nc and,
 * with gauges, <prefix>_ts.nc (src/GPU/netcdfTH.cu, src/GPU/netcdfSeries.cu). */
int thy_run_netcdf(const thy_problem *p, const char *problem_name, const char *prefix, thy_stats *stats);

/* The Okada stage alone on device memory, replacing
 *   void aplicarOkada(...)                       src/GPU/Deformacion.cu:118-143
 * d_state1 is the reference's device state (double2 (h, H) per cell,
 * dimensionless, nx*ny), d_eta_initial its eta_initial field (may be NULL);
 * fault holds the 10 problem-file values (time lon lat depth_km length_km
 * width_km strike dip rake slip_m); the stations are lon0 + i*dlon,
 * lat0 + j*dlat; H is the depth scale; crop_flag / crop_value as in
 * thy_problem.  Computes U_Z in FP64, crops, then H -= U_Z/H_scale and
 * eta_initial += U_Z/H_scale.  Runs on the caller's current device and
 * `stream` (a cudaStream_t, NULL = default stream); allocates its nx*ny
 * doubles of scratch with cudaMalloc and returns after the stream is idle. */
int thy_apply_okada(int nx, int ny, double lon0, double dlon, double lat0, double dlat, const double *fault,
                    double H, int crop_flag, double crop_value, void *d_state1, double *d_eta_initial, void *stream);

/* thy_apply_okada without any device allocation.  No counterpart in the
 * reference: it serves callers that cannot call cudaMalloc (the GPU's memory
 * is owned by a caching or budgeted allocator, or an allocation's implicit
 * device-wide synchronisation is not allowed where they run).  Its scratch
 * is a fixed array inside the library, THY_OKADA_NOALLOC_MAX_CELLS doubles
 * (8 MiB) held by every GPU that loads the library until the process exits;
 * larger grids return THY_ERR_TOO_LARGE.  The first call on a device looks
 * up that array's device address, so it should come before any stream
 * capture; after a device reset (cudaDeviceReset) the addresses are looked
 * up again by the next call, which then counts as a first call.  The call
 * only enqueues the work on `stream`.  All calls share the scratch: calls
 * whose work overlaps on the GPU race. */
#define THY_OKADA_NOALLOC_MAX_CELLS (1 << 20)
int thy_apply_okada_noalloc(int nx, int ny, double lon0, double dlon, double lat0, double dlat, const double *fault,
                            double H, int crop_flag, double crop_value, void *d_state1, double *d_eta_initial,
                            void *stream);

/* Step-level access for benchmarking: set up a problem on the device, run
 * `steps` time steps (Okada applied first), report the device time of the
 * stepping kernels.  No outputs are produced. */
typedef struct thy_session thy_session;
int thy_session_open(const thy_problem *p, thy_session **out);
int thy_session_steps(thy_session *s, long long steps, double *device_ms, long long *steps_done);
int thy_session_fetch(thy_session *s, float *max_height, float *eta, float *ux, float *uy);
/* average device time (ms) of the phase-1 (mass + diagnostics) and phase-2
 * (momentum + dt) launches over `steps` individually launched steps */
int thy_session_profile(thy_session *s, long long steps, double *phase1_ms, double *phase2_ms);
/* the same, per launch: ms_per_launch[6] = deep phase 1, general phase 1,
   deep/general classification, deep phase 2, general phase 2, step controller */
int thy_session_profile_launches(thy_session *s, long long steps, double *ms_per_launch);
long long thy_session_launches(const thy_session *s);   /* stepping kernels launched so far */
/* work units (112 x 16-cell half tiles) x steps so far, of which stepped by
   the deep-water kernels, and skipped as settled dry land */
int thy_session_tiles(const thy_session *s, long long *tiles, long long *deep_tiles, long long *dry_tiles);
double thy_session_time(const thy_session *s);    /* simulated time (s) */
/* step (real steps of the run) until the autotuner has decided the tiling
   for this problem's work size, at most max_steps; *steps_done: steps taken */
int thy_session_tune(thy_session *s, long long max_steps, long long *steps_done);
int thy_session_tiling(const thy_session *s, thy_tiling *t);   /* tiling of the last chunk */
/* 1 when the tiling for the session's current work (its last chunk's deep
   and general units per step) is decided (*best set), 0 while tuning */
int thy_session_tuned(const thy_session *s, thy_tiling *best);
void thy_session_close(thy_session *s);
/* Test hook for failure detection: with `what` = 1 the deep-water kernels
   issue none of this session's staging copies, so their bounded waits
   (four seconds of global time) run out, the step stops and thy_session_steps
   returns THY_ERR_TIMEOUT with the device context still usable; 0 turns it
   off.  Nothing faults, traps or hangs. */
int thy_session_inject(thy_session *s, int what);

/* Autotuner of the warp tilings.  Every full chunk of a run (of any entry
   point) is timed as one sample of the tiling it ran with; the search, per
   device and work of a step (ceil log2 of its deep units and of its general
   units, estimated from each scenario's previous chunk), is coordinate
   descent over deep phase 2, deep phase 1 and the general kernel.
   Environment: THY_TILING="d1,d2,g" forces a tiling, THY_TUNE=0 keeps the
   default, THY_TUNE_CACHE=<file> keeps decided tilings across processes. */
int thy_tiling_force(const thy_tiling *t);          /* NULL: autotune again */
/* 1 when the tiling for steps of deep_units deep and general_units general
   work units is decided on the current device (*best set), 0 while tuning
   (*best: the incumbent) */
int thy_tiling_tuned(double deep_units, double general_units, thy_tiling *best);
void thy_tuner_clear(void);                         /* forget every decision of this process */

/* Multi-scenario runtime (batched and serving use): scenarios submitted at
   any time are admitted in order under an HBM budget and stepped together -
   one work list over all their tiles, one CUDA graph per chunk of steps -
   and retired as they finish, each with its own dt, time and events.  A
   scenario's results are identical alone (thy_run) and in any mix.  A
   scenario whose state turns non-finite is retired with THY_ERR_NONFINITE
   while the others continue. */
typedef struct thy_server thy_server;
typedef struct thy_server_opts {
    long long hbm_budget_bytes;   /* device memory for scenario state (0: 90 % of the free memory) */
    int max_scenarios;            /* scenarios resident at once (0: 256) */
    int device;
    long long chunk_cells;        /* cells stepped per chunk: the resident scenario submitted first,
                                     then those with the least remaining work (cells x remaining
                                     steps), until their cells reach this (0: 2^24, one 4096^2 grid;
                                     < 0: all); a scenario of at least half this many cells is
                                     stepped only when submitted first, and then alone, and
                                     queued requests are admitted after it */
} thy_server_opts;
typedef struct thy_server_stats {
    long long submitted, admitted, completed, failed, cancelled, rejected;
    long long chunks;             /* graph launches */
    int queued, running;
    long long hbm_in_use, hbm_budget;
    double device_ms;             /* device time of the chunks */
    double cell_updates;          /* of retired scenarios */
} thy_server_stats;
/* completion callback, from thy_server_progress / drain / cancel / close:
   status THY_OK, THY_ERR_NONFINITE, THY_ERR_CANCELLED or a set-up error;
   stats may be NULL for a request that never ran.  For the request's
   thy_stats: setup_seconds = time queued, loop_seconds = time admitted,
   total_seconds = submission to result. */
typedef void (*thy_done_fn)(void *user, long long request, int status, const thy_stats *stats);
int thy_server_open(const thy_server_opts *opts, thy_server **out);
/* queues a request; `p` and `o` must stay valid until its callback (nothing
   is copied before admission); THY_ERR_BUDGET if it can never fit */
int thy_server_submit(thy_server *s, const thy_problem *p, const thy_outputs *o, thy_done_fn done, void *user,
                      long long *request);
int thy_server_cancel(thy_server *s, long long request);   /* queued: now; running: at the next progress */
/* admits, performs due events, runs one chunk of steps for every running
   scenario and retires the finished ones; *active = queued + running */
int thy_server_progress(thy_server *s, int *active);
int thy_server_drain(thy_server *s);                        /* progress until nothing is queued or running */
int thy_server_get_stats(const thy_server *s, thy_server_stats *out);
void thy_server_close(thy_server *s);                       /* cancels what is left */

#ifdef __cplusplus
}
#endif

#endif /* THYSEA_H */
