// Host-side engine: device state of scenarios, the graph-captured time loop
// and its event handling.  Shared by thy_run (one scenario), the session
// API (benchmarking) and the batch / server runtimes (many scenarios in one
// persistent launch).
#pragma once
#include <cstdint>
#include <memory>
#include <string>
#include <utility>
#include <vector>

#include <cuda_runtime.h>

#include "../../../include/thysea.h"
#include "../kernels/device.cuh"
#include "../kernels/kernels.h"
#include "tuner.h"

namespace thy {

#define THY_CK(expr)                                                          \
    do {                                                                      \
        cudaError_t _e = (expr);                                              \
        if (_e != cudaSuccess) {                                              \
            set_last_cuda_error(_e, #expr, __FILE__, __LINE__);               \
            return (_e == cudaErrorMemoryAllocation) ? THY_ERR_GPU_MEMORY : THY_ERR_CUDA; \
        }                                                                     \
    } while (0)

void set_last_cuda_error(cudaError_t e, const char *what, const char *file, int line);
const char *last_error_text();

// Device bytes one scenario of nx*ny cells needs (fields, row tables, control,
// Okada scratch when it has faults).
size_t scenario_bytes(int nx, int ny, bool has_faults);

class OutputPipe;   // asynchronous snapshot / gauge delivery (engine.cu)

// One scenario on the device.
struct DevScenario {
    int nx = 0, ny = 0, pitch = 0;
    size_t plane = 0;              // floats per field plane
    float *fields = nullptr;       // 10 planes: eta0 eta1 qx0 qx1 qy0 qy1 dep emax arr eini
    float *rows = nullptr;         // row tables
    double *def = nullptr;         // Okada scratch (nx*ny doubles)
    unsigned int *maxbits = nullptr;
    int *d_cells = nullptr;        // gauge cells
    float *d_gauge = nullptr;      // 4 floats per gauge
    float *d_gring = nullptr;      // kGaugeRing device samples x 4 floats per gauge (desc.gauge_ring)
    double *d_gring_t = nullptr;   // their times (desc.gauge_ring_t)
    float2 *d_gminmax = nullptr;   // per gauge extremes of eta (desc.gauge_minmax)
    unsigned gauges_read = 0;      // device samples handed to the outputs so far
    float *d_out = nullptr;        // 3 planes nx*ny for snapshots / outputs
    double *fault_times_d = nullptr;
    UnitSum *usum = nullptr;       // 2 parities x 2 ntiles unit depth summaries (desc.usum)
    unsigned char *dry_age = nullptr;   // 2 ntiles (desc.dry_age)
    float *gmax = nullptr;              // 2 ntiles depth steps per unit (desc.unit_gmax)
    TmaMap *tmaps = nullptr;       // kNumMaps tensor maps of the field planes (desc.tmap)
    float4 *rowpack = nullptr;     // ny+1 packed row metrics (desc.rowpack)
    ScenarioCtl *ctl = nullptr;    // device control block (owned by the batch slot)
    cudaStream_t ast = nullptr;    // stream the buffers were allocated on (stream-ordered pool)
    ScenarioDev desc{};            // descriptor (device pointers), host copy
    // problem data kept on the host
    double Hs = 1, Qs = 1, Ts = 1, Hmin = 0, Ls = 1;
    double lon0 = 0, dlon = 0, lat0 = 0, dlat = 0;
    double t_end = 0, save_nc = -1, save_ts = -1;
    long long max_steps = -1;
    int crop_flag = 0;
    double crop_value = 0;
    std::vector<double> faults;    // 10 per fault, sorted by time
    std::vector<int> cells;        // gauge cells
    int okada_flag = 0;
    // host mirror of the control block
    ScenarioCtl hctl{};
    // run bookkeeping
    int snapshots = 0, series = 0;
    double first_dt_s = 0;
    // work mix of the last chunk it stepped (per step): deep units, skipped
    // dry units; the autotuner's key for the chunks that follow
    double mix_deep = 0, mix_dry = 0;
    bool mix_known = false;
    std::unique_ptr<OutputPipe> pipe;   // created at the first snapshot / gauge sample

    long long units() const { return (long long)desc.tiles_x * ((ny + kHalfRows - 1) / kHalfRows); }   // work units
    DevScenario();
    ~DevScenario();
    int setup(const thy_problem *p, cudaStream_t st);   // allocate, upload, initial dt
    int upload_ctl(cudaStream_t st);
    int download_ctl(cudaStream_t st);                   // async into hctl (pinned by the batch)
    int apply_due_faults(cudaStream_t st);               // faults with time <= t (the loop's first action)
    cudaError_t invalidate_tile_minima(cudaStream_t st);
    int encode_tensor_maps(cudaStream_t st);
    int extract(int field, float *host_out, cudaStream_t st);
    int open_outputs(const thy_outputs *o, cudaStream_t st);
    int snapshot(const thy_outputs *o, cudaStream_t st);
    int sample_gauges(const thy_outputs *o, cudaStream_t st);
    int read_device_gauges(const thy_outputs *o, cudaStream_t st);   // the controller's samples since the last call
    int finish(const thy_outputs *o, cudaStream_t st);
};

// A set of scenarios stepped together: one work list over all their tiles,
// one CUDA graph of `chunk` steps (kLaunchesPerStep launches per step) per
// warp tiling the autotuner has run it with (tuner.h).
struct Batch {
    std::vector<DevScenario *> members;
    ScenarioDev *d_table = nullptr;
    int2 *d_work = nullptr;
    int *d_nwork = nullptr;
    int2 *d_work0 = nullptr;           // work list of scenarios joining (their initial dt)
    int *d_nwork0 = nullptr;
    int *d_lists = nullptr;            // deep / general lists of the current step (StepLaunch::lists)
    int *d_claims = nullptr;           // StepLaunch::claims
    ScenarioCtl *d_ctl = nullptr;      // slots
    ScenarioCtl *h_ctl = nullptr;      // pinned mirror
    int capacity = 0;
    int work_capacity = 0;
    int nwork = 0;
    int chunk = 16;
    int device = 0;
    Tiling tiling;                     // of gexec
    // step graphs captured for the current capacity, per tiling and length:
    // the full chunk, and one step, launched as often as a shorter chunk
    // needs (a session's last steps, the steps before an event)
    struct Graph {
        Tiling tiling;
        int len;
        cudaGraphExec_t exec;
    };
    std::vector<Graph> graphs;
    long long tune_samples = 0;        // chunks timed for the autotuner
    cudaStream_t st = nullptr;
    cudaStream_t st_side = nullptr;    // second branch of the captured graph (deep-water kernels)
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    cudaGraphExec_t gexec = nullptr;   // graph of the current tiling
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    double device_ms = 0;
    long long launches = 0;
    long long chunks_run = 0;          // graph launches
    long long captures = 0;            // graphs captured
    double capture_s = 0;              // host time spent capturing and instantiating them
    bool owns_stream = false;          // st was created for the batch (pooled batches of thy_run)
    void reset_counters();             // the per-run counters above, and the tuning samples

    ~Batch();
    int init(int capacity, int max_work, cudaStream_t stream);
    int attach(DevScenario *s);      // gives s a control slot
    int detach(DevScenario *s);
    // upload the member table and the work list (of the members with
    // selected[slot] != 0, all of them without a selection) and classify
    int update(const std::vector<char> *selected = nullptr);
    // (re)capture the `len`-step graph of `tiling` for the current capacity
    // (len 0: the full chunk, which becomes gexec)
    int capture(int len = 0);
    int use_tiling(const Tiling &t);  // switch graphs (capturing the tiling's graph if it has none)
    void drop_graphs();
    int rebuild();                    // update(), and capture() when there is no graph yet
    int initial_dt_of(DevScenario *s);   // initial dt of one member (phase 0 over its units only)
    // `len` steps (0 or more than `chunk`: the full chunk, one graph launch;
    // fewer: the 1-step graph launched len times) + control download
    // (synchronous); the tiling is the autotuner's pick, and a full timed
    // chunk is one of its samples
    int run_chunk(bool timed, int len = 0);
    // steps a member can take before its next event or its end, estimated
    // from its current dt (at least 1)
    static long long steps_to_event(const DevScenario &s);
    // the chunk length for `steps` steps: at most `chunk`, at least 1
    int chunk_for(long long steps) const;
    // the autotuner's key of the next chunk: this device, the deep and
    // general units per step estimated from each stepping member's last
    // chunk (members with status running; every member when all_members);
    // *known: each of them has been measured
    TuneKey tune_key(bool *known = nullptr, bool all_members = false) const;
    StepLaunch params() const;
    int reset_lists();               // classify again: after the host changed a member's state
};

// Single-scenario batches of thy_run, kept per device between runs with
// their buffers, stream and captured graphs, so that a run of a grid size the
// process has run before captures no graph.  A lease hands a batch with at
// least `max_work` work items to one caller at a time.
Batch *lease_run_batch(int device, int max_work, int *rc);
void return_run_batch(Batch *b, bool healthy);   // healthy = false: destroy it instead

int ensure_device();
int device_sm_count();
// the THY_ERR_* code of a scenario the controller stopped as failed
int failure_code(const ScenarioCtl &c);
// page-locked host blocks, reused across runs (engine.cu)
cudaError_t pinned_alloc(void **p, size_t bytes);
void pinned_free(void *p);

}  // namespace thy
