// Host engine of the B200 stepper: device state of a scenario, the batch
// (work list + CUDA graph of stepping kernels), the event-driven time loop
// of src/GPU/ShallowWater.cu:396-450 and the C ABI entry points thy_run /
// thy_session_* / thy_device_*.
//
// The time loop stays on the device: dt, the simulated time and the event
// checks live in a per-scenario control block updated by the controller
// launch that ends each step, so steps are launched in graph chunks with one host
// synchronisation per chunk instead of one blocking copy per step.  When an
// event is due (fault time, snapshot time, gauge time) the controller pauses
// the scenario; later launches of the chunk do nothing for it, and the host
// performs the event exactly at that step before resuming.
#include "engine.h"
#include "tuner.h"

#include <cuda.h>

#include <algorithm>
#include <chrono>
#include <cstdlib>
#include <condition_variable>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <cmath>
#include <cstdio>
#include <cstring>

namespace thy {

namespace {
thread_local char g_err[512] = "";
int g_device = 0;
bool g_configured[64] = {};
int g_sms[64] = {};
}  // namespace

void set_last_cuda_error(cudaError_t e, const char *what, const char *file, int line)
{
    snprintf(g_err, sizeof(g_err), "%s (%s) at %s:%d", cudaGetErrorString(e), what, file, line);
}

const char *last_error_text() { return g_err; }

int ensure_device()
{
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        cudaGetLastError();
        return THY_ERR_NO_DEVICE;
    }
    if (g_device >= n) return THY_ERR_INVALID;
    THY_CK(cudaSetDevice(g_device));
    if (!g_configured[g_device]) {
        THY_CK(configure_step_kernels());
        THY_CK(preload_output_kernels());
        THY_CK(preload_okada_kernels());
        // device buffers come from the stream-ordered default pool; freed
        // memory stays in the pool for the next scenario instead of going
        // back to the driver
        cudaMemPool_t pool;
        THY_CK(cudaDeviceGetDefaultMemPool(&pool, g_device));
        unsigned long long keep = ~0ull;
        THY_CK(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
        THY_CK(cudaDeviceGetAttribute(&g_sms[g_device], cudaDevAttrMultiProcessorCount, g_device));
        g_configured[g_device] = true;
    }
    return THY_OK;
}

int device_sm_count() { return g_sms[g_device] > 0 ? g_sms[g_device] : 148; }

int failure_code(const ScenarioCtl &c)
{
    if (c.errors & 2u) return THY_ERR_TIMEOUT;
    if (c.errors & 4u) return THY_ERR_CUDA;
    return THY_ERR_NONFINITE;
}

// Page-locked host blocks reused across runs.  Pinning and unpinning are
// driver calls that synchronise the device, and unpinning a block was seen to
// stall a run's release for over half a second; freed blocks are kept by
// power-of-two size class (up to kPinnedKeep bytes in all) and handed out
// again.  Blocks are portable: any device of the process may copy to them.
namespace {
constexpr size_t kPinnedKeep = (size_t)2 << 30;
std::mutex g_pin_mu;
std::multimap<size_t, void *> g_pin_free;          // size class -> free block
std::unordered_map<void *, size_t> g_pin_class;    // every block handed out -> its size class
size_t g_pin_kept = 0;
}  // namespace

cudaError_t pinned_alloc(void **p, size_t bytes)
{
    size_t cls = 4096;
    while (cls < bytes) cls <<= 1;
    {
        std::lock_guard<std::mutex> lk(g_pin_mu);
        auto it = g_pin_free.find(cls);
        if (it != g_pin_free.end()) {
            *p = it->second;
            g_pin_free.erase(it);
            g_pin_kept -= cls;
            g_pin_class[*p] = cls;
            return cudaSuccess;
        }
    }
    const cudaError_t e = cudaHostAlloc(p, cls, cudaHostAllocPortable);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lk(g_pin_mu);
    g_pin_class[*p] = cls;
    return cudaSuccess;
}

void pinned_free(void *p)
{
    if (!p) return;
    {
        std::lock_guard<std::mutex> lk(g_pin_mu);
        auto it = g_pin_class.find(p);
        if (it != g_pin_class.end()) {
            const size_t cls = it->second;
            g_pin_class.erase(it);
            if (g_pin_kept + cls <= kPinnedKeep) {
                g_pin_free.emplace(cls, p);
                g_pin_kept += cls;
                return;
            }
        }
    }
    cudaFreeHost(p);
}

static int round_up(int a, int b) { return (a + b - 1) / b * b; }

size_t scenario_bytes(int nx, int ny, bool has_faults)
{
    const size_t pitch = (size_t)round_up(nx, 32);
    size_t b = 10 * pitch * ny * sizeof(float);          // fields
    b += (size_t)(5 * ny + 1) * sizeof(float);           // row tables
    b += 3 * (size_t)nx * ny * sizeof(float);            // output staging
    b += 2 * (size_t)((nx + 2 * kTileX - 1) / kTileX) * ((ny + kTileY - 1) / kTileY) * (2 * sizeof(UnitSum) + 1 + sizeof(float));
    b += kNumMaps * sizeof(TmaMap) + (size_t)(ny + 1) * sizeof(float4);
    if (has_faults) b += (size_t)nx * ny * sizeof(double);
    return b + 4096 + kGaugeRing * sizeof(double);   // (gauges: 4 + 16 kGaugeRing + 8 bytes per point, not counted)
}

// ---------------------------------------------------------------------------
// DevScenario
// ---------------------------------------------------------------------------

DevScenario::DevScenario() = default;

DevScenario::~DevScenario()
{
    pipe.reset();   // joins the writer before the buffers go
    if (fields) cudaFreeAsync(fields, ast);
    if (rows) cudaFreeAsync(rows, ast);
    if (def) cudaFreeAsync(def, ast);
    if (maxbits) cudaFreeAsync(maxbits, ast);
    if (d_cells) cudaFreeAsync(d_cells, ast);
    if (d_gauge) cudaFreeAsync(d_gauge, ast);
    if (d_gring) cudaFreeAsync(d_gring, ast);
    if (d_gring_t) cudaFreeAsync(d_gring_t, ast);
    if (d_gminmax) cudaFreeAsync(d_gminmax, ast);
    if (d_out) cudaFreeAsync(d_out, ast);
    if (fault_times_d) cudaFreeAsync(fault_times_d, ast);
    if (usum) cudaFreeAsync(usum, ast);
    if (dry_age) cudaFreeAsync(dry_age, ast);
    if (gmax) cudaFreeAsync(gmax, ast);
    if (tmaps) cudaFreeAsync(tmaps, ast);
    if (rowpack) cudaFreeAsync(rowpack, ast);
}

int DevScenario::setup(const thy_problem *p, cudaStream_t st)
{
    if (!p || p->nx < 2 || p->ny < 2 || !p->h || !p->Hs || !p->area_cos || !p->dlon || !p->dlat || !p->lon || !p->lat)
        return THY_ERR_INVALID;
    ast = st;
    nx = p->nx;
    ny = p->ny;
    pitch = round_up(nx, 32);
    plane = (size_t)pitch * ny;
    if (plane >= (size_t)1 << 31) return THY_ERR_INVALID;   // cell offsets are 32-bit in the kernels
    const size_t n = (size_t)nx * ny;
    Hs = p->H;
    Qs = p->Q;
    Ts = p->T;
    Ls = p->L;
    Hmin = p->Hmin;
    t_end = p->t_end;
    save_nc = p->save_nc;
    save_ts = (p->npoints > 0) ? p->save_ts : -1.0;
    max_steps = p->max_steps;
    crop_flag = p->crop_flag;
    crop_value = p->crop_value;
    okada_flag = p->okada_flag;
    lon0 = p->lon[0];
    lat0 = p->lat[0];
    dlon = (p->lon[nx - 1] - p->lon[0]) / (nx - 1);
    dlat = (p->lat[ny - 1] - p->lat[0]) / (ny - 1);
    faults.assign(p->faults ? p->faults : (const double *)nullptr,
                  p->faults ? p->faults + 10 * (size_t)std::max(p->nfaults, 0) : nullptr);
    cells.assign(p->point_cell ? p->point_cell : (const int *)nullptr,
                 p->point_cell ? p->point_cell + std::max(p->npoints, 0) : nullptr);
    const int nf = (int)(faults.size() / 10);

    THY_CK(cudaMallocAsync(&fields, 10 * plane * sizeof(float), st));
    THY_CK(cudaMallocAsync(&rows, (size_t)(5 * ny + 1) * sizeof(float), st));
    THY_CK(cudaMallocAsync(&d_out, 3 * n * sizeof(float), st));
    if (nf > 0) {
        THY_CK(cudaMallocAsync(&def, n * sizeof(double), st));
        THY_CK(cudaMallocAsync(&maxbits, sizeof(unsigned int), st));
        THY_CK(cudaMallocAsync(&fault_times_d, nf * sizeof(double), st));
        std::vector<double> tf(nf);
        for (int i = 0; i < nf; i++) tf[i] = faults[10 * i];
        THY_CK(cudaMemcpyAsync(fault_times_d, tf.data(), nf * sizeof(double), cudaMemcpyHostToDevice, st));
        THY_CK(cudaStreamSynchronize(st));
    }
    if (!cells.empty()) {
        // gauge cells, the ring of device samples and the extremes of eta
        // (1e30 / -1e30 before the first sample; -9999 outside the grid)
        const size_t np = cells.size();
        THY_CK(cudaMallocAsync(&d_cells, np * sizeof(int), st));
        THY_CK(cudaMallocAsync(&d_gauge, 4 * np * sizeof(float), st));
        THY_CK(cudaMallocAsync(&d_gring, (size_t)kGaugeRing * 4 * np * sizeof(float), st));
        THY_CK(cudaMallocAsync(&d_gring_t, kGaugeRing * sizeof(double), st));
        THY_CK(cudaMallocAsync(&d_gminmax, np * sizeof(float2), st));
        THY_CK(cudaMemcpyAsync(d_cells, cells.data(), np * sizeof(int), cudaMemcpyHostToDevice, st));
        std::vector<float2> mm(np);
        for (size_t i = 0; i < np; i++) mm[i] = cells[i] < 0 ? make_float2(-9999.0f, -9999.0f) : make_float2(1e30f, -1e30f);
        THY_CK(cudaMemcpyAsync(d_gminmax, mm.data(), np * sizeof(float2), cudaMemcpyHostToDevice, st));
        THY_CK(cudaStreamSynchronize(st));
    }
    gauges_read = 0;

    // per-row metric terms: computed in FP64, stored once as FP32
    {
        std::vector<float> r((size_t)(5 * ny + 1));
        float *cosr = r.data(), *ilc = cosr + ny, *ar = ilc + ny, *dlo = ar + ny, *dla = dlo + ny + 1;
        for (int y = 0; y < ny; y++) {
            const double area = p->area_cos[2 * y], c = p->area_cos[2 * y + 1];
            cosr[y] = (float)c;
            ilc[y] = (float)(p->dlat[y] / c);
            ar[y] = (float)area;
            dla[y] = (float)p->dlat[y];
        }
        for (int y = 0; y <= ny; y++) dlo[y] = (float)p->dlon[y];
        std::vector<float4> pk((size_t)ny + 1);
        for (int y = 0; y <= ny; y++) {
            const bool cell = y < ny;
            pk[y] = make_float4(cell ? cosr[y] : 1.f, cell ? ilc[y] : 0.f, cell ? ar[y] : 1.f, dlo[y]);
        }
        THY_CK(cudaMallocAsync(&rowpack, pk.size() * sizeof(float4), st));
        THY_CK(cudaMemcpyAsync(rows, r.data(), r.size() * sizeof(float), cudaMemcpyHostToDevice, st));
        THY_CK(cudaMemcpyAsync(rowpack, pk.data(), pk.size() * sizeof(float4), cudaMemcpyHostToDevice, st));
        THY_CK(cudaStreamSynchronize(st));
        desc.rowpack = rowpack;
        desc.row.cosphi = rows;
        desc.row.ilcos = rows + ny;
        desc.row.area = rows + 2 * ny;
        desc.row.dlon = rows + 3 * ny;
        desc.row.dlat = rows + 4 * ny + 1;
    }

    desc.nx = nx;
    desc.ny = ny;
    desc.pitch = pitch;
    desc.periodic = (std::fabs(p->border_left - 2.0) < 2.220446049250313e-16) &&
                    (std::fabs(p->border_right - 2.0) < 2.220446049250313e-16);
    desc.x_org = tile_origin(nx, desc.periodic != 0, p->sponge_left, p->sponge_right);
    desc.tiles_x = (nx - desc.x_org + kTileX - 1) / kTileX;
    desc.tiles_y = (ny + kTileY - 1) / kTileY;
    desc.ntiles = desc.tiles_x * desc.tiles_y;
    THY_CK(cudaMallocAsync(&usum, 4 * (size_t)desc.ntiles * sizeof(UnitSum), st));
    THY_CK(cudaMallocAsync(&dry_age, 2 * (size_t)desc.ntiles, st));
    THY_CK(cudaMallocAsync(&gmax, 2 * (size_t)desc.ntiles * sizeof(float), st));
    desc.usum[0] = usum;
    desc.usum[1] = usum + 2 * desc.ntiles;
    desc.dry_age = dry_age;
    desc.unit_gmax = gmax;
    desc.b_up = (float)p->border_up;
    desc.b_low = (float)p->border_low;
    desc.b_left = (float)p->border_left;
    desc.b_right = (float)p->border_right;
    desc.sp_up = p->sponge_up;
    desc.sp_low = p->sponge_low;
    desc.sp_left = p->sponge_left;
    desc.sp_right = p->sponge_right;
    desc.cfl = (float)p->cfl;
    desc.eps_h = (float)p->eps_h;
    desc.eps_h64 = p->eps_h;
    desc.hpos = (float)p->hpos;
    desc.cvis = (float)p->cvis;
    desc.mf0 = (float)p->mf0;
    desc.vmax = (float)p->vmax;
    desc.dif_at = (float)p->dif_at;
    desc.sea = 0.f;
    desc.gauge_cells = d_cells;
    desc.ngauges = (int)cells.size();
    desc.gauge_ring = d_gring;
    desc.gauge_ring_t = d_gring_t;
    desc.gauge_minmax = d_gminmax;
    desc.Hs = Hs;
    desc.Qs = Qs;
    for (int k = 0; k < 2; k++) {
        desc.eta[k] = fields + (0 + k) * plane;
        desc.qx[k] = fields + (2 + k) * plane;
        desc.qy[k] = fields + (4 + k) * plane;
    }
    desc.dep = fields + 6 * plane;
    desc.eta_max = fields + 7 * plane;
    desc.arr = fields + 8 * plane;
    desc.eta_ini = fields + 9 * plane;
    if (const int rc = encode_tensor_maps(st)) return rc;

    // dimensionless double state -> FP32 device state
    {
        double *tmp = nullptr;
        const bool hasq = p->qx && p->qy;
        THY_CK(cudaMallocAsync(&tmp, (hasq ? 4 : 2) * n * sizeof(double), st));
        THY_CK(cudaMemcpyAsync(tmp, p->h, n * sizeof(double), cudaMemcpyHostToDevice, st));
        THY_CK(cudaMemcpyAsync(tmp + n, p->Hs, n * sizeof(double), cudaMemcpyHostToDevice, st));
        if (hasq) {
            THY_CK(cudaMemcpyAsync(tmp + 2 * n, p->qx, n * sizeof(double), cudaMemcpyHostToDevice, st));
            THY_CK(cudaMemcpyAsync(tmp + 3 * n, p->qy, n * sizeof(double), cudaMemcpyHostToDevice, st));
        }
        launch_init_state(&desc, nullptr, tmp, tmp + n, hasq ? tmp + 2 * n : nullptr, hasq ? tmp + 3 * n : nullptr, Hmin, st);
        THY_CK(cudaGetLastError());
        THY_CK(invalidate_tile_minima(st));
        THY_CK(cudaStreamSynchronize(st));
        cudaFreeAsync(tmp, st);
    }

    std::memset(&hctl, 0, sizeof(hctl));
    hctl.t = 0.0;
    hctl.dt = 0.0;
    hctl.t_end = t_end;
    hctl.save_nc = save_nc;
    hctl.next_nc = 0.0;
    hctl.save_ts = save_ts;
    hctl.next_ts = 0.0;
    hctl.T = Ts;
    hctl.step = 0;
    hctl.max_steps = max_steps;
    hctl.status = kRunning;
    hctl.parity = 0;
    hctl.fault_next = 0;
    hctl.jumping = 0;
    hctl.nfaults = nf;
    hctl.fault_times = fault_times_d;
    hctl.dt_bits = 0x7f7fffffu;
    hctl.tiles_done = 0;
    hctl.errors = 0;
    return THY_OK;
}

// 2D tensor maps of the field planes for the deep-water kernels' TMA
// staging: state planes boxed kStageW x kStageRows, diagnostics kTileX x
// kHalfRows, zero fill outside the grid.  A grid with fewer than three tiles
// in either direction has no deep tile and gets no maps.
// The driver's encoder is looked up through the runtime, so the library has
// no link-time dependency on libcuda.
using EncodeTiledFn = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                   const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_tiled_fn()
{
    static EncodeTiledFn fn = nullptr;
    if (!fn) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(p);
        else
            cudaGetLastError();
    }
    return fn;
}

int DevScenario::encode_tensor_maps(cudaStream_t st)
{
    desc.tmap = nullptr;
    if (desc.tiles_x < 3 || desc.tiles_y < 3) return THY_OK;
    static_assert(sizeof(TmaMap) == sizeof(CUtensorMap), "opaque map size");
    const EncodeTiledFn encode = encode_tiled_fn();
    if (!encode) {
        set_last_cuda_error(cudaErrorSymbolNotFound, "cuTensorMapEncodeTiled entry point", __FILE__, __LINE__);
        return THY_ERR_CUDA;
    }
    CUtensorMap h[kNumMaps];
    float *base[kNumMaps] = {desc.eta[0], desc.eta[1], desc.qx[0], desc.qx[1], desc.qy[0], desc.qy[1],
                             desc.dep, desc.eta_max, desc.arr, desc.eta_ini};
    for (int k = 0; k < kNumMaps; k++) {
        const bool diag = k >= kMapEtaMax;
        const cuuint64_t dims[2] = {(cuuint64_t)nx, (cuuint64_t)ny};
        const cuuint64_t strides[1] = {(cuuint64_t)pitch * sizeof(float)};
        const cuuint32_t box[2] = {(cuuint32_t)(diag ? kTileX : kStageW), (cuuint32_t)(diag ? kHalfRows : kStageRows)};
        const cuuint32_t estr[2] = {1, 1};
        const CUresult r = encode(&h[k], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, base[k], dims, strides, box,
                                                  estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                                  CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                                                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS) {
            char what[64];
            snprintf(what, sizeof(what), "cuTensorMapEncodeTiled returned %d", (int)r);
            set_last_cuda_error(cudaErrorInvalidValue, what, __FILE__, __LINE__);
            return THY_ERR_CUDA;
        }
    }
    THY_CK(cudaMallocAsync(&tmaps, kNumMaps * sizeof(TmaMap), st));
    THY_CK(cudaMemcpyAsync(tmaps, h, kNumMaps * sizeof(TmaMap), cudaMemcpyHostToDevice, st));
    THY_CK(cudaStreamSynchronize(st));
    desc.tmap = tmaps;
    return THY_OK;
}

// The state changed outside phase 1: no unit counts as deep or dry until
// phase 1 has measured the depth summaries again (all-ones bytes are NaN
// floats) and the dry count starts again.
cudaError_t DevScenario::invalidate_tile_minima(cudaStream_t st)
{
    cudaError_t e = cudaMemsetAsync(usum, 0xff, 4 * (size_t)desc.ntiles * sizeof(UnitSum), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(dry_age, 0, 2 * (size_t)desc.ntiles, st);
    if (e == cudaSuccess) {
        // the depths changed (set-up, a fault): their steps per unit again
        launch_unit_gmax(&desc, st);
        e = cudaGetLastError();
    }
    return e;
}

int DevScenario::upload_ctl(cudaStream_t st)
{
    THY_CK(cudaMemcpyAsync(ctl, &hctl, sizeof(ScenarioCtl), cudaMemcpyHostToDevice, st));
    return THY_OK;
}

int DevScenario::download_ctl(cudaStream_t st)
{
    THY_CK(cudaMemcpyAsync(&hctl, ctl, sizeof(ScenarioCtl), cudaMemcpyDeviceToHost, st));
    return THY_OK;
}

// src/GPU/ShallowWater.cu:125-147: every fault whose time has been reached
int DevScenario::apply_due_faults(cudaStream_t st)
{
    const int nf = (int)(faults.size() / 10);
    while (hctl.fault_next < nf && hctl.t * Ts >= faults[10 * hctl.fault_next]) {
        const double *f = &faults[10 * hctl.fault_next];
        OkadaFault of{f[1], f[2], f[3], f[4], f[5], f[6], f[7], f[8], f[9]};
        launch_okada(&desc, def, lon0, dlon, lat0, dlat, of, Hs, st);
        if (crop_flag == 1) launch_absmax(def, (long long)nx * ny, maxbits, st);
        // the apply kernel reads the parity from the control block
        THY_CK(cudaMemcpyAsync(ctl, &hctl, sizeof(ScenarioCtl), cudaMemcpyHostToDevice, st));
        launch_apply_deformation(&desc, def, crop_flag, crop_value, maxbits, st);
        THY_CK(cudaGetLastError());
        THY_CK(invalidate_tile_minima(st));
        hctl.fault_next++;
    }
    return THY_OK;
}

int DevScenario::extract(int field, float *host_out, cudaStream_t st)
{
    const size_t n = (size_t)nx * ny;
    launch_extract(&desc, field, hctl.parity, d_out, Hs, Qs, Hmin, st);
    THY_CK(cudaGetLastError());
    THY_CK(cudaMemcpyAsync(host_out, d_out, n * sizeof(float), cudaMemcpyDeviceToHost, st));
    THY_CK(cudaStreamSynchronize(st));
    return THY_OK;
}

// ---------------------------------------------------------------------------
// Asynchronous delivery of snapshots and gauge samples.  The reference
// extracts, copies (blocking) and writes each snapshot inside its time loop
// (src/GPU/ShallowWater.cu:398-421), so the GPU waits for the host.  Here
// the extraction kernels go on the stepping stream (they read exactly the
// state of that step, before the next steps are enqueued), the copy into a
// page-locked host slot goes on a copy stream, and one writer thread hands
// the slots to the caller's callbacks in event order while the GPU steps
// on.  Snapshots use two slots of 3 fields (the first is d_out), gauge
// samples eight slots of 4 floats per gauge; a producer that finds no free
// slot waits for the writer.
// ---------------------------------------------------------------------------
class OutputPipe {
public:
    static constexpr int kSnapSlots = 2, kTsSlots = 8;

    ~OutputPipe()
    {
        drain();
        {
            std::lock_guard<std::mutex> lk(m_);
            stop_ = true;
        }
        cv_.notify_all();
        if (writer_.joinable()) writer_.join();
        for (int k = 0; k < kSnapSlots; k++) {
            if (snap_ready_[k]) cudaEventDestroy(snap_ready_[k]);
            if (snap_copied_[k]) cudaEventDestroy(snap_copied_[k]);
        }
        for (int k = 0; k < kTsSlots; k++) {
            if (ts_ready_[k]) cudaEventDestroy(ts_ready_[k]);
            if (ts_copied_[k]) cudaEventDestroy(ts_copied_[k]);
        }
        if (d_snap1_) cudaFreeAsync(d_snap1_, alloc_st_);
        if (d_ts_) cudaFreeAsync(d_ts_, alloc_st_);
        pinned_free(h_snap_);
        pinned_free(h_ts_);
        if (copy_st_) cudaStreamDestroy(copy_st_);
    }

    int init(DevScenario *s, const thy_outputs *o, cudaStream_t st)
    {
        s_ = s;
        o_ = o;
        alloc_st_ = st;
        n_ = (size_t)s->nx * s->ny;
        np_ = (int)s->cells.size();
        THY_CK(cudaStreamCreateWithFlags(&copy_st_, cudaStreamNonBlocking));
        if (o && o->on_snapshot && s->save_nc >= 0.0) {
            THY_CK(cudaMallocAsync(&d_snap1_, 3 * n_ * sizeof(float), st));
            THY_CK(pinned_alloc(reinterpret_cast<void **>(&h_snap_), kSnapSlots * 3 * n_ * sizeof(float)));
            for (int k = 0; k < kSnapSlots; k++) {
                THY_CK(cudaEventCreateWithFlags(&snap_ready_[k], cudaEventDisableTiming));
                THY_CK(cudaEventCreateWithFlags(&snap_copied_[k], cudaEventDisableTiming));
            }
        }
        if (np_ > 0) {
            THY_CK(cudaMallocAsync(&d_ts_, kTsSlots * 4 * (size_t)np_ * sizeof(float), st));
            THY_CK(pinned_alloc(reinterpret_cast<void **>(&h_ts_), kTsSlots * 4 * (size_t)np_ * sizeof(float)));
            for (int k = 0; k < kTsSlots; k++) {
                THY_CK(cudaEventCreateWithFlags(&ts_ready_[k], cudaEventDisableTiming));
                THY_CK(cudaEventCreateWithFlags(&ts_copied_[k], cudaEventDisableTiming));
            }
        }
        writer_ = std::thread([this] { run(); });
        return THY_OK;
    }

    bool snapshots_on() const { return h_snap_ != nullptr; }

    // Extracts eta, ux, uy of the current state into a free slot and queues its delivery.
    int snapshot(int index, double time_s, cudaStream_t st)
    {
        const int k = acquire(snap_busy_, kSnapSlots);
        float *d = (k == 0) ? s_->d_out : d_snap1_;
        for (int f = 0; f < 3; f++)
            launch_extract(&s_->desc, kFieldEta + f, s_->hctl.parity, d + f * n_, s_->Hs, s_->Qs, s_->Hmin, st);
        THY_CK(cudaGetLastError());
        THY_CK(cudaEventRecord(snap_ready_[k], st));
        THY_CK(cudaStreamWaitEvent(copy_st_, snap_ready_[k], 0));
        THY_CK(cudaMemcpyAsync(h_snap_ + k * 3 * n_, d, 3 * n_ * sizeof(float), cudaMemcpyDeviceToHost, copy_st_));
        THY_CK(cudaEventRecord(snap_copied_[k], copy_st_));
        push(Job{0, index, time_s, k, {}});
        return THY_OK;
    }

    // Queues the delivery of a gauge sample the device already took (4
    // floats per gauge, copied here).
    void gauges_taken(int index, double time_s, const float *g4)
    {
        Job j{2, index, time_s, -1};
        j.data.assign(g4, g4 + 4 * (size_t)np_);
        push(j);
    }

    // Samples the gauges of the current state into a free slot and queues its delivery.
    int gauges(int index, double time_s, cudaStream_t st)
    {
        const int k = acquire(ts_busy_, kTsSlots);
        float *d = d_ts_ + k * 4 * (size_t)np_;
        launch_gauges(&s_->desc, s_->hctl.parity, s_->d_cells, np_, d, true, st);
        THY_CK(cudaGetLastError());
        THY_CK(cudaEventRecord(ts_ready_[k], st));
        THY_CK(cudaStreamWaitEvent(copy_st_, ts_ready_[k], 0));
        THY_CK(cudaMemcpyAsync(h_ts_ + k * 4 * (size_t)np_, d, 4 * (size_t)np_ * sizeof(float),
                               cudaMemcpyDeviceToHost, copy_st_));
        THY_CK(cudaEventRecord(ts_copied_[k], copy_st_));
        push(Job{1, index, time_s, k, {}});
        return THY_OK;
    }

    // Waits until every queued delivery has been handed to the callbacks.
    int drain()
    {
        std::unique_lock<std::mutex> lk(m_);
        cv_.wait(lk, [this] { return q_.empty() && !busy_; });
        return error_;
    }

private:
    struct Job {
        int kind;     // 0 snapshot, 1 gauges in a slot, 2 gauges in `data`
        int index;
        double time;
        int slot;
        std::vector<float> data;
    };

    int acquire(bool *busy, int n)
    {
        std::unique_lock<std::mutex> lk(m_);
        for (;;) {
            for (int k = 0; k < n; k++)
                if (!busy[k]) {
                    busy[k] = true;
                    return k;
                }
            cv_.wait(lk);
        }
    }

    void push(Job j)
    {
        {
            std::lock_guard<std::mutex> lk(m_);
            q_.push_back(std::move(j));
        }
        cv_.notify_all();
    }

    void run()
    {
        for (;;) {
            Job j;
            {
                std::unique_lock<std::mutex> lk(m_);
                cv_.wait(lk, [this] { return stop_ || !q_.empty(); });
                if (q_.empty()) return;
                j = std::move(q_.front());
                q_.pop_front();
                busy_ = true;
            }
            deliver(j);
            {
                std::lock_guard<std::mutex> lk(m_);
                if (j.kind < 2) (j.kind == 0 ? snap_busy_ : ts_busy_)[j.slot] = false;
                busy_ = false;
            }
            cv_.notify_all();
        }
    }

    void deliver(const Job &j)
    {
        if (j.kind == 0) {
            if (cudaEventSynchronize(snap_copied_[j.slot]) != cudaSuccess) {
                set_error();
                return;
            }
            const float *h = h_snap_ + j.slot * 3 * n_;
            o_->on_snapshot(o_->user, j.index, j.time, h, h + n_, h + 2 * n_);
            return;
        }
        const float *g;
        if (j.kind == 1) {
            if (cudaEventSynchronize(ts_copied_[j.slot]) != cudaSuccess) {
                set_error();
                return;
            }
            g = h_ts_ + j.slot * 4 * (size_t)np_;
        } else {
            g = j.data.data();
        }
        // (the extremes of eta are folded on the device with every sample)
        std::vector<float> e(np_), ux(np_), uy(np_);
        for (int i = 0; i < np_; i++) {
            e[i] = g[4 * i];
            ux[i] = g[4 * i + 1];
            uy[i] = g[4 * i + 2];
        }
        if (o_ && o_->on_series) o_->on_series(o_->user, j.index, j.time, e.data(), ux.data(), uy.data());
    }

    void set_error()
    {
        cudaGetLastError();
        std::lock_guard<std::mutex> lk(m_);
        error_ = THY_ERR_CUDA;
    }

    DevScenario *s_ = nullptr;
    const thy_outputs *o_ = nullptr;
    cudaStream_t alloc_st_ = nullptr, copy_st_ = nullptr;
    size_t n_ = 0;
    int np_ = 0;
    float *d_snap1_ = nullptr, *d_ts_ = nullptr, *h_snap_ = nullptr, *h_ts_ = nullptr;
    cudaEvent_t snap_ready_[kSnapSlots] = {}, snap_copied_[kSnapSlots] = {};
    cudaEvent_t ts_ready_[kTsSlots] = {}, ts_copied_[kTsSlots] = {};
    bool snap_busy_[kSnapSlots] = {}, ts_busy_[kTsSlots] = {};
    std::thread writer_;
    std::mutex m_;
    std::condition_variable cv_;
    std::deque<Job> q_;
    bool stop_ = false, busy_ = false;
    int error_ = THY_OK;
};

int DevScenario::open_outputs(const thy_outputs *o, cudaStream_t st)
{
    if (pipe) return THY_OK;
    if (!o || (!(o->on_snapshot && save_nc >= 0.0) && cells.empty())) return THY_OK;
    pipe.reset(new OutputPipe());
    return pipe->init(this, o, st);
}

int DevScenario::snapshot(const thy_outputs *o, cudaStream_t st)
{
    int rc;
    if (o && o->on_snapshot) {
        if ((rc = open_outputs(o, st))) return rc;
        if (pipe && pipe->snapshots_on() && (rc = pipe->snapshot(snapshots, hctl.t * Ts, st))) return rc;
    }
    snapshots++;
    return THY_OK;
}

int DevScenario::sample_gauges(const thy_outputs *o, cudaStream_t st)
{
    int rc;
    if (!cells.empty()) {
        if ((rc = open_outputs(o, st))) return rc;
        if (pipe && (rc = pipe->gauges(series, hctl.t * Ts, st))) return rc;
    }
    series++;
    return THY_OK;
}

// Gauge samples the step controller took since the last call (at most
// kGaugeRing: the host reads them after every chunk), handed to the output
// pipe in time order, before any event the host performs at the chunk's end.
int DevScenario::read_device_gauges(const thy_outputs *o, cudaStream_t st)
{
    const unsigned n = hctl.gauge_count - gauges_read;
    if (n == 0 || cells.empty()) return THY_OK;
    if (n > (unsigned)kGaugeRing) return THY_ERR_INVALID;   // more samples than the ring holds: not read in time
    const size_t np = cells.size();
    std::vector<float> ring((size_t)kGaugeRing * 4 * np);
    double ring_t[kGaugeRing];
    THY_CK(cudaMemcpyAsync(ring.data(), d_gring, ring.size() * sizeof(float), cudaMemcpyDeviceToHost, st));
    THY_CK(cudaMemcpyAsync(ring_t, d_gring_t, sizeof(ring_t), cudaMemcpyDeviceToHost, st));
    THY_CK(cudaStreamSynchronize(st));
    int rc;
    if ((rc = open_outputs(o, st))) return rc;
    for (unsigned k = gauges_read; k != hctl.gauge_count; k++) {
        const unsigned slot = k % kGaugeRing;
        if (pipe) pipe->gauges_taken(series, ring_t[slot], ring.data() + (size_t)slot * 4 * np);
        series++;
    }
    gauges_read = hctl.gauge_count;
    return THY_OK;
}

int DevScenario::finish(const thy_outputs *o, cudaStream_t st)
{
    int rc;
    // every snapshot and gauge sample is delivered before the final fields
    if (pipe && (rc = pipe->drain())) return rc;
    if (!o) return THY_OK;
    if (o->max_height && (rc = extract(kFieldMaxHeight, o->max_height, st))) return rc;
    if (o->arrival && (rc = extract(kFieldArrival, o->arrival, st))) return rc;
    if (o->deformed_bathy && (rc = extract(kFieldDeformed, o->deformed_bathy, st))) return rc;
    if (o->eta && (rc = extract(kFieldEta, o->eta, st))) return rc;
    if (o->ux && (rc = extract(kFieldUx, o->ux, st))) return rc;
    if (o->uy && (rc = extract(kFieldUy, o->uy, st))) return rc;
    const int np = (int)cells.size();
    if (np > 0 && (o->series_min || o->series_max || o->series_bathy)) {
        std::vector<float> g(4 * (size_t)np);
        std::vector<float2> mm(np);
        // the depths of the final state (not a sample: no fold) and the extremes
        launch_gauges(&desc, hctl.parity, d_cells, np, d_gauge, false, st);
        THY_CK(cudaGetLastError());
        THY_CK(cudaMemcpyAsync(g.data(), d_gauge, g.size() * sizeof(float), cudaMemcpyDeviceToHost, st));
        THY_CK(cudaMemcpyAsync(mm.data(), d_gminmax, np * sizeof(float2), cudaMemcpyDeviceToHost, st));
        THY_CK(cudaStreamSynchronize(st));
        for (int i = 0; i < np; i++) {
            if (o->series_min) o->series_min[i] = mm[i].x;
            if (o->series_max) o->series_max[i] = mm[i].y;
            if (o->series_bathy) o->series_bathy[i] = g[4 * i + 3];
        }
    }
    return THY_OK;
}

// ---------------------------------------------------------------------------
// Batch
// ---------------------------------------------------------------------------

Batch::~Batch()
{
    drop_graphs();
    if (d_table) cudaFreeAsync(d_table, st);
    if (d_work) cudaFreeAsync(d_work, st);
    if (d_nwork) cudaFreeAsync(d_nwork, st);
    if (d_work0) cudaFreeAsync(d_work0, st);
    if (d_nwork0) cudaFreeAsync(d_nwork0, st);
    if (d_lists) cudaFreeAsync(d_lists, st);
    if (d_claims) cudaFreeAsync(d_claims, st);
    if (d_ctl) cudaFreeAsync(d_ctl, st);
    pinned_free(h_ctl);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (ev_fork) cudaEventDestroy(ev_fork);
    if (ev_join) cudaEventDestroy(ev_join);
    if (st_side) cudaStreamDestroy(st_side);
    if (owns_stream && st) cudaStreamDestroy(st);
}

void Batch::reset_counters()
{
    device_ms = 0;
    launches = 0;
    chunks_run = 0;
    captures = 0;
    capture_s = 0;
    tune_samples = 0;
}

namespace {
struct RunPool {
    std::mutex mu;
    std::vector<std::pair<Batch *, bool>> batches;   // (batch, leased)
};
// never destroyed: batches still held at process exit are left to the driver
RunPool &run_pool()
{
    static RunPool *p = new RunPool();
    return *p;
}
constexpr size_t kRunPoolMax = 8;   // idle batches kept per process
}  // namespace

Batch *lease_run_batch(int device, int max_work, int *rc)
{
    *rc = THY_OK;
    RunPool &P = run_pool();
    {
        std::lock_guard<std::mutex> g(P.mu);
        // the smallest idle batch of this device that holds the work, within
        // 16x of it (grids follow the capacity)
        int best = -1;
        for (int i = 0; i < (int)P.batches.size(); i++) {
            Batch *b = P.batches[i].first;
            if (P.batches[i].second || b->device != device || b->work_capacity < max_work ||
                b->work_capacity > 16 * std::max(max_work, 64))
                continue;
            if (best < 0 || b->work_capacity < P.batches[best].first->work_capacity) best = i;
        }
        if (best >= 0) {
            P.batches[best].second = true;
            Batch *b = P.batches[best].first;
            b->reset_counters();
            return b;
        }
    }
    Batch *b = new Batch();
    cudaStream_t st = nullptr;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        delete b;
        *rc = THY_ERR_CUDA;
        return nullptr;
    }
    b->owns_stream = true;
    if ((*rc = b->init(1, max_work, st))) {
        b->st = st;
        delete b;
        return nullptr;
    }
    std::lock_guard<std::mutex> g(P.mu);
    P.batches.emplace_back(b, true);
    return b;
}

void return_run_batch(Batch *b, bool healthy)
{
    if (!b) return;
    RunPool &P = run_pool();
    Batch *drop = nullptr;
    {
        std::lock_guard<std::mutex> g(P.mu);
        for (size_t i = 0; i < P.batches.size(); i++)
            if (P.batches[i].first == b) {
                if (!healthy) {
                    P.batches.erase(P.batches.begin() + i);
                    drop = b;
                } else {
                    P.batches[i].second = false;
                }
                break;
            }
        if (!drop) {
            // keep at most kRunPoolMax idle batches: drop the oldest idle one
            size_t idle = 0;
            for (auto &e : P.batches) idle += e.second ? 0 : 1;
            if (idle > kRunPoolMax)
                for (size_t i = 0; i < P.batches.size(); i++)
                    if (!P.batches[i].second) {
                        drop = P.batches[i].first;
                        P.batches.erase(P.batches.begin() + i);
                        break;
                    }
        }
    }
    if (drop) {
        cudaStreamSynchronize(drop->st);
        delete drop;
    }
}

int Batch::init(int cap, int max_work, cudaStream_t stream)
{
    capacity = cap;
    work_capacity = max_work;
    st = stream;
    THY_CK(cudaGetDevice(&device));
    THY_CK(cudaMallocAsync(&d_table, cap * sizeof(ScenarioDev), st));
    THY_CK(cudaMallocAsync(&d_ctl, cap * sizeof(ScenarioCtl), st));
    THY_CK(pinned_alloc(reinterpret_cast<void **>(&h_ctl), cap * sizeof(ScenarioCtl)));
    THY_CK(cudaMallocAsync(&d_work, std::max(max_work, 1) * sizeof(int2), st));
    THY_CK(cudaMallocAsync(&d_nwork, sizeof(int), st));
    THY_CK(cudaMallocAsync(&d_work0, std::max(max_work, 1) * sizeof(int2), st));
    THY_CK(cudaMallocAsync(&d_nwork0, sizeof(int), st));
    THY_CK(cudaMallocAsync(&d_lists, (2 + 4 * (size_t)std::max(max_work, 1)) * sizeof(int), st));
    THY_CK(cudaMemsetAsync(d_lists, 0, 2 * sizeof(int), st));
    THY_CK(cudaMallocAsync(&d_claims, 4 * sizeof(int), st));
    THY_CK(cudaMemsetAsync(d_claims, 0, 4 * sizeof(int), st));
    THY_CK(cudaEventCreate(&ev0));
    THY_CK(cudaEventCreate(&ev1));
    THY_CK(cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming));
    THY_CK(cudaEventCreateWithFlags(&ev_join, cudaEventDisableTiming));
    THY_CK(cudaStreamCreateWithFlags(&st_side, cudaStreamNonBlocking));
    std::vector<ScenarioCtl> z(cap);
    for (auto &c : z) { std::memset(&c, 0, sizeof(c)); c.status = kIdle; }
    THY_CK(cudaMemcpyAsync(d_ctl, z.data(), cap * sizeof(ScenarioCtl), cudaMemcpyHostToDevice, st));
    THY_CK(cudaStreamSynchronize(st));
    members.assign(cap, nullptr);
    return THY_OK;
}

int Batch::attach(DevScenario *s)
{
    for (int i = 0; i < capacity; i++) {
        if (!members[i]) {
            members[i] = s;
            s->ctl = d_ctl + i;
            s->desc.ctl = s->ctl;
            return THY_OK;
        }
    }
    return THY_ERR_BUDGET;
}

int Batch::detach(DevScenario *s)
{
    for (int i = 0; i < capacity; i++)
        if (members[i] == s) {
            members[i] = nullptr;
            ScenarioCtl z;
            std::memset(&z, 0, sizeof(z));
            z.status = kIdle;
            THY_CK(cudaMemcpyAsync(d_ctl + i, &z, sizeof(z), cudaMemcpyHostToDevice, st));
            s->ctl = nullptr;
        }
    return THY_OK;
}

int Batch::update(const std::vector<char> *selected)
{
    std::vector<ScenarioDev> table(capacity);
    std::vector<int2> work;
    for (int i = 0; i < capacity; i++) {
        if (!members[i]) continue;
        table[i] = members[i]->desc;
        if (selected && !(*selected)[i]) continue;
        for (int t = 0; t < members[i]->desc.ntiles; t++) work.push_back(make_int2(i, t));
    }
    if ((int)work.size() > work_capacity) {
        // the captured graph holds the list pointers: grow, then recapture
        cudaFreeAsync(d_work, st);
        cudaFreeAsync(d_work0, st);
        cudaFreeAsync(d_lists, st);
        d_lists = nullptr;
        work_capacity = (int)work.size();
        THY_CK(cudaMallocAsync(&d_work, work_capacity * sizeof(int2), st));
        THY_CK(cudaMallocAsync(&d_work0, work_capacity * sizeof(int2), st));
        THY_CK(cudaMallocAsync(&d_lists, (2 + 4 * (size_t)work_capacity) * sizeof(int), st));
        drop_graphs();
    }
    nwork = (int)work.size();
    THY_CK(cudaMemcpyAsync(d_table, table.data(), capacity * sizeof(ScenarioDev), cudaMemcpyHostToDevice, st));
    if (nwork) THY_CK(cudaMemcpyAsync(d_work, work.data(), nwork * sizeof(int2), cudaMemcpyHostToDevice, st));
    THY_CK(cudaMemcpyAsync(d_nwork, &nwork, sizeof(int), cudaMemcpyHostToDevice, st));
    THY_CK(cudaStreamSynchronize(st));
    return reset_lists();
}

void Batch::drop_graphs()
{
    for (auto &g : graphs) cudaGraphExecDestroy(g.exec);
    graphs.clear();
    gexec = nullptr;
}

int Batch::use_tiling(const Tiling &t)
{
    if (gexec && t == tiling) return THY_OK;
    tiling = t;
    for (auto &g : graphs)
        if (g.tiling == t && g.len == chunk) {
            gexec = g.exec;
            return THY_OK;
        }
    return capture();
}

// Grids depend on the work-list capacity and the tiling only, so a graph
// survives changes of the member set (the kernels read the table and the
// lists from device memory).
int Batch::capture(int len)
{
    if (len <= 0 || len > chunk) len = chunk;
    const auto t_cap = std::chrono::steady_clock::now();
    for (size_t i = 0; i < graphs.size(); i++)
        if (graphs[i].tiling == tiling && graphs[i].len == len) {
            if (graphs[i].exec == gexec) gexec = nullptr;
            cudaGraphExecDestroy(graphs[i].exec);
            graphs.erase(graphs.begin() + i);
            break;
        }
    if (len == chunk) gexec = nullptr;
    // Each phase's general and deep-water kernels step disjoint tiles and
    // share only atomically updated scenario fields, so they are two
    // branches of the graph: the deep tiles fill the SMs the general
    // kernel's last wave leaves idle.
    const StepLaunch L = params();
    cudaGraph_t g;
    cudaGraphExec_t exec = nullptr;
    THY_CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    for (int k = 0; k < len; k++) {
        for (int ph = 0; ph < 2; ph++) {
            THY_CK(cudaEventRecord(ev_fork, st));
            THY_CK(cudaStreamWaitEvent(st_side, ev_fork, 0));
            launch_step_kernel(3 * ph + 1, L, st);        // general
            launch_step_kernel(3 * ph, L, st_side);       // deep
            THY_CK(cudaEventRecord(ev_join, st_side));
            THY_CK(cudaStreamWaitEvent(st, ev_join, 0));
            if (ph == 0) launch_step_kernel(2, L, st);   // classification for phase 2 and the next phase 1
        }
        launch_step_kernel(5, L, st);                     // controller
    }
    THY_CK(cudaStreamEndCapture(st, &g));
    cudaError_t e = cudaGraphInstantiate(&exec, g, 0);
    cudaGraphDestroy(g);
    THY_CK(e);
    graphs.push_back(Graph{tiling, len, exec});
    if (len == chunk) gexec = exec;
    captures++;
    capture_s += std::chrono::duration<double>(std::chrono::steady_clock::now() - t_cap).count();
    return THY_OK;
}

long long Batch::steps_to_event(const DevScenario &s)
{
    const ScenarioCtl &c = s.hctl;
    double horizon = c.t_end;
    if (c.save_nc >= 0.0) horizon = std::min(horizon, c.next_nc);
    // (gauge times do not: the controller samples the gauges on the device)
    const int nf = (int)(s.faults.size() / 10);
    if (c.fault_next < nf) horizon = std::min(horizon, s.faults[10 * c.fault_next] / s.Ts);
    long long n = (c.dt > 0.0) ? (long long)std::ceil((horizon - c.t) / c.dt) : 1;
    if (c.max_steps >= 0) n = std::min(n, c.max_steps - c.step);
    return std::max(1ll, n);
}

int Batch::chunk_for(long long steps) const { return (int)std::max(1ll, std::min<long long>(steps, chunk)); }

int Batch::rebuild()
{
    int rc;
    if ((rc = update())) return rc;
    // the graphs of the tiling the first chunk will take (the tuner's pick for
    // the work now attached), a full chunk and one step, so that no capture
    // falls into the time loop of a run whose work needs no tuning
    bool sampling = false, known = false;
    if ((rc = use_tiling(tuner_pick(tune_key(&known), &sampling)))) return rc;
    for (const auto &g : graphs)
        if (g.tiling == tiling && g.len == 1) return THY_OK;
    return capture(1);
}

StepLaunch Batch::params() const
{
    StepLaunch L;
    L.scen = d_table;
    L.work = d_work;
    L.nwork = d_nwork;
    L.lists = d_lists;
    L.claims = d_claims;
    L.cap = 2 * work_capacity;   // lists hold work units (two per work-list entry)
    L.tiling = tiling;
    // general kernel: persistent, one wave of warps that claim their tasks
    // (4 strips x row groups per unit; 4 warps a CTA), no more CTAs than the
    // tasks of a full list; deep kernels: persistent, one wave
    const int sms = device_sm_count();
    L.grid = std::max(1, std::min(2 * work_capacity * general_ng(tiling.general),
                                  sms * std::max(1, step_blocks_per_sm(tiling.general))));
    L.deep_grid[0] = std::max(1, std::min(2 * work_capacity, sms * std::max(1, deep_blocks_per_sm(1, tiling.deep1))));
    L.deep_grid[1] = std::max(1, std::min(2 * work_capacity, sms * std::max(1, deep_blocks_per_sm(2, tiling.deep2))));
    L.classify_grid = std::max(1, std::min((2 * work_capacity + 127) / 128, 8 * device_sm_count()));
    L.nslots = capacity;
    return L;
}

int Batch::reset_lists()
{
    launch_lists_current(params(), st);
    THY_CK(cudaGetLastError());
    return THY_OK;
}

TuneKey Batch::tune_key(bool *known, bool all_members) const
{
    double deep = 0, general = 0;
    bool all = true;
    for (auto *m : members)
        if (m && (all_members || m->hctl.status == kRunning)) {
            deep += m->mix_deep;
            general += std::max(0.0, (double)m->units() - m->mix_deep - m->mix_dry);
            all = all && m->mix_known;
        }
    if (known) *known = all;
    return TuneKey{device, tune_bucket(deep), tune_bucket(general)};
}

int Batch::run_chunk(bool timed, int len)
{
    int rc;
    bool sampling = false, known = false;
    if (len <= 0 || len > chunk) len = chunk;
    const TuneKey key = tune_key(&known);
    if ((rc = use_tiling(tuner_pick(key, &sampling)))) return rc;
    // a full chunk is one graph launch; a shorter one launches the 1-step
    // graph `len` times (two captures per tiling in all)
    cudaGraphExec_t exec = gexec;
    int repeat = 1;
    if (len != chunk) {
        exec = nullptr;
        for (auto &g : graphs)
            if (g.tiling == tiling && g.len == 1) exec = g.exec;
        if (!exec) {
            if ((rc = capture(1))) return rc;
            exec = graphs.back().exec;
        }
        repeat = len;
    }
    // a sample needs a chunk in which every running member steps `chunk`
    // times (no member reaches its end or an event before the chunk's last
    // step, none fails) and whose work mix was known beforehand
    struct Before {
        long long step;
        unsigned long long deep, dry;
    };
    std::vector<Before> b0(capacity, Before{-1, 0, 0});
    long long running = 0;
    for (int i = 0; i < capacity; i++)
        if (members[i] && members[i]->hctl.status == kRunning) {
            b0[i] = Before{members[i]->hctl.step, members[i]->hctl.units_deep, members[i]->hctl.units_dry};
            running++;
        }
    if (timed) THY_CK(cudaEventRecord(ev0, st));
    for (int i = 0; i < repeat; i++) THY_CK(cudaGraphLaunch(exec, st));
    if (timed) THY_CK(cudaEventRecord(ev1, st));
    THY_CK(cudaMemcpyAsync(h_ctl, d_ctl, capacity * sizeof(ScenarioCtl), cudaMemcpyDeviceToHost, st));
    THY_CK(cudaStreamSynchronize(st));
    float ms = 0;
    if (timed) {
        THY_CK(cudaEventElapsedTime(&ms, ev0, ev1));
        device_ms += ms;
    }
    launches += (long long)kLaunchesPerStep * len;
    chunks_run++;
    bool full = running > 0 && len == chunk;
    double stepped = 0;   // deep + general units stepped in the chunk
    for (int i = 0; i < capacity; i++) {
        DevScenario *m = members[i];
        if (!m) continue;
        m->hctl = h_ctl[i];
        if (b0[i].step < 0) continue;
        const long long k = m->hctl.step - b0[i].step;
        if (m->hctl.status == kFailed || k != chunk) full = false;
        if (k > 0) {
            const double deep = (double)(m->hctl.units_deep - b0[i].deep);
            const double dry = (double)(m->hctl.units_dry - b0[i].dry);
            m->mix_deep = deep / k;
            m->mix_dry = dry / k;
            m->mix_known = true;
            stepped += std::max(0.0, (double)m->units() * k - dry);
        }
    }
    if (timed && sampling && full && known && stepped > 0) {
        tuner_sample(key, tiling, (double)ms / stepped);
        tune_samples++;
    }
    return THY_OK;
}

// Truncation of a member's initial dt to its first fault time
// (src/GPU/ShallowWater.cu:382-391).
static void truncate_initial_dt(DevScenario *s)
{
    double dt = s->hctl.dt, t = s->hctl.t, T = s->Ts;
    const int nf = (int)(s->faults.size() / 10);
    int jumping = 0;
    if (nf > 0) {
        const double *tf0 = &s->faults[0];
        if (tf0[0] < 2.220446049250313e-16) {
            int k = 1;
            while (k < nf && !(std::fabs(s->faults[10 * k] - tf0[0]) > 2.220446049250313e-16)) k++;
            if (k < nf && (t + dt) * T > s->faults[10 * k]) { dt = s->faults[10 * k] / T - t; jumping = 1; }
        } else if ((t + dt) * T > tf0[0]) {
            dt = tf0[0] / T - t;
            jumping = 1;
        }
    }
    s->hctl.dt = dt;
    s->hctl.jumping = jumping;
    s->first_dt_s = dt * T;
}

// Initial dt of every member (src/GPU/Timestep.cu:11-33) and the truncation
// to the first fault time.
static int initial_dt(Batch &b)
{
    int rc;
    for (auto *s : b.members)
        if (s && (rc = s->upload_ctl(b.st))) return rc;
    launch_initial_dt(b.params(), b.st);
    THY_CK(cudaGetLastError());
    THY_CK(cudaMemcpyAsync(b.h_ctl, b.d_ctl, b.capacity * sizeof(ScenarioCtl), cudaMemcpyDeviceToHost, b.st));
    THY_CK(cudaStreamSynchronize(b.st));
    for (int i = 0; i < b.capacity; i++) {
        DevScenario *s = b.members[i];
        if (!s) continue;
        s->hctl = b.h_ctl[i];
        truncate_initial_dt(s);
    }
    return THY_OK;
}

// Initial dt of one member that joins a running batch: phase 0 over its own
// units (a work list of its tiles), the other members untouched.
int Batch::initial_dt_of(DevScenario *s)
{
    int slot = -1;
    for (int i = 0; i < capacity; i++)
        if (members[i] == s) slot = i;
    if (slot < 0) return THY_ERR_INVALID;
    std::vector<int2> w(s->desc.ntiles);
    for (int t = 0; t < s->desc.ntiles; t++) w[t] = make_int2(slot, t);
    const int n = (int)w.size();
    if (n > work_capacity) return THY_ERR_INVALID;
    int rc;
    if ((rc = s->upload_ctl(st))) return rc;
    THY_CK(cudaMemcpyAsync(d_work0, w.data(), n * sizeof(int2), cudaMemcpyHostToDevice, st));
    THY_CK(cudaMemcpyAsync(d_nwork0, &n, sizeof(int), cudaMemcpyHostToDevice, st));
    StepLaunch L = params();
    L.work = d_work0;
    L.nwork = d_nwork0;
    launch_initial_dt(L, st);
    THY_CK(cudaGetLastError());
    THY_CK(cudaMemcpyAsync(&h_ctl[slot], d_ctl + slot, sizeof(ScenarioCtl), cudaMemcpyDeviceToHost, st));
    THY_CK(cudaStreamSynchronize(st));
    s->hctl = h_ctl[slot];
    truncate_initial_dt(s);
    return THY_OK;
}

// Host side of one loop iteration's events (src/GPU/ShallowWater.cu:398-421);
// *changed: a fault deformed the state.
int handle_events_ex(DevScenario &s, const thy_outputs *o, cudaStream_t st, bool *changed)
{
    int rc;
    const int f0 = s.hctl.fault_next;
    if ((rc = s.apply_due_faults(st))) return rc;
    if (changed) *changed = s.hctl.fault_next != f0;
    if (s.save_nc >= 0.0 && s.hctl.t >= s.hctl.next_nc) {
        s.hctl.next_nc += s.save_nc;
        if ((rc = s.snapshot(o, st))) return rc;
    }
    if (s.save_ts >= 0.0 && s.hctl.t >= s.hctl.next_ts) {
        s.hctl.next_ts += s.save_ts;
        if ((rc = s.sample_gauges(o, st))) return rc;
    }
    return THY_OK;
}

}  // namespace thy

using namespace thy;

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------

extern "C" const char *thy_version(void) { return "thysea-b200 1.0 (Tsunami-HySEA 1.3.0 scheme)"; }

extern "C" const char *thy_strerror(int code)
{
    switch (code) {
    case THY_OK: return "ok";
    case THY_ERR_GPU_MEMORY: return "not enough GPU memory";
    case THY_ERR_HOST: return "host memory or output file error";
    case THY_ERR_INVALID: return "invalid argument";
    case THY_ERR_CUDA: return last_error_text()[0] ? last_error_text() : "CUDA error";
    case THY_ERR_NO_DEVICE: return "there is no CUDA device";
    case THY_ERR_NONFINITE: return "the state or the time step became non-finite";
    case THY_ERR_TIMEOUT: return "a bounded wait on the device ran out (a staging copy did not land)";
    case THY_ERR_BUDGET: return "scenario does not fit the HBM budget";
    case THY_ERR_CANCELLED: return "request cancelled";
    case THY_ERR_TOO_LARGE: return "grid exceeds the allocation-free entry point's maximum of 1048576 cells";
    default: return "unknown error";
    }
}

extern "C" int thy_device_count(void)
{
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}

// Page-locks (and releases) host memory the caller owns, e.g. the problem's
// FP64 arrays and the output fields, so that the copies of thy_run run at
// full link speed.
extern "C" int thy_host_register(void *p, size_t bytes)
{
    int rc = ensure_device();
    if (rc) return rc;
    if (!p || bytes == 0) return THY_ERR_INVALID;
    THY_CK(cudaHostRegister(p, bytes, cudaHostRegisterDefault));
    return THY_OK;
}

extern "C" int thy_host_unregister(void *p)
{
    if (!p) return THY_ERR_INVALID;
    THY_CK(cudaHostUnregister(p));
    return THY_OK;
}

extern "C" int thy_set_device(int device)
{
    if (device < 0 || device >= 64) return THY_ERR_INVALID;
    g_device = device;
    return THY_OK;
}

extern "C" int thy_run(const thy_problem *p, const thy_outputs *o, thy_stats *stats)
{
    int rc = ensure_device();
    if (rc) return rc;
    if (!p) return THY_ERR_INVALID;
    const auto t_start = std::chrono::steady_clock::now();
    if (stats) std::memset(stats, 0, sizeof(*stats));
    int device = 0;
    THY_CK(cudaGetDevice(&device));
    Batch *bp = lease_run_batch(device, (p->nx / kTileX + 2) * (p->ny / kTileY + 2), &rc);
    if (!bp) return rc;
    Batch &b = *bp;
    cudaStream_t st = b.st;
    auto t0 = std::chrono::steady_clock::now();
    auto t_release = t0;
    double event_s = 0;
    {
        DevScenario s;
        if ((rc = b.attach(&s))) goto out;
        if ((rc = s.setup(p, st))) goto out;
        s.desc.ctl = s.ctl;
        if ((rc = b.rebuild())) goto out;
        // the delivery of snapshots and gauge samples (writer thread,
        // page-locked slots, copy stream) is set up before the loop, as the
        // reference creates its output files before its loop
        if ((rc = s.open_outputs(o, st))) goto out;
        t0 = std::chrono::steady_clock::now();
        if (stats) stats->setup_seconds = std::chrono::duration<double>(t0 - t_start).count();
        if ((rc = initial_dt(b))) goto out;
        if (stats) stats->initial_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        for (;;) {
            if (!(s.hctl.t < s.t_end)) break;
            if (s.max_steps >= 0 && s.hctl.step >= s.max_steps) break;
            if (s.hctl.status == kFailed) { rc = failure_code(s.hctl); goto out; }
            {
                const auto te = std::chrono::steady_clock::now();
                bool changed = false;
                if ((rc = handle_events_ex(s, o, st, &changed))) goto out;
                if (changed && (rc = b.reset_lists())) goto out;
                event_s += std::chrono::duration<double>(std::chrono::steady_clock::now() - te).count();
            }
            s.hctl.status = kRunning;
            s.hctl.events = 0;
            if ((rc = s.upload_ctl(st))) goto out;
            // chunks no longer than the steps left before the next event (as
            // far as the current dt tells), so that few launches find the
            // scenario paused
            do {
                if ((rc = b.run_chunk(true, b.chunk_for(Batch::steps_to_event(s))))) goto out;
                if ((rc = s.read_device_gauges(o, st))) goto out;
            } while (s.hctl.status == kRunning);
            if (s.hctl.status == kFailed) { rc = failure_code(s.hctl); goto out; }
        }
        {
            auto t1 = std::chrono::steady_clock::now();
            if (stats) {
                stats->steps = s.hctl.step;
                stats->final_time_s = s.hctl.t * s.Ts;
                stats->first_dt_s = s.first_dt_s;
                stats->loop_seconds = std::chrono::duration<double>(t1 - t0).count();
                stats->device_loop_ms = b.device_ms;
                stats->kernel_launches = b.launches;
                stats->snapshots = s.snapshots;
                stats->series_samples = s.series;
                stats->tiles = s.hctl.step * (long long)s.units();
                stats->deep_tiles = (long long)s.hctl.units_deep;
                stats->dry_tiles = (long long)s.hctl.units_dry;
                stats->tiling = thy_tiling{b.tiling.deep1, b.tiling.deep2, b.tiling.general};
                stats->tune_samples = b.tune_samples;
                stats->chunks = b.chunks_run;
                stats->graph_captures = b.captures;
                stats->capture_seconds = b.capture_s;
                stats->event_seconds = event_s;
            }
        }
        {
            const auto t2 = std::chrono::steady_clock::now();
            rc = s.finish(o, st);
            if (stats)
                stats->output_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t2).count();
        }
    out:
        t_release = std::chrono::steady_clock::now();
        b.detach(&s);
    }
    {
        // the batch goes back to the pool unless the run ended in a CUDA
        // error (its state is then unknown); its stream is idle
        const bool healthy = cudaStreamSynchronize(st) == cudaSuccess && rc != THY_ERR_CUDA && rc != THY_ERR_TIMEOUT;
        if (!healthy) cudaGetLastError();
        return_run_batch(bp, healthy);
    }
    if (stats) {
        const auto t_end = std::chrono::steady_clock::now();
        stats->release_seconds = std::chrono::duration<double>(t_end - t_release).count();
        stats->total_seconds = std::chrono::duration<double>(t_end - t_start).count();
    }
    return rc;
}

// ---------------------------------------------------------------------------
// sessions: step-level access for benchmarking
// ---------------------------------------------------------------------------

struct thy_session {
    cudaStream_t st = nullptr;
    DevScenario s;
    Batch b;
};

extern "C" int thy_session_open(const thy_problem *p, thy_session **out)
{
    int rc = ensure_device();
    if (rc) return rc;
    if (!p || !out) return THY_ERR_INVALID;
    thy_session *S = new thy_session();
    THY_CK(cudaStreamCreateWithFlags(&S->st, cudaStreamNonBlocking));
    thy_problem q = *p;
    q.save_nc = -1.0;
    q.save_ts = -1.0;
    q.max_steps = 0;
    if ((rc = S->b.init(1, (p->nx / kTileX + 2) * (p->ny / kTileY + 2), S->st)) || (rc = S->b.attach(&S->s)) ||
        (rc = S->s.setup(&q, S->st)) || (rc = S->b.rebuild()) || (rc = initial_dt(S->b)) ||
        (rc = S->s.apply_due_faults(S->st)) || (rc = S->b.reset_lists())) {
        cudaStream_t st = S->st;
        delete S;
        cudaStreamDestroy(st);
        return rc;
    }
    *out = S;
    return THY_OK;
}

extern "C" int thy_session_steps(thy_session *S, long long steps, double *device_ms, long long *steps_done)
{
    if (!S) return THY_ERR_INVALID;
    DevScenario &s = S->s;
    const long long start = s.hctl.step;
    const double ms0 = S->b.device_ms;
    int rc;
    s.hctl.max_steps = start + steps;
    if (s.hctl.t < s.t_end && steps > 0) {
        s.hctl.status = kRunning;
        s.hctl.events = 0;
        if ((rc = s.upload_ctl(S->st))) return rc;
        // exactly `steps` steps' launches: full chunks, then power-of-two
        // chunks for the rest (a scenario that reaches its end or a fault
        // time earlier stops there)
        do {
            if ((rc = S->b.run_chunk(true, S->b.chunk_for(start + steps - s.hctl.step)))) return rc;
        } while (s.hctl.status == kRunning && s.hctl.step < start + steps);
    }
    if (device_ms) *device_ms = S->b.device_ms - ms0;
    if (steps_done) *steps_done = s.hctl.step - start;
    return s.hctl.status == kFailed ? failure_code(s.hctl) : THY_OK;
}

// Per-kernel device time: `steps` steps launched one kernel at a time with
// CUDA events around each launch on the session's stream.  ms_per_launch
// receives the average duration (ms) of each of the kLaunchesPerStep launches
// of a step (deep phase 1, general phase 1, classification, deep phase 2,
// general phase 2, controller).
extern "C" int thy_session_profile_launches(thy_session *S, long long steps, double *ms_per_launch)
{
    if (!S || steps <= 0) return THY_ERR_INVALID;
    DevScenario &s = S->s;
    Batch &b = S->b;
    constexpr int NL = kLaunchesPerStep;
    const StepLaunch L = b.params();
    int rc;
    s.hctl.max_steps = s.hctl.step + steps;
    s.hctl.status = kRunning;
    s.hctl.events = 0;
    if ((rc = s.upload_ctl(S->st))) return rc;
    std::vector<cudaEvent_t> ev((NL + 1) * steps);
    for (auto &e : ev) THY_CK(cudaEventCreate(&e));
    for (long long k = 0; k < steps; k++) {
        for (int j = 0; j < NL; j++) {
            THY_CK(cudaEventRecord(ev[(NL + 1) * k + j], S->st));
            launch_step_kernel(j, L, S->st);
        }
        THY_CK(cudaEventRecord(ev[(NL + 1) * k + NL], S->st));
    }
    THY_CK(cudaGetLastError());
    THY_CK(cudaStreamSynchronize(S->st));
    double t[NL] = {};
    for (long long k = 0; k < steps; k++)
        for (int j = 0; j < NL; j++) {
            float a = 0;
            THY_CK(cudaEventElapsedTime(&a, ev[(NL + 1) * k + j], ev[(NL + 1) * k + j + 1]));
            t[j] += a;
        }
    for (auto &e : ev) cudaEventDestroy(e);
    b.launches += (long long)NL * steps;
    if ((rc = s.download_ctl(S->st))) return rc;
    THY_CK(cudaStreamSynchronize(S->st));
    if (ms_per_launch)
        for (int j = 0; j < NL; j++) ms_per_launch[j] = t[j] / steps;
    return s.hctl.status == kFailed ? failure_code(s.hctl) : THY_OK;
}

// Average device time of phase 1 and phase 2 (each the sum of its launches).
extern "C" int thy_session_profile(thy_session *S, long long steps, double *phase1_ms, double *phase2_ms)
{
    double t[kLaunchesPerStep] = {};
    const int rc = thy_session_profile_launches(S, steps, t);
    if (phase1_ms) *phase1_ms = t[0] + t[1] + t[2];
    if (phase2_ms) *phase2_ms = t[3] + t[4] + t[5];
    return rc;
}

extern "C" long long thy_session_launches(const thy_session *S) { return S ? S->b.launches : 0; }

extern "C" int thy_session_tiles(const thy_session *S, long long *tiles, long long *deep_tiles, long long *dry_tiles)
{
    if (!S) return THY_ERR_INVALID;
    if (tiles) *tiles = S->s.hctl.step * (long long)S->s.units();
    if (deep_tiles) *deep_tiles = (long long)S->s.hctl.units_deep;
    if (dry_tiles) *dry_tiles = (long long)S->s.hctl.units_dry;
    return THY_OK;
}

extern "C" int thy_session_fetch(thy_session *S, float *max_height, float *eta, float *ux, float *uy)
{
    if (!S) return THY_ERR_INVALID;
    thy_outputs o;
    std::memset(&o, 0, sizeof(o));
    o.max_height = max_height;
    o.eta = eta;
    o.ux = ux;
    o.uy = uy;
    return S->s.finish(&o, S->st);
}

extern "C" double thy_session_time(const thy_session *S) { return S ? S->s.hctl.t * S->s.Ts : 0.0; }

extern "C" int thy_session_inject(thy_session *S, int what)
{
    if (!S || what < 0 || what > 1) return THY_ERR_INVALID;
    S->s.hctl.inject = what;
    return S->s.upload_ctl(S->st);
}

extern "C" int thy_session_tune(thy_session *S, long long max_steps, long long *steps_done)
{
    if (!S || max_steps < 0) return THY_ERR_INVALID;
    long long done = 0;
    int rc = THY_OK;
    while (done < max_steps && S->s.hctl.t < S->s.t_end) {
        // the session's scenario waits between calls (its status is not
        // running): its key counts it all the same
        bool known = false;
        const TuneKey key = S->b.tune_key(&known, true);
        if (known && tuner_decided(key, nullptr)) break;
        long long k = 0;
        if ((rc = thy_session_steps(S, std::min<long long>(S->b.chunk, max_steps - done), nullptr, &k))) break;
        if (k <= 0) break;
        done += k;
    }
    if (steps_done) *steps_done = done;
    return rc;
}

extern "C" int thy_session_tiling(const thy_session *S, thy_tiling *t)
{
    if (!S || !t) return THY_ERR_INVALID;
    *t = thy_tiling{S->b.tiling.deep1, S->b.tiling.deep2, S->b.tiling.general};
    return THY_OK;
}

extern "C" int thy_session_tuned(const thy_session *S, thy_tiling *best)
{
    if (!S) return THY_ERR_INVALID;
    bool known = false;
    const TuneKey key = S->b.tune_key(&known, true);
    Tiling t;
    const bool done = tuner_decided(key, &t);
    if (best) *best = thy_tiling{t.deep1, t.deep2, t.general};
    return (known && done) ? 1 : 0;
}

static bool tiling_ok(const thy_tiling *t)
{
    return t->deep1 >= 0 && t->deep1 < kTilingVariants && t->deep2 >= 0 && t->deep2 < kTilingVariants &&
           t->general >= 0 && t->general < kTilingVariants;
}

extern "C" int thy_tiling_force(const thy_tiling *t)
{
    if (!t) {
        tuner_force(nullptr);
        return THY_OK;
    }
    if (!tiling_ok(t)) return THY_ERR_INVALID;
    Tiling x;
    x.deep1 = t->deep1;
    x.deep2 = t->deep2;
    x.general = t->general;
    tuner_force(&x);
    return THY_OK;
}

extern "C" int thy_tiling_tuned(double deep_units, double general_units, thy_tiling *best)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) dev = 0;
    Tiling t;
    const bool done = tuner_decided(TuneKey{dev, tune_bucket(deep_units), tune_bucket(general_units)}, &t);
    if (best) *best = thy_tiling{t.deep1, t.deep2, t.general};
    return done ? 1 : 0;
}

extern "C" void thy_tuner_clear(void) { tuner_clear(); }

extern "C" void thy_session_close(thy_session *S)
{
    if (!S) return;
    cudaStream_t st = S->st;
    delete S;
    if (st) cudaStreamDestroy(st);
}
