// C ABI of the Okada stage on its own: the reference's aplicarOkada()
// (src/GPU/Deformacion.cu:118-143) on device memory in the reference's state
// layout (double2 (h, H) per cell, dimensionless): the FP64 vertical
// deformation of one fault, optional relative / absolute cropping, then
// H -= U_Z and eta_initial += U_Z (src/GPU/Deformacion.cu:38-53).
//
// Two entry points run the same kernels and differ only in where the
// scratch (the nx*ny deformation field and one word for the cropping
// maximum) lives: thy_apply_okada takes it from cudaMalloc for the call;
// thy_apply_okada_noalloc uses the fixed-size device arrays below, for
// callers that must not allocate device memory at all.
#include <mutex>

#include <cuda.h>

#include "engine.h"

namespace thy {

// Scratch of thy_apply_okada_noalloc.  File-scope device arrays: every GPU
// that loads the library holds them (8 MiB + 4 bytes) until the process
// exits, and every call shares them.
static __device__ __align__(256) double g_okada_scratch[THY_OKADA_NOALLOC_MAX_CELLS];
static __device__ __align__(256) unsigned int g_okada_scratch_max;

namespace {
// Device addresses of the two arrays, looked up once per device and context:
// a device reset (cudaDeviceReset) or a new primary context can load the
// module at other addresses, so a cached address is only used while the
// context it was looked up in is still the current one.
struct ScratchAddr {
    CUcontext ctx = nullptr;
    double *def = nullptr;
    unsigned int *max = nullptr;
};
std::mutex g_scratch_mu;
ScratchAddr g_scratch[64];

using CtxGetCurrentFn = CUresult (*)(CUcontext *);
CtxGetCurrentFn ctx_get_current_fn()
{
    static CtxGetCurrentFn fn = nullptr;
    if (!fn) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<CtxGetCurrentFn>(p);
        else
            cudaGetLastError();
    }
    return fn;
}
}  // namespace

__global__ void okada_kernel(int nx, int ny, double *__restrict__ def, double lon0, double dlon, double lat0,
                             double dlat, OkadaFault f, double Hs);
__global__ void absmax_kernel(const double *__restrict__ def, long long n, unsigned int *max_bits);

__global__ void apply_deformation_reference_layout(long long n, double2 *__restrict__ state,
                                                   double *__restrict__ eta_initial, const double *__restrict__ def,
                                                   int crop_flag, double crop_value,
                                                   const unsigned int *__restrict__ max_bits)
{
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    double U = def[i];
    if (crop_flag == 1) {
        if (fabs(U) < crop_value * (double)__uint_as_float(*max_bits)) U = 0.0;
    } else if (crop_flag == 2) {
        if (fabs(U) < crop_value) U = 0.0;
    }
    state[i].y -= U;
    if (eta_initial) eta_initial[i] += U;
}

// Enqueues the Okada stage on `st` with caller-provided scratch: def holds
// def_cells doubles (at least nx*ny, else THY_ERR_TOO_LARGE before any
// work), max_bits one word.
int enqueue_okada_reference_layout(int nx, int ny, double lon0, double dlon, double lat0, double dlat,
                                   const double *fault, double H, int crop_flag, double crop_value, double2 *state,
                                   double *eta_initial, double *def, size_t def_cells, unsigned int *max_bits,
                                   cudaStream_t st)
{
    const long long n = (long long)nx * ny;
    if (n > (long long)def_cells) return THY_ERR_TOO_LARGE;
    OkadaFault f{fault[1], fault[2], fault[3], fault[4], fault[5], fault[6], fault[7], fault[8], fault[9]};
    dim3 block(32, 4), grid((nx + 31) / 32, (ny + 3) / 4);
    okada_kernel<<<grid, block, 0, st>>>(nx, ny, def, lon0, dlon, lat0, dlat, f, H);
    THY_CK(cudaMemsetAsync(max_bits, 0, sizeof(unsigned int), st));
    if (crop_flag == 1) absmax_kernel<<<296, 256, 0, st>>>(def, n, max_bits);
    apply_deformation_reference_layout<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(n, state, eta_initial, def,
                                                                                  crop_flag, crop_value, max_bits);
    THY_CK(cudaGetLastError());
    return THY_OK;
}

int check_okada_args(int nx, int ny, const double *fault, int crop_flag, const void *state)
{
    if (nx < 2 || ny < 2 || !fault || !state || crop_flag < 0 || crop_flag > 2) return THY_ERR_INVALID;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return THY_ERR_NO_DEVICE;
    }
    return THY_OK;
}

}  // namespace thy

using namespace thy;

extern "C" int thy_apply_okada(int nx, int ny, double lon0, double dlon, double lat0, double dlat, const double *fault,
                               double H, int crop_flag, double crop_value, void *d_state1, double *d_eta_initial,
                               void *stream)
{
    int rc = check_okada_args(nx, ny, fault, crop_flag, d_state1);
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    double *def = nullptr;
    unsigned int *mx = nullptr;
    const size_t n = (size_t)nx * ny;
    THY_CK(cudaMalloc(&def, n * sizeof(double)));
    if (cudaMalloc(&mx, sizeof(unsigned int)) != cudaSuccess) {
        cudaFree(def);
        return THY_ERR_GPU_MEMORY;
    }
    rc = enqueue_okada_reference_layout(nx, ny, lon0, dlon, lat0, dlat, fault, H, crop_flag, crop_value,
                                        (double2 *)d_state1, d_eta_initial, def, n, mx, st);
    cudaError_t e = cudaStreamSynchronize(st);
    cudaFree(def);
    cudaFree(mx);
    if (rc) return rc;
    THY_CK(e);
    return THY_OK;
}

// Same computation with the library's fixed device scratch instead of a
// cudaMalloc: for callers that cannot allocate device memory (a caching or
// budgeted allocator owns the GPU, or an allocation's implicit device-wide
// synchronisation is not acceptable).  Up to THY_OKADA_NOALLOC_MAX_CELLS
// cells; larger grids return THY_ERR_TOO_LARGE before any work.  The first
// call on a device looks up the scratch's device address there
// (cudaGetSymbolAddress), so make that first call before any stream capture;
// after a device reset the next call looks it up again (and is then again a
// first call).  The work is only enqueued on `stream`.  The scratch is shared
// by every call and keeps the last call's contents (the cropping maximum is
// cleared at the start of each call); calls whose work overlaps on the GPU
// (other streams, other host threads) race on it.
extern "C" int thy_apply_okada_noalloc(int nx, int ny, double lon0, double dlon, double lat0, double dlat,
                                       const double *fault, double H, int crop_flag, double crop_value,
                                       void *d_state1, double *d_eta_initial, void *stream)
{
    // the size first, before anything touches the device
    if (nx > 0 && ny > 0 && (long long)nx * ny > (long long)THY_OKADA_NOALLOC_MAX_CELLS) return THY_ERR_TOO_LARGE;
    int rc = check_okada_args(nx, ny, fault, crop_flag, d_state1);
    if (rc) return rc;
    int dev = 0;
    THY_CK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return THY_ERR_INVALID;
    // the context the work will run in (none yet before the runtime's first
    // use of the device: the look-up below creates it)
    CtxGetCurrentFn get_ctx = ctx_get_current_fn();
    if (!get_ctx) return THY_ERR_CUDA;
    CUcontext ctx = nullptr;
    if (get_ctx(&ctx) != CUDA_SUCCESS) return THY_ERR_CUDA;
    double *def;
    unsigned int *mx;
    {
        std::lock_guard<std::mutex> lock(g_scratch_mu);
        ScratchAddr &a = g_scratch[dev];
        if (!ctx || a.ctx != ctx || !a.def || !a.max) {
            void *pd = nullptr, *pm = nullptr;
            THY_CK(cudaGetSymbolAddress(&pd, g_okada_scratch));
            THY_CK(cudaGetSymbolAddress(&pm, g_okada_scratch_max));
            if (!ctx && (get_ctx(&ctx) != CUDA_SUCCESS || !ctx)) return THY_ERR_CUDA;
            a.ctx = ctx;
            a.def = (double *)pd;
            a.max = (unsigned int *)pm;
        }
        def = a.def;
        mx = a.max;
    }
    return enqueue_okada_reference_layout(nx, ny, lon0, dlon, lat0, dlat, fault, H, crop_flag, crop_value,
                                          (double2 *)d_state1, d_eta_initial, def, THY_OKADA_NOALLOC_MAX_CELLS, mx,
                                          (cudaStream_t)stream);
}
