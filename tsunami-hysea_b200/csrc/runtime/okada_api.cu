// C ABI of the Okada stage on its own: the reference's aplicarOkada()
// (src/GPU/Deformacion.cu:118-143) on device memory in the reference's state
// layout (double2 (h, H) per cell, dimensionless): the FP64 vertical
// deformation of one fault, optional relative / absolute cropping, then
// H -= U_Z and eta_initial += U_Z (src/GPU/Deformacion.cu:38-53).
#include "engine.h"

namespace thy {

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
// nx*ny doubles, max_bits one word.
int enqueue_okada_reference_layout(int nx, int ny, double lon0, double dlon, double lat0, double dlat,
                                   const double *fault, double H, int crop_flag, double crop_value, double2 *state,
                                   double *eta_initial, double *def, unsigned int *max_bits, cudaStream_t st)
{
    const long long n = (long long)nx * ny;
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
                                        (double2 *)d_state1, d_eta_initial, def, mx, st);
    cudaError_t e = cudaStreamSynchronize(st);
    cudaFree(def);
    cudaFree(mx);
    if (rc) return rc;
    THY_CK(e);
    return THY_OK;
}
