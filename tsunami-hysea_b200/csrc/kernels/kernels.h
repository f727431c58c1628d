// Launch wrappers of the device kernels (host-callable, no CUDA types beyond
// cudaStream_t / int2 in the signatures).
#pragma once
#include <cstddef>
#include <cuda_runtime.h>

namespace thy {

struct ScenarioDev;

constexpr int kStepThreads = 128;           // 4 warps = 4 column strips per tile
constexpr int kTileX = 28 * (kStepThreads / 32);   // tile width: 28 output columns per warp
constexpr int kTileY = 32;                  // tile height: rows one warp marches through

// Grid column where tile 0 starts: 0 or a negative multiple of 4 above
// -kTileX (tile 0 then holds its last 4 .. 108 columns), so that the deep
// kernels' boxes at x0 - 4 and x0 stay 16-byte aligned.  Tiles that reach
// within two cells of the left or right boundary, or into a sponge layer,
// take the general kernel, whose cost is one warp per 28-column strip holding
// a cell; the origin is the first of the 28 aligned shifts that minimises
// those strips (origin 0 when no shift does better).  Periodic grids and
// grids narrower than 2 kTileX + 4 keep origin 0.
inline int tile_origin(int nx, bool periodic, int sp_left, int sp_right)
{
    if (periodic || nx < 2 * kTileX + 4) return 0;
    const int need_l = sp_left > 2 ? sp_left : 2, need_r = sp_right > 2 ? sp_right : 2;
    int best = 0, best_cost = -1;
    for (int org = 0; org > -kTileX; org -= 4) {
        const int tiles = (nx - org + kTileX - 1) / kTileX;
        int cost = 0;
        for (int t = 0; t < tiles; t++) {
            const int x0 = org + t * kTileX;
            if (x0 >= need_l && x0 + kTileX <= nx - need_r) continue;   // may run deep
            for (int k = 0; k < kTileX / 28; k++) cost += (x0 + 28 * k + 28 > 0 && x0 + 28 * k < nx) ? 1 : 0;
        }
        if (best_cost < 0 || cost < best_cost) {
            best_cost = cost;
            best = org;
        }
    }
    return best;
}

// Warp tilings of the stepping kernels, picked per workload by the autotuner
// (runtime/tuner.cu).  A work unit is always kTileX x kHalfRows cells, its
// column strips marched by warps; a tiling says into how many row groups a
// unit's rows are split (deep kernels: compute warps per CTA = 4 x groups of
// the variant, and the CTAs an SM keeps resident follow; general kernel: one
// warp task per strip and row group).  Every cell's arithmetic is the same
// under every tiling (a warp recomputes the y edge above its first row from
// the same inputs), so results do not depend on the tiling.  Variant 0 is the
// default.
constexpr int kTilingVariants = 3;
struct Tiling {
    int deep1 = 0, deep2 = 0, general = 0;   // variant of deep phase 1, deep phase 2, the general kernel
    bool operator==(const Tiling &o) const { return deep1 == o.deep1 && deep2 == o.deep2 && general == o.general; }
    bool operator!=(const Tiling &o) const { return !(*this == o); }
};
// compute warps per CTA = 4 x deep_ng: deep phase 1 {3, 2, 4} (4 column strips
// x that many row groups), deep phase 2 {2, 1, 4} (2 column strips of column
// pairs x twice that many row groups); general {2, 1, 8} row groups (one warp
// task per strip and row group; 8 groups of 2 rows for short chains)
__host__ __device__ constexpr int deep_ng(int phase, int v)
{
    return phase == 1 ? (v == 0 ? 3 : v == 1 ? 2 : 4) : (v == 0 ? 2 : v == 1 ? 1 : 4);
}
// resident CTAs per SM the deep kernels are compiled for: phase 1 is held to
// two by its staging buffers; phase 2 (its lanes hold two columns) two, three
// or one as its registers allow
__host__ __device__ constexpr int deep_minb(int phase, int v) { return phase == 1 ? 2 : (v == 0 ? 2 : v == 1 ? 3 : 1); }
__host__ __device__ constexpr int general_ng(int v) { return v == 0 ? 2 : v == 1 ? 1 : 8; }

// step.cu
cudaError_t configure_step_kernels();
int step_blocks_per_sm(int general_variant);
// Launch parameters of the stepping kernels of a batch.
struct StepLaunch {
    const ScenarioDev *scen;   // scenario table (nslots entries)
    const int2 *work;          // work list: (scenario slot, tile)
    const int *nwork;          // its length (device)
    int *lists;                // deep / general lists of the step: 2 counts + 2 x cap indices
    int *claims;               // units claimed beyond the first wave by deep phase 1 / 2 and the general
                               // kernel of phase 1 / 2 (zeroed by classification)
    int cap;                   // list capacity (>= work-list length)
    int grid;                  // general kernel grid
    int deep_grid[2];          // persistent deep kernel grids, phase 1 and 2
    int classify_grid;
    int nslots;
    Tiling tiling;
};

// The kLaunchesPerStep launches of a time step, in order: 0 deep phase 1,
// 1 general phase 1, 2 work-list classification, 3 deep phase 2, 4 general
// phase 2, 5 step controller.  Launches 0/1 and 3/4 may run concurrently.
constexpr int kLaunchesPerStep = 6;
void launch_step_kernel(int k, const StepLaunch &L, cudaStream_t st);
void launch_initial_dt(const StepLaunch &L, cudaStream_t st);
// lists for the current states of the work list's scenarios (from the host,
// before a chunk: after the work list or a state changed)
void launch_lists_current(const StepLaunch &L, cudaStream_t st);
// init_extract.cu: the step controller of every slot (launch 5 of a step)
void launch_controller(const StepLaunch &L, cudaStream_t st);
// init_extract.cu: per-unit depth steps (ScenarioDev::unit_gmax), after the
// depths change
void launch_unit_gmax(const ScenarioDev *s_host, cudaStream_t st);
// init_extract.cu / okada.cu: load their kernels now rather than at first use
cudaError_t preload_output_kernels();
cudaError_t preload_okada_kernels();
int deep_blocks_per_sm(int phase, int variant);

// init.cu: double-precision host state (reference layout, dimensionless) to
// the FP32 device state; metrics initialised as in src/GPU/ShallowWater.cu:305-309
void launch_init_state(const ScenarioDev *s_host, const ScenarioDev *s_dev, const double *h, const double *Hs,
                       const double *qx, const double *qy, double Hmin, cudaStream_t st);

// okada.cu: FP64 Okada deformation of one fault into a double scratch field,
// |U_Z| max (for relative cropping), crop and apply
struct OkadaFault {
    double lon_c, lat_c, depth_c, length, width, strike, dip, rake, slip;
};
void launch_okada(const ScenarioDev *s_host, double *def, double lon0, double dlon, double lat0, double dlat,
                  const OkadaFault &f, double Hs, cudaStream_t st);
void launch_absmax(const double *def, long long n, unsigned int *max_bits, cudaStream_t st);
void launch_apply_deformation(const ScenarioDev *s_host, const double *def, int crop_flag, double crop_value,
                              const unsigned int *max_bits, cudaStream_t st);

// extract.cu: dimensional output fields (src/GPU/netcdf_kernel.cu)
enum Field { kFieldEta = 0, kFieldUx = 1, kFieldUy = 2, kFieldMaxHeight = 3, kFieldArrival = 4, kFieldDeformed = 5 };
void launch_extract(const ScenarioDev *s_host, int field, int parity, float *out, double Hs, double Qs, double Hmin,
                    cudaStream_t st);
// gauges: eta (m), ux, uy (m/s) and depth at nP cells (cell index or -1);
// fold_minmax: a sample of the series, its eta folded into the scenario's
// gauge extremes (not for the final read of the depths)
void launch_gauges(const ScenarioDev *s_host, int parity, const int *cells, int nP, float *out4, bool fold_minmax,
                   cudaStream_t st);

}  // namespace thy
