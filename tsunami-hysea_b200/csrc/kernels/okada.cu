// Okada seafloor deformation on the GPU, in FP64 (the dislocation formulas
// cancel strongly near the fault; FP32 would lose centimetres of uplift).
//
// Per cell (src/GPU/Deformacion.cu:55-116): station coordinates on the
// lon/lat lattice lon0 + i*dlon, lat0 + j*dlat; Gauss-Krueger projection
// about the fault centre (src/GPU/prtoxy.cu:33-54); rotation by the strike;
// vertical surface displacement of a rectangular dislocation (Okada 1985,
// BSSA 75(4), closed-form surface solution, which the reference's DC3D of
// Okada 1992 equals at z = 0) divided by the depth scale.  Then optional
// relative / absolute cropping and the update bathymetry -= U_Z,
// eta_initial += U_Z (src/GPU/Deformacion.cu:13-53,118-143); the water depth
// h is unchanged, so the surface rises by U_Z.
#include "device.cuh"
#include "kernels.h"

namespace thy {

__device__ void gauss_krueger(double lat, double lon, double lat0, double lon0, double &x, double &y)
{
    // reference constants: Bessel-type ellipsoid a = 6378.16 km, e^2 = 0.0066946053,
    // e'^2 = 0.0067397251, a(1-e^2) = 6335.4607362597517 km, 57.29578 deg/rad,
    // 6 * 57.29578^2 and pi/180 rounded to single precision
    const double deg = 0.017453292371619689;
    const double rlat = lat * deg, slat = sin(rlat), clat = cos(rlat);
    const double v2 = clat * 0.0067397251 * clat + 1.0;
    const double dl = lon - lon0;
    const double ph1 = lat + v2 * 0.5 * dl * dl * slat * clat * deg;
    const double s1 = sin(ph1 * deg), s2 = sin((ph1 + lat0) * 0.5 * deg);
    const double d = sqrt(1.0 - s2 * 0.0066946053 * s2);
    const double rm = 6335.4607362597517 / (d * (d * d));
    const double rn = 6378.16 / sqrt(1.0 - s1 * 0.0066946053 * s1);
    y = (ph1 - lat0) / (57.29578 / rm);
    x = dl * clat / (57.29578 / rn) * (dl * dl * cos(rlat * 2.0) / 19696.838434850401 + 1.0);
}

// u_z at the surface; x along strike, y across (km), d centroid depth (km),
// fault length L and width W (km) centred on the reference point, U1
// strike-slip and U2 dip-slip (m).  mu/(lambda+mu) = 1/2 (alpha = 2/3).
__device__ double okada_uz(double x, double y, double d, double dip_deg, double L, double W, double U1, double U2)
{
    const double two_pi = 6.283185307179586, eps = 1e-6, k = 0.5;
    double sd = sin(dip_deg * (two_pi / 360.0)), cd = cos(dip_deg * (two_pi / 360.0));
    if (fabs(cd) < eps) { cd = 0.0; sd = (sd > 0.0) ? 1.0 : -1.0; }
    double xi[2] = {x + 0.5 * L, x - 0.5 * L};
    if (fabs(xi[0]) < eps) xi[0] = 0.0;
    if (fabs(xi[1]) < eps) xi[1] = 0.0;
    const double p = y * cd + d * sd;
    double q = y * sd - d * cd;
    double et[2] = {p + 0.5 * W, p - 0.5 * W};
    if (fabs(q) < eps) q = 0.0;
    if (fabs(et[0]) < eps) et[0] = 0.0;
    if (fabs(et[1]) < eps) et[1] = 0.0;
    if ((q == 0.0) && ((xi[0] * xi[1] <= 0.0 && et[0] * et[1] == 0.0) || (et[0] * et[1] <= 0.0 && xi[0] * xi[1] == 0.0)))
        return 0.0;
    int kxi[2] = {0, 0}, ket[2] = {0, 0};
    {
        const double r12 = sqrt(xi[0] * xi[0] + et[1] * et[1] + q * q);
        const double r21 = sqrt(xi[1] * xi[1] + et[0] * et[0] + q * q);
        const double r22 = sqrt(xi[1] * xi[1] + et[1] * et[1] + q * q);
        if (xi[0] < 0.0 && r21 + xi[1] < eps) kxi[0] = 1;
        if (xi[0] < 0.0 && r22 + xi[1] < eps) kxi[1] = 1;
        if (et[0] < 0.0 && r12 + et[1] < eps) ket[0] = 1;
        if (et[0] < 0.0 && r22 + et[1] < eps) ket[1] = 1;
    }
    double uz = 0.0;
#pragma unroll
    for (int kk = 0; kk < 2; kk++) {
#pragma unroll
        for (int j = 0; j < 2; j++) {
            const double sgn = (j + kk == 1) ? -1.0 : 1.0;
            const double X = xi[j], E = et[kk];
            const double R = sqrt(X * X + E * E + q * q);
            if (R == 0.0) continue;
            const double dt = E * sd - q * cd;
            const double theta = (q == 0.0) ? 0.0 : atan(X * E / (q * R));
            const double inv_rx = kxi[kk] ? 0.0 : 1.0 / (R + X);
            double inv_re, ln_re;
            if (ket[j]) { inv_re = 0.0; ln_re = -log(R - E); }
            else { inv_re = 1.0 / (R + E); ln_re = log(R + E); }
            double I4, I5;
            if (cd != 0.0) {
                const double Xs = sqrt(X * X + q * q);
                I4 = k / cd * (log(R + dt) - sd * ln_re);
                I5 = (X == 0.0) ? 0.0 : k * 2.0 / cd * atan((E * (Xs + q * cd) + Xs * (R + Xs) * sd) / (X * (R + Xs) * cd));
            } else {
                I4 = -k * q / (R + dt);
                I5 = -k * X * sd / (R + dt);
            }
            const double fss = dt * q / R * inv_re + q * sd * inv_re + I4 * sd;
            const double fds = dt * q / R * inv_rx + sd * theta - I5 * sd * cd;
            uz += sgn * (-U1 / two_pi * fss - U2 / two_pi * fds);
        }
    }
    return uz;
}

__global__ void okada_kernel(int nx, int ny, double *__restrict__ def, double lon0, double dlon, double lat0, double dlat,
                             OkadaFault f, double Hs)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= nx || y >= ny) return;
    const double rad = M_PI / 180.0;
    const double lon = lon0 + x * dlon, lat = lat0 + y * dlat;
    const double ss = sin(rad * f.strike), cs = cos(rad * f.strike);
    double xp, yp;
    gauss_krueger(lat, lon, f.lat_c, f.lon_c, xp, yp);
    const double uz = okada_uz(xp * ss + yp * cs, -xp * cs + yp * ss, f.depth_c, f.dip, f.length, f.width,
                               f.slip * cos(rad * f.rake), f.slip * sin(rad * f.rake));
    def[(size_t)y * nx + x] = uz / Hs;
}

void launch_okada(const ScenarioDev *s_host, double *def, double lon0, double dlon, double lat0, double dlat,
                  const OkadaFault &f, double Hs, cudaStream_t st)
{
    dim3 block(32, 4);
    dim3 grid((s_host->nx + 31) / 32, (s_host->ny + 3) / 4);
    okada_kernel<<<grid, block, 0, st>>>(s_host->nx, s_host->ny, def, lon0, dlon, lat0, dlat, f, Hs);
}

// max over cells of (float)|U_Z| as float bits (non-negative floats order as unsigned)
__global__ void absmax_kernel(const double *__restrict__ def, long long n, unsigned int *max_bits)
{
    float m = 0.f;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        m = fmaxf(m, (float)fabs(def[i]));
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    __shared__ float red[8];
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 1; k < (int)(blockDim.x >> 5); k++) m = fmaxf(m, red[k]);
        atomicMax(max_bits, __float_as_uint(m));
    }
}

void launch_absmax(const double *def, long long n, unsigned int *max_bits, cudaStream_t st)
{
    cudaMemsetAsync(max_bits, 0, sizeof(unsigned int), st);
    absmax_kernel<<<296, 256, 0, st>>>(def, n, max_bits);
}

__global__ void apply_deformation_kernel(ScenarioDev s, const double *__restrict__ def, int crop_flag, double crop_value,
                                         const unsigned int *__restrict__ max_bits)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    if (x >= s.nx || y >= s.ny) return;
    double U = def[(size_t)y * s.nx + x];
    if (crop_flag == 1) {
        const double thr = crop_value * (double)__uint_as_float(*max_bits);
        if (fabs(U) < thr) U = 0.0;
    } else if (crop_flag == 2) {
        if (fabs(U) < crop_value) U = 0.0;
    }
    const int p = s.ctl->parity;
    const size_t idx = (size_t)y * s.pitch + x;
    const float eta = s.eta[p][idx], dep = s.dep[idx];
    const double h = (double)eta + (double)dep;   // exact in double
    const float dep_n = (float)((double)dep - U);
    // eta and the depth are rounded independently: deriving eta from the
    // rounded depth would quantise the surface to an ulp of the depth
    // (0.24 mm at 4 km); h absorbs that rounding instead (6e-8 relative)
    float eta_n = (float)((double)eta + U);
    if (h == 0.0 || !((double)eta_n + (double)dep_n > 0.0)) eta_n = -dep_n;   // dry stays dry, exactly
    s.dep[idx] = dep_n;
    s.eta[p][idx] = eta_n;
    s.eta_ini[idx] = (float)((double)s.eta_ini[idx] + U);
}

void launch_apply_deformation(const ScenarioDev *s_host, const double *def, int crop_flag, double crop_value,
                              const unsigned int *max_bits, cudaStream_t st)
{
    dim3 grid((s_host->nx + 255) / 256, s_host->ny);
    apply_deformation_kernel<<<grid, 256, 0, st>>>(*s_host, def, crop_flag, crop_value, max_bits);
}

cudaError_t preload_okada_kernels()
{
    cudaFuncAttributes a;
    cudaError_t e;
    if ((e = cudaFuncGetAttributes(&a, okada_kernel)) || (e = cudaFuncGetAttributes(&a, absmax_kernel)) ||
        (e = cudaFuncGetAttributes(&a, apply_deformation_kernel)))
        return e;
    return cudaSuccess;
}

}  // namespace thy
