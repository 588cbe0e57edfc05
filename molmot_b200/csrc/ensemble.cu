// ensemble.cu -- device reductions over trajectory ensembles: per-time-bin
// statistics of the particles still inside the trap and histograms, the
// heavy parts of molmot/mot/analysis.py (sigma_vs_time :128-192,
// temperature_vs_time :195-246, density_vs_time :249-287, gaussian_fit /
// maxwell_boltzmann_fit_1d histograms :28-125).  C-ABI: mm_ensemble_stats,
// mm_histogram.
//
// Layout: a quantity x of particle p at time index j is x[p * stride + j]
// (the [N][n_steps] trajectory arrays of mm_traj_run with ndim = 1, or one
// column of any row-major array).
#include <stdio.h>
#include <algorithm>
#include "common.cuh"

namespace {

constexpr int kStatThreads = 256;

// Deterministic block sum (fixed tree over the block's threads).
template <int NV>
__device__ void block_sum(double (&v)[NV], double *sh)
{
    const int tid = threadIdx.x;
#pragma unroll
    for (int k = 0; k < NV; k++) sh[k * kStatThreads + tid] = v[k];
    __syncthreads();
    for (int s = kStatThreads / 2; s > 0; s >>= 1) {
        if (tid < s)
#pragma unroll
            for (int k = 0; k < NV; k++) sh[k * kStatThreads + tid] += sh[k * kStatThreads + tid + s];
        __syncthreads();
    }
#pragma unroll
    for (int k = 0; k < NV; k++) v[k] = sh[k * kStatThreads];
    __syncthreads();
}

// One CTA per time bin.  Pass 1: count, sum z, sum v, sum v^2 over the
// particles with |z| < r_alive; pass 2: squared deviations from the means
// (two-pass, as numpy.std).  out[bin] = {n, mean_z, mean_v, var_z, var_v, mean_v2}.
__global__ void __launch_bounds__(kStatThreads)
ensemble_stats_kernel(const double *z, const double *v, long long n, long long stride,
                      const long long *idx, double r_alive, double *out)
{
    __shared__ double sh[4 * kStatThreads];
    const long long j = idx[blockIdx.x];
    double a[4] = {0.0, 0.0, 0.0, 0.0};
    for (long long p = threadIdx.x; p < n; p += kStatThreads) {
        const double zp = z[p * stride + j];
        if (fabs(zp) < r_alive) {
            const double vp = v[p * stride + j];
            a[0] += 1.0;
            a[1] += zp;
            a[2] += vp;
            a[3] = fma(vp, vp, a[3]);
        }
    }
    block_sum<4>(a, sh);
    const double cnt = a[0];
    const double mz = cnt > 0.0 ? a[1] / cnt : 0.0, mv = cnt > 0.0 ? a[2] / cnt : 0.0;
    double b[2] = {0.0, 0.0};
    for (long long p = threadIdx.x; p < n; p += kStatThreads) {
        const double zp = z[p * stride + j];
        if (fabs(zp) < r_alive) {
            const double dz = zp - mz, dv = v[p * stride + j] - mv;
            b[0] = fma(dz, dz, b[0]);
            b[1] = fma(dv, dv, b[1]);
        }
    }
    block_sum<2>(b, sh);
    if (threadIdx.x == 0) {
        double *o = out + (size_t)blockIdx.x * 6;
        o[0] = cnt;
        o[1] = mz;
        o[2] = mv;
        o[3] = cnt > 0.0 ? b[0] / cnt : 0.0;
        o[4] = cnt > 0.0 ? b[1] / cnt : 0.0;
        o[5] = cnt > 0.0 ? a[3] / cnt : 0.0;
    }
}

// numpy.histogram with equal bins on [lo, hi] (numpy/lib/_histograms_impl.py,
// the equal-width branch): index = trunc(((x - lo) / (hi - lo)) * bins), the
// value hi in the last bin, then the two corrections against the edges of
// numpy.linspace(lo, hi, bins + 1) -- edges[k] = k * ((hi - lo) / bins) + lo,
// edges[bins] = hi -- so every value lands between its bin's edges.  Values
// outside [lo, hi] and NaNs are not counted.  Explicit roundings reproduce
// numpy's uncontracted arithmetic.
__global__ void histogram_kernel(const double *x, long long n, long long stride, double lo, double hi,
                                 int bins, unsigned long long *counts)
{
    const double delta = __dsub_rn(hi, lo);
    const double step = __ddiv_rn(delta, (double)bins);
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const double xi = x[i * stride];
        if (!(xi >= lo && xi <= hi)) continue;
        int k = (int)__dmul_rn(__ddiv_rn(__dsub_rn(xi, lo), delta), (double)bins);
        if (k >= bins) k = bins - 1;
        const double e0 = __dadd_rn(__dmul_rn((double)k, step), lo);
        const double e1 = (k + 1 == bins) ? hi : __dadd_rn(__dmul_rn((double)(k + 1), step), lo);
        if (xi < e0) k--;
        else if (xi >= e1 && k != bins - 1) k++;
        atomicAdd(&counts[k], 1ull);
    }
}

}  // namespace

extern "C" int mm_ensemble_stats(const double *z, const double *v, int64_t n_particles, int64_t stride,
                                 const int64_t *time_index, int32_t n_bins, double r_alive, double *out,
                                 void *stream)
{
    if (!z || !v || !time_index || !out) { mm_set_error("z, v, time_index and out are required"); return -1; }
    if (n_particles < 0 || stride < 1 || n_bins < 0) { mm_set_error("bad sizes"); return -1; }
    if (n_bins == 0) return 0;
    ensemble_stats_kernel<<<n_bins, kStatThreads, 0, (cudaStream_t)stream>>>(
        z, v, n_particles, stride, (const long long *)time_index, r_alive, out);
    return mm_cuda_check(cudaGetLastError(), "ensemble_stats_kernel launch") ? -3 : 0;
}

extern "C" int mm_histogram(const double *x, int64_t n, int64_t stride, double lo, double hi, int32_t bins,
                            uint64_t *counts, void *stream)
{
    if (!x || !counts) { mm_set_error("x and counts are required"); return -1; }
    if (n < 0 || stride < 1 || bins < 1 || !(hi > lo)) { mm_set_error("bad histogram arguments"); return -1; }
    cudaStream_t st = (cudaStream_t)stream;
    if (mm_cuda_check(cudaMemsetAsync(counts, 0, sizeof(uint64_t) * bins, st), "cudaMemsetAsync")) return -3;
    if (n == 0) return 0;
    const long long blocks = std::min<long long>((n + 255) / 256, 148 * 16);
    histogram_kernel<<<(unsigned)blocks, 256, 0, st>>>(x, n, stride, lo, hi, bins,
                                                       (unsigned long long *)counts);
    return mm_cuda_check(cudaGetLastError(), "histogram_kernel launch") ? -3 : 0;
}
