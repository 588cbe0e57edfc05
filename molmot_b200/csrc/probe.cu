// probe.cu -- FMA-throughput probe used as the roofline denominator of the
// force kernels, which are bound by the FP64 / FP32 CUDA-core pipes (no
// tensor-core work exists on this path).  Each thread runs 8 independent
// FMA chains in registers; one FMA counts as 2 FLOP.
#include "common.cuh"

namespace {

template <class T>
__global__ void __launch_bounds__(256) fma_probe_kernel(T *sink, long long iters, T a, T b)
{
    T x0 = (T)threadIdx.x, x1 = x0 + (T)1, x2 = x0 + (T)2, x3 = x0 + (T)3;
    T x4 = x0 + (T)4, x5 = x0 + (T)5, x6 = x0 + (T)6, x7 = x0 + (T)7;
    for (long long i = 0; i < iters; i++) {
        x0 = fma(x0, a, b); x1 = fma(x1, a, b); x2 = fma(x2, a, b); x3 = fma(x3, a, b);
        x4 = fma(x4, a, b); x5 = fma(x5, a, b); x6 = fma(x6, a, b); x7 = fma(x7, a, b);
    }
    const T s = ((x0 + x1) + (x2 + x3)) + ((x4 + x5) + (x6 + x7));
    if (s == (T)-12345.678) sink[0] = s;  // keeps the chains live, never true in practice
}

}  // namespace

// which: 0 = FP64, 1 = FP32.  Writes elapsed milliseconds and the FLOP count.
extern "C" MM_API int mm_peak_probe(int32_t which, int64_t iters, double *ms_out, double *flops_out,
                                    void *stream)
{
    if (!ms_out || !flops_out || iters < 1) { mm_set_error("mm_peak_probe: bad arguments"); return -1; }
    int dev = 0, nsm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    cudaStream_t st = (cudaStream_t)stream;
    const int blocks = nsm * 8, threads = 256;
    void *sink = nullptr;
    if (mm_cuda_check(cudaMalloc(&sink, 16), "cudaMalloc")) return -3;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, st);
    if (which == 0)
        fma_probe_kernel<double><<<blocks, threads, 0, st>>>((double *)sink, iters, 0.999999, 1e-7);
    else
        fma_probe_kernel<float><<<blocks, threads, 0, st>>>((float *)sink, iters, 0.999999f, 1e-7f);
    cudaEventRecord(e1, st);
    int rc = mm_cuda_check(cudaEventSynchronize(e1), "mm_peak_probe") ? -3 : 0;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(sink);
    *ms_out = ms;
    *flops_out = 2.0 * 8.0 * (double)iters * blocks * threads;
    return rc;
}
