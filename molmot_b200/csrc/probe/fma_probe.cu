// fma_probe.cu -- FMA-throughput probe: a measurement aid of bench.py, built
// into its own library (libmolmot_probe.so), not part of the product ABI.
// It gives the roofline denominators of the force kernels, which are bound by
// the FP64 / FP32 CUDA-core pipes (no tensor-core work exists on this path).
// Each thread runs 8 independent FMA chains in registers; one FMA counts as
// 2 FLOP.
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

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

int fail(cudaError_t e, const char *what)
{
    if (e == cudaSuccess) return 0;
    fprintf(stderr, "fma_peak_probe: %s: %s\n", what, cudaGetErrorString(e));
    return -3;
}

}  // namespace

// which: 0 = FP64, 1 = FP32.  Runs the FMA loop on every SM of the current
// device on `stream`, synchronises, and writes the elapsed milliseconds and
// the FLOP count.  Returns 0, -1 for bad arguments, -3 for a CUDA error.
extern "C" __attribute__((visibility("default"))) int fma_peak_probe(int32_t which, int64_t iters,
                                                                     double *ms_out, double *flops_out,
                                                                     void *stream)
{
    if (!ms_out || !flops_out || iters < 1 || which < 0 || which > 1) return -1;
    int dev = 0, nsm = 0;
    if (fail(cudaGetDevice(&dev), "cudaGetDevice")) return -3;
    if (fail(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev), "cudaDeviceGetAttribute"))
        return -3;
    cudaStream_t st = (cudaStream_t)stream;
    const int blocks = nsm * 8, threads = 256;
    void *sink = nullptr;
    if (fail(cudaMalloc(&sink, 16), "cudaMalloc")) return -3;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, st);
    if (which == 0)
        fma_probe_kernel<double><<<blocks, threads, 0, st>>>((double *)sink, iters, 0.999999, 1e-7);
    else
        fma_probe_kernel<float><<<blocks, threads, 0, st>>>((float *)sink, iters, 0.999999f, 1e-7f);
    cudaEventRecord(e1, st);
    int rc = fail(cudaGetLastError(), "launch");
    if (!rc) rc = fail(cudaEventSynchronize(e1), "cudaEventSynchronize");
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(sink);
    *ms_out = ms;
    *flops_out = 2.0 * 8.0 * (double)iters * blocks * threads;
    return rc;
}
