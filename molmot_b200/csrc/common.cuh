// common.cuh -- shared definitions of the molmot_b200 CUDA library (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <math.h>
#include <memory>
#include <vector>

#include "../../include/molmot_b200.h"

// 2.0 * pi as the reference spells it (molmot/obe/rate_equations_jit.py:35):
// doubling (double)pi is exact, so x * MM_TWO_PI == (x * 2.0) * pi bit for bit.
#define MM_PI 3.141592653589793
#define MM_TWO_PI 6.283185307179586
// hbar hard-coded in molmot/obe/rate_equations_jit.py:27
#define MM_HBAR_JIT 1.0545718e-34

// status bits written per point
#define MM_ST_PIVOT 1
#define MM_ST_NONFINITE 2
#define MM_ST_ZERO_POP 4

// Host-side error reporting (capi.cu).
void mm_set_error(const char *fmt, ...);
int mm_cuda_check(cudaError_t e, const char *what);

// Device-resident molecule ("pack"): one allocation, fixed offsets.
struct mm_pack {
    int n_g, n_e, n_s;
    double Gamma, k, mass;
    int has3d;
    int device;
    double *buf;     // device
    size_t n_buf;    // doubles
    // offsets (in doubles) into buf
    size_t oE, ozd, od2, oBR, oZre, oZim, oZe, oTdm;
    std::vector<unsigned char> act;  // host: d2[g][e][q] >= 1e-15 (active triple pattern)
    std::vector<double> h_br;        // host: branching ratios BR[e][g]
};

// Device-resident parameter sets of beams.
struct mm_beams {
    int n_sets, n_b;
    double gamma_eff;
    int has3d;
    int device;
    double *kdir, *freq, *s0, *bgrad, *khat, *radius;  // device
    int32_t *pol;                                       // device
    int view;  // 1: the arrays belong to another handle (mm_beams_view)
    std::shared_ptr<std::vector<int32_t>> h_pol_store;  // host copy of pol (shared by views)
    const int32_t *h_pol;                               // this handle's first set in it
};

// Parameters of the 1D force kernels (passed by value).
struct ForceParams {
    int n_g, n_e, n_b, n_sets;
    double Gamma, k, hbar, geff;
    const double *E, *zd, *d2, *BR;
    const double *kdir, *freq, *s0, *bgrad;
    const int32_t *pol;
    int layout;
    long long nv, nz, pps, n_points;
    const double *v, *z;
    double *F, *R, *pop;
    int32_t *status;
    int uniform_fb;
};

// Parameters of the fused 1D trajectory kernels (passed by value).
struct TrajParams {
    double dt, z_escape, mass;
    long long n_particles, n_steps;
    int ndim;         // 1: along z;  3: per-axis model (x, y, z)
    int n_avg;        // parameter sets averaged per force evaluation (RF MOT: 2 phases)
    long long i_eq;   // first step whose v^2 enters vsq_sum (temperature); < 0: off
    const double *z0, *v0;          // [N][ndim]
    double *z_final, *v_final;      // [N][ndim]
    double *z_traj, *v_traj;        // [N][n_steps][ndim] or null
    int32_t *n_actual;              // [N]
    double *vsq_sum, *n_samp;       // [N] or null
};

__device__ __forceinline__ double mm_group_sum(double x, int G)
{
    for (int o = G >> 1; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    return x;
}

__device__ __forceinline__ int mm_group_or(int x, int G)
{
    for (int o = G >> 1; o > 0; o >>= 1) x |= __shfl_xor_sync(0xffffffffu, x, o);
    return x;
}

__device__ __forceinline__ float mm_group_sumf(float x, int G)
{
    for (int o = G >> 1; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    return x;
}
