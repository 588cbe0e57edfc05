// large.cuh -- host entry of the shared-memory 1D kernels (large.cu) for
// molecules beyond the register-resident classes of force1d.cu.
#pragma once
#include "common.cuh"

// Register-resident classes of force1d.cu: n_ground <= 12 and n_excited <= 4.
inline bool mm_register_class(int n_g, int n_e) { return n_g <= 12 && n_e <= 4; }

// Force maps of mm_force_batch (P filled and validated as there); reduced:
// populations from the excited-chain solve (every set must pass its
// structural checks), else the elimination.
int mm_large_force(const ForceParams &P, long long pps, bool reduced, cudaStream_t st);

// mm_force_adjoint's elimination adjoint (grad rows [n][2 n_beams + 1]).
int mm_large_adjoint(const ForceParams &P, long long pps, double *grad, cudaStream_t st);

// mm_traj_run's trajectories with the plain FP64 force.
int mm_large_traj(const ForceParams &P, const TrajParams &T, cudaStream_t st);
