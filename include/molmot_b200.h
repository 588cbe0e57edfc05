/*
 * molmot_b200.h -- C ABI of the B200 rate-equation steady-state force library.
 *
 * Plain C: opaque handles, plain pointers and sizes, integer return codes.
 * All array arguments of the compute calls are DEVICE pointers owned by the
 * caller; `stream` is a cudaStream_t passed as void* (NULL = legacy default
 * stream).  Calls are stream-ordered and do not synchronise the host unless
 * stated.  Handles are immutable after creation and may be shared between
 * host threads.
 *
 * Return codes: 0 ok; < 0 argument or CUDA error (see mm_last_error()).
 * Per-point numerical conditions go to the optional status array
 * (bit 1: a pivot below 1e-30 was skipped, bit 2: non-finite result,
 *  bit 4: every population clamped to zero).
 *
 * Each entry point names the reference interface it replaces (paths within
 * the molmot project).
 */
#ifndef MOLMOT_B200_H
#define MOLMOT_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define MM_API __attribute__((visibility("default")))
#else
#define MM_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define MM_MAX_GROUND 48
#define MM_MAX_EXCITED 16
#define MM_MAX_BEAMS 32

/* precision of the force kernels */
#define MM_PREC_FP64 0         /* plain FP64, reference operation order */
#define MM_PREC_FP32_REFINE 1  /* FP32-bulk: FP32 Lorentzians with FP64 sums, populations in FP64
                                  through the excited-state chain (reduced.cuh), one point or
                                  particle per thread (the name is kept for the ABI) */
#define MM_PREC_FP64_REDUCED 2 /* mm_force_batch and mm_force_adjoint: FP64 rates in the plain
                                  form's operation order, populations from the same FP64
                                  excited-chain solve as MM_PREC_FP32_REFINE (agrees with
                                  MM_PREC_FP64 to rounding) */

/* point layouts of mm_force_batch */
#define MM_LAYOUT_POINTS 0 /* v[i], z[i]; point i belongs to set i / points_per_set */
#define MM_LAYOUT_GRID 1   /* per set the outer product v[nv] x z[nz], index (set*nv+iv)*nz+iz */

typedef struct mm_pack mm_pack;
typedef struct mm_beams mm_beams;

/* Molecule description (host pointers, copied by mm_pack_create).
 * Replaces molmot/molecules/sroh.py:87-174 MolecularData as consumed by
 * molmot_cuda/rate_equations_cuda.py:399-441 CUDAMolData. */
typedef struct {
    int32_t n_ground, n_excited;
    const double *energies;      /* [n_g + n_e] Hz                                 */
    const double *d_squared;     /* [n_g][n_e][3] |tdm|^2, q = sigma-, pi, sigma+   */
    const double *zeeman_z_diag; /* [n_g + n_e] Zeeman diagonal (Gamma/2pi per G)  */
    double Gamma;                /* rad/s                                          */
    double k;                    /* 1/m                                            */
    double mass;                 /* kg                                             */
    /* 3D model only (may be NULL for 1D use): ground Zeeman blocks and |tdm| */
    const double *zeeman_ground_re; /* [3][n_g][n_g] x, y, z real parts          */
    const double *zeeman_ground_im; /* [3][n_g][n_g] imaginary parts             */
    const double *zeeman_excited_z; /* [n_e] Re diag of zeeman_z excited block   */
    const double *tdm_abs;          /* [n_g][n_e][3] |tdm[g, n_g+e, q]|          */
} mm_mol_desc;

/* Parameter sets of beams (host pointers, copied by mm_beams_create).
 * Each of n_sets sets has n_beams beams.  Replaces the LaserBeam lists of
 * molmot/obe/fields.py:22-58 (kdir_z, freq_offset, polarization, s0) plus
 * the per-call B_gradient of molmot/obe/rate_equations_jit.py:148. */
typedef struct {
    int32_t n_beams;
    const double *kdir;       /* [n_sets][n_beams] z-projection of k (1D)          */
    const double *freq;       /* [n_sets][n_beams] absolute frequency, Hz          */
    const int32_t *pol;       /* [n_sets][n_beams] 0, 1, 2                         */
    const double *s0;         /* [n_sets][n_beams] saturation parameter            */
    const double *b_gradient; /* [n_sets] T/m                                      */
    double gamma_eff;         /* Gamma_eff_factor (same for all sets)              */
    /* 3D model only (may be NULL): unit k vectors and 1/e^2 radii (<= 0: plane wave) */
    const double *khat;       /* [n_sets][n_beams][3]                              */
    const double *radius;     /* [n_sets][n_beams]                                 */
} mm_beam_desc;

typedef struct {
    int32_t precision;        /* MM_PREC_*                                         */
    int32_t layout;           /* MM_LAYOUT_*                                       */
    int64_t points_per_set;   /* MM_LAYOUT_POINTS                                  */
    int64_t nv, nz;           /* MM_LAYOUT_GRID                                    */
    double hbar;              /* J s; <= 0 selects 1.0545718e-34 (the JIT value)   */
    int32_t uniform_fallback; /* 1: p = 1/n_g when every population clamps to 0
                                 (reference CUDA / Python); 0: keep zeros (JIT)   */
    int32_t reserved;
} mm_batch_opts;

/* Last error message of the calling host thread ("" if none). */
MM_API const char *mm_last_error(void);

/* Library version string. */
MM_API const char *mm_version(void);

/* Upload a molecule; replaces CUDAMolData molecule transfer
 * (molmot_cuda/rate_equations_cuda.py:399-441). */
MM_API int mm_pack_create(const mm_mol_desc *desc, mm_pack **out);
MM_API int mm_pack_destroy(mm_pack *pack);

/* Upload n_sets parameter sets of beams; replaces CUDAMolData beam transfer
 * (molmot_cuda/rate_equations_cuda.py:370-397, 427-441). */
MM_API int mm_beams_create(const mm_beam_desc *desc, int32_t n_sets, mm_beams **out);
MM_API int mm_beams_destroy(mm_beams *beams);

/* A handle for the parameter sets [first_set, first_set + n_sets) of `parent`
 * that shares the parent's device arrays (no device allocation or copy), so a
 * long batch can be computed in chunks, e.g. to overlap each chunk's
 * device->host copy with the next chunk's computation.  No counterpart in the
 * reference.  Destroy it with mm_beams_destroy before the parent. */
MM_API int mm_beams_view(const mm_beams *parent, int32_t first_set, int32_t n_sets, mm_beams **out);

/*
 * Steady-state force, populations and scattering rate for a batch of points.
 * Replaces solve_rate_equations_batch (molmot_cuda/rate_equations_cuda.py:448-544,
 * kernel :51-277) and, point by point, _rate_eq_core
 * (molmot/obe/rate_equations_jit.py:18-145).
 * v, z: device arrays (layout per opts).  Outputs: F[n], R[n] (R nullable),
 * pop[n][n_ground] (nullable), status[n] (nullable), n = total points.
 * Molecules up to MM_MAX_GROUND x MM_MAX_EXCITED: those with n_ground <= 12
 * and n_excited <= 4 run the register-resident kernels; larger ones run
 * shared-memory kernels (a group of 16 or 32 lanes per point) in FP64 for
 * every precision -- the reference's elimination for MM_PREC_FP64, the
 * excited-chain solve for the other precisions when every set passes its
 * structural checks (else the elimination).
 */
MM_API int mm_force_batch(const mm_pack *pack, const mm_beams *beams, const double *v,
                   const double *z, int64_t n_points, const mm_batch_opts *opts,
                   double *F, double *R, double *pop, int32_t *status, void *stream);

/*
 * Steady-state force and its gradient with respect to each beam's frequency
 * and saturation parameter and the set's B' (FP64 form).  Implicit
 * differentiation through the steady state: one transposed solve per point
 * with the elimination's own factors (M'^T lambda = dF/dp), on the fixed set
 * of unclamped populations.  No counterpart in the reference (new on this
 * path); the reference computes these only by finite differences of
 * _rate_eq_core.  grad: [n][2 n_beams + 1] rows
 * (dF/dfreq_b, b = 0..n_beams-1; dF/ds0_b; dF/dB'), Newton per Hz, per unit
 * s0 and per T/m.  Same layouts as mm_force_batch.
 * opts->precision: MM_PREC_FP64 (the elimination adjoint) or
 * MM_PREC_FP64_REDUCED (the adjoint of the excited-chain solve, one point per
 * thread; when any set fails the reduced form's structural checks the whole
 * batch runs the elimination adjoint).  Other precisions are rejected.
 * Molecules beyond n_ground 12 / n_excited 4 run the elimination adjoint in
 * shared memory (group of 16 or 32 lanes per point) for both precisions.
 */
MM_API int mm_force_adjoint(const mm_pack *pack, const mm_beams *beams, const double *v,
                            const double *z, int64_t n_points, const mm_batch_opts *opts,
                            double *F, double *grad, void *stream);

/*
 * Uneven batches: many different molecules (n_ground 2..48, n_excited 1..16),
 * each with its own beam set and number of points.  No single counterpart in
 * the reference, which handles one molecule per CUDAMolData
 * (molmot_cuda/rate_equations_cuda.py:399-441) and launches per call.
 */
typedef struct mm_bank mm_bank;
typedef struct mm_uneven_plan mm_uneven_plan;

/* Upload n_mol molecules (1D fields of mm_mol_desc) into one device bank. */
MM_API int mm_bank_create(const mm_mol_desc *mols, int32_t n_mol, mm_bank **out);
MM_API int mm_bank_destroy(mm_bank *bank);

typedef struct {
    int32_t warps_per_cta[3]; /* per size class (n_g <= 16, <= 32, <= 48); <= 0: default */
    int32_t chunk_groups;     /* points per work item, in CTA widths; <= 0: 8          */
} mm_uneven_opts;

/* Work plan: molecule m owns points [point_offsets[m], point_offsets[m+1])
 * (host array of n_mol + 1).  Allocates the plan's task lists and counters. */
MM_API int mm_uneven_plan_create(const mm_bank *bank, const int64_t *point_offsets,
                                 const mm_uneven_opts *opts, mm_uneven_plan **out);
MM_API int mm_uneven_plan_destroy(mm_uneven_plan *plan);

/* Forces of every point (device arrays v, z, F [n], R and status nullable).
 * beams: one set per molecule.  persistent = 1: one persistent launch per
 * size class drawing work items from the plan's counters (reset on `stream`
 * by this call, so the whole call can be captured in a CUDA graph);
 * persistent = 0: one CTA per work item.  hbar <= 0: 1.0545718e-34. */
MM_API int mm_uneven_force(const mm_uneven_plan *plan, const mm_beams *beams, const double *v,
                           const double *z, double hbar, int32_t uniform_fallback,
                           int32_t persistent, double *F, double *R, int32_t *status,
                           void *stream);

/*
 * mm_uneven_force_static: the same forces as mm_uneven_force (persistent = 1)
 * with no plan and no allocation of any kind.  It has no counterpart in the
 * reference.  It is for callers that cannot allocate when they ask for
 * forces: a point layout that changes every call (adaptive sampling, an
 * ensemble losing particles) would otherwise create and destroy a plan per
 * call, and cudaFree synchronises the whole device; a host application that
 * has handed the device memory to its own pool has none left to allocate.
 * The work list and work counters live in a fixed 1 MiB array in the
 * library's device memory (per GPU), so a batch may make at most 43,680 work
 * items (point chunks of chunk_groups CTA widths); a larger one is refused
 * with an error naming the limit.  The counters are zeroed on `stream` by
 * every call.  The first call on each GPU (and the first after a reset of
 * its context) looks up the array's device address (cudaGetSymbolAddress);
 * make that first call before any stream capture on that GPU.  Calls share
 * the array and host staging arrays: two calls race unless the second is
 * ordered after the first on the GPU -- issued on the same stream, or on a
 * stream that waits on an event recorded after the first call -- and calls
 * from two host threads at once race on the host arrays.
 */
MM_API int mm_uneven_force_static(const mm_bank *bank, const mm_beams *beams,
                                  const int64_t *point_offsets, const mm_uneven_opts *opts,
                                  const double *v, const double *z, double hbar,
                                  int32_t uniform_fallback, double *F, double *R,
                                  int32_t *status, void *stream);

/* Options of mm_traj_run. */
typedef struct {
    int32_t ndim;      /* 1: along z; 3: per-axis model of trajectories.py:78-156        */
    int32_t n_avg;     /* 1: beam set 0; 2: average of sets 0 and 1 (RF MOT phases)      */
    int64_t n_steps;   /* samples per trajectory, the initial one included               */
    double dt;         /* s                                                              */
    double r_escape;   /* m: |z| (ndim 1) or |r| (ndim 3) beyond which a particle stops  */
    int64_t i_eq;      /* first step whose v^2 enters vsq_sum (with vsq_sum non-NULL)    */
    int32_t precision; /* MM_PREC_*                                                      */
    int32_t reserved;
    double hbar;       /* J s; <= 0 selects 1.0545718e-34                                */
} mm_traj_opts;

/*
 * Independent trajectories, one launch for all steps.  ndim = 1 replaces
 * traj_kernel / simulate_trajectories_cuda (molmot_cuda/trajectories_cuda.py:44-280,
 * 305-426) and _trajectory_1d_jit (molmot/propagation/trajectories_jit.py:18-58);
 * ndim = 3 replaces simulate_trajectories_3d (molmot/propagation/trajectories.py:78-156);
 * with vsq_sum / n_samp it also accumulates the sums of monte_carlo_temperature
 * (molmot/propagation/trajectories.py:159-229).  Arrays are [N][ndim]
 * (r_traj / v_traj: [N][n_steps][ndim], nullable; vsq_sum / n_samp: [N], nullable).
 * Molecules beyond n_ground 12 / n_excited 4 run the plain FP64 force in
 * shared memory (group of 16 or 32 lanes per particle) for both precisions.
 */
MM_API int mm_traj_run(const mm_pack *pack, const mm_beams *beams, const mm_traj_opts *opts,
                       const double *r0, const double *v0, int64_t n_particles,
                       double *r_final, double *v_final, int32_t *n_actual, double *r_traj,
                       double *v_traj, double *vsq_sum, double *n_samp, void *stream);

/* Options of mm_traj_grad_run. */
#define MM_TGRAD_MAX_PAR 8
typedef struct {
    int64_t n_steps;     /* Euler steps in this call                                          */
    int64_t step0;       /* absolute step index of the state passed in (0 for a new run)      */
    int64_t ckpt_every;  /* with ckpt non-NULL: save the state after every ckpt_every-th step  */
    double dt;           /* s                                                                 */
    double r_escape;     /* m: |r| beyond which a particle stops                              */
    double hbar;         /* J s; <= 0 selects 1.0545718e-34                                   */
    uint64_t seed;       /* Philox key of the recoil kicks                                    */
    int32_t kicks;       /* != 0: photon-recoil kicks, held fixed under differentiation       */
    int32_t n_par;       /* parameters theta_k, 1..MM_TGRAD_MAX_PAR                           */
    int32_t freq_par[MM_MAX_BEAMS]; /* parameter whose value adds to beam b's frequency, or -1 */
    int32_t s0_par[MM_MAX_BEAMS];   /* parameter whose value adds to beam b's s0, or -1        */
    int32_t bprime_par;  /* parameter that adds to B', or -1                                  */
    int32_t reserved;
} mm_tgrad_opts;

/*
 * Trajectories of the per-axis 3D MOT model (molmot/propagation/
 * trajectories.py:78-156; the model of mm_traj_run with ndim = 3, beam set 0)
 * carried with their tangents d(r, v)/d theta_k (forward mode, the force's
 * gradient from the FP64-reduced adjoint each step).  Optional photon-recoil
 * kicks as in mm_traj3d_run, with N ~ Poisson((R_x + R_y + R_z) dt) events per
 * step.  No counterpart in the reference (new on this path).
 * state [N][6 + 6 n_par] (device, in/out): r[3], v[3], dr[3][n_par], dv[3][n_par];
 * n_actual [N] (device, in/out; 0 for a new run): the absolute step a particle
 * stopped at, or step0 + n_steps.  ckpt [n_steps / ckpt_every][N][6 + 6 n_par]
 * (nullable): the state after steps ckpt_every, 2 ckpt_every, ... of the call;
 * passing checkpoint c back as state with step0 + (c + 1) ckpt_every resumes
 * the run bit for bit.  Beam set 0 must pass the reduced form's structural
 * checks (every ground state pumped, excited chain strongly connected), and
 * the molecule must fit the register-resident class (n_ground <= 12,
 * n_excited <= 4).
 */
MM_API int mm_traj_grad_run(const mm_pack *pack, const mm_beams *beams, const mm_tgrad_opts *opts,
                            int64_t n_particles, double *state, int32_t *n_actual, double *ckpt,
                            void *stream);

/* Options of mm_traj3d_grad_run. */
typedef struct {
    int64_t n_steps;     /* as mm_traj3d_run: step0 = 0 applies the first half kick and runs updates
                            j = 1 .. n_steps - 1; step0 > 0 runs updates j = step0 .. step0 + n_steps - 1 */
    int64_t step0;       /* absolute index of the first update (0 for a new run)                   */
    int64_t ckpt_every;  /* with ckpt non-NULL: the state after every update j with j % ckpt_every == 0;
                            resume from it with step0 = j + 1                                     */
    double dt;           /* s                                                                     */
    double r_escape;     /* m: |r| beyond which a particle stops                                  */
    double hbar;         /* J s; <= 0 selects CODATA 1.054571817e-34 (the 3D reference's value)  */
    double gap_tol;      /* relative ground Zeeman eigenvalue gap below which the eigenbasis
                            derivative is undefined (status MM_ST_DEGENERATE); <= 0 selects 1e-9 */
    uint64_t seed;       /* Philox key of the recoil kicks (mm_traj3d_run's)                      */
    int32_t kicks;       /* != 0: recoil kicks, held fixed under differentiation                  */
    int32_t n_par;       /* parameters theta_k, 1..MM_TGRAD_MAX_PAR                               */
    int32_t freq_par[MM_MAX_BEAMS]; /* parameter whose value adds to beam b's frequency, or -1     */
    int32_t s0_par[MM_MAX_BEAMS];   /* parameter whose value adds to beam b's s0, or -1            */
    int32_t bprime_par;  /* parameter that adds to B', or -1                                      */
    int32_t reserved;
} mm_t3grad_opts;

#define MM_ST_DEGENERATE 8 /* status bit of mm_traj3d_grad_run: a step met a degenerate ground
                              Zeeman spectrum (gap below gap_tol), where d(force)/d(position)
                              is not defined; the terms through that pair were dropped */

/*
 * The 3D leapfrog ensemble of mm_traj3d_run (MOTSimulator3D.simulate_trajectory_3d,
 * molmot/mot/simulator_3d.py:443-504; beam set 0, its bits and recoil kicks) carried with
 * its tangents d(r, v)/d theta_k (forward mode) through the 24-beam force, the field
 * dependence of the ground Zeeman eigenbasis included (first-order perturbation theory of
 * the eigenvectors, defined for a non-degenerate spectrum; the reference's SrOH spectrum is
 * degenerate and is flagged).  No counterpart in the reference (new on this path).
 * state [N][6 + 6 n_par] (in/out): r[3], v_half[3], dr[3][n_par], dv_half[3][n_par]; for
 * step0 = 0 pass v0 and the initial tangents (zero for initial conditions that do not depend
 * on theta) in place of v_half.  vsync [N][3 + 3 n_par] (out): the synchronised velocity of
 * the last update and its tangent (mean kinetic energy gradients: m v . dv).  n_actual [N]
 * (in/out; 0 for a new run), status [N] (out), n_events [N] (nullable).  ckpt
 * [mm_traj3d_grad_checkpoints(step0, n_steps, ckpt_every)][N][6 + 6 n_par] (nullable).
 * Molecules up to 16 ground and 8 excited states.
 */
MM_API int mm_traj3d_grad_run(const mm_pack *pack, const mm_beams *beams, const mm_t3grad_opts *opts,
                              int64_t n_particles, double *state, double *vsync, int32_t *n_actual,
                              int32_t *status, int32_t *n_events, double *ckpt, void *stream);

/* Number of checkpoints one mm_traj3d_grad_run call writes. */
MM_API int64_t mm_traj3d_grad_checkpoints(int64_t step0, int64_t n_steps, int64_t ckpt_every);

/*
 * N independent 1D trajectories with symplectic Euler, one beam set (set 0).
 * Replaces traj_kernel / simulate_trajectories_cuda
 * (molmot_cuda/trajectories_cuda.py:44-280, 305-426) and
 * _trajectory_1d_jit (molmot/propagation/trajectories_jit.py:18-58).
 * z_traj / v_traj: [N][n_steps] or NULL.  n_actual: [N] steps run.
 */
MM_API int mm_traj1d_run(const mm_pack *pack, const mm_beams *beams, const double *z0,
                  const double *v0, int64_t n_particles, double dt, int64_t n_steps,
                  double z_escape, const mm_batch_opts *opts, double *z_final,
                  double *v_final, int32_t *n_actual, double *z_traj, double *v_traj,
                  void *stream);

/*
 * 3D steady-state force at points (r[i], v[i]) (arrays [n][3]); point i uses
 * beam set i / points_per_set.  Replaces rate_eq_force_3d
 * (molmot/mot/simulator_3d.py:168-365) and rate_eq_force_3d_batch
 * (molmot_cuda/simulator_3d_cuda.py:666-754; that kernel's Jacobi eigensolver
 * is replaced by a correct one).  Needs a pack with the 3D fields and beam
 * sets with khat; molecules up to 16 ground and 8 excited states.  hbar <= 0 selects CODATA 1.054571817e-34 (the 3D
 * reference path's value).  Outputs: F[n][3], R[n] (nullable),
 * pop[n][n_ground] (nullable), status[n] (nullable).
 */
MM_API int mm_force3d_batch(const mm_pack *pack, const mm_beams *beams, const double *r,
                            const double *v, int64_t n_points, int64_t points_per_set, double hbar,
                            double *F, double *R, double *pop, int32_t *status, void *stream);

/*
 * 3D leapfrog ensemble, one launch for all steps (beam set 0).  Replaces
 * MOTSimulator3D.simulate_trajectory_3d / simulate_ensemble_3d
 * (molmot/mot/simulator_3d.py:443-532) and simulate_ensemble_3d_cuda
 * (molmot_cuda/simulator_3d_cuda.py:890-973).  step0 = 0: v0 is the initial
 * velocity and the first half kick is applied; step0 > 0 resumes a run:
 * r0 / v0 are r_out / vh_out of the previous call (checkpoint).  kicks != 0
 * adds photon-recoil kicks: N ~ Poisson(R dt) events per step, 2N isotropic
 * kicks of hbar k / m, random numbers from Philox4x32-10 keyed by seed with
 * counter (particle, step, draw, 0) -- reproducible across checkpoints.
 * Outputs [N][3]: r_out, vh_out (half-step velocity), v_out (synchronised,
 * nullable); n_actual[N]; r_traj / v_traj [N][n_steps][3] (nullable);
 * ke[N] = m |v|^2 / 2 at the end (nullable); n_events[N] (nullable).
 */
MM_API int mm_traj3d_run(const mm_pack *pack, const mm_beams *beams, const double *r0,
                         const double *v0, int64_t n_particles, int64_t step0, int64_t n_steps,
                         double dt, double r_escape, int32_t kicks, uint64_t seed, double hbar,
                         double *r_out, double *vh_out, double *v_out, int32_t *n_actual,
                         double *r_traj, double *v_traj, double *ke, int32_t *n_events,
                         void *stream);

/*
 * Per-time-bin statistics of a trajectory ensemble (the reductions of
 * sigma_vs_time, temperature_vs_time and density_vs_time,
 * molmot/mot/analysis.py:128-287).  z, v: device arrays, value of particle p
 * at time index j at [p * stride + j]; time_index: device array of n_bins
 * indices.  Particles with |z| < r_alive count.  out (device, [n_bins][6]):
 * count, mean z, mean v, variance of z, variance of v (population, two-pass),
 * mean v^2.
 */
MM_API int mm_ensemble_stats(const double *z, const double *v, int64_t n_particles, int64_t stride,
                             const int64_t *time_index, int32_t n_bins, double r_alive, double *out,
                             void *stream);

/*
 * numpy.histogram of x[i * stride], i < n, with `bins` equal bins on [lo, hi]
 * (the histograms of gaussian_fit and maxwell_boltzmann_fit_1d,
 * molmot/mot/analysis.py:28-125).  counts: device array of bins uint64,
 * overwritten.
 */
MM_API int mm_histogram(const double *x, int64_t n, int64_t stride, double lo, double hi, int32_t bins,
                        uint64_t *counts, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* MOLMOT_B200_H */
