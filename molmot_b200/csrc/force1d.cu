// force1d.cu -- batched 1D steady-state force and fused 1D trajectory
// kernels, and their C-ABI entry points (mm_force_batch, mm_force_adjoint,
// mm_traj_run, mm_traj1d_run, mm_traj_grad_run).
//
// One CTA works on one parameter set: its prologue stages the molecule and
// the set's beams into shared memory and compacts the active
// (ground, beam, excited) triples; then its threads stream over the set's
// points.
//  * Plain FP64 form: the reference's elimination (rate_core.cuh).  Force
//    maps (force_plain_kernel) and the adjoint (force_plain_adjoint_kernel):
//    rates one point per thread into a shared table, then the elimination
//    on groups of 2 (force) or 4 (adjoint, which keeps L) lanes per point,
//    then (adjoint) the gradient passes one point per thread.  Trajectories
//    (traj1d_kernel): a particle per group of G = 4 lanes (solve_point).
//  * FP32-bulk and FP64-reduced forms (force_reduced_kernel,
//    traj1d_reduced_kernel): one point or particle per thread (two points
//    per thread for FP32 force maps without populations), populations from
//    the excited-state chain (reduced.cuh).
#include <stdio.h>
#include <algorithm>
#include "rate_core.cuh"
#include "reduced.cuh"
#include "kicks.cuh"
#include "large.cuh"

namespace {

constexpr int kThreads = 128;

// Plain FP64 force maps in two phases per round of TH points (one per thread):
//  1. each thread computes its point's saturated rates R[g,e] and force terms
//     F_g (reduced_rates<F64>: the reference's detuning chain and products,
//     rate_equations_jit.py:58-90; the triples of a ground state run excited-
//     state-major, beams ascending, so R[g,e] has the reference's summation
//     order and F_g, s_g differ from it in rounding only) into a shared table;
//  2. groups of G lanes solve the TH points' population systems from the
//     table (group_factor: the reference's elimination with partial
//     pivoting, without keeping L), TH / G points at a time; lane t builds
//     its columns k = c*G + t of M' straight from the table.
// Every record of the triple table is read by all threads at once
// (broadcast), and the rates need no lane-to-lane exchange.  Rate table: per
// ground state k, R[k][e] for e < NEMAX and F_k, each a row of TH doubles (a
// thread's point in column p); rows of consecutive k sit 8 doubles apart
// modulo 16, so the lanes of a group reading consecutive k of the same
// point, 32 / G groups at once, take the minimum two wavefronts.
// G = 2 (kPlainG): 6 columns per lane for SrOH.  Against 4 lanes per point
// it halves the work every lane repeats for its group (multipliers, pivot
// tests, shuffles); on 1024 SrOH sets x 256 x 256 it took 38.8 ms against
// 54.8 ms at G = 4 and 75.7 ms for the former one-pass kernel (4 lanes per
// point computing rates and elimination together).
template <int NGMAX, int NEMAX, bool EXACT, int PAD, int TH, int G>
__global__ void __launch_bounds__(TH, (TH <= 64 ? 4 : 2))
force_plain_kernel(ForceParams P)
{
    using GS = GroupShape<NGMAX, NEMAX, G>;
    constexpr int CPL = GS::CPL;
    constexpr int RBS = (NEMAX + 1) * TH + 8;
    static_assert(((NEMAX + 1) * TH) % 16 == 0, "rate-table rows 8 doubles off a 16-double multiple");
    extern __shared__ __align__(16) unsigned char sm[];
    RedLayout<NGMAX, NEMAX> Ly;
    Ly.build(P.n_b);
    double *fds = (double *)(sm + Ly.total);   // [n_b][TH]: Doppler-shifted beam frequencies
    double *rtab = fds + (size_t)P.n_b * TH;   // [NGMAX][RBS]
    const int tid = threadIdx.x, lane = tid & 31, t = lane % G, gbase = lane - t, group = tid / G;
    const int n_g = EXACT ? NGMAX : P.n_g;
    const int n_e = EXACT ? NEMAX : P.n_e;
    const double gh2 = (P.Gamma / 2.0) * (P.Gamma / 2.0);
    const long long pts_per_set = (P.layout == MM_LAYOUT_GRID) ? P.nv * P.nz : P.pps;
    for (int set = blockIdx.y; set < P.n_sets; set += gridDim.y) {
        const long long set_first = (long long)set * pts_per_set;
        long long set_count = pts_per_set;
        if (set_first + set_count > P.n_points) set_count = P.n_points - set_first;
        if (set_count <= 0) continue;  // uniform over the CTA
        RedView S;
        __syncthreads();
        build_reduced_tables<NGMAX, NEMAX, PAD, true>(P, set, sm, Ly, S);
        const double Bg = P.bgrad[set];
        const long long chunk = (set_count + gridDim.x - 1) / gridDim.x;
        const long long start = (long long)blockIdx.x * chunk;
        const long long end = min(start + chunk, set_count);
        for (long long base = start; base < end; base += TH) {
            // ---- phase 1: rates of point base + tid ----
            if (base + tid < end) {
                const long long ip = base + tid;
                double v, z;
                if (P.layout == MM_LAYOUT_GRID) {
                    v = P.v[ip / P.nz];
                    z = P.z[ip % P.nz];
                } else {
                    v = P.v[set_first + ip];
                    z = P.z[set_first + ip];
                }
                RateCtx<NEMAX> C;
                C.B = __dmul_rn(__dmul_rn(Bg, z), 1e4);
                C.vf = 0.0f;
                C.Bf = 0.0f;
                C.fd = fds + tid;
                C.stride = TH;
                for (int b = 0; b < P.n_b; b++)
                    fds[b * TH + tid] = __dadd_rn(S.freq[b], __ddiv_rn(__dmul_rn(S.ck[b], v), MM_TWO_PI));
#pragma unroll
                for (int e = 0; e < NEMAX; e++)
                    C.Ese[e] = (e < n_e) ? __dadd_rn(S.E[n_g + e],
                                                     __ddiv_rn(__dmul_rn(__dmul_rn(C.B, S.zde[e]), P.Gamma), MM_TWO_PI))
                                         : 0.0;
                for (int g = 0; g < n_g; g++) {
                    double Re[NEMAX], f, s;
                    reduced_rates<NEMAX, PAD, true>(S, g, C, gh2, Re, f, s);
                    // saturation correction 1/(1 + s_total[g]) (rate_equations_jit.py:85-90)
                    const double sat = mm_rcp(1.0 + s);
                    double *row = rtab + (size_t)g * RBS + tid;
#pragma unroll
                    for (int e = 0; e < NEMAX; e++) row[e * TH] = Re[e] * sat;
                    row[NEMAX * TH] = f * sat;
                }
            }
            __syncthreads();
            // ---- phase 2: population systems, TH / G points per pass ----
#pragma unroll 1
            for (int q = 0; q < G; q++) {
                const int p = q * (TH / G) + group;
                const long long ip = base + p;
                // warps whose points all lie beyond the chunk skip the pass (lanes of
                // a partly filled warp solve whatever the table holds, unused)
                if (!__any_sync(0xffffffffu, ip < end)) continue;
                // columns of M' straight from the rate table (one column's rates live at a time)
                double A[CPL][NGMAX], invU[CPL], xs[CPL];
#pragma unroll
                for (int c = 0; c < CPL; c++) {
                    const int k = c * G + t;
                    const bool own = EXACT ? (k < NGMAX) : (k < n_g);
                    const double *row = rtab + (size_t)(own ? k : 0) * RBS + p;
                    double Rc[NEMAX], rs = 0.0;
#pragma unroll
                    for (int e = 0; e < NEMAX; e++) {
                        Rc[e] = own ? row[e * TH] : 0.0;
                        rs += Rc[e];
                    }
#pragma unroll
                    for (int r = 0; r < NGMAX; r++) {
                        double br[NEMAX];
#pragma unroll
                        for (int e = 0; e < NEMAX; e++) br[e] = (r < n_g && e < n_e) ? S.brt[r * NEMAX + e] : 0.0;
                        A[c][r] = mprime_entry<NGMAX, NEMAX, G, EXACT>(n_g, r, k, Rc, rs, br);
                    }
                }
                int prows[NGMAX];
                bool swapped;
                int stat = 0;
                group_factor<NGMAX, NEMAX, G, EXACT, false>(P, t, gbase, A, invU, prows, swapped, xs, stat);
                double Rk[CPL], Fk[CPL];
#pragma unroll
                for (int c = 0; c < CPL; c++) {
                    const int k = c * G + t;
                    const bool own = EXACT ? (k < NGMAX) : (k < n_g);
                    const double *row = rtab + (size_t)(own ? k : 0) * RBS + p;
                    double rs = 0.0;
#pragma unroll
                    for (int e = 0; e < NEMAX; e++) rs += own ? row[e * TH] : 0.0;
                    Rk[c] = rs;
                    Fk[c] = own ? row[NEMAX * TH] : 0.0;
                }
                PointOut o = group_finish<NGMAX, NEMAX, G, EXACT>(P, t, xs, Fk, Rk, stat);
                if (!isfinite(o.F)) stat |= MM_ST_NONFINITE;
                o.status = mm_group_or(stat, G);
                if (ip < end) {
                    const long long gi = set_first + ip;
                    if (t == 0) {
                        P.F[gi] = o.F;
                        if (P.R) P.R[gi] = o.R;
                        if (P.status) P.status[gi] = o.status;
                    }
                    if (P.pop) {
#pragma unroll
                        for (int c = 0; c < CPL; c++) {
                            const int k = c * G + t;
                            if (k < P.n_g) P.pop[gi * P.n_g + k] = xs[c];
                        }
                    }
                }
            }
            __syncthreads();  // the next round rewrites the rate table
        }
    }
}

// The plain form's force and its gradient (implicit differentiation through
// the steady state) in three phases per round of
// TH points:
//  1. one thread per point: saturated rates into the rate table, as
//     force_plain_kernel, plus each ground state's saturation factor;
//  2. groups of G lanes: the elimination keeping L (group_factor), the
//     populations and force (group_finish), and the multipliers lambda and nu
//     of the transposed solve (group_lambda); also, per ground state,
//     T_g = sum over its triples of (p_g hk_b - mu[g,e]) rate_bge, which
//     equals p_g F_g - sum_e mu[g,e] R[g,e] from the table's own sums.  p_g,
//     lambda_g and T_g replace rate rows 0, 1 and the force row of the
//     point's column, nu goes to its own table;
//  3. one thread per point: one pass over each ground state's triples
//     (dF/dtheta = sum (p_g hk_b - mu[g,e]) d rate_bge / dtheta, with
//     mu[g,e] = p_g (nu_e - lambda_g [g < n_g - 1]); the saturation term
//     through T_g) into the thread's own accumulators (no atomics; a fixed
//     summation order).
// grad row layout per point: [dF/dfreq_0 .. dF/dfreq_{nb-1}, dF/ds0_0 ..
// dF/ds0_{nb-1}, dF/dB'].
template <int NGMAX, int NEMAX, bool EXACT, int PAD, int TH, int G>
__global__ void __launch_bounds__(TH, (TH <= 64 ? 3 : 2))
force_plain_adjoint_kernel(ForceParams P, double *grad)
{
    using GS = GroupShape<NGMAX, NEMAX, G>;
    constexpr int CPL = GS::CPL;
    constexpr int RBS = (NEMAX + 2) * TH + 8;  // rows: R[k][e] sat, F_k sat, sat_k
    static_assert(((NEMAX + 2) * TH) % 16 == 0, "rate-table rows 8 doubles off a 16-double multiple");
    extern __shared__ __align__(16) unsigned char sm[];
    RedLayout<NGMAX, NEMAX> Ly;
    Ly.build(P.n_b, true);
    const int nb = P.n_b, gw = 2 * nb + 1;
    double *fds = (double *)(sm + Ly.total);      // [n_b][TH]
    double *gas = fds + (size_t)nb * TH;          // [2 n_b][TH]: dF/dfreq_b, dF/ds0_b
    double *nut = gas + (size_t)2 * nb * TH;      // [NEMAX][TH]
    double *rtab = nut + (size_t)NEMAX * TH;      // [NGMAX][RBS]
    const int tid = threadIdx.x, lane = tid & 31, t = lane % G, gbase = lane - t, group = tid / G;
    const int n_g = EXACT ? NGMAX : P.n_g;
    const int n_e = EXACT ? NEMAX : P.n_e;
    const double gh = P.Gamma / 2.0, gh2 = gh * gh, geff = P.geff;
    const long long pts_per_set = (P.layout == MM_LAYOUT_GRID) ? P.nv * P.nz : P.pps;
    for (int set = blockIdx.y; set < P.n_sets; set += gridDim.y) {
        const long long set_first = (long long)set * pts_per_set;
        long long set_count = pts_per_set;
        if (set_first + set_count > P.n_points) set_count = P.n_points - set_first;
        if (set_count <= 0) continue;  // uniform over the CTA
        RedView S;
        __syncthreads();
        build_reduced_tables<NGMAX, NEMAX, PAD, true>(P, set, sm, Ly, S);
        const double Bg = P.bgrad[set];
        const long long chunk = (set_count + gridDim.x - 1) / gridDim.x;
        const long long start = (long long)blockIdx.x * chunk;
        const long long end = min(start + chunk, set_count);
        for (long long base = start; base < end; base += TH) {
            const bool mine = base + tid < end;
            double v = 0.0, z = 0.0;
            RateCtx<NEMAX> C;
            if (mine) {
                const long long ip = base + tid;
                if (P.layout == MM_LAYOUT_GRID) {
                    v = P.v[ip / P.nz];
                    z = P.z[ip % P.nz];
                } else {
                    v = P.v[set_first + ip];
                    z = P.z[set_first + ip];
                }
            }
            C.B = __dmul_rn(__dmul_rn(Bg, z), 1e4);
            C.vf = 0.0f;
            C.Bf = 0.0f;
            C.fd = fds + tid;
            C.stride = TH;
#pragma unroll
            for (int e = 0; e < NEMAX; e++)
                C.Ese[e] = (e < n_e) ? __dadd_rn(S.E[n_g + e],
                                                 __ddiv_rn(__dmul_rn(__dmul_rn(C.B, S.zde[e]), P.Gamma), MM_TWO_PI))
                                     : 0.0;
            // ---- phase 1: rates ----
            if (mine) {
                for (int b = 0; b < nb; b++)
                    fds[b * TH + tid] = __dadd_rn(S.freq[b], __ddiv_rn(__dmul_rn(S.ck[b], v), MM_TWO_PI));
                for (int g = 0; g < n_g; g++) {
                    double Re[NEMAX], f, s;
                    reduced_rates<NEMAX, PAD, true>(S, g, C, gh2, Re, f, s);
                    const double sat = mm_rcp(1.0 + s);  // rate_equations_jit.py:85-90
                    double *row = rtab + (size_t)g * RBS + tid;
#pragma unroll
                    for (int e = 0; e < NEMAX; e++) row[e * TH] = Re[e] * sat;
                    row[NEMAX * TH] = f * sat;
                    row[(NEMAX + 1) * TH] = sat;
                }
            }
            __syncthreads();
            // ---- phase 2: elimination, populations, multipliers ----
#pragma unroll 1
            for (int q = 0; q < G; q++) {
                const int p = q * (TH / G) + group;
                const long long ip = base + p;
                if (!__any_sync(0xffffffffu, ip < end)) continue;
                double A[CPL][NGMAX], invU[CPL], xs[CPL], Rk[CPL], Fk[CPL];
#pragma unroll
                for (int c = 0; c < CPL; c++) {
                    const int k = c * G + t;
                    const bool own = EXACT ? (k < NGMAX) : (k < n_g);
                    const double *row = rtab + (size_t)(own ? k : 0) * RBS + p;
                    double Rc[NEMAX], rs = 0.0;
#pragma unroll
                    for (int e = 0; e < NEMAX; e++) {
                        Rc[e] = own ? row[e * TH] : 0.0;
                        rs += Rc[e];
                    }
                    Rk[c] = rs;
                    Fk[c] = own ? row[NEMAX * TH] : 0.0;
#pragma unroll
                    for (int r = 0; r < NGMAX; r++) {
                        double br[NEMAX];
#pragma unroll
                        for (int e = 0; e < NEMAX; e++) br[e] = (r < n_g && e < n_e) ? S.brt[r * NEMAX + e] : 0.0;
                        A[c][r] = mprime_entry<NGMAX, NEMAX, G, EXACT>(n_g, r, k, Rc, rs, br);
                    }
                }
                int prows[NGMAX];
                bool swapped;
                int stat = 0;
                group_factor<NGMAX, NEMAX, G, EXACT, true>(P, t, gbase, A, invU, prows, swapped, xs, stat);
                PointOut o = group_finish<NGMAX, NEMAX, G, EXACT>(P, t, xs, Fk, Rk, stat);
                double wv[NGMAX], nu[NEMAX];
                group_lambda<NGMAX, NEMAX, G, EXACT>(P, S.brt, 1, NEMAX, t, gbase, A, invU, prows, swapped, Fk,
                                                     wv, nu);
                if (!isfinite(o.F)) stat |= MM_ST_NONFINITE;
                o.status = mm_group_or(stat, G);
                // T_k = sum over k's triples of (p_k hk_b - mu[k,e]) rate_bke
                //     = p_k F_k - sum_e mu[k,e] R[k,e]   (F_k, R[k,e] saturated)
                double Tk[CPL], lk[CPL];
#pragma unroll
                for (int c = 0; c < CPL; c++) {
                    const int k = c * G + t;
                    const bool own = EXACT ? (k < NGMAX) : (k < n_g);
                    const double *row = rtab + (size_t)(own ? k : 0) * RBS + p;
                    double lam = 0.0;
#pragma unroll
                    for (int g = 0; g < NGMAX; g++)
                        if (g == k) lam = wv[g];
                    lk[c] = lam;
                    double T = xs[c] * Fk[c];
#pragma unroll
                    for (int e = 0; e < NEMAX; e++) {
                        const double mue = xs[c] * (nu[e] - ((k < n_g - 1) ? lam : 0.0));
                        T = fma(-mue, own ? row[e * TH] : 0.0, T);
                    }
                    Tk[c] = T;
                }
                __syncwarp();
                // p_k, lambda_k and T_k over rows 0, 1 and NEMAX (F) of the point's column
#pragma unroll
                for (int c = 0; c < CPL; c++) {
                    const int k = c * G + t;
                    if (EXACT ? (k < NGMAX) : (k < n_g)) {
                        double *row = rtab + (size_t)k * RBS + p;
                        row[0] = xs[c];
                        row[TH] = lk[c];
                        row[NEMAX * TH] = Tk[c];
                    }
                }
                if (t == 0) {
#pragma unroll
                    for (int e = 0; e < NEMAX; e++) nut[e * TH + p] = nu[e];
                    if (ip < end) {
                        const long long gi = set_first + ip;
                        P.F[gi] = o.F;
                        if (P.R) P.R[gi] = o.R;
                        if (P.status) P.status[gi] = o.status;
                    }
                }
            }
            __syncthreads();
            // ---- phase 3: gradient passes over the triples ----
            if (mine) {
                const long long gi = set_first + base + tid;
                for (int i = 0; i < 2 * nb; i++) gas[i * TH + tid] = 0.0;
                double nue[NEMAX];
#pragma unroll
                for (int e = 0; e < NEMAX; e++) nue[e] = nut[e * TH + tid];
                double gB = 0.0;
                const double igh2 = 1.0 / gh2;
                for (int g = 0; g < n_g; g++) {
                    const double *row = rtab + (size_t)g * RBS + tid;
                    const double pk = row[0], lamk = row[TH], sat = row[(NEMAX + 1) * TH];
                    const double Cs = row[NEMAX * TH] * sat;  // T_g sat (saturation term)
                    const double Esg = fma(C.B, S.czd[g], S.E[g]);
#pragma unroll
                    for (int e = 0; e < NEMAX; e++) {
                        const double mue = pk * (nue[e] - ((g < n_g - 1) ? lamk : 0.0));
                        const double ddB = (e < n_e) ? -z * 1e4 * (P.zd[n_g + e] - P.zd[g]) * P.Gamma : 0.0;
                        const int i1 = S.offs[g * NEMAX + e + 1];
                        for (int i = S.offs[g * NEMAX + e]; i < i1; i++) {
                            const TripD tr = ((const TripD *)S.trip)[i];
                            const double om = __dsub_rn(C.Ese[e], Esg);
                            const double de = __dmul_rn(__dsub_rn(fds[tr.b * TH + tid], om), MM_TWO_PI);
                            const double L = gh2 * mm_rcp1(fma(de, de, gh2));  // feeds the gradient only
                            const double rate = tr.c1 * L * sat;
                            const double w = pk * tr.hk - mue;
                            const double Q = w * rate - Cs * tr.c2 * L;
                            const double dLL = -2.0 * de * L * igh2;  // (dL/d delta) / L
                            gas[tr.b * TH + tid] += Q * dLL * MM_TWO_PI;
                            gas[(nb + tr.b) * TH + tid] += S.d2t[i] * L * (w * gh * geff * sat - Cs);
                            gB = fma(Q * dLL, ddB, gB);
                        }
                    }
                }
                for (int i = 0; i < 2 * nb; i++) grad[gi * gw + i] = gas[i * TH + tid];
                grad[gi * gw + 2 * nb] = gB;
            }
            __syncthreads();  // the next round rewrites the tables
        }
    }
}


// FP32-bulk form: one point per thread, populations from the reduced
// (excited-manifold) solve of reduced.cuh.  One CTA per parameter set at a
// time; its prologue builds the set's triple tables in shared memory, then the
// threads stream over the set's points.
#ifndef MM_RED_THREADS
#define MM_RED_THREADS 128
#endif
#ifndef MM_RED_MINB
#define MM_RED_MINB 4
#endif

constexpr int kRedThreads = MM_RED_THREADS;
// The FP32 form's two-point path needs ~166 registers: 3 CTAs per SM
// (24.0 ms per 2.68e8 points, against 27.3 ms for one point per thread at 4).
constexpr int kRedMinBlocks32 = 3;

template <int NGMAX, int NEMAX, bool EXACT, int PAD, bool F64>
__global__ void __launch_bounds__(kRedThreads, F64 ? MM_RED_MINB : kRedMinBlocks32)
force_reduced_kernel(ForceParams P)
{
    extern __shared__ __align__(16) unsigned char sm[];
    RedLayout<NGMAX, NEMAX> Ly;
    Ly.build(P.n_b);
    const long long pts_per_set = (P.layout == MM_LAYOUT_GRID) ? P.nv * P.nz : P.pps;
    for (int set = blockIdx.y; set < P.n_sets; set += gridDim.y) {
        const long long set_first = (long long)set * pts_per_set;
        long long set_count = pts_per_set;
        if (set_first + set_count > P.n_points) set_count = P.n_points - set_first;
        if (set_count <= 0) continue;  // uniform over the CTA
        RedView S;
        __syncthreads();
        build_reduced_tables<NGMAX, NEMAX, PAD, F64>(P, set, sm, Ly, S);
        const double Bg = P.bgrad[set];
        double *fd = (double *)(sm + Ly.total) + threadIdx.x;  // FP64 form: n_b slots, stride blockDim.x
        const long long chunk = (set_count + gridDim.x - 1) / gridDim.x;
        const long long start = (long long)blockIdx.x * chunk;
        const long long end = min(start + chunk, set_count);
        const bool idx32 = P.layout == MM_LAYOUT_GRID && end <= 0x7fffffffll;
        if constexpr (!F64) {
            // FP32 form without populations: two points per thread (ip, ip + blockDim.x)
            if (!P.pop && S.valid) {
                auto load = [&](long long ip, double &v, double &z) {
                    if (idx32) {  // 32-bit division for grids below 2^31 points per set
                        const unsigned iu = (unsigned)ip, nz = (unsigned)P.nz;
                        const unsigned iv = iu / nz;
                        v = P.v[iv];
                        z = P.z[iu - iv * nz];
                    } else if (P.layout == MM_LAYOUT_GRID) {
                        v = P.v[ip / P.nz];
                        z = P.z[ip % P.nz];
                    } else {
                        v = P.v[set_first + ip];
                        z = P.z[set_first + ip];
                    }
                };
                for (long long ip0 = start + threadIdx.x; ip0 < end; ip0 += 2 * blockDim.x) {
                    const long long ip1 = ip0 + blockDim.x;
                    double v[2], z[2];
                    load(ip0, v[0], z[0]);
                    const bool two = ip1 < end;
                    if (two) load(ip1, v[1], z[1]);
                    if (two && isfinite(v[0]) && isfinite(z[0]) && isfinite(v[1]) && isfinite(z[1])) {
                        RedOut o[2];
                        reduced_point2<NGMAX, NEMAX, EXACT, PAD>(P, S, v, z, Bg, o);
                        P.F[set_first + ip0] = o[0].F;
                        P.F[set_first + ip1] = o[1].F;
                        if (P.R) { P.R[set_first + ip0] = o[0].R; P.R[set_first + ip1] = o[1].R; }
                        if (P.status) { P.status[set_first + ip0] = o[0].status; P.status[set_first + ip1] = o[1].status; }
                    } else {
                        for (int h = 0; h < (two ? 2 : 1); h++) {
                            const long long gi = set_first + (h ? ip1 : ip0);
                            const RedOut o = reduced_point<NGMAX, NEMAX, EXACT, PAD, F64>(P, S, v[h], z[h], Bg,
                                                                                           nullptr, fd, blockDim.x);
                            P.F[gi] = o.F;
                            if (P.R) P.R[gi] = o.R;
                            if (P.status) P.status[gi] = o.status;
                        }
                    }
                }
                continue;
            }
        }
        for (long long ip = start + threadIdx.x; ip < end; ip += blockDim.x) {
            double v, z;
            if (idx32) {  // 32-bit division for grids below 2^31 points per set
                const unsigned iu = (unsigned)ip, nz = (unsigned)P.nz;
                const unsigned iv = iu / nz;
                v = P.v[iv];
                z = P.z[iu - iv * nz];
            } else if (P.layout == MM_LAYOUT_GRID) {
                v = P.v[ip / P.nz];
                z = P.z[ip % P.nz];
            } else {
                v = P.v[set_first + ip];
                z = P.z[set_first + ip];
            }
            const long long gi = set_first + ip;
            double *pop = P.pop ? P.pop + gi * P.n_g : nullptr;
            const RedOut o = reduced_point<NGMAX, NEMAX, EXACT, PAD, F64>(P, S, v, z, Bg, pop, fd, blockDim.x);
            P.F[gi] = o.F;
            if (P.R) P.R[gi] = o.R;
            if (P.status) P.status[gi] = o.status;
        }
    }
}

// FP64-reduced adjoint: the FP64-reduced force and its gradient (same row
// layout as force_plain_adjoint_kernel), one point per thread.  The host launches it
// only when every set passes the reduced form's structural checks.  Shared
// scratch per thread: Doppler-shifted frequencies, dF/dfreq_b and dF/ds0_b
// (3 n_b doubles, stride blockDim.x).
template <int NGMAX, int NEMAX, bool EXACT, int PAD>
__global__ void __launch_bounds__(kRedThreads, 2)
force_reduced_adjoint_kernel(ForceParams P, double *grad)
{
    extern __shared__ __align__(16) unsigned char sm[];
    RedLayout<NGMAX, NEMAX> Ly;
    Ly.build(P.n_b, true);
    const long long pts_per_set = (P.layout == MM_LAYOUT_GRID) ? P.nv * P.nz : P.pps;
    const int nb = P.n_b, gw = 2 * nb + 1, st = blockDim.x;
    double *fd = (double *)(sm + Ly.total) + threadIdx.x;
    double *gf = fd + (size_t)nb * st, *gs = gf + (size_t)nb * st;
    for (int set = blockIdx.y; set < P.n_sets; set += gridDim.y) {
        const long long set_first = (long long)set * pts_per_set;
        long long set_count = pts_per_set;
        if (set_first + set_count > P.n_points) set_count = P.n_points - set_first;
        if (set_count <= 0) continue;
        RedView S;
        __syncthreads();
        build_reduced_tables<NGMAX, NEMAX, PAD, true>(P, set, sm, Ly, S);
        const double Bg = P.bgrad[set];
        const int32_t *pol = P.pol + (size_t)set * nb;
        const long long chunk = (set_count + gridDim.x - 1) / gridDim.x;
        const long long start = (long long)blockIdx.x * chunk;
        const long long end = min(start + chunk, set_count);
        for (long long ip = start + threadIdx.x; ip < end; ip += st) {
            double v, z;
            if (P.layout == MM_LAYOUT_GRID) {
                v = P.v[ip / P.nz];
                z = P.z[ip % P.nz];
            } else {
                v = P.v[set_first + ip];
                z = P.z[set_first + ip];
            }
            const long long gi = set_first + ip;
            double *row = grad + gi * gw;
            if (!(isfinite(v) && isfinite(z))) {
                const double nan = __longlong_as_double(0x7ff8000000000000ll);
                P.F[gi] = nan;
                if (P.status) P.status[gi] = MM_ST_NONFINITE;
                for (int i = 0; i < gw; i++) row[i] = nan;
                continue;
            }
            for (int b = 0; b < nb; b++) {
                gf[b * st] = 0.0;
                gs[b * st] = 0.0;
            }
            double gBG;
            const RedOut o = reduced_adjoint_point<NGMAX, NEMAX, EXACT, PAD>(P, S, pol, v, z, Bg, fd, st,
                                                                             gf, gs, gBG);
            P.F[gi] = o.F;
            if (P.status) P.status[gi] = o.status;
            for (int b = 0; b < nb; b++) {
                row[b] = gf[b * st];
                row[nb + b] = gs[b * st];
            }
            row[2 * nb] = gBG * (z * 1e4);  // dB/dB' = z 1e4
        }
    }
}


// Fused trajectories, one particle per group, all steps in one launch.
//  ndim = 1: symplectic Euler along z (molmot/propagation/trajectories_jit.py:18-58,
//            molmot_cuda/trajectories_cuda.py:44-280):
//            v_j = v_{j-1} + F(v_{j-1}, z_{j-1})/m dt; z_j = z_{j-1} + v_j dt;
//            stop when |z| > z_escape (n_actual = j, the rest of the row repeats).
//  ndim = 3: the per-axis model of molmot/propagation/trajectories.py:78-156:
//            F_z = F(v_z, z), F_x = F(v_x, -x/2), F_y = F(v_y, -y/2), the same Euler
//            update per axis, stop when |r| > z_escape.  F(v, -x/2) is computed as
//            F at coordinate x with gradient -B'/2 (bit-identical product).
//  n_avg = 2: force = 0.5 (F_set0 + F_set1), the RF MOT time average
//            (molmot/mot/simulator.py:49-90; the sets carry +B' and -B').
//  vsq_sum / n_samp: sums of v^2 over steps j >= i_eq that did not escape
//            (molmot/propagation/trajectories.py:159-229, monte_carlo_temperature).
// The integrator uses explicit round-to-nearest operations so it matches the
// reference's uncontracted arithmetic.
template <int NGMAX, int NEMAX, int G, bool EXACT>
__global__ void __launch_bounds__(kThreads, 3)
traj1d_kernel(ForceParams P, TrajParams T)
{
    using GS = GroupShape<NGMAX, NEMAX, G>;
    extern __shared__ __align__(16) unsigned char sm[];
    SmemLayout Ly;
    const int ngroups = kThreads / G;
    Ly.build(P.n_g, P.n_e, P.n_b, GS::CPL, ngroups);
    const int lane = threadIdx.x & 31, t = lane % G, gbase = lane - t;
    const int group = threadIdx.x / G;
    double *scr = (double *)(sm + Ly.scratch) + (size_t)group * Ly.scratch_per_group;
    double *fd = scr, *Ese = scr + P.n_b;
    SetView S[2];
    double Bg[2];
    for (int a = 0; a < T.n_avg; a++) {
        build_set_tables<G, GS::CPL>(P, a, sm + a * Ly.total, Ly, S[a]);
        Bg[a] = P.bgrad[a];
    }
    const int nd = T.ndim;
    const long long ip = (long long)blockIdx.x * ngroups + group;
    const bool valid = ip < T.n_particles;
    double x[3] = {0.0, 0.0, 0.0}, u[3] = {0.0, 0.0, 0.0};
    for (int d = 0; d < nd; d++) {
        x[d] = valid ? T.z0[ip * nd + d] : 0.0;
        u[d] = valid ? T.v0[ip * nd + d] : 0.0;
    }
    long long na = T.n_steps;
    bool done = !valid;
    double vsq = 0.0, nsamp = 0.0;
    const long long row = ip * T.n_steps * nd;
    if (valid && T.z_traj && t == 0)
        for (int d = 0; d < nd; d++) { T.z_traj[row + d] = x[d]; T.v_traj[row + d] = u[d]; }
    for (long long j = 1; j < T.n_steps; j++) {
        if (__all_sync(0xffffffffu, done)) break;
        double acc[3];
        for (int d = 0; d < nd; d++) {
            // axis multipliers of B' in the per-axis model: x, y see -B'/2, z sees B'
            const double mult = (nd == 3 && d < 2) ? -0.5 : 1.0;
            double F = 0.0;
            for (int a = 0; a < T.n_avg; a++) {
                double xs[GS::CPL];
                const PointOut o = solve_point<NGMAX, NEMAX, G, EXACT>(
                    P, S[a], fd, Ese, t, gbase, u[d], x[d], Bg[a] * mult, xs);
                F = (a == 0) ? o.F : __dadd_rn(F, o.F);
            }
            if (T.n_avg == 2) F = 0.5 * F;
            acc[d] = __ddiv_rn(F, T.mass);
        }
        if (!done) {
            double r2 = 0.0;
            for (int d = 0; d < nd; d++) {
                u[d] = __dadd_rn(u[d], __dmul_rn(acc[d], T.dt));
                x[d] = __dadd_rn(x[d], __dmul_rn(u[d], T.dt));
                r2 = fma(x[d], x[d], r2);
            }
            if (T.z_traj && t == 0)
                for (int d = 0; d < nd; d++) {
                    T.z_traj[row + j * nd + d] = x[d];
                    T.v_traj[row + j * nd + d] = u[d];
                }
            const bool esc = (nd == 1) ? (fabs(x[0]) > T.z_escape) : (sqrt(r2) > T.z_escape);
            if (esc) {
                na = j;
                done = true;
                if (T.z_traj && t == 0)
                    for (long long s = j + 1; s < T.n_steps; s++)
                        for (int d = 0; d < nd; d++) {
                            T.z_traj[row + s * nd + d] = x[d];
                            T.v_traj[row + s * nd + d] = u[d];
                        }
            } else if (T.i_eq >= 0 && j >= T.i_eq) {
                for (int d = 0; d < nd; d++) vsq = __dadd_rn(vsq, __dmul_rn(u[d], u[d]));
                nsamp += 1.0;
            }
        }
    }
    if (valid && t == 0) {
        for (int d = 0; d < nd; d++) { T.z_final[ip * nd + d] = x[d]; T.v_final[ip * nd + d] = u[d]; }
        T.n_actual[ip] = (int32_t)na;
        if (T.vsq_sum) { T.vsq_sum[ip] = vsq; T.n_samp[ip] = nsamp; }
    }
}

// FP32-bulk trajectories: one particle per thread, the force of every step
// from reduced_point (reduced.cuh); the same integrator, escape rule, RF
// averaging, per-axis model and v^2 sums as traj1d_kernel.
template <int NGMAX, int NEMAX, bool EXACT, int PAD>
__global__ void __launch_bounds__(kRedThreads, MM_RED_MINB)
traj1d_reduced_kernel(ForceParams P, TrajParams T)
{
    extern __shared__ __align__(16) unsigned char sm[];
    RedLayout<NGMAX, NEMAX> Ly;
    Ly.build(P.n_b);
    RedView S0, S1;
    build_reduced_tables<NGMAX, NEMAX, PAD, false>(P, 0, sm, Ly, S0);
    S1 = S0;
    if (T.n_avg == 2) build_reduced_tables<NGMAX, NEMAX, PAD, false>(P, 1, sm + Ly.total, Ly, S1);
    const double Bg0 = P.bgrad[0], Bg1 = (T.n_avg == 2) ? P.bgrad[1] : 0.0;
    const int nd = T.ndim;
    const long long ip = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = ip < T.n_particles;
    double x[3] = {0.0, 0.0, 0.0}, u[3] = {0.0, 0.0, 0.0};
    for (int d = 0; d < nd; d++) {
        x[d] = valid ? T.z0[ip * nd + d] : 0.0;
        u[d] = valid ? T.v0[ip * nd + d] : 0.0;
    }
    long long na = T.n_steps;
    bool done = !valid;
    double vsq = 0.0, nsamp = 0.0;
    const long long row = ip * T.n_steps * nd;
    if (valid && T.z_traj)
        for (int d = 0; d < nd; d++) { T.z_traj[row + d] = x[d]; T.v_traj[row + d] = u[d]; }
    for (long long j = 1; j < T.n_steps; j++) {
        if (__all_sync(0xffffffffu, done)) break;
        if (done) continue;
        double acc[3];
        for (int d = 0; d < nd; d++) {
            // axis multipliers of B' in the per-axis model: x, y see -B'/2, z sees B'
            const double mult = (nd == 3 && d < 2) ? -0.5 : 1.0;
            double F = reduced_point<NGMAX, NEMAX, EXACT, PAD>(P, S0, u[d], x[d], Bg0 * mult, nullptr).F;
            if (T.n_avg == 2)
                F = 0.5 * __dadd_rn(F, reduced_point<NGMAX, NEMAX, EXACT, PAD>(P, S1, u[d], x[d], Bg1 * mult,
                                                                                nullptr).F);
            acc[d] = __ddiv_rn(F, T.mass);
        }
        double r2 = 0.0;
        for (int d = 0; d < nd; d++) {
            u[d] = __dadd_rn(u[d], __dmul_rn(acc[d], T.dt));
            x[d] = __dadd_rn(x[d], __dmul_rn(u[d], T.dt));
            r2 = fma(x[d], x[d], r2);
        }
        if (T.z_traj)
            for (int d = 0; d < nd; d++) {
                T.z_traj[row + j * nd + d] = x[d];
                T.v_traj[row + j * nd + d] = u[d];
            }
        const bool esc = (nd == 1) ? (fabs(x[0]) > T.z_escape) : (sqrt(r2) > T.z_escape);
        if (esc) {
            na = j;
            done = true;
            if (T.z_traj)
                for (long long s2 = j + 1; s2 < T.n_steps; s2++)
                    for (int d = 0; d < nd; d++) {
                        T.z_traj[row + s2 * nd + d] = x[d];
                        T.v_traj[row + s2 * nd + d] = u[d];
                    }
        } else if (T.i_eq >= 0 && j >= T.i_eq) {
            for (int d = 0; d < nd; d++) vsq = __dadd_rn(vsq, __dmul_rn(u[d], u[d]));
            nsamp += 1.0;
        }
    }
    if (valid) {
        for (int d = 0; d < nd; d++) { T.z_final[ip * nd + d] = x[d]; T.v_final[ip * nd + d] = u[d]; }
        T.n_actual[ip] = (int32_t)na;
        if (T.vsq_sum) { T.vsq_sum[ip] = vsq; T.n_samp[ip] = nsamp; }
    }
}

// Trajectory tangents of the per-axis 3D model (molmot/propagation/
// trajectories.py:78-156: symplectic Euler per axis, F_x = F(v_x, x) at
// gradient -B'/2, F_y likewise, F_z = F(v_z, z) at B', escape at
// |r| > r_escape) with respect to parameters theta_k (beam frequency groups,
// s0 groups, B').  Forward mode; the force's gradient at each step comes from
// reduced_adjoint_point (FP64-reduced form):
//   dF_a/dtheta_k = sum_{b: freq_par[b] = k} dF/dfreq_b + sum_{b: s0_par[b] = k} dF/ds0_b
//                   + [k = B'] dF/dB mult_a x_a 1e4 + dF/dv Tv_ak + dF/dx Tx_ak,
//   dF/dv = sum_b dF/dfreq_b ck_b / 2pi (ck_b = -k kdir_b),  dF/dx = dF/dB B' mult_a 1e4,
//   Tv_ak += dt (dF_a/dtheta_k) / m,  Tx_ak += dt Tv_ak,
// mult_a = -1/2 for x and y, 1 for z.  Recoil kicks (kicks != 0): N ~
// Poisson((R_x + R_y + R_z) dt) events per step, 2N isotropic kicks of
// hbar k / m (kicks.cuh, counters (particle, absolute step)); under
// differentiation they are held fixed (the derivative at fixed noise: event
// counts and directions do not move with theta).  Per particle four axis
// slots (x, y, z and an idle one) of kTgSub lanes; with kTgSub > 1 the lanes
// of an axis split the ground states of each force-and-gradient solve and
// add their partial sums with shuffles (reduced_adjoint_point<..., NL>),
// then hold the axis' state alike.  One lane per axis was the fastest on
// 4096 SrOH particles x 1000 steps (33.5 ms; two lanes 38.2 ms, four 49.5 ms:
// the split adds shuffles and leaves fewer particles per warp).  The lanes of a particle share the kick's
// total rate and the escape radius through shuffles; every lane of the warp
// executes all of these unconditionally, including lanes without a particle,
// the idle slot and particles that stopped (they solve the point (0, 0)).
// State row per particle (width 6 + 6 n_par): r[3], v[3], Tr[3][n_par],
// Tv[3][n_par].
struct TgParams {
    double dt, r_escape, mass, v_rec;
    long long n_particles, n_steps, step0, ckpt_every;
    int n_par, kicks, bprime_par;
    unsigned long long seed;
    signed char freq_par[MM_MAX_BEAMS], s0_par[MM_MAX_BEAMS];
    double *state;      // [N][6 + 6 n_par], in/out
    int32_t *n_actual;  // [N], in/out: the absolute step a particle stopped at
    double *ckpt;       // [n_steps / ckpt_every][N][6 + 6 n_par] or null
};

constexpr int kTgMaxPar = MM_TGRAD_MAX_PAR;
constexpr int kTgThreads = 128;
constexpr int kTgSub = 1;             // lanes per axis (each takes every kTgSub-th ground state)
constexpr int kTgLanes = 4 * kTgSub;  // lanes per particle: x, y, z and an idle slot
constexpr int kTgBofs = (MM_MAX_BEAMS + 4) / 4 * 4;  // beam offsets (ints), a multiple of 4

template <int NGMAX, int NEMAX, bool EXACT, int PAD, bool KEEP>
__global__ void __launch_bounds__(kTgThreads, 2)
traj_grad_kernel(ForceParams P, TgParams T)
{
    extern __shared__ __align__(16) unsigned char sm[];
    RedLayout<NGMAX, NEMAX> Ly;
    Ly.build(P.n_b, true);
    RedView S;
    build_reduced_tables<NGMAX, NEMAX, PAD, true>(P, 0, sm, Ly, S);
    const int nb = P.n_b, st = blockDim.x, np = T.n_par, W = 6 + 6 * np;
    double *fd = (double *)(sm + Ly.total) + threadIdx.x;
    double *gf = fd + (size_t)nb * st, *gs = gf + (size_t)nb * st;
    double *keep = gs + (size_t)nb * st;  // KEEP: NGMAX kKeepSlots slots per thread
    // KEEP: the triples in beam-major order (reduced_adjoint_point's gradient pass)
    // (the same address on every thread: after the per-thread regions, which
    // are counted from the shared base, not from this thread's slot)
    int *bofs = (int *)((double *)(sm + Ly.total) + (size_t)(3 * nb + NGMAX * kKeepSlots<NEMAX>) * st);
    int *bidx = bofs + kTgBofs;
    if constexpr (KEEP) {
        if (threadIdx.x == 0) {
            const TripD *tr = (const TripD *)S.trip;
            int k = 0;
            for (int b = 0; b < nb; b++) {
                bofs[b] = k;
                for (int g = 0; g < P.n_g; g++)
                    for (int e = 0; e < P.n_e; e++)
                        for (int i = S.offs[g * NEMAX + e]; i < S.offs[g * NEMAX + e + 1]; i++)
                            if (!tr[i].pad && tr[i].b == b) bidx[k++] = i | (g << 16) | (e << 24);
            }
            bofs[nb] = k;
        }
        __syncthreads();
    }
    const int tl = threadIdx.x % kTgLanes;
    const int a = tl / kTgSub, jsub = tl % kTgSub;  // axis slot, sub-lane
    const bool axis = a < 3;
    const long long ip = ((long long)blockIdx.x * blockDim.x + threadIdx.x) / kTgLanes;
    const bool valid = ip < T.n_particles;
    const double mult = (a < 2) ? -0.5 : 1.0;
    const double Bg = P.bgrad[0] * mult;  // the per-axis model's product (mm_traj_run)
    // sum over the particle's axis slots (the same sub-lane of each slot)
    auto axis_sum = [](double v) {
        v += __shfl_xor_sync(0xffffffffu, v, kTgSub);
        return v + __shfl_xor_sync(0xffffffffu, v, 2 * kTgSub);
    };
    double x = 0.0, u = 0.0, Tx[kTgMaxPar], Tv[kTgMaxPar];
    double *row = T.state + (valid ? ip : 0) * W;
#pragma unroll
    for (int k = 0; k < kTgMaxPar; k++) {
        const bool on = valid && axis && k < np;
        Tx[k] = on ? row[6 + a * np + k] : 0.0;
        Tv[k] = on ? row[6 + 3 * np + a * np + k] : 0.0;
    }
    if (valid && axis) {
        x = row[a];
        u = row[3 + a];
    }
    auto write_row = [&](double *dst) {
        if (valid && axis && jsub == 0) {
            dst[a] = x;
            dst[3 + a] = u;
#pragma unroll
            for (int k = 0; k < kTgMaxPar; k++)  // compile-time indices keep Tx, Tv in registers
                if (k < np) {
                    dst[6 + a * np + k] = Tx[k];
                    dst[6 + 3 * np + a * np + k] = Tv[k];
                }
        }
    };
    // a particle already beyond r_escape stopped in an earlier call (the sum
    // runs on every lane: it is a warp collective)
    const double r2_0 = axis_sum(x * x);
    const bool stopped = !valid || sqrt(r2_0) > T.r_escape;
    bool done = stopped;
    long long na = -1;
    long long n_ck = 0;
    const long long jend = T.step0 + T.n_steps;
    long long j = T.step0 + 1;
    for (; j <= jend; j++) {
        if (__all_sync(0xffffffffu, done)) break;
        double F = 0.0, R = 0.0, dth[kTgMaxPar];
#pragma unroll
        for (int k = 0; k < kTgMaxPar; k++) dth[k] = 0.0;
        // the solve is shared by the axis' sub-lanes (warp collectives inside):
        // every lane takes part, stopped particles and the idle slot at (0, 0)
        const bool act = !done && axis;
        for (int b = 0; b < nb; b++) {
            gf[b * st] = 0.0;
            gs[b * st] = 0.0;
        }
        double gBG;
        const RedOut o = reduced_adjoint_point<NGMAX, NEMAX, EXACT, PAD, kTgSub, KEEP>(
            P, S, P.pol, act ? u : 0.0, act ? x : 0.0, Bg, fd, st, gf, gs, gBG, jsub, keep, bofs, bidx);
        if (act) {
            F = o.F;
            R = o.R;
            double dv = 0.0;
            for (int b = 0; b < nb; b++) dv = fma(gf[b * st], S.ck[b], dv);
            const double dFdv = dv / MM_TWO_PI, dFdx = gBG * (Bg * 1e4);
#pragma unroll
            for (int k = 0; k < kTgMaxPar; k++) dth[k] = fma(dFdv, Tv[k], dFdx * Tx[k]);
            for (int b = 0; b < nb; b++) {
                const int kf = T.freq_par[b], ks = T.s0_par[b];
#pragma unroll
                for (int k = 0; k < kTgMaxPar; k++) {
                    if (k == kf) dth[k] += gf[b * st];
                    if (k == ks) dth[k] += gs[b * st];
                }
            }
#pragma unroll
            for (int k = 0; k < kTgMaxPar; k++)
                if (k == T.bprime_par) dth[k] = fma(gBG, mult * x * 1e4, dth[k]);
        }
        // warp collectives below: every lane, every iteration
        double kick[3] = {0.0, 0.0, 0.0};
        if (T.kicks) {  // uniform over the grid
            const double Rt = axis_sum(act ? R : 0.0);
            if (!done) recoil_kick(T.seed, (unsigned)ip, (unsigned)j, Rt * T.dt, T.v_rec, kick);
        }
        if (act) {
            const double acc = __ddiv_rn(F, T.mass);
            u = __dadd_rn(u, __dmul_rn(acc, T.dt));
            if (T.kicks) u = __dadd_rn(u, (a == 0) ? kick[0] : (a == 1) ? kick[1] : kick[2]);  // no run-time index
            x = __dadd_rn(x, __dmul_rn(u, T.dt));
            const double im = T.dt / T.mass;
#pragma unroll
            for (int k = 0; k < kTgMaxPar; k++) {
                Tv[k] = fma(dth[k], im, Tv[k]);
                Tx[k] = fma(Tv[k], T.dt, Tx[k]);
            }
        }
        const double r2 = axis_sum(x * x);
        if (!done && sqrt(r2) > T.r_escape) {
            na = j;
            done = true;
        }
        if (T.ckpt && (j - T.step0) % T.ckpt_every == 0) {
            write_row(T.ckpt + ((size_t)n_ck * T.n_particles + (valid ? ip : 0)) * W);
            n_ck++;
        }
    }
    // checkpoints after the whole warp stopped: the frozen state
    if (T.ckpt)
        for (; j <= jend; j++)
            if ((j - T.step0) % T.ckpt_every == 0) {
                write_row(T.ckpt + ((size_t)n_ck * T.n_particles + (valid ? ip : 0)) * W);
                n_ck++;
            }
    write_row(row);
    if (valid && tl == 0) {
        if (na >= 0) T.n_actual[ip] = (int32_t)na;
        else if (!stopped) T.n_actual[ip] = (int32_t)jend;
    }
}

// Size classes: (NGMAX, NEMAX, G, EXACT).
template <int NGMAX, int NEMAX, int G, bool EXACT>
struct Class {
    static constexpr int ng = NGMAX, ne = NEMAX, g = G;
    static constexpr bool exact = EXACT;
};

template <class C>
size_t smem_bytes(const ForceParams &P)
{
    SmemLayout Ly;
    Ly.build(P.n_g, P.n_e, P.n_b, GroupShape<C::ng, C::ne, C::g>::CPL, kThreads / C::g);
    return Ly.total;
}

constexpr int kPlainThreads = 64;
constexpr int kPlainG = 2;  // lanes per point in the elimination

template <class C, int PAD>
int launch_plain(const ForceParams &P, long long pts_per_set, cudaStream_t st)
{
    constexpr int TH = kPlainThreads;
    auto kern = force_plain_kernel<C::ng, C::ne, C::exact, PAD, TH, kPlainG>;
    RedLayout<C::ng, C::ne> Ly;
    Ly.build(P.n_b);
    const size_t sb = Ly.total + sizeof(double) * ((size_t)P.n_b * TH + (size_t)C::ng * ((C::ne + 1) * TH + 8));
    if (sb > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sb);
        if (mm_cuda_check(e, "cudaFuncSetAttribute")) return -3;
    }
    int dev = 0, nsm = 148, per_sm = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, TH, sb);
    if (per_sm < 1) per_sm = 1;
    // enough CTAs to fill the GPU a few times over, at least 8 rounds of TH points each
    const long long want = (long long)nsm * per_sm * 4;
    long long gx = std::max<long long>(1, want / std::max(1, P.n_sets));
    gx = std::min(gx, std::max<long long>(1, (pts_per_set + TH * 8 - 1) / (TH * 8)));
    gx = std::min<long long>(gx, 1 << 20);
    dim3 grid((unsigned)gx, (unsigned)std::min(P.n_sets, 65535));
    kern<<<grid, TH, sb, st>>>(P);
    return mm_cuda_check(cudaGetLastError(), "force_plain_kernel launch") ? -3 : 0;
}

template <class C, int PAD, bool F64>
int launch_reduced(const ForceParams &P, long long pts_per_set, cudaStream_t st)
{
    auto kern = force_reduced_kernel<C::ng, C::ne, C::exact, PAD, F64>;
    RedLayout<C::ng, C::ne> Ly;
    Ly.build(P.n_b);
    const size_t sb = Ly.total + (F64 ? sizeof(double) * P.n_b * kRedThreads : 0);
    if (sb > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sb);
        if (mm_cuda_check(e, "cudaFuncSetAttribute")) return -3;
    }
    int dev = 0, nsm = 148, per_sm = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kRedThreads, sb);
    if (per_sm < 1) per_sm = 1;
    // enough CTAs to fill the GPU a few times over, at least 8 points per thread
    const long long want = (long long)nsm * per_sm * 4;
    long long gx = std::max<long long>(1, want / std::max(1, P.n_sets));
    gx = std::min(gx, std::max<long long>(1, (pts_per_set + kRedThreads * 8 - 1) / (kRedThreads * 8)));
    gx = std::min<long long>(gx, 1 << 20);
    dim3 grid((unsigned)gx, (unsigned)std::min(P.n_sets, 65535));
    kern<<<grid, kRedThreads, sb, st>>>(P);
    return mm_cuda_check(cudaGetLastError(), "force_reduced_kernel launch") ? -3 : 0;
}

template <class C, int PAD>
int launch_traj_reduced(const ForceParams &P, const TrajParams &T, cudaStream_t st)
{
    auto kern = traj1d_reduced_kernel<C::ng, C::ne, C::exact, PAD>;
    RedLayout<C::ng, C::ne> Ly;
    Ly.build(P.n_b);
    const size_t sb = Ly.total * T.n_avg;
    if (sb > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sb);
        if (mm_cuda_check(e, "cudaFuncSetAttribute")) return -3;
    }
    const long long gx = (T.n_particles + kRedThreads - 1) / kRedThreads;
    kern<<<(unsigned)gx, kRedThreads, sb, st>>>(P, T);
    return mm_cuda_check(cudaGetLastError(), "traj1d_reduced_kernel launch") ? -3 : 0;
}


// rounds of 96 points: 2 CTAs per SM (the tables take 93 KB for SrOH); on
// 1024 sets x 66 stencil points this took 0.257 ms against 0.287 ms with
// rounds of 64 (3 CTAs per SM, but a second round for 2 points of every
// set) and 0.432 ms with rounds of 128 (one CTA per SM)
constexpr int kPlainAdjThreads = 96;
constexpr int kPlainAdjG = 4;

template <class C, int PAD>
int launch_plain_adjoint(const ForceParams &P, double *grad, cudaStream_t st)
{
    constexpr int TH = kPlainAdjThreads;
    auto kern = force_plain_adjoint_kernel<C::ng, C::ne, C::exact, PAD, TH, kPlainAdjG>;
    RedLayout<C::ng, C::ne> Ly;
    Ly.build(P.n_b, true);
    const size_t sb = Ly.total + sizeof(double) * ((size_t)3 * P.n_b * TH + (size_t)C::ne * TH +
                                                   (size_t)C::ng * ((C::ne + 2) * TH + 8));
    if (sb > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sb);
        if (mm_cuda_check(e, "cudaFuncSetAttribute")) return -3;
    }
    int dev = 0, nsm = 148, per_sm = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, TH, sb);
    if (per_sm < 1) per_sm = 1;
    const long long pts_per_set = (P.layout == MM_LAYOUT_GRID) ? P.nv * P.nz : P.pps;
    const long long want = (long long)nsm * per_sm * 4;
    long long gx = std::max<long long>(1, want / std::max(1, P.n_sets));
    gx = std::min(gx, std::max<long long>(1, (pts_per_set + TH * 4 - 1) / (TH * 4)));
    gx = std::min<long long>(gx, 1 << 20);
    dim3 grid((unsigned)gx, (unsigned)std::min(P.n_sets, 65535));
    kern<<<grid, TH, sb, st>>>(P, grad);
    return mm_cuda_check(cudaGetLastError(), "force_plain_adjoint_kernel launch") ? -3 : 0;
}

template <class C, int PAD>
int launch_reduced_adjoint(const ForceParams &P, double *grad, cudaStream_t st)
{
    auto kern = force_reduced_adjoint_kernel<C::ng, C::ne, C::exact, PAD>;
    RedLayout<C::ng, C::ne> Ly;
    Ly.build(P.n_b, true);
    const size_t sb = Ly.total + sizeof(double) * 3 * P.n_b * kRedThreads;
    if (sb > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sb);
        if (mm_cuda_check(e, "cudaFuncSetAttribute")) return -3;
    }
    int dev = 0, nsm = 148, per_sm = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kRedThreads, sb);
    if (per_sm < 1) per_sm = 1;
    const long long pts_per_set = (P.layout == MM_LAYOUT_GRID) ? P.nv * P.nz : P.pps;
    const long long want = (long long)nsm * per_sm * 4;
    long long gx = std::max<long long>(1, want / std::max(1, P.n_sets));
    gx = std::min(gx, std::max<long long>(1, (pts_per_set + kRedThreads * 4 - 1) / (kRedThreads * 4)));
    gx = std::min<long long>(gx, 1 << 20);
    dim3 grid((unsigned)gx, (unsigned)std::min(P.n_sets, 65535));
    kern<<<grid, kRedThreads, sb, st>>>(P, grad);
    return mm_cuda_check(cudaGetLastError(), "force_reduced_adjoint_kernel launch") ? -3 : 0;
}

template <class C, int PAD>
int launch_traj_grad(const ForceParams &P, const TgParams &T, cudaStream_t st)
{
    const long long gx = ((long long)kTgLanes * T.n_particles + kTgThreads - 1) / kTgThreads;
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    // an ensemble of at most one CTA per SM keeps each ground state's rate sums
    // from the adjoint point's first pass in shared memory (the second pass
    // then skips the rates); larger ensembles keep two CTAs per SM instead
    auto go = [&](auto keepc) -> int {
        constexpr bool KEEP = decltype(keepc)::value;
        auto kern = traj_grad_kernel<C::ng, C::ne, C::exact, PAD, KEEP>;
        RedLayout<C::ng, C::ne> Ly;
        Ly.build(P.n_b, true);
        const size_t slots = (size_t)C::ng * C::ne * ((P.n_b + kRedPad - 1) / kRedPad * kRedPad);
        const size_t sb = Ly.total + sizeof(double) * (3 * (size_t)P.n_b + (KEEP ? C::ng * kKeepSlots<C::ne> : 0)) * kTgThreads +
                          (KEEP ? sizeof(int) * (kTgBofs + slots) : 0);
        if (sb > 48 * 1024) {
            cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sb);
            if (mm_cuda_check(e, "cudaFuncSetAttribute")) return -3;
        }
        kern<<<(unsigned)gx, kTgThreads, sb, st>>>(P, T);
        return mm_cuda_check(cudaGetLastError(), "traj_grad_kernel launch") ? -3 : 0;
    };
    if (gx <= nsm) return go(std::true_type{});
    return go(std::false_type{});
}

template <class C>
int launch_traj(const ForceParams &P, const TrajParams &T, cudaStream_t st)
{
    auto kern = traj1d_kernel<C::ng, C::ne, C::g, C::exact>;
    const size_t sb = smem_bytes<C>(P) * T.n_avg;
    if (sb > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sb);
        if (mm_cuda_check(e, "cudaFuncSetAttribute")) return -3;
    }
    const int ngroups = kThreads / C::g;
    const long long gx = (T.n_particles + ngroups - 1) / ngroups;
    kern<<<(unsigned)gx, kThreads, sb, st>>>(P, T);
    return mm_cuda_check(cudaGetLastError(), "traj1d_kernel launch") ? -3 : 0;
}

// List granule of the reduced kernel for a batch: kRedPad when padding every
// (ground, excited) triple list to a multiple of kRedPad adds at most a quarter
// to the batch's triples, else 1.  The triple count of a pair is
// sum_q active[g][e][q] * (beams of the set with polarisation q), from the
// host copies kept in the handles.
int reduced_list_granule(const mm_pack *pack, const mm_beams *beams)
{
    const int n_g = pack->n_g, n_e = pack->n_e, n_b = beams->n_b;
    long long n_raw = 0, n_pad = 0;
    for (int s = 0; s < beams->n_sets; s++) {
        int npol[3] = {0, 0, 0};
        for (int b = 0; b < n_b; b++) npol[beams->h_pol[(size_t)s * n_b + b]]++;
        for (int i = 0; i < n_g * n_e; i++) {
            const unsigned char *a = &pack->act[(size_t)i * 3];
            const int c = a[0] * npol[0] + a[1] * npol[1] + a[2] * npol[2];
            n_raw += c;
            n_pad += (c + kRedPad - 1) / kRedPad * kRedPad;
        }
    }
    return (4 * n_pad <= 5 * n_raw) ? kRedPad : 1;
}

// True when every set of the batch passes the reduced form's structural
// checks (the host twin of build_reduced_tables' flags[0]): every ground state
// has a triple, and the excited chain e' -> e (e' decays to a ground state
// that a beam of the set excites to e) is strongly connected.
bool reduced_sets_valid(const mm_pack *pack, const mm_beams *beams, int first, int count)
{
    const int n_g = pack->n_g, n_e = pack->n_e, n_b = beams->n_b;
    if (n_e > 32) return false;
    std::vector<int> cnt((size_t)n_g * n_e);
    for (int s = first; s < first + count; s++) {
        int npol[3] = {0, 0, 0};
        for (int b = 0; b < n_b; b++) npol[beams->h_pol[(size_t)s * n_b + b]]++;
        for (int i = 0; i < n_g * n_e; i++) {
            const unsigned char *a = &pack->act[(size_t)i * 3];
            cnt[i] = a[0] * npol[0] + a[1] * npol[1] + a[2] * npol[2];
        }
        for (int g = 0; g < n_g; g++) {
            int c = 0;
            for (int e = 0; e < n_e; e++) c += cnt[g * n_e + e];
            if (c == 0) return false;
        }
        unsigned T[32];
        for (int i = 0; i < n_e; i++) {
            unsigned ti = 1u << i;
            for (int g = 0; g < n_g; g++)
                if (pack->h_br[(size_t)i * n_g + g] > 0.0)
                    for (int j = 0; j < n_e; j++)
                        if (cnt[g * n_e + j] > 0) ti |= 1u << j;
            T[i] = ti;
        }
        for (int k = 0; k < n_e; k++)
            for (int i = 0; i < n_e; i++)
                if (T[i] >> k & 1u) T[i] |= T[k];
        const unsigned all = (n_e == 32) ? ~0u : (1u << n_e) - 1u;
        for (int i = 0; i < n_e; i++)
            if ((T[i] & all) != all) return false;
    }
    return true;
}

bool reduced_all_valid(const mm_pack *pack, const mm_beams *beams)
{
    return reduced_sets_valid(pack, beams, 0, beams->n_sets);
}

// Size-class dispatch.  SrOH (12 ground, 4 excited) has an exact class.
template <class F>
int dispatch_class(int n_g, int n_e, F &&f)
{
    if (n_g == 12 && n_e == 4) return f(Class<12, 4, 4, true>{});   // SrOH
    if (n_g <= 12 && n_e <= 4) return f(Class<12, 4, 4, false>{});
    mm_set_error("molecule size n_ground=%d n_excited=%d: this entry point runs the register-"
                 "resident kernels only (n_ground <= 12, n_excited <= 4)", n_g, n_e);
    return -1;
}

int fill_params(const mm_pack *pack, const mm_beams *beams, const mm_batch_opts *opts,
                ForceParams &P)
{
    if (!pack || !beams) { mm_set_error("null pack or beams handle"); return -1; }
    if (beams->n_b < 1 || beams->n_b > MM_MAX_BEAMS) {
        mm_set_error("n_beams=%d out of range [1, %d]", beams->n_b, MM_MAX_BEAMS);
        return -1;
    }
    P.n_g = pack->n_g; P.n_e = pack->n_e; P.n_b = beams->n_b; P.n_sets = beams->n_sets;
    P.Gamma = pack->Gamma; P.k = pack->k;
    P.hbar = (opts && opts->hbar > 0) ? opts->hbar : MM_HBAR_JIT;
    P.geff = beams->gamma_eff;
    P.E = pack->buf + pack->oE; P.zd = pack->buf + pack->ozd;
    P.d2 = pack->buf + pack->od2; P.BR = pack->buf + pack->oBR;
    P.kdir = beams->kdir; P.freq = beams->freq; P.s0 = beams->s0; P.bgrad = beams->bgrad;
    P.pol = beams->pol;
    P.uniform_fb = opts ? opts->uniform_fallback : 0;
    return 0;
}

}  // namespace

static int prepare_batch(const mm_pack *pack, const mm_beams *beams, const double *v,
                         const double *z, int64_t n_points, const mm_batch_opts *opts, double *F,
                         ForceParams &P, long long &pps);

extern "C" int mm_force_adjoint(const mm_pack *pack, const mm_beams *beams, const double *v,
                                const double *z, int64_t n_points, const mm_batch_opts *opts,
                                double *F, double *grad, void *stream)
{
    ForceParams P;
    long long pps;
    const int rc = prepare_batch(pack, beams, v, z, n_points, opts, F, P, pps);
    if (rc <= 0) return rc;
    if (!grad) { mm_set_error("grad must be non-null"); return -1; }
    if (opts->precision != MM_PREC_FP64 && opts->precision != MM_PREC_FP64_REDUCED) {
        mm_set_error("the adjoint runs in the FP64 and FP64-reduced forms only");
        return -1;
    }
    P.R = nullptr; P.pop = nullptr; P.status = nullptr;
    cudaStream_t st = (cudaStream_t)stream;
    // beyond the register classes: the shared-memory elimination adjoint (both precisions)
    if (!mm_register_class(P.n_g, P.n_e)) return mm_large_adjoint(P, pps, grad, st);
    // FP64-reduced: the reduced adjoint when every set is structurally valid,
    // else the elimination adjoint for the whole batch
    const bool red = opts->precision == MM_PREC_FP64_REDUCED && reduced_all_valid(pack, beams);
    return dispatch_class(P.n_g, P.n_e, [&](auto C) -> int {
        using CT = decltype(C);
        const bool pad = reduced_list_granule(pack, beams) == kRedPad;
        if (!red) return pad ? launch_plain_adjoint<CT, kRedPad>(P, grad, st) : launch_plain_adjoint<CT, 1>(P, grad, st);
        return pad ? launch_reduced_adjoint<CT, kRedPad>(P, grad, st) : launch_reduced_adjoint<CT, 1>(P, grad, st);
    });
}

// Validates a batch call and fills P; returns 1 to launch, 0 for an empty
// batch, < 0 on error.
static int prepare_batch(const mm_pack *pack, const mm_beams *beams, const double *v,
                         const double *z, int64_t n_points, const mm_batch_opts *opts, double *F,
                         ForceParams &P, long long &pps)
{
    if (fill_params(pack, beams, opts, P)) return -1;
    if (!opts) { mm_set_error("opts is required"); return -1; }
    if (n_points < 0) { mm_set_error("n_points < 0"); return -1; }
    if (n_points == 0) return 0;  // an empty batch may pass null arrays
    if (!v || !z || !F) { mm_set_error("v, z and F must be non-null"); return -1; }
    P.layout = opts->layout;
    P.nv = opts->nv; P.nz = opts->nz; P.pps = opts->points_per_set;
    if (opts->layout == MM_LAYOUT_GRID) {
        if (opts->nv < 1 || opts->nz < 1) { mm_set_error("grid layout needs nv, nz >= 1"); return -1; }
        pps = opts->nv * opts->nz;
        if (n_points != pps * (long long)beams->n_sets) {
            mm_set_error("grid layout: n_points=%lld != n_sets*nv*nz=%lld", (long long)n_points,
                         pps * (long long)beams->n_sets);
            return -1;
        }
    } else if (opts->layout == MM_LAYOUT_POINTS) {
        pps = opts->points_per_set > 0 ? opts->points_per_set : n_points;
        P.pps = pps;
        if ((n_points + pps - 1) / pps > beams->n_sets) {
            mm_set_error("points layout: %lld points at %lld per set need more than %d sets",
                         (long long)n_points, pps, beams->n_sets);
            return -1;
        }
    } else {
        mm_set_error("unknown layout %d", opts->layout);
        return -1;
    }
    if (opts->precision != MM_PREC_FP64 && opts->precision != MM_PREC_FP32_REFINE &&
        opts->precision != MM_PREC_FP64_REDUCED) {
        mm_set_error("unknown precision %d", opts->precision);
        return -1;
    }
    P.n_points = n_points;
    P.v = v; P.z = z; P.F = F;
    return 1;
}

extern "C" int mm_force_batch(const mm_pack *pack, const mm_beams *beams, const double *v,
                              const double *z, int64_t n_points, const mm_batch_opts *opts,
                              double *F, double *R, double *pop, int32_t *status, void *stream)
{
    ForceParams P;
    long long pps;
    const int prc = prepare_batch(pack, beams, v, z, n_points, opts, F, P, pps);
    if (prc <= 0) return prc;
    P.R = R; P.pop = pop; P.status = status;
    const int prec = opts->precision;
    cudaStream_t st = (cudaStream_t)stream;
    // beyond the register classes: the shared-memory kernels in FP64 for every
    // precision (the plain form's elimination, or the excited-chain solve for
    // the other forms when every set passes its structural checks)
    if (!mm_register_class(P.n_g, P.n_e))
        return mm_large_force(P, pps, prec != MM_PREC_FP64 && reduced_all_valid(pack, beams), st);
    return dispatch_class(P.n_g, P.n_e, [&](auto C) -> int {
        using CT = decltype(C);
        const bool pad = reduced_list_granule(pack, beams) == kRedPad;
        if (prec == MM_PREC_FP64) return pad ? launch_plain<CT, kRedPad>(P, pps, st) : launch_plain<CT, 1>(P, pps, st);
        if (prec == MM_PREC_FP64_REDUCED)
            return pad ? launch_reduced<CT, kRedPad, true>(P, pps, st) : launch_reduced<CT, 1, true>(P, pps, st);
        return pad ? launch_reduced<CT, kRedPad, false>(P, pps, st) : launch_reduced<CT, 1, false>(P, pps, st);
    });
}

extern "C" int mm_traj_run(const mm_pack *pack, const mm_beams *beams, const mm_traj_opts *topt,
                           const double *r0, const double *v0, int64_t n_particles,
                           double *r_final, double *v_final, int32_t *n_actual, double *r_traj,
                           double *v_traj, double *vsq_sum, double *n_samp, void *stream)
{
    if (!topt) { mm_set_error("trajectory options are required"); return -1; }
    mm_batch_opts bo = {};
    bo.precision = topt->precision;
    bo.hbar = topt->hbar;
    ForceParams P;
    if (fill_params(pack, beams, &bo, P)) return -1;
    if (n_particles > 0 && (!r0 || !v0 || !r_final || !v_final || !n_actual)) {
        mm_set_error("r0, v0, r_final, v_final and n_actual must be non-null");
        return -1;
    }
    if ((r_traj == nullptr) != (v_traj == nullptr)) { mm_set_error("r_traj and v_traj go together"); return -1; }
    if ((vsq_sum == nullptr) != (n_samp == nullptr)) { mm_set_error("vsq_sum and n_samp go together"); return -1; }
    if (n_particles < 0 || topt->n_steps < 1) { mm_set_error("n_particles >= 0 and n_steps >= 1 required"); return -1; }
    if (topt->ndim != 1 && topt->ndim != 3) { mm_set_error("ndim must be 1 or 3"); return -1; }
    if (topt->n_avg < 1 || topt->n_avg > 2 || topt->n_avg > beams->n_sets) {
        mm_set_error("n_avg=%d must be 1 or 2 and <= n_sets=%d", topt->n_avg, beams->n_sets);
        return -1;
    }
    if (topt->precision != MM_PREC_FP64 && topt->precision != MM_PREC_FP32_REFINE) {
        mm_set_error("unknown precision %d", topt->precision);
        return -1;
    }
    if (n_particles == 0) return 0;
    P.layout = MM_LAYOUT_POINTS; P.nv = P.nz = 0; P.pps = 1; P.n_points = 0;
    P.v = P.z = nullptr; P.F = P.R = P.pop = nullptr; P.status = nullptr;
    TrajParams T;
    T.dt = topt->dt; T.z_escape = topt->r_escape; T.mass = pack->mass;
    T.n_particles = n_particles; T.n_steps = topt->n_steps;
    T.ndim = topt->ndim; T.n_avg = topt->n_avg; T.i_eq = vsq_sum ? topt->i_eq : -1;
    T.z0 = r0; T.v0 = v0; T.z_final = r_final; T.v_final = v_final;
    T.z_traj = r_traj; T.v_traj = v_traj; T.n_actual = n_actual;
    T.vsq_sum = vsq_sum; T.n_samp = n_samp;
    const bool fp32 = topt->precision == MM_PREC_FP32_REFINE;
    cudaStream_t st = (cudaStream_t)stream;
    // beyond the register classes: the plain FP64 force from the shared-memory kernel
    if (!mm_register_class(P.n_g, P.n_e)) return mm_large_traj(P, T, st);
    return dispatch_class(P.n_g, P.n_e, [&](auto C) -> int {
        using CT = decltype(C);
        if (!fp32) return launch_traj<CT>(P, T, st);
        return reduced_list_granule(pack, beams) == kRedPad ? launch_traj_reduced<CT, kRedPad>(P, T, st)
                                                            : launch_traj_reduced<CT, 1>(P, T, st);
    });
}

extern "C" int mm_traj_grad_run(const mm_pack *pack, const mm_beams *beams, const mm_tgrad_opts *opts,
                                int64_t n_particles, double *state, int32_t *n_actual, double *ckpt,
                                void *stream)
{
    if (!opts) { mm_set_error("trajectory-gradient options are required"); return -1; }
    mm_batch_opts bo = {};
    bo.precision = MM_PREC_FP64_REDUCED;
    bo.hbar = opts->hbar;
    ForceParams P;
    if (fill_params(pack, beams, &bo, P)) return -1;
    if (n_particles < 0 || opts->n_steps < 0 || opts->step0 < 0) {
        mm_set_error("n_particles, n_steps and step0 must be >= 0");
        return -1;
    }
    if (opts->step0 + opts->n_steps > 0x7fffffffll) { mm_set_error("step indices exceed 2^31 - 1"); return -1; }
    if (opts->n_par < 1 || opts->n_par > MM_TGRAD_MAX_PAR) {
        mm_set_error("n_par=%d out of range [1, %d]", opts->n_par, MM_TGRAD_MAX_PAR);
        return -1;
    }
    for (int b = 0; b < beams->n_b; b++)
        if (opts->freq_par[b] < -1 || opts->freq_par[b] >= opts->n_par || opts->s0_par[b] < -1 ||
            opts->s0_par[b] >= opts->n_par) {
            mm_set_error("beam %d: parameter index out of range [-1, n_par)", b);
            return -1;
        }
    if (opts->bprime_par < -1 || opts->bprime_par >= opts->n_par) {
        mm_set_error("bprime_par out of range [-1, n_par)");
        return -1;
    }
    if (ckpt && opts->ckpt_every < 1) { mm_set_error("ckpt needs ckpt_every >= 1"); return -1; }
    if (!reduced_sets_valid(pack, beams, 0, 1)) {
        mm_set_error("beam set 0 fails the reduced form's structural checks (a ground state no beam "
                     "pumps, or an excited chain that is not strongly connected)");
        return -1;
    }
    if (n_particles == 0 || opts->n_steps == 0) return 0;
    if (!state || !n_actual) { mm_set_error("state and n_actual must be non-null"); return -1; }
    P.layout = MM_LAYOUT_POINTS; P.nv = P.nz = 0; P.pps = 1; P.n_points = 0;
    P.v = P.z = nullptr; P.F = P.R = P.pop = nullptr; P.status = nullptr;
    TgParams T;
    T.dt = opts->dt; T.r_escape = opts->r_escape; T.mass = pack->mass;
    T.v_rec = P.hbar * P.k / pack->mass;
    T.n_particles = n_particles; T.n_steps = opts->n_steps; T.step0 = opts->step0;
    T.ckpt_every = ckpt ? opts->ckpt_every : 0;
    T.n_par = opts->n_par; T.kicks = opts->kicks ? 1 : 0; T.bprime_par = opts->bprime_par;
    T.seed = opts->seed;
    for (int b = 0; b < MM_MAX_BEAMS; b++) {
        T.freq_par[b] = (signed char)(b < beams->n_b ? opts->freq_par[b] : -1);
        T.s0_par[b] = (signed char)(b < beams->n_b ? opts->s0_par[b] : -1);
    }
    T.state = state; T.n_actual = n_actual; T.ckpt = ckpt;
    cudaStream_t st = (cudaStream_t)stream;
    return dispatch_class(P.n_g, P.n_e, [&](auto C) -> int {
        using CT = decltype(C);
        return reduced_list_granule(pack, beams) == kRedPad ? launch_traj_grad<CT, kRedPad>(P, T, st)
                                                            : launch_traj_grad<CT, 1>(P, T, st);
    });
}

extern "C" int mm_traj1d_run(const mm_pack *pack, const mm_beams *beams, const double *z0,
                             const double *v0, int64_t n_particles, double dt, int64_t n_steps,
                             double z_escape, const mm_batch_opts *opts, double *z_final,
                             double *v_final, int32_t *n_actual, double *z_traj, double *v_traj,
                             void *stream)
{
    mm_traj_opts T = {};
    T.ndim = 1;
    T.n_avg = 1;
    T.n_steps = n_steps;
    T.dt = dt;
    T.r_escape = z_escape;
    T.i_eq = -1;
    T.precision = opts ? opts->precision : MM_PREC_FP64;
    T.hbar = opts ? opts->hbar : 0.0;
    return mm_traj_run(pack, beams, &T, z0, v0, n_particles, z_final, v_final, n_actual, z_traj,
                       v_traj, nullptr, nullptr, stream);
}
