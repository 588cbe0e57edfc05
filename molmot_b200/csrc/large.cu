// large.cu -- the drop-in 1D entry points (mm_force_batch, mm_force_adjoint,
// mm_traj_run) for molecules beyond the register-resident kernel classes of
// force1d.cu (n_ground > 12 or n_excited > 4), up to 48 ground and 16
// excited states, as the reference's kernel compiles for any molecule size
// (molmot_cuda/rate_equations_cuda.py:287-320) and its numba core takes any
// MolecularData (molmot/obe/rate_equations_jit.py:18-145).
//
// A group of G lanes (16 for n_ground <= 16, else 32) solves one point with
// the molecule's tables and the population system in shared memory
// (sm_point, smem_solve.cuh).  The CTA stages the molecule once and the
// parameter set's beams per set; force maps run one CTA row per set with the
// set's points split over gridDim.x like force_kernel; trajectories run one
// particle per group with every step's solve in the same launch.
#include <algorithm>
#include "smem_solve.cuh"
#include "large.cuh"

namespace {

template <int NGMAX, int NEMAX, int G>
struct LClass {
    static constexpr int ng = NGMAX, ne = NEMAX, g = G;
    static constexpr int warps = (G == 16) ? 4 : 2;
};
using LC0 = LClass<16, 16, 16>;
using LC1 = LClass<32, 16, 32>;
using LC2 = LClass<48, 16, 32>;

template <int NGMAX, int NEMAX, bool RED, bool ADJ>
size_t large_smem(int groups, int n_sets_staged)
{
    using W = SmWorkLayout<NGMAX, NEMAX, RED, ADJ>;
    return sizeof(double) * ((size_t)SmMolLayout<NGMAX, NEMAX>::doubles + (size_t)n_sets_staged * kSmBeamDoubles +
                             (size_t)groups * W::doubles) +
           sizeof(int) * ((size_t)n_sets_staged * kSmBeamInts + (size_t)groups * W::ints);
}

// Shared-memory carve-up: molecule | beam sets | group workspaces | beam ints | group ints.
template <int NGMAX, int NEMAX, bool RED, bool ADJ>
struct LSmem {
    double *mol, *beams, *groups;
    int *beam_ints, *group_ints;
    __device__ LSmem(unsigned char *raw, int n_groups, int n_sets_staged)
    {
        using W = SmWorkLayout<NGMAX, NEMAX, RED, ADJ>;
        mol = (double *)raw;
        beams = mol + SmMolLayout<NGMAX, NEMAX>::doubles;
        groups = beams + (size_t)n_sets_staged * kSmBeamDoubles;
        beam_ints = (int *)(groups + (size_t)n_groups * W::doubles);
        group_ints = beam_ints + n_sets_staged * kSmBeamInts;
    }
};

// Force maps (and, with ADJ, the elimination adjoint's gradient rows), same
// layouts and outputs as force_kernel / force_adjoint_kernel.  Points with a
// non-finite v or z are solved at (0, 0) so the group keeps step with the
// warp's shuffles, and then written as NaN with the non-finite status bit.
template <int NGMAX, int NEMAX, int G, bool RED, bool ADJ>
__global__ void __launch_bounds__(128)
large_force_kernel(ForceParams P, double *grad)
{
    extern __shared__ __align__(16) unsigned char sm[];
    const int groups = blockDim.x / G;
    LSmem<NGMAX, NEMAX, RED, ADJ> L(sm, groups, 1);
    const int t = (threadIdx.x & 31) % G, group = threadIdx.x / G;
    using WL = SmWorkLayout<NGMAX, NEMAX, RED, ADJ>;
    const SmWork W = sm_work<NGMAX, NEMAX, RED, ADJ>(L.groups + (size_t)group * WL::doubles,
                                                     L.group_ints + (size_t)group * WL::ints);
    SmMol M;
    sm_stage_mol<NGMAX, NEMAX>(P.E, P.n_g, P.n_e, P.Gamma, L.mol, M);
    const long long pts_per_set = (P.layout == MM_LAYOUT_GRID) ? P.nv * P.nz : P.pps;
    const int nb = P.n_b, gw = 2 * nb + 1;
    for (int set = blockIdx.y; set < P.n_sets; set += gridDim.y) {
        const long long set_first = (long long)set * pts_per_set;
        long long set_count = pts_per_set;
        if (set_first + set_count > P.n_points) set_count = P.n_points - set_first;
        if (set_count <= 0) continue;  // uniform over the CTA
        SmBeam Bm;
        __syncthreads();
        const size_t o = (size_t)set * nb;
        sm_stage_beams(P.kdir + o, P.freq + o, P.s0 + o, P.pol + o, nb, P.bgrad[set], P.k, P.hbar, P.Gamma,
                       L.beams, L.beam_ints, Bm);
        __syncthreads();
        const long long chunk = (set_count + gridDim.x - 1) / gridDim.x;
        const long long start = (long long)blockIdx.x * chunk;
        const long long end = min(start + chunk, set_count);
        for (long long base = start; base < end; base += groups) {
            const long long ip = base + group;
            const bool valid = ip < end;
            const long long ipc = valid ? ip : start;
            double v, z;
            if (P.layout == MM_LAYOUT_GRID) {
                v = P.v[ipc / P.nz];
                z = P.z[ipc % P.nz];
            } else {
                v = P.v[set_first + ipc];
                z = P.z[set_first + ipc];
            }
            const bool fin = isfinite(v) && isfinite(z);
            const long long gi = set_first + ipc;
            double *pop = (valid && fin && P.pop) ? P.pop + gi * P.n_g : nullptr;
            const SmOut r = sm_point<NGMAX, NEMAX, G, RED, ADJ>(M, Bm, W, t, fin ? v : 0.0, fin ? z : 0.0,
                                                                Bm.Bg, P.geff, P.uniform_fb, pop);
            if (valid) {
                const double nan = __longlong_as_double(0x7ff8000000000000ll);
                if (t == 0) {
                    P.F[gi] = fin ? r.F : nan;
                    if (P.R) P.R[gi] = fin ? r.R : nan;
                    if (P.status) P.status[gi] = fin ? r.status : MM_ST_NONFINITE;
                }
                if (!fin && P.pop)
                    for (int g = t; g < P.n_g; g += G) P.pop[gi * P.n_g + g] = nan;
                if constexpr (ADJ) {
                    double *row = grad + gi * gw;
                    for (int i = t; i < 2 * nb; i += G) row[i] = fin ? W.gacc[i] : nan;
                    if (t == 0) row[2 * nb] = fin ? r.gB : nan;
                }
            }
            __syncwarp();
        }
    }
}

// Fused trajectories, one particle per group: the integrator, escape rule,
// per-axis model, RF averaging and v^2 sums of traj1d_kernel (force1d.cu),
// with each force from the elimination (the plain FP64 form).
template <int NGMAX, int NEMAX, int G>
__global__ void __launch_bounds__(128)
large_traj_kernel(ForceParams P, TrajParams T)
{
    extern __shared__ __align__(16) unsigned char sm[];
    const int groups = blockDim.x / G;
    LSmem<NGMAX, NEMAX, false, false> L(sm, groups, 2);
    const int t = (threadIdx.x & 31) % G, group = threadIdx.x / G;
    using WL = SmWorkLayout<NGMAX, NEMAX, false, false>;
    const SmWork W = sm_work<NGMAX, NEMAX, false, false>(L.groups + (size_t)group * WL::doubles, nullptr);
    SmMol M;
    SmBeam Bm[2];
    sm_stage_mol<NGMAX, NEMAX>(P.E, P.n_g, P.n_e, P.Gamma, L.mol, M);
    for (int a = 0; a < T.n_avg; a++) {
        const size_t o = (size_t)a * P.n_b;
        sm_stage_beams(P.kdir + o, P.freq + o, P.s0 + o, P.pol + o, P.n_b, P.bgrad[a], P.k, P.hbar, P.Gamma,
                       L.beams + a * kSmBeamDoubles, L.beam_ints + a * kSmBeamInts, Bm[a]);
    }
    __syncthreads();
    const int nd = T.ndim;
    const long long ip = (long long)blockIdx.x * groups + group;
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
            // a stopped particle (or an empty group) solves a finite dummy point so
            // the group keeps step with the warp's shuffles
            const bool fin = !done && isfinite(u[d]) && isfinite(x[d]);
            double F = 0.0;
            for (int a = 0; a < T.n_avg; a++) {
                const SmOut r = sm_point<NGMAX, NEMAX, G, false>(M, Bm[a], W, t, fin ? u[d] : 0.0,
                                                                 fin ? x[d] : 0.0, Bm[a].Bg * mult, P.geff,
                                                                 P.uniform_fb, nullptr);
                F = (a == 0) ? r.F : __dadd_rn(F, r.F);
            }
            if (T.n_avg == 2) F = 0.5 * F;
            if (!fin) F = __longlong_as_double(0x7ff8000000000000ll);
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

template <class C>
int large_class_of(int n_g, int n_e, C &&f)
{
    if (n_g < 2 || n_g > 48 || n_e < 1 || n_e > 16) {
        mm_set_error("molecule size n_ground=%d n_excited=%d outside 2..48 / 1..16", n_g, n_e);
        return -1;
    }
    if (n_g <= 16) return f(LC0{});
    if (n_g <= 32) return f(LC1{});
    return f(LC2{});
}

template <class KernT>
int set_smem(KernT kern, size_t sb)
{
    int dev = 0, smax = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&smax, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (sb > (size_t)smax) {
        mm_set_error("the shared-memory kernel needs %zu bytes of shared memory (limit %d)", sb, smax);
        return -1;
    }
    if (sb > 48 * 1024 &&
        mm_cuda_check(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sb),
                      "cudaFuncSetAttribute"))
        return -3;
    return 0;
}

template <class C, bool RED, bool ADJ>
int launch_large_force(const ForceParams &P, long long pps, double *grad, cudaStream_t st)
{
    auto kern = large_force_kernel<C::ng, C::ne, C::g, RED, ADJ>;
    const int threads = 32 * C::warps, groups = threads / C::g;
    const size_t sb = large_smem<C::ng, C::ne, RED, ADJ>(groups, 1);
    if (int rc = set_smem(kern, sb)) return rc;
    int dev = 0, nsm = 148, per_sm = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, sb);
    if (per_sm < 1) per_sm = 1;
    // enough CTAs to fill the GPU a few times over, at least 8 points per group
    const long long want = (long long)nsm * per_sm * 4;
    long long gx = std::max<long long>(1, want / std::max(1, P.n_sets));
    gx = std::min(gx, std::max<long long>(1, (pps + (long long)groups * 8 - 1) / ((long long)groups * 8)));
    gx = std::min<long long>(gx, 1 << 20);
    dim3 grid((unsigned)gx, (unsigned)std::min(P.n_sets, 65535));
    kern<<<grid, threads, sb, st>>>(P, grad);
    return mm_cuda_check(cudaGetLastError(), "large_force_kernel launch") ? -3 : 0;
}

}  // namespace

int mm_large_force(const ForceParams &P, long long pps, bool reduced, cudaStream_t st)
{
    return large_class_of(P.n_g, P.n_e, [&](auto C) -> int {
        using CT = decltype(C);
        return reduced ? launch_large_force<CT, true, false>(P, pps, nullptr, st)
                       : launch_large_force<CT, false, false>(P, pps, nullptr, st);
    });
}

int mm_large_adjoint(const ForceParams &P, long long pps, double *grad, cudaStream_t st)
{
    return large_class_of(P.n_g, P.n_e, [&](auto C) -> int {
        using CT = decltype(C);
        return launch_large_force<CT, false, true>(P, pps, grad, st);
    });
}

int mm_large_traj(const ForceParams &P, const TrajParams &T, cudaStream_t st)
{
    return large_class_of(P.n_g, P.n_e, [&](auto C) -> int {
        using CT = decltype(C);
        auto kern = large_traj_kernel<CT::ng, CT::ne, CT::g>;
        const int threads = 32 * CT::warps, groups = threads / CT::g;
        const size_t sb = large_smem<CT::ng, CT::ne, false, false>(groups, 2);
        if (int rc = set_smem(kern, sb)) return rc;
        const long long gx = (T.n_particles + groups - 1) / groups;
        kern<<<(unsigned)gx, threads, sb, st>>>(P, T);
        return mm_cuda_check(cudaGetLastError(), "large_traj_kernel launch") ? -3 : 0;
    });
}
