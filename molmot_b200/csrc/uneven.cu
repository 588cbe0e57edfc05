// uneven.cu -- steady-state forces for a batch of different molecules
// (n_ground up to 48, n_excited up to 16), each with its own parameter set
// and its own number of points, in persistent kernels that draw work from an
// atomic counter.  C-ABI: mm_bank_*, mm_uneven_plan_*, mm_uneven_force.
//
// Same algorithm and exactness as rate_core.cuh (molmot/obe/rate_equations_jit.py:18-145).
// The population matrix lives in shared memory: a group of G lanes
// (16 or 32) per point, lanes covering consecutive columns so every
// row-wise access is conflict-free; the pivot search is a group-wide argmax
// (first maximum, as the reference's strict-greater scan); factors are
// stored below the diagonal.
//
// Work: the plan cuts every molecule's points into chunks of a few CTA
// widths and sorts the chunks of each size class by decreasing cost
// (n_g^3 + triples); a CTA takes the next chunk from the class counter,
// stages that molecule and its beams in shared memory, and its groups sweep
// the chunk's points.
#include <stdio.h>
#include <string.h>
#include <algorithm>
#include <vector>
#include "smem_solve.cuh"

struct mm_bank {
    int n_mol;
    int device;
    std::vector<int> ng, ne;          // host copies
    std::vector<long long> off;
    int *d_ng, *d_ne;
    long long *d_off;
    double *d_gam, *d_k, *d_mass;
    double *buf;                      // per molecule: E[n_s], zd[n_s], d2[n_g n_e 3], BR[n_e n_g]
};

struct UnevenTask {
    int mol, pad;
    long long p0, p1;
};

struct mm_uneven_plan {
    const mm_bank *bank;
    long long n_points;
    int n_mol;
    int wpc[3];                        // warps per CTA per class
    int n_tasks[3];
    UnevenTask *d_tasks[3];
    int *d_counter;                    // [3], reset by every mm_uneven_force
    int *d_valid;                      // [n_mol]: the reduced solve applies (set per call)
    std::vector<UnevenTask> h_tasks[3];
};

namespace {

struct UnevenParams {
    const int *ng, *ne;
    const long long *off;
    const double *gam, *kw, *buf;
    int n_b;
    const double *kdir, *freq, *s0, *bgrad;
    const int32_t *pol;
    double geff, hbar;
    int uniform_fb;
    const double *v, *z;
    double *F, *R;
    int32_t *status;
    const UnevenTask *tasks;
    int n_tasks;
    int *counter;
    int persistent;
    // valid[m] = 1: molecule m is solved by the reduced kernels; the
    // elimination kernels then take only molecules with valid[m] = 0.
    // nullptr: the elimination kernels take every molecule.
    const int *valid;
};

template <int NGMAX, int NEMAX, bool RED = false>
struct ULayout {
    using W = SmWorkLayout<NGMAX, NEMAX, RED>;
    static constexpr int mol_doubles = SmMolLayout<NGMAX, NEMAX>::doubles;
    static size_t bytes(int groups)
    {
        return sizeof(double) * (size_t)(mol_doubles + kSmBeamDoubles + groups * W::doubles) +
               sizeof(int) * (kSmBeamInts + 8);
    }
};

// RED: the populations from the excited-state chain (see reduced.cuh for the
// identity).  Molecules the reduction does not cover (valid[m] = 0) are left
// to the elimination kernels (RED = false).  The point solve is sm_point
// (smem_solve.cuh).
template <int NGMAX, int NEMAX, int G, bool RED>
__global__ void __launch_bounds__(256)
uneven_kernel(UnevenParams P)
{
    using Ly = ULayout<NGMAX, NEMAX, RED>;
    extern __shared__ __align__(16) unsigned char smraw[];
    double *smd = (double *)smraw;
    double *molsm = smd, *beamsm = molsm + Ly::mol_doubles, *grp0 = beamsm + kSmBeamDoubles;
    const int groups = blockDim.x / G;
    int *pol = (int *)(grp0 + (size_t)groups * Ly::W::doubles);
    int *sint = pol + kSmBeamInts;  // [0] task

    const int lane = threadIdx.x & 31, t = lane % G;
    const int group = threadIdx.x / G;
    const SmWork W = sm_work<NGMAX, NEMAX, RED>(grp0 + (size_t)group * Ly::W::doubles, nullptr);

    for (int it = 0;; it++) {
        __syncthreads();
        if (threadIdx.x == 0)
            sint[0] = P.persistent ? atomicAdd(P.counter, 1) : (it == 0 ? (int)blockIdx.x : P.n_tasks);
        __syncthreads();
        const int task = sint[0];
        if (task >= P.n_tasks) break;
        const UnevenTask T = P.tasks[task];
        const int m = T.mol;
        if (P.valid && (RED ? !P.valid[m] : P.valid[m])) continue;  // uniform over the CTA
        SmMol M;
        SmBeam Bm;
        sm_stage_mol<NGMAX, NEMAX>(P.buf + P.off[m], P.ng[m], P.ne[m], P.gam[m], molsm, M);
        const size_t o = (size_t)m * P.n_b;
        sm_stage_beams(P.kdir + o, P.freq + o, P.s0 + o, P.pol + o, P.n_b, P.bgrad[m], P.kw[m], P.hbar,
                       P.gam[m], beamsm, pol, Bm);
        __syncthreads();
        for (long long base = T.p0; base < T.p1; base += groups) {
            const long long ip = base + group;
            const bool valid = ip < T.p1;
            const long long gi = valid ? ip : T.p0;
            const SmOut r = sm_point<NGMAX, NEMAX, G, RED>(M, Bm, W, t, P.v[gi], P.z[gi], Bm.Bg, P.geff,
                                                           P.uniform_fb, nullptr);
            if (valid && t == 0) {
                P.F[gi] = r.F;
                if (P.R) P.R[gi] = r.R;
                if (P.status) P.status[gi] = r.status;
            }
        }
    }
}

// valid[m] = 1 when the excited-state chain reduction applies to molecule m
// with its beam set: every ground state has an active (beam, excited) pair,
// and the chain of excited states (e' -> e when e' decays to a ground state
// that some beam excites to e) is strongly connected, so its stationary
// vector is unique and the state reduction never meets a zero outflow.
__global__ void uneven_valid_kernel(UnevenParams P, int n_mol, int *valid)
{
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= n_mol) return;
    const int n_g = P.ng[m], n_e = P.ne[m], n_s = n_g + n_e, n_b = P.n_b;
    const double *mb = P.buf + P.off[m];
    const double *d2 = mb + 2 * n_s, *BR = d2 + n_g * n_e * 3;
    const int32_t *pol = P.pol + (size_t)m * n_b;
    int ok = 1;
    unsigned T[MM_MAX_EXCITED];
    for (int e = 0; e < n_e; e++) T[e] = 0u;
    for (int g = 0; g < n_g; g++) {
        unsigned act = 0u;  // excited states that some beam drives from g
        for (int e = 0; e < n_e; e++)
            for (int b = 0; b < n_b; b++)
                if (d2[(g * n_e + e) * 3 + pol[b]] >= 1e-15) act |= 1u << e;
        if (!act) ok = 0;
        for (int e = 0; e < n_e; e++)
            if (BR[e * n_g + g] > 0.0) T[e] |= act;
    }
    // reachability closure (Floyd-Warshall on bit masks)
    for (int e = 0; e < n_e; e++) T[e] |= 1u << e;
    for (int k = 0; k < n_e; k++)
        for (int i = 0; i < n_e; i++)
            if (T[i] >> k & 1u) T[i] |= T[k];
    const unsigned all = (n_e >= 32) ? 0xffffffffu : ((1u << n_e) - 1u);
    for (int e = 0; e < n_e; e++)
        if ((T[e] & all) != all) ok = 0;
    valid[m] = ok;
}

template <int NGMAX, int NEMAX, int G>
struct UClass {
    static constexpr int ng = NGMAX, ne = NEMAX, g = G;
};
using UC0 = UClass<16, 16, 16>;
using UC1 = UClass<32, 16, 32>;
using UC2 = UClass<48, 16, 32>;

int class_of(int n_g, int n_e)
{
    if (n_e > 16 || n_g > 48) return -1;
    if (n_g <= 16) return 0;
    if (n_g <= 32) return 1;
    return 2;
}

template <class C, bool RED = false>
int launch_class(const UnevenParams &P0, const mm_uneven_plan *plan, int cls, int persistent,
                 cudaStream_t st)
{
    if (plan->n_tasks[cls] == 0) return 0;
    UnevenParams P = P0;
    P.tasks = plan->d_tasks[cls];
    P.n_tasks = plan->n_tasks[cls];
    P.counter = plan->d_counter + cls;
    P.persistent = persistent;
    const int threads = 32 * plan->wpc[cls];
    const int groups = threads / C::g;
    auto kern = uneven_kernel<C::ng, C::ne, C::g, RED>;
    const size_t sb = ULayout<C::ng, C::ne, RED>::bytes(groups);
    int dev0 = 0, smax = 0;
    cudaGetDevice(&dev0);
    cudaDeviceGetAttribute(&smax, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev0);
    if (sb > (size_t)smax) {
        mm_set_error("size class %d at %d warps per CTA needs %zu bytes of shared memory (limit %d)", cls,
                     plan->wpc[cls], sb, smax);
        return -1;
    }
    if (mm_cuda_check(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sb),
                      "cudaFuncSetAttribute"))
        return -3;
    int grid = P.n_tasks;
    if (persistent) {
        int dev = 0, nsm = 148, per_sm = 1;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, sb);
        grid = std::min(P.n_tasks, nsm * std::max(per_sm, 1));
    }
    kern<<<grid, threads, sb, st>>>(P);
    return mm_cuda_check(cudaGetLastError(), "uneven_kernel launch") ? -3 : 0;
}

}  // namespace

extern "C" int mm_bank_create(const mm_mol_desc *mols, int32_t n_mol, mm_bank **out)
{
    if (!out) { mm_set_error("out is null"); return -1; }
    *out = nullptr;
    if (!mols || n_mol < 1) { mm_set_error("need at least one molecule"); return -1; }
    mm_bank *bk = new mm_bank();
    bk->n_mol = n_mol;
    cudaGetDevice(&bk->device);
    std::vector<double> h, gam(n_mol), kw(n_mol), mass(n_mol);
    bk->ng.resize(n_mol); bk->ne.resize(n_mol); bk->off.resize(n_mol);
    for (int m = 0; m < n_mol; m++) {
        const mm_mol_desc &d = mols[m];
        const int n_g = d.n_ground, n_e = d.n_excited, n_s = n_g + n_e;
        if (!d.energies || !d.d_squared || !d.zeeman_z_diag || class_of(n_g, n_e) < 0 || n_g < 2 ||
            n_e < 1 || !(d.Gamma > 0) || !(d.k > 0)) {
            mm_set_error("molecule %d: incomplete or out of range (n_ground 2..48, n_excited 1..16)", m);
            delete bk;
            return -1;
        }
        bk->ng[m] = n_g; bk->ne[m] = n_e; bk->off[m] = (long long)h.size();
        gam[m] = d.Gamma; kw[m] = d.k; mass[m] = d.mass;
        h.insert(h.end(), d.energies, d.energies + n_s);
        h.insert(h.end(), d.zeeman_z_diag, d.zeeman_z_diag + n_s);
        h.insert(h.end(), d.d_squared, d.d_squared + n_g * n_e * 3);
        // branching ratios in the reference's summation order
        for (int ie = 0; ie < n_e; ie++) {
            double total = 0.0;
            for (int ig = 0; ig < n_g; ig++)
                for (int q = 0; q < 3; q++) total += d.d_squared[(ig * n_e + ie) * 3 + q];
            for (int ig = 0; ig < n_g; ig++) {
                double s = 0.0;
                for (int q = 0; q < 3; q++) s += d.d_squared[(ig * n_e + ie) * 3 + q];
                h.push_back(total > 1e-30 ? s / total : 0.0);
            }
        }
    }
    for (double x : h)
        if (!isfinite(x)) { mm_set_error("molecule data contains a non-finite value"); delete bk; return -1; }
    auto up = [](auto **dst, const auto *src, size_t n) -> int {
        if (mm_cuda_check(cudaMalloc((void **)dst, n * sizeof(**dst)), "cudaMalloc")) return -3;
        return mm_cuda_check(cudaMemcpy(*dst, src, n * sizeof(**dst), cudaMemcpyHostToDevice), "cudaMemcpy") ? -3 : 0;
    };
    int rc = 0;
    rc |= up(&bk->d_ng, bk->ng.data(), n_mol);
    rc |= up(&bk->d_ne, bk->ne.data(), n_mol);
    rc |= up(&bk->d_off, bk->off.data(), n_mol);
    rc |= up(&bk->d_gam, gam.data(), n_mol);
    rc |= up(&bk->d_k, kw.data(), n_mol);
    rc |= up(&bk->d_mass, mass.data(), n_mol);
    rc |= up(&bk->buf, h.data(), h.size());
    if (rc) { mm_bank_destroy(bk); return -3; }
    *out = bk;
    return 0;
}

extern "C" int mm_bank_destroy(mm_bank *bk)
{
    if (!bk) return 0;
    cudaFree(bk->d_ng); cudaFree(bk->d_ne); cudaFree(bk->d_off); cudaFree(bk->d_gam);
    cudaFree(bk->d_k); cudaFree(bk->d_mass); cudaFree(bk->buf);
    delete bk;
    return 0;
}

extern "C" int mm_uneven_plan_create(const mm_bank *bank, const int64_t *point_offsets,
                                     const mm_uneven_opts *opts, mm_uneven_plan **out)
{
    if (!out) { mm_set_error("out is null"); return -1; }
    *out = nullptr;
    if (!bank || !point_offsets) { mm_set_error("bank and point_offsets are required"); return -1; }
    const int n_mol = bank->n_mol;
    if (point_offsets[0] != 0) { mm_set_error("point_offsets[0] must be 0"); return -1; }
    for (int m = 0; m < n_mol; m++)
        if (point_offsets[m + 1] < point_offsets[m]) { mm_set_error("point_offsets must not decrease"); return -1; }
    mm_uneven_plan *p = new mm_uneven_plan();
    p->bank = bank;
    p->n_mol = n_mol;
    p->n_points = point_offsets[n_mol];
    const int G[3] = {16, 32, 32};
    for (int c = 0; c < 3; c++) {
        int w = opts ? opts->warps_per_cta[c] : 0;
        if (w <= 0) w = c == 0 ? 4 : 2;
        if (w > 8) { mm_set_error("warps_per_cta must be <= 8"); delete p; return -1; }
        p->wpc[c] = w;
    }
    const int chunk_groups = (opts && opts->chunk_groups > 0) ? opts->chunk_groups : 8;
    std::vector<std::pair<double, UnevenTask>> tk[3];
    for (int m = 0; m < n_mol; m++) {
        const int c = class_of(bank->ng[m], bank->ne[m]);
        const long long chunk = (long long)(32 * p->wpc[c] / G[c]) * chunk_groups;
        const double cost = (double)bank->ng[m] * bank->ng[m] * bank->ng[m] +
                            8.0 * bank->ng[m] * bank->ne[m] * 8;
        for (long long a = point_offsets[m]; a < point_offsets[m + 1]; a += chunk) {
            UnevenTask t;
            t.mol = m; t.pad = 0; t.p0 = a;
            t.p1 = std::min<long long>(a + chunk, point_offsets[m + 1]);
            tk[c].push_back({cost * (double)(t.p1 - t.p0), t});
        }
    }
    int rc = 0;
    for (int c = 0; c < 3; c++) {
        std::stable_sort(tk[c].begin(), tk[c].end(),
                         [](const auto &a, const auto &b) { return a.first > b.first; });
        for (auto &x : tk[c]) p->h_tasks[c].push_back(x.second);
        p->n_tasks[c] = (int)p->h_tasks[c].size();
        p->d_tasks[c] = nullptr;
        if (p->n_tasks[c]) {
            rc |= mm_cuda_check(cudaMalloc((void **)&p->d_tasks[c], sizeof(UnevenTask) * p->n_tasks[c]), "cudaMalloc");
            if (!rc)
                rc |= mm_cuda_check(cudaMemcpy(p->d_tasks[c], p->h_tasks[c].data(),
                                               sizeof(UnevenTask) * p->n_tasks[c], cudaMemcpyHostToDevice),
                                    "cudaMemcpy");
        }
    }
    rc |= mm_cuda_check(cudaMalloc((void **)&p->d_counter, 3 * sizeof(int)), "cudaMalloc");
    rc |= mm_cuda_check(cudaMalloc((void **)&p->d_valid, sizeof(int) * n_mol), "cudaMalloc");
    if (rc) { mm_uneven_plan_destroy(p); return -3; }
    *out = p;
    return 0;
}

extern "C" int mm_uneven_plan_destroy(mm_uneven_plan *p)
{
    if (!p) return 0;
    for (int c = 0; c < 3; c++) cudaFree(p->d_tasks[c]);
    cudaFree(p->d_counter);
    cudaFree(p->d_valid);
    delete p;
    return 0;
}

extern "C" int mm_uneven_force(const mm_uneven_plan *plan, const mm_beams *beams, const double *v,
                               const double *z, double hbar, int32_t uniform_fallback,
                               int32_t persistent, double *F, double *R, int32_t *status,
                               void *stream)
{
    if (!plan || !beams || !v || !z || !F) { mm_set_error("plan, beams, v, z and F are required"); return -1; }
    if (beams->n_sets != plan->n_mol) {
        mm_set_error("beams must hold one parameter set per molecule (%d), got %d", plan->n_mol,
                     beams->n_sets);
        return -1;
    }
    if (plan->n_points == 0) return 0;
    const mm_bank *bk = plan->bank;
    UnevenParams P;
    P.ng = bk->d_ng; P.ne = bk->d_ne; P.off = bk->d_off; P.gam = bk->d_gam; P.kw = bk->d_k;
    P.buf = bk->buf;
    P.n_b = beams->n_b; P.kdir = beams->kdir; P.freq = beams->freq; P.s0 = beams->s0;
    P.bgrad = beams->bgrad; P.pol = beams->pol; P.geff = beams->gamma_eff;
    P.hbar = hbar > 0 ? hbar : MM_HBAR_JIT;
    P.uniform_fb = uniform_fallback;
    P.v = v; P.z = z; P.F = F; P.R = R; P.status = status;
    P.valid = plan->d_valid;
    cudaStream_t st = (cudaStream_t)stream;
    // which molecules the reduction covers, then the reduced kernels, then the
    // elimination kernels for the rest (each pass draws from zeroed counters)
    uneven_valid_kernel<<<(plan->n_mol + 127) / 128, 128, 0, st>>>(P, plan->n_mol, plan->d_valid);
    if (mm_cuda_check(cudaGetLastError(), "uneven_valid_kernel launch")) return -3;
    if (mm_cuda_check(cudaMemsetAsync(plan->d_counter, 0, 3 * sizeof(int), st), "cudaMemsetAsync"))
        return -3;
    int rc = launch_class<UC2, true>(P, plan, 2, persistent, st);
    if (!rc) rc = launch_class<UC1, true>(P, plan, 1, persistent, st);
    if (!rc) rc = launch_class<UC0, true>(P, plan, 0, persistent, st);
    if (!rc && mm_cuda_check(cudaMemsetAsync(plan->d_counter, 0, 3 * sizeof(int), st), "cudaMemsetAsync"))
        return -3;
    if (!rc) rc = launch_class<UC2>(P, plan, 2, persistent, st);
    if (!rc) rc = launch_class<UC1>(P, plan, 1, persistent, st);
    if (!rc) rc = launch_class<UC0>(P, plan, 0, persistent, st);
    return rc;
}

// ---------------------------------------------------------------------------
// mm_uneven_force_static: mm_uneven_force without a plan and without any
// allocation.  The work list and the three work counters live in a fixed
// array in the module's device memory (one copy per GPU, held until the
// process exits); the host side stages the work list in fixed host arrays.
// Capacity: MM_STATIC_SCRATCH_BYTES = 1 MiB, i.e. kStaticMaxTasks = 43,680
// work items (each covers chunk_groups x groups-per-CTA points).
// Calls share that array and the host arrays.  Two calls race unless the
// second is ordered after the first on the GPU (the same stream, or a wait
// on an event recorded after the first call), and calls from two host
// threads race on the host arrays.
#define MM_STATIC_SCRATCH_BYTES (1u << 20)
static __device__ __align__(256) unsigned char g_uneven_scratch[MM_STATIC_SCRATCH_BYTES];

namespace {
constexpr size_t kScratchHead = 256;  // int counters[3] at offset 0, work list from here
constexpr int kStaticMaxTasks = (int)((MM_STATIC_SCRATCH_BYTES - kScratchHead) / sizeof(UnevenTask));
constexpr int kMaxDevices = 64;
UnevenTask h_st_tasks[kStaticMaxTasks];   // in creation order
UnevenTask h_st_sorted[kStaticMaxTasks];  // in launch order
double h_st_cost[kStaticMaxTasks];
int h_st_order[kStaticMaxTasks];
// Device address of g_uneven_scratch per device ordinal, with the id of the
// context it was looked up in: after cudaDeviceReset the module is loaded
// again in a new context, possibly at another address, so the address is
// looked up again whenever the current context is a different one.
struct ScratchAddr {
    unsigned long long ctx_id;
    void *ptr;
};
ScratchAddr g_scratch_dev[kMaxDevices];

// Id of the calling thread's current CUDA context (driver entry points
// cuCtxGetCurrent / cuCtxGetId, resolved through the runtime so the library
// does not link libcuda); 0 when no context is current.
int current_context_id(unsigned long long *id)
{
    typedef int (*GetCurrent)(void **);
    typedef int (*GetId)(void *, unsigned long long *);
    static GetCurrent get_current = nullptr;
    static GetId get_id = nullptr;
    if (!get_current || !get_id) {
        void *a = nullptr, *b = nullptr;
        cudaDriverEntryPointQueryResult qa, qb;
        if (mm_cuda_check(cudaGetDriverEntryPoint("cuCtxGetCurrent", &a, cudaEnableDefault, &qa),
                          "cudaGetDriverEntryPoint(cuCtxGetCurrent)") ||
            mm_cuda_check(cudaGetDriverEntryPoint("cuCtxGetId", &b, cudaEnableDefault, &qb),
                          "cudaGetDriverEntryPoint(cuCtxGetId)"))
            return -3;
        if (qa != cudaDriverEntryPointSuccess || qb != cudaDriverEntryPointSuccess || !a || !b) {
            mm_set_error("the driver does not provide cuCtxGetCurrent / cuCtxGetId");
            return -3;
        }
        get_current = (GetCurrent)a;
        get_id = (GetId)b;
    }
    void *ctx = nullptr;
    if (get_current(&ctx) != 0) { mm_set_error("cuCtxGetCurrent failed"); return -3; }
    *id = 0;
    if (ctx && get_id(ctx, id) != 0) { mm_set_error("cuCtxGetId failed"); return -3; }
    return 0;
}
}  // namespace

extern "C" int mm_uneven_force_static(const mm_bank *bank, const mm_beams *beams,
                                      const int64_t *point_offsets, const mm_uneven_opts *opts,
                                      const double *v, const double *z, double hbar,
                                      int32_t uniform_fallback, double *F, double *R,
                                      int32_t *status, void *stream)
{
    if (!bank || !beams || !point_offsets || !v || !z || !F) {
        mm_set_error("bank, beams, point_offsets, v, z and F are required");
        return -1;
    }
    const int n_mol = bank->n_mol;
    if (beams->n_sets != n_mol) {
        mm_set_error("beams must hold one parameter set per molecule (%d), got %d", n_mol, beams->n_sets);
        return -1;
    }
    if (point_offsets[0] != 0) { mm_set_error("point_offsets[0] must be 0"); return -1; }
    for (int m = 0; m < n_mol; m++)
        if (point_offsets[m + 1] < point_offsets[m]) { mm_set_error("point_offsets must not decrease"); return -1; }
    int dev = 0;
    if (mm_cuda_check(cudaGetDevice(&dev), "cudaGetDevice")) return -3;
    if (dev < 0 || dev >= kMaxDevices) { mm_set_error("device ordinal %d is above %d", dev, kMaxDevices - 1); return -1; }
    // set-up: the array's device address, looked up on the first call on this
    // device and again after a context reset (the host name of the array is
    // not a device address)
    unsigned long long ctx = 0;
    if (current_context_id(&ctx)) return -3;
    if (!g_scratch_dev[dev].ptr || ctx == 0 || ctx != g_scratch_dev[dev].ctx_id) {
        void *p = nullptr;
        if (mm_cuda_check(cudaGetSymbolAddress(&p, g_uneven_scratch), "cudaGetSymbolAddress")) return -3;
        if (current_context_id(&ctx)) return -3;  // the lookup makes the primary context current
        g_scratch_dev[dev].ptr = p;
        g_scratch_dev[dev].ctx_id = ctx;
    }
    mm_uneven_plan plan;  // a view of the fixed array; owns no memory
    plan.bank = bank;
    plan.n_mol = n_mol;
    plan.n_points = point_offsets[n_mol];
    const int G[3] = {16, 32, 32};
    long long chunk[3];
    const int chunk_groups = (opts && opts->chunk_groups > 0) ? opts->chunk_groups : 8;
    for (int c = 0; c < 3; c++) {
        int w = opts ? opts->warps_per_cta[c] : 0;
        if (w <= 0) w = c == 0 ? 4 : 2;
        if (w > 8) { mm_set_error("warps_per_cta must be <= 8"); return -1; }
        plan.wpc[c] = w;
        chunk[c] = (long long)(32 * w / G[c]) * chunk_groups;
    }
    long long n_items = 0;
    for (int m = 0; m < n_mol; m++) {
        const long long c = chunk[class_of(bank->ng[m], bank->ne[m])];
        n_items += (point_offsets[m + 1] - point_offsets[m] + c - 1) / c;
    }
    if (n_items > kStaticMaxTasks) {
        mm_set_error("mm_uneven_force_static: the batch makes %lld work items, above the %d that fit "
                     "its fixed %u-byte scratch; raise chunk_groups, split the batch, or use "
                     "mm_uneven_force", n_items, kStaticMaxTasks, (unsigned)MM_STATIC_SCRATCH_BYTES);
        return -1;
    }
    if (plan.n_points == 0) return 0;
    // work items of each class, largest cost first (ties in creation order, as
    // the plan's stable sort); std::sort works in place
    int base = 0;
    for (int c = 0; c < 3; c++) {
        int n = 0;
        for (int m = 0; m < n_mol; m++) {
            if (class_of(bank->ng[m], bank->ne[m]) != c) continue;
            const double cost = (double)bank->ng[m] * bank->ng[m] * bank->ng[m] +
                                8.0 * bank->ng[m] * bank->ne[m] * 8;
            for (long long a = point_offsets[m]; a < point_offsets[m + 1]; a += chunk[c]) {
                UnevenTask &t = h_st_tasks[base + n];
                t.mol = m; t.pad = 0; t.p0 = a;
                t.p1 = std::min<long long>(a + chunk[c], point_offsets[m + 1]);
                h_st_cost[base + n] = cost * (double)(t.p1 - t.p0);
                h_st_order[base + n] = base + n;
                n++;
            }
        }
        std::sort(h_st_order + base, h_st_order + base + n, [](int a, int b) {
            return h_st_cost[a] > h_st_cost[b] || (h_st_cost[a] == h_st_cost[b] && a < b);
        });
        for (int i = base; i < base + n; i++) h_st_sorted[i] = h_st_tasks[h_st_order[i]];
        plan.n_tasks[c] = n;
        base += n;
    }
    unsigned char *scr = (unsigned char *)g_scratch_dev[dev].ptr;
    UnevenTask *d_tasks = (UnevenTask *)(scr + kScratchHead);
    for (int c = 0, b = 0; c < 3; b += plan.n_tasks[c], c++) plan.d_tasks[c] = d_tasks + b;
    plan.d_counter = (int *)scr;
    cudaStream_t st = (cudaStream_t)stream;
    // the host arrays are pageable: the copy has taken them before it returns
    if (mm_cuda_check(cudaMemcpyAsync(d_tasks, h_st_sorted, sizeof(UnevenTask) * base,
                                      cudaMemcpyHostToDevice, st), "cudaMemcpyAsync"))
        return -3;
    // the work counters must start at zero on every call
    if (mm_cuda_check(cudaMemsetAsync(plan.d_counter, 0, 3 * sizeof(int), st), "cudaMemsetAsync"))
        return -3;
    UnevenParams P;
    P.ng = bank->d_ng; P.ne = bank->d_ne; P.off = bank->d_off; P.gam = bank->d_gam; P.kw = bank->d_k;
    P.buf = bank->buf;
    P.n_b = beams->n_b; P.kdir = beams->kdir; P.freq = beams->freq; P.s0 = beams->s0;
    P.bgrad = beams->bgrad; P.pol = beams->pol; P.geff = beams->gamma_eff;
    P.hbar = hbar > 0 ? hbar : MM_HBAR_JIT;
    P.uniform_fb = uniform_fallback;
    P.v = v; P.z = z; P.F = F; P.R = R; P.status = status;
    P.valid = nullptr;  // the elimination kernels take every molecule
    int rc = launch_class<UC2>(P, &plan, 2, 1, st);
    if (!rc) rc = launch_class<UC1>(P, &plan, 1, 1, st);
    if (!rc) rc = launch_class<UC0>(P, &plan, 0, 1, st);
    return rc;
}
