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
#include "rate_core.cuh"

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

constexpr int NBU = MM_MAX_BEAMS;

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
    static constexpr int LDA = NGMAX + 1;
    static constexpr int LDK = NEMAX + 1;
    // row stride of the rates Rm[g][e]: lanes own consecutive ground states,
    // so an odd stride keeps their row accesses in distinct banks
    static constexpr int LDR = NEMAX + 1;
    // per CTA
    static constexpr int mol_doubles = 2 * (NGMAX + NEMAX) + NGMAX * NEMAX * 3 + NEMAX * NGMAX + NGMAX;
    static constexpr int beam_doubles = 5 * NBU;
    // per group
    // elimination: A, Rm, bv, xv, invU, Fk, Rk, Esg, fd, Ese
    // reduced:     Rm (scaled rates), K, Fk, Rk, Esg, w, phi, fd, Ese, cw, cf, rs, pi
    static constexpr int grp_raw = RED ? NGMAX * LDR + NEMAX * LDK + 5 * NGMAX + NBU + 5 * NEMAX
                                       : NGMAX * LDA + NGMAX * LDR + 6 * NGMAX + NBU + NEMAX;
    // two 16-lane groups of a warp read the same offsets of their own region:
    // a stride of 16 banks past a multiple of 128 bytes keeps those reads
    // conflict-free (a multiple of 128 bytes would put both in the same banks)
    static constexpr int grp_doubles = (grp_raw + 15) / 16 * 16 + 8;
    static size_t bytes(int groups)
    {
        return sizeof(double) * (size_t)(mol_doubles + beam_doubles + groups * grp_doubles) +
               sizeof(int) * (NBU + 8);
    }
};

__device__ __forceinline__ double gsum(double x, int G)
{
    for (int o = G >> 1; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    return x;
}

// RED: the populations from the excited-state chain (see reduced.cuh for the
// identity): each group scales its rates by 1/r_g, forms K = A^T BR^T
// (n_e x n_e) and the two n_e-vectors in shared memory, reduces the chain
// cooperatively and writes F and R.  Molecules the reduction does not cover
// (valid[m] = 0) are left to the elimination kernels (RED = false).
template <int NGMAX, int NEMAX, int G, bool RED>
__global__ void __launch_bounds__(256)
uneven_kernel(UnevenParams P)
{
    using Ly = ULayout<NGMAX, NEMAX, RED>;
    constexpr int LDA = Ly::LDA, LDK = Ly::LDK, LDR = Ly::LDR;
    extern __shared__ __align__(16) unsigned char smraw[];
    double *smd = (double *)smraw;
    // molecule
    double *E = smd, *zd = E + NGMAX + NEMAX, *d2s = zd + NGMAX + NEMAX;
    double *BR = d2s + NGMAX * NEMAX * 3, *czd = BR + NEMAX * NGMAX;
    // beams
    double *freq = czd + NGMAX, *ck = freq + NBU, *hk = ck + NBU, *s0 = hk + NBU, *c1 = s0 + NBU;
    const int groups = blockDim.x / G;
    double *grp0 = c1 + NBU;
    int *pol = (int *)(grp0 + (size_t)groups * Ly::grp_doubles);
    int *sint = pol + NBU;  // [0] task, [1] n_g, [2] n_e

    const int lane = threadIdx.x & 31, t = lane % G;
    const int group = threadIdx.x / G;
    double *W = grp0 + (size_t)group * Ly::grp_doubles;
    double *A, *Rm, *bv, *xv, *invU, *Fk, *Rk, *Esg, *fd, *Ese;
    double *Kc = nullptr, *wg = nullptr, *ph = nullptr, *cw = nullptr, *cf = nullptr, *rsv = nullptr,
           *piv = nullptr;
    if constexpr (RED) {
        Rm = W; Kc = Rm + NGMAX * LDR; Fk = Kc + NEMAX * LDK; Rk = Fk + NGMAX; Esg = Rk + NGMAX;
        wg = Esg + NGMAX; ph = wg + NGMAX; fd = ph + NGMAX; Ese = fd + NBU;
        cw = Ese + NEMAX; cf = cw + NEMAX; rsv = cf + NEMAX; piv = rsv + NEMAX;
        A = bv = xv = invU = nullptr;
    } else {
        A = W; Rm = A + NGMAX * LDA; bv = Rm + NGMAX * LDR; xv = bv + NGMAX;
        invU = xv + NGMAX; Fk = invU + NGMAX; Rk = Fk + NGMAX; Esg = Rk + NGMAX;
        fd = Esg + NGMAX; Ese = fd + NBU;
    }
    const int n_b = P.n_b;

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
        const int n_g = P.ng[m], n_e = P.ne[m], n_s = n_g + n_e;
        const double Gam = P.gam[m], kw = P.kw[m];
        const double *mb = P.buf + P.off[m];
        for (int i = threadIdx.x; i < n_s; i += blockDim.x) { E[i] = mb[i]; zd[i] = mb[n_s + i]; }
        // |d|^2 transposed to [e][q][g]: the lanes of a group own consecutive
        // ground states, so their reads of one (e, q) are consecutive doubles
        for (int i = threadIdx.x; i < n_g * n_e * 3; i += blockDim.x) {
            const int k = i / (n_e * 3), r = i - k * (n_e * 3);
            d2s[r * NGMAX + k] = mb[2 * n_s + i];  // r = e * 3 + q
        }
        // branching ratios transposed to [g][e]: the chain build's lanes read
        // consecutive excited states of one ground state
        for (int i = threadIdx.x; i < n_e * n_g; i += blockDim.x) {
            const int e = i / n_g, g = i - e * n_g;
            BR[g * NEMAX + e] = mb[2 * n_s + n_g * n_e * 3 + i];
        }
        for (int i = threadIdx.x; i < n_g; i += blockDim.x) czd[i] = mb[n_s + i] * Gam / MM_TWO_PI;
        const double gh = Gam / 2.0, gh2 = gh * gh;
        for (int b = threadIdx.x; b < n_b; b += blockDim.x) {
            const size_t o = (size_t)m * n_b + b;
            freq[b] = P.freq[o];
            ck[b] = __dmul_rn(-kw, P.kdir[o]);
            hk[b] = __dmul_rn(__dmul_rn(P.hbar, kw), P.kdir[o]);
            s0[b] = P.s0[o];
            c1[b] = __dmul_rn(gh, P.s0[o]);
            pol[b] = P.pol[o];
        }
        __syncthreads();
        const double Bg = P.bgrad[m];

        for (long long base = T.p0; base < T.p1; base += groups) {
            const long long ip = base + group;
            const bool valid = ip < T.p1;
            const long long gi = valid ? ip : T.p0;
            const double v = P.v[gi], z = P.z[gi];
            int stat = 0;
            const double B = __dmul_rn(__dmul_rn(Bg, z), 1e4);
            __syncwarp();
            for (int b = t; b < n_b; b += G)
                fd[b] = __dadd_rn(freq[b], __ddiv_rn(__dmul_rn(ck[b], v), MM_TWO_PI));
            for (int e = t; e < n_e; e += G)
                Ese[e] = __dadd_rn(E[n_g + e], __ddiv_rn(__dmul_rn(__dmul_rn(B, zd[n_g + e]), Gam), MM_TWO_PI));
            for (int k = t; k < n_g; k += G) Esg[k] = fma(B, czd[k], E[k]);
            __syncwarp();
            // rates of ground states k = t, t + G, ... (rows of Rm owned by this lane)
            for (int k = t; k < n_g; k += G) {
                double s = 0.0, f = 0.0;
                double Racc[NEMAX];  // per excited state, in registers (compile-time index)
#pragma unroll
                for (int e = 0; e < NEMAX; e++) Racc[e] = 0.0;
                const double Eg = Esg[k];
                for (int b = 0; b < n_b; b++) {
                    const int q = pol[b];
                    const double fdb = fd[b], c1b = c1[b], hkb = hk[b], s0b = s0[b];
#pragma unroll
                    for (int e = 0; e < NEMAX; e++) {
                        if (e >= n_e) break;
                        const double d2 = d2s[(e * 3 + q) * NGMAX + k];
                        if (d2 < 1e-15) continue;
                        const double om = __dsub_rn(Ese[e], Eg);
                        const double de = __dmul_rn(__dsub_rn(fdb, om), MM_TWO_PI);
                        const double L = gh2 * mm_rcp(fma(de, de, gh2));
                        const double ru = c1b * d2 * P.geff * L;
                        Racc[e] += ru;
                        f = fma(hkb, ru, f);
                        s = fma(s0b * d2, L, s);
                    }
                }
                const double sat = mm_rcp(1.0 + s);
                double rs = 0.0;
#pragma unroll
                for (int e = 0; e < NEMAX; e++) {
                    if (e < n_e) {
                        const double r = Racc[e] * sat;
                        Rm[k * LDR + e] = r;
                        rs += r;
                    }
                }
                Fk[k] = f * sat;
                Rk[k] = rs;
            }
            __syncwarp();
            if constexpr (RED) {
                // a_ge = R[g,e] / r_g, w_g = 1 / r_g, phi_g = F_g / r_g (lane per ground state)
                for (int k = t; k < n_g; k += G) {
                    const double inv = mm_rcp(Rk[k]);  // r_g > 0: every ground state is pumped
                    for (int e = 0; e < n_e; e++) Rm[k * LDR + e] *= inv;
                    wg[k] = inv;
                    ph[k] = Fk[k] * inv;
                }
                __syncwarp();
                // K[e][e'] = sum_g a_ge BR[e', g]; cw, cf, rs: sums of BR[e', g] w_g, phi_g, 1
                for (int idx = t; idx < n_e * n_e; idx += G) {
                    const int e = idx / n_e, e2 = idx - e * n_e;
                    double a = 0.0;
                    for (int g = 0; g < n_g; g++) a = fma(Rm[g * LDR + e], BR[g * NEMAX + e2], a);
                    Kc[e * LDK + e2] = a;
                }
                for (int e2 = t; e2 < n_e; e2 += G) {
                    double a = 0.0, b = 0.0, c = 0.0;
                    for (int g = 0; g < n_g; g++) {
                        const double br = BR[g * NEMAX + e2];
                        a = fma(br, wg[g], a);
                        b = fma(br, ph[g], b);
                        c += br;
                    }
                    cw[e2] = a;
                    cf[e2] = b;
                    rsv[e2] = c;
                }
                __syncwarp();
                // state reduction of the chain, Q[i][j] = K[j][i] (probability i -> j)
                bool ok = true;
                for (int k = n_e - 1; k >= 1; k--) {
                    double S = 0.0;
                    for (int j = 0; j < k; j++) S += Kc[j * LDK + k];
                    ok = ok && (S > 0.0);
                    const double inv = mm_rcp(S > 0.0 ? S : 1.0);
                    __syncwarp();
                    for (int i = t; i < k; i += G) Kc[k * LDK + i] *= inv;
                    __syncwarp();
                    for (int idx = t; idx < k * k; idx += G) {
                        const int i = idx / k, j = idx - i * k;
                        Kc[j * LDK + i] = fma(Kc[k * LDK + i], Kc[j * LDK + k], Kc[j * LDK + i]);
                    }
                    __syncwarp();
                }
                double nrm = 0.0, fn = 0.0, rn = 0.0;
                if (t == 0) {
                    piv[0] = 1.0;
                    for (int k = 1; k < n_e; k++) {
                        double a = 0.0;
                        for (int i = 0; i < k; i++) a = fma(piv[i], Kc[k * LDK + i], a);
                        piv[k] = a;
                    }
                    for (int e = 0; e < n_e; e++) {
                        nrm = fma(cw[e], piv[e], nrm);
                        fn = fma(cf[e], piv[e], fn);
                        rn = fma(rsv[e], piv[e], rn);
                    }
                    const double in = mm_rcp(nrm);
                    const double Fo = fn * in, Ro = rn * in;
                    int st = 0;
                    if (!ok || !isfinite(Fo)) st |= MM_ST_NONFINITE;
                    if (valid) {
                        P.F[gi] = Fo;
                        if (P.R) P.R[gi] = Ro;
                        if (P.status) P.status[gi] = st;
                    }
                }
                __syncwarp();
            } else {
                // population matrix M' (rows i, columns j), right-hand side e_last
                for (int i = 0; i < n_g; i++) {
                    for (int j = t; j < n_g; j += G) {
                        double a = (i == j) ? -Rk[j] : 0.0;
                        for (int e = 0; e < n_e; e++) a = fma(Rm[j * LDR + e], BR[i * NEMAX + e], a);
                        A[i * LDA + j] = (i == n_g - 1) ? 1.0 : a;
                    }
                }
                for (int i = t; i < n_g; i += G) bv[i] = (i == n_g - 1) ? 1.0 : 0.0;
                __syncwarp();
                // elimination with partial pivoting
                for (int col = 0; col < n_g; col++) {
                    double best = -1.0;
                    int brow = n_g;
                    for (int r = col + t; r < n_g; r += G) {
                        const double a = fabs(A[r * LDA + col]);
                        if (a > best) { best = a; brow = r; }
                    }
                    for (int o = G >> 1; o > 0; o >>= 1) {
                        const double ob = __shfl_xor_sync(0xffffffffu, best, o);
                        const int orow = __shfl_xor_sync(0xffffffffu, brow, o);
                        if (ob > best || (ob == best && orow < brow)) { best = ob; brow = orow; }
                    }
                    const int prow = brow;
                    if (prow != col) {
                        for (int j = t; j < n_g; j += G) {
                            const double tmp = A[col * LDA + j];
                            A[col * LDA + j] = A[prow * LDA + j];
                            A[prow * LDA + j] = tmp;
                        }
                        if (t == 0) { const double tb = bv[col]; bv[col] = bv[prow]; bv[prow] = tb; }
                    }
                    __syncwarp();
                    const double pv = A[col * LDA + col];
                    const double ap = fabs(pv);
                    const double y = mm_rcp(ap >= 1e-30 ? pv : 1.0);
                    const double inv_e = (ap < 1e-30) ? 0.0 : y;
                    if (ap < 1e-30) stat |= MM_ST_PIVOT;
                    if (t == 0) invU[col] = (ap > 1e-30) ? y : 0.0;
                    for (int r = col + 1 + t; r < n_g; r += G) A[r * LDA + col] *= inv_e;
                    __syncwarp();
                    for (int r = col + 1; r < n_g; r++) {
                        const double f = A[r * LDA + col];
                        for (int j = col + 1 + t; j < n_g; j += G)
                            A[r * LDA + j] = fma(-f, A[col * LDA + j], A[r * LDA + j]);
                    }
                    for (int r = col + 1 + t; r < n_g; r += G)
                        bv[r] = fma(-A[r * LDA + col], bv[col], bv[r]);
                    __syncwarp();
                }
                // back substitution
                for (int i = n_g - 1; i >= 0; i--) {
                    double part = 0.0;
                    for (int j = i + 1 + t; j < n_g; j += G) part = fma(A[i * LDA + j], xv[j], part);
                    part = gsum(part, G);
                    const double xi = (bv[i] - part) * invU[i];
                    __syncwarp();
                    if (t == 0) xv[i] = xi;
                    __syncwarp();
                }
                // clamp, normalise, force
                double tot = 0.0, Fs = 0.0, Rs = 0.0;
                for (int i = t; i < n_g; i += G) {
                    const double p = xv[i] > 0.0 ? xv[i] : 0.0;
                    tot += p;
                    Fs = fma(p, Fk[i], Fs);
                    Rs = fma(p, Rk[i], Rs);
                }
                // uniform-population sums, reduced outside the branch (both 16-lane groups
                // of a warp take every shuffle)
                double fu = 0.0, ru = 0.0;
                for (int i = t; i < n_g; i += G) { fu += Fk[i]; ru += Rk[i]; }
                tot = gsum(tot, G);
                Fs = gsum(Fs, G);
                Rs = gsum(Rs, G);
                fu = gsum(fu, G);
                ru = gsum(ru, G);
                double Fo, Ro;
                if (tot > 0.0) {
                    const double it = mm_rcp(tot);
                    Fo = Fs * it;
                    Ro = Rs * it;
                } else {
                    stat |= MM_ST_ZERO_POP;
                    Fo = P.uniform_fb ? fu / n_g : 0.0;
                    Ro = P.uniform_fb ? ru / n_g : 0.0;
                }
                if (!isfinite(Fo)) stat |= MM_ST_NONFINITE;
                for (int o = G >> 1; o > 0; o >>= 1) stat |= __shfl_xor_sync(0xffffffffu, stat, o);
                if (valid && t == 0) {
                    P.F[gi] = Fo;
                    if (P.R) P.R[gi] = Ro;
                    if (P.status) P.status[gi] = stat;
                }
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
