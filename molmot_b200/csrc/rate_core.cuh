// rate_core.cuh -- the steady-state rate-equation solve for one point,
// executed cooperatively by a group of G consecutive lanes (sm_100a).
//
// Algorithm (molmot/obe/rate_equations_jit.py:18-145, the numba core):
//   Es[i]   = E[i] + B*zd[i]*Gamma/(2 pi),  B = B'*z*1e4 (Gauss)
//   delta   = (freq_b + doppler_b - (Es[e] - Es[g])) * 2 pi
//   L       = (Gamma/2)^2 / (delta^2 + (Gamma/2)^2)
//   R[g,e] += (Gamma/2) s0 d2 L Geff,  s[g] += s0 d2 L,  F[g] += hbar k kdir rate
//   R, F   *= 1/(1+s[g])
//   M[g,k]  = sum_e R[k,e] BR[e,g] - delta_gk sum_e R[g,e];  last row := 1
//   solve M p = e_last by Gaussian elimination with partial pivoting,
//   clamp p >= 0, normalise, F = sum p F, R = sum p R.
//
// Work split inside a group: lane t owns ground states k = c*G + t
// (slot c = 0 .. CPL-1): it computes their rates and holds column k of the
// augmented matrix [M | b] in registers (b is column NGMAX, owned by lane
// NGMAX % G).  Pivot search is lane-local (the owner of the pivot column);
// the pivot row and the elimination factors are broadcast with shuffles.
// Row swaps are predicated register moves, taken only when some group of
// the warp pivots (warp-uniform branch).
//
// Exactness: the detuning chain (Es, doppler, omega, delta) and the
// Lorentzian use the reference's operations in its order with explicit
// round-to-nearest intrinsics (no FMA contraction), because E_e ~ 4.3e14 Hz
// makes delta a difference of nearly equal numbers.  Reductions, the matrix
// build and the elimination use FMA; they agree with the reference to
// rounding (about 1e-15 of max|F|).
#pragma once
#include "common.cuh"
#include <type_traits>

// Compile-time loop: f(std::integral_constant<int, I>) for I in [B, E).  Keeps
// every register-array index a constant so the matrix stays in registers.
template <int B, int E, class Fn>
__device__ __forceinline__ void static_for(Fn &&f)
{
    if constexpr (B < E) {
        f(std::integral_constant<int, B>{});
        static_for<B + 1, E>(f);
    }
}

// Active (ground k, beam b, excited e) triple of one parameter set.
struct Trip64 {
    double c1;  // (Gamma/2 * s0_b) * d2       -> rate = (c1 * L) * Geff
    double c2;  // s0_b * d2                   -> saturation term c2 * L
    int b, e;
};
struct Trip32 {
    float d0;   // freq_b - (E_e - E_g), FP64 then rounded         (Hz)
    float dzd;  // (zd_e - zd_g) * Gamma / (2 pi)                   (Hz per G)
    float c1;   // (Gamma/2) s0 d2 Geff
    float c2;   // s0 d2
    int b, e;
};

// Shared-memory view of one parameter set's tables.
struct SetView {
    const double *E, *zd, *BR;
    const double *freq, *ck, *hk;   // per beam: freq, (-k)*kdir, (hbar*k)*kdir
    const float *kdf, *hkf;         // per beam (FP32 form): (-k kdir)/(2 pi), hbar k kdir
    const int *cnt, *off, *maxcnt;  // per ground state / per slot
    const Trip64 *t64;
    const Trip32 *t32;
};

// Byte layout of the dynamic shared memory of the 1D force kernels.
struct SmemLayout {
    size_t E, zd, BR, freq, ck, hk, kdf, hkf, cnt, off, maxcnt, trip, scratch, total;
    int ntrip_max, scratch_per_group;  // doubles per group

    __host__ __device__ static size_t al(size_t x) { return (x + 15) & ~size_t(15); }

    __host__ __device__ void build(int n_g, int n_e, int n_b, int cpl, int ngroups, bool fp32)
    {
        const int n_s = n_g + n_e;
        size_t o = 0;
        E = o;   o = al(o + sizeof(double) * n_s);
        zd = o;  o = al(o + sizeof(double) * n_s);
        BR = o;  o = al(o + sizeof(double) * n_e * n_g);
        freq = o; o = al(o + sizeof(double) * n_b);
        ck = o;  o = al(o + sizeof(double) * n_b);
        hk = o;  o = al(o + sizeof(double) * n_b);
        kdf = o; o = al(o + sizeof(float) * n_b);
        hkf = o; o = al(o + sizeof(float) * n_b);
        cnt = o; o = al(o + sizeof(int) * n_g);
        off = o; o = al(o + sizeof(int) * n_g);
        maxcnt = o; o = al(o + sizeof(int) * cpl);
        ntrip_max = n_g * n_b * n_e;
        trip = o; o = al(o + (fp32 ? sizeof(Trip32) : sizeof(Trip64)) * (size_t)ntrip_max);
        scratch_per_group = n_b + n_e;
        scratch = o; o = al(o + sizeof(double) * (size_t)scratch_per_group * ngroups);
        total = o;
    }
};

// Build the parameter-set tables (all threads of the CTA participate).
template <int G, int CPL, bool FP32>
__device__ void build_set_tables(const ForceParams &P, int set, unsigned char *sm,
                                 const SmemLayout &Ly, SetView &S)
{
    const int n_g = P.n_g, n_e = P.n_e, n_b = P.n_b, n_s = n_g + n_e;
    double *E = (double *)(sm + Ly.E), *zd = (double *)(sm + Ly.zd), *BR = (double *)(sm + Ly.BR);
    double *freq = (double *)(sm + Ly.freq), *ck = (double *)(sm + Ly.ck), *hk = (double *)(sm + Ly.hk);
    float *kdf = (float *)(sm + Ly.kdf), *hkf = (float *)(sm + Ly.hkf);
    int *cnt = (int *)(sm + Ly.cnt), *off = (int *)(sm + Ly.off), *maxcnt = (int *)(sm + Ly.maxcnt);
    Trip64 *t64 = (Trip64 *)(sm + Ly.trip);
    Trip32 *t32 = (Trip32 *)(sm + Ly.trip);
    const int tid = threadIdx.x, nt = blockDim.x;
    const double *kdir = P.kdir + (size_t)set * n_b, *fr = P.freq + (size_t)set * n_b;
    const double *s0 = P.s0 + (size_t)set * n_b;
    const int32_t *pol = P.pol + (size_t)set * n_b;

    for (int i = tid; i < n_s; i += nt) { E[i] = P.E[i]; zd[i] = P.zd[i]; }
    for (int i = tid; i < n_e * n_g; i += nt) BR[i] = P.BR[i];
    for (int b = tid; b < n_b; b += nt) {
        freq[b] = fr[b];
        ck[b] = __dmul_rn(-P.k, kdir[b]);                       // -k_wave * kdir
        hk[b] = __dmul_rn(__dmul_rn(P.hbar, P.k), kdir[b]);     // hbar * k_wave * kdir
        kdf[b] = (float)__ddiv_rn(ck[b], MM_TWO_PI);
        hkf[b] = (float)hk[b];
    }
    // count active triples per ground state (d2 >= 1e-15, rate_equations_jit.py:67-69)
    for (int k = tid; k < n_g; k += nt) {
        int c = 0;
        for (int b = 0; b < n_b; b++)
            for (int e = 0; e < n_e; e++)
                if (P.d2[(k * n_e + e) * 3 + pol[b]] >= 1e-15) c++;
        cnt[k] = c;
    }
    __syncthreads();
    if (tid == 0) {
        int o = 0;
        for (int k = 0; k < n_g; k++) { off[k] = o; o += cnt[k]; }
        for (int c = 0; c < CPL; c++) {
            int m = 0;
            for (int t = 0; t < G; t++) {
                const int k = c * G + t;
                if (k < n_g && cnt[k] > m) m = cnt[k];
            }
            maxcnt[c] = m;
        }
    }
    __syncthreads();
    const double gh = P.Gamma / 2.0;
    for (int k = tid; k < n_g; k += nt) {
        int o = off[k];
        // order (b ascending, e ascending) = the reference's accumulation order
        for (int b = 0; b < n_b; b++)
            for (int e = 0; e < n_e; e++) {
                const double d2 = P.d2[(k * n_e + e) * 3 + pol[b]];
                if (d2 < 1e-15) continue;
                if (!FP32) {
                    Trip64 tr;
                    tr.c1 = __dmul_rn(__dmul_rn(gh, s0[b]), d2);
                    tr.c2 = __dmul_rn(s0[b], d2);
                    tr.b = b; tr.e = e;
                    t64[o++] = tr;
                } else {
                    Trip32 tr;
                    tr.d0 = (float)(fr[b] - (P.E[n_g + e] - P.E[k]));
                    tr.dzd = (float)((P.zd[n_g + e] - P.zd[k]) * P.Gamma / MM_TWO_PI);
                    tr.c1 = (float)(gh * s0[b] * d2 * P.geff);
                    tr.c2 = (float)(s0[b] * d2);
                    tr.b = b; tr.e = e;
                    t32[o++] = tr;
                }
            }
    }
    __syncthreads();
    S.E = E; S.zd = zd; S.BR = BR; S.freq = freq; S.ck = ck; S.hk = hk; S.kdf = kdf; S.hkf = hkf;
    S.cnt = cnt; S.off = off; S.maxcnt = maxcnt; S.t64 = t64; S.t32 = t32;
}

// Result of one point, replicated in every lane of the group except xs.
struct PointOut {
    double F, R;
    int status;
};

template <int NGMAX, int NEMAX, int G>
struct GroupShape {
    static constexpr int AUGS = NGMAX / G;  // slot of the augmented column
    static constexpr int AUGL = NGMAX % G;  // lane of the augmented column
    static constexpr int CPL = AUGS + 1;    // slots per lane
};

// Solve one point.  xs[c] receives p[c*G + t] for the owned columns.
// fd / Ese: this group's scratch (n_b + n_e doubles) in shared memory.
template <int NGMAX, int NEMAX, int G, bool FP32>
__device__ __forceinline__ PointOut solve_point(const ForceParams &P, const SetView &S, double *fd,
                                                double *Ese, int t, int gbase, double v, double z,
                                                double Bgrad,
                                                double (&xs)[GroupShape<NGMAX, NEMAX, G>::CPL])
{
    using GS = GroupShape<NGMAX, NEMAX, G>;
    constexpr int CPL = GS::CPL, AUGS = GS::AUGS, AUGL = GS::AUGL;
    constexpr unsigned FULL = 0xffffffffu;
    const int n_g = P.n_g, n_e = P.n_e, n_b = P.n_b;
    const double Gam = P.Gamma;
    const double gh = Gam / 2.0;
    const double gh2 = gh * gh;
    int stat = 0;

    // ---------------- rates of the owned ground states ----------------
    double R[CPL][NEMAX];
    double Fk[CPL], Rk[CPL];
#pragma unroll
    for (int c = 0; c < CPL; c++) {
        Fk[c] = 0.0; Rk[c] = 0.0;
#pragma unroll
        for (int e = 0; e < NEMAX; e++) R[c][e] = 0.0;
    }
    const double B_gauss = __dmul_rn(__dmul_rn(Bgrad, z), 1e4);
    __syncwarp();
    if (!FP32) {
        // per-beam laser frequency seen by the moving molecule, per-excited Es
        for (int b = t; b < n_b; b += G)
            fd[b] = __dadd_rn(S.freq[b], __ddiv_rn(__dmul_rn(S.ck[b], v), MM_TWO_PI));
        for (int e = t; e < n_e; e += G)
            Ese[e] = __dadd_rn(S.E[n_g + e],
                               __ddiv_rn(__dmul_rn(__dmul_rn(B_gauss, S.zd[n_g + e]), Gam), MM_TWO_PI));
        __syncwarp();
#pragma unroll
        for (int c = 0; c < CPL; c++) {
            if (c * G >= NGMAX) continue;  // slot holds no ground state for any lane
            const int k = c * G + t;
            const bool own = k < n_g;
            const int kk = own ? k : 0;
            const double Esg = __dadd_rn(S.E[kk], __ddiv_rn(__dmul_rn(__dmul_rn(B_gauss, S.zd[kk]), Gam),
                                                         MM_TWO_PI));
            const int cntk = own ? S.cnt[kk] : 0;
            const int o = S.off[kk];
            double s = 0.0, f = 0.0;
            const int mc = S.maxcnt[c];
            for (int i = 0; i < mc; i++) {
                if (i < cntk) {
                    const Trip64 tr = S.t64[o + i];
                    const double om = __dsub_rn(Ese[tr.e], Esg);
                    const double de = __dmul_rn(__dsub_rn(fd[tr.b], om), MM_TWO_PI);
                    const double L = __ddiv_rn(gh2, __dadd_rn(__dmul_rn(de, de), gh2));
                    const double ru = __dmul_rn(__dmul_rn(tr.c1, L), P.geff);
#pragma unroll
                    for (int e = 0; e < NEMAX; e++)
                        if (e == tr.e) R[c][e] = __dadd_rn(R[c][e], ru);
                    f = fma(S.hk[tr.b], ru, f);
                    s = __dadd_rn(s, __dmul_rn(tr.c2, L));
                }
            }
            // saturation correction 1/(1 + s_total[g]) (rate_equations_jit.py:85-90)
            const double sat = __ddiv_rn(1.0, __dadd_rn(1.0, s));
            double rs = 0.0;
#pragma unroll
            for (int e = 0; e < NEMAX; e++) {
                R[c][e] = __dmul_rn(R[c][e], sat);
                rs = __dadd_rn(rs, R[c][e]);
            }
            Rk[c] = rs;
            Fk[c] = f * sat;
        }
    } else {
        // FP32 bulk: delta/2pi = d0 + v kdf_b - B dzd, all in FP32 (d0 from FP64)
        const float Bf = (float)B_gauss, vf = (float)v;
        const float gh2f = (float)gh2;
        const float twopif = 6.2831855f;
#pragma unroll
        for (int c = 0; c < CPL; c++) {
            if (c * G >= NGMAX) continue;
            const int k = c * G + t;
            const bool own = k < n_g;
            const int kk = own ? k : 0;
            const int cntk = own ? S.cnt[kk] : 0;
            const int o = S.off[kk];
            float s = 0.f, f = 0.f;
            float Rf[NEMAX];
#pragma unroll
            for (int e = 0; e < NEMAX; e++) Rf[e] = 0.f;
            const int mc = S.maxcnt[c];
            for (int i = 0; i < mc; i++) {
                if (i < cntk) {
                    const Trip32 tr = S.t32[o + i];
                    float x = fmaf(S.kdf[tr.b], vf, tr.d0);
                    x = fmaf(-Bf, tr.dzd, x);
                    const float de = x * twopif;
                    const float L = __fdividef(gh2f, fmaf(de, de, gh2f));
                    const float ru = tr.c1 * L;
#pragma unroll
                    for (int e = 0; e < NEMAX; e++)
                        if (e == tr.e) Rf[e] += ru;
                    f = fmaf(S.hkf[tr.b], ru, f);
                    s = fmaf(tr.c2, L, s);
                }
            }
            const float sat = 1.0f / (1.0f + s);
            double rs = 0.0;
#pragma unroll
            for (int e = 0; e < NEMAX; e++) {
                R[c][e] = (double)(Rf[e] * sat);
                rs += R[c][e];
            }
            Rk[c] = rs;
            Fk[c] = (double)(f * sat);
        }
    }

    // ---------------- columns of [M' | b] ----------------
    double A[CPL][NGMAX];
#pragma unroll
    for (int c = 0; c < CPL; c++) {
        const int j = c * G + t;
#pragma unroll
        for (int r = 0; r < NGMAX; r++) {
            double a = 0.0;
            if (c * G < NGMAX && j < n_g) {
                if (r < n_g) {
                    a = (r == j) ? -Rk[c] : 0.0;
#pragma unroll
                    for (int e = 0; e < NEMAX; e++)
                        if (e < n_e) a = fma(R[c][e], S.BR[e * n_g + r], a);
                    if (r == n_g - 1) a = 1.0;  // normalisation row
                }
            } else if (j < NGMAX) {
                a = (r == j) ? 1.0 : 0.0;       // identity padding beyond n_g
            } else if (j == NGMAX) {
                a = (r == n_g - 1) ? 1.0 : 0.0; // right-hand side e_last
            }
            A[c][r] = a;
        }
    }

    // ---------------- LU with partial pivoting ----------------
    int prows[NGMAX];
    bool swapped = false;
    static_for<0, NGMAX>([&](auto colc) {
        constexpr int col = decltype(colc)::value;
        prows[col] = col;
        if (col < n_g) {
            constexpr int own = col % G, lc = col / G;
            int prow = col;
            if (t == own) {
                double mx = fabs(A[lc][col]);
#pragma unroll
                for (int r = col + 1; r < NGMAX; r++) {
                    if (r < n_g) {
                        const double av = fabs(A[lc][r]);
                        if (av > mx) { mx = av; prow = r; }
                    }
                }
            }
            prow = __shfl_sync(FULL, prow, gbase + own);
            prows[col] = prow;
            if (__any_sync(FULL, prow != col)) {
                swapped = true;
#pragma unroll
                for (int c = 0; c < CPL; c++)
#pragma unroll
                    for (int r = col + 1; r < NGMAX; r++)
                        if (r == prow) { const double tmp = A[c][col]; A[c][col] = A[c][r]; A[c][r] = tmp; }
            }
            double inv = 0.0;
            if (t == own) {
                const double pv = A[lc][col];
                if (fabs(pv) < 1e-30) stat |= MM_ST_PIVOT;
                else inv = 1.0 / pv;
            }
#pragma unroll
            for (int r = col + 1; r < NGMAX; r++) {
                if (r < n_g) {
                    double f = 0.0;
                    if (t == own) { f = A[lc][r] * inv; A[lc][r] = f; }  // keep L factor
                    f = __shfl_sync(FULL, f, gbase + own);
#pragma unroll
                    for (int c = 0; c < CPL; c++) {
                        const int j = c * G + t;
                        if (j > col && j <= NGMAX) A[c][r] = fma(-f, A[c][col], A[c][r]);
                    }
                }
            }
        }
    });

    // ---------------- back substitution ----------------
#pragma unroll
    for (int c = 0; c < CPL; c++) xs[c] = 0.0;
    static_for<0, NGMAX>([&](auto iic) {
        constexpr int i = NGMAX - 1 - decltype(iic)::value;
        if (i < n_g) {
            double part = 0.0;
#pragma unroll
            for (int c = 0; c < CPL; c++) {
                const int j = c * G + t;
                if (j > i && j < n_g) part = fma(A[c][i], xs[c], part);
            }
            part = mm_group_sum(part, G);
            const double bi = __shfl_sync(FULL, A[AUGS][i], gbase + AUGL);
            constexpr int own = i % G, li = i / G;
            if (t == own) {
                const double d = A[li][i];
                if (fabs(d) > 1e-30) xs[li] = (bi - part) / d;
                else { xs[li] = 0.0; stat |= MM_ST_PIVOT; }
            }
        }
    });

    if (FP32) {
        // ---------- one FP64 residual-refinement step: M' dx = e_last - M' x ----------
        // M' x uses the low-rank form M = BR^T R^T - diag(sum_e R): w_e = sum_k R[k,e] x_k.
        double w[NEMAX];
#pragma unroll
        for (int e = 0; e < NEMAX; e++) {
            double a = 0.0;
#pragma unroll
            for (int c = 0; c < CPL; c++) {
                const int j = c * G + t;
                if (c * G < NGMAX && j < n_g) a = fma(R[c][e], xs[c], a);
            }
            w[e] = (e < n_e) ? mm_group_sum(a, G) : 0.0;
        }
        double sx = 0.0;
#pragma unroll
        for (int c = 0; c < CPL; c++) {
            const int j = c * G + t;
            if (j < n_g) sx += xs[c];
        }
        sx = mm_group_sum(sx, G);
        // residual of row g, evaluated by the lane owning column g
        double rr[CPL];
#pragma unroll
        for (int c = 0; c < CPL; c++) {
            const int g = c * G + t;
            double r = 0.0;
            if (c * G < NGMAX && g < n_g) {
                if (g == n_g - 1) r = 1.0 - sx;
                else {
                    double mx = -Rk[c] * xs[c];
#pragma unroll
                    for (int e = 0; e < NEMAX; e++)
                        if (e < n_e) mx = fma(S.BR[e * n_g + g], w[e], mx);
                    r = -mx;
                }
            }
            rr[c] = r;
        }
        if (__any_sync(FULL, swapped)) {
            // general permutation: gather the residual in every lane, apply the swaps
            double rfull[NGMAX];
#pragma unroll
            for (int g = 0; g < NGMAX; g++) {
                const int own = g % G, lg = g / G;
                rfull[g] = __shfl_sync(FULL, rr[lg], gbase + own);
            }
#pragma unroll
            for (int col = 0; col < NGMAX; col++) {
#pragma unroll
                for (int r = col + 1; r < NGMAX; r++)
                    if (r == prows[col]) { const double tmp = rfull[col]; rfull[col] = rfull[r]; rfull[r] = tmp; }
            }
#pragma unroll
            for (int c = 0; c < CPL; c++) {
#pragma unroll
                for (int g = 0; g < NGMAX; g++)
                    if (g == c * G + t) rr[c] = rfull[g];
            }
        }
        // forward substitution with unit-lower L (factors stored below the diagonal)
        static_for<0, NGMAX>([&](auto ic) {
            constexpr int i = decltype(ic)::value;
            if (i < n_g) {
                double part = 0.0;
#pragma unroll
                for (int c = 0; c < CPL; c++) {
                    const int j = c * G + t;
                    if (j < i) part = fma(A[c][i], rr[c], part);
                }
                part = mm_group_sum(part, G);
                constexpr int own = i % G, li = i / G;
                if (t == own) rr[li] -= part;
            }
        });
        // backward substitution with U
        double dx[CPL];
#pragma unroll
        for (int c = 0; c < CPL; c++) dx[c] = 0.0;
        static_for<0, NGMAX>([&](auto iic) {
            constexpr int i = NGMAX - 1 - decltype(iic)::value;
            if (i < n_g) {
                double part = 0.0;
#pragma unroll
                for (int c = 0; c < CPL; c++) {
                    const int j = c * G + t;
                    if (j > i && j < n_g) part = fma(A[c][i], dx[c], part);
                }
                part = mm_group_sum(part, G);
                constexpr int own = i % G, li = i / G;
                if (t == own) {
                    const double d = A[li][i];
                    dx[li] = (fabs(d) > 1e-30) ? (rr[li] - part) / d : 0.0;
                }
            }
        });
#pragma unroll
        for (int c = 0; c < CPL; c++) xs[c] += dx[c];
    }

    // ---------------- clamp, normalise, force ----------------
    double tot = 0.0;
#pragma unroll
    for (int c = 0; c < CPL; c++) {
        const int j = c * G + t;
        if (j < n_g) { if (xs[c] < 0.0) xs[c] = 0.0; }
        else xs[c] = 0.0;
        tot += xs[c];
    }
    tot = mm_group_sum(tot, G);
    if (tot > 0.0) {
#pragma unroll
        for (int c = 0; c < CPL; c++) xs[c] = xs[c] / tot;
    } else {
        stat |= MM_ST_ZERO_POP;
        if (P.uniform_fb) {
            const double u = 1.0 / (double)n_g;
#pragma unroll
            for (int c = 0; c < CPL; c++) xs[c] = (c * G + t < n_g) ? u : 0.0;
        }
    }
    double F = 0.0, Rs = 0.0;
#pragma unroll
    for (int c = 0; c < CPL; c++) {
        if (c * G < NGMAX && c * G + t < n_g) {
            F = fma(xs[c], Fk[c], F);
            Rs = fma(xs[c], Rk[c], Rs);
        }
    }
    PointOut out;
    out.F = mm_group_sum(F, G);
    out.R = mm_group_sum(Rs, G);
    if (!isfinite(out.F)) stat |= MM_ST_NONFINITE;
    out.status = mm_group_or(stat, G);
    return out;
}
