// smem_solve.cuh -- the steady-state solve of one point by a group of G
// lanes (16 or 32) with the molecule's tables and the population system in
// shared memory: molecules up to 48 ground and 16 excited states.  Used by
// the uneven batches (uneven.cu) and by the drop-in 1D entry points for
// molecules beyond the register-resident classes (large.cu).
//
// Same model and exactness as rate_core.cuh (molmot/obe/rate_equations_jit.py
// :18-145): the detuning chain in the reference's operation order with
// explicit round-to-nearest operations, FMA and Newton reciprocals elsewhere.
// Two population solves:
//  * elimination (RED = false): the reference's Gaussian elimination with
//    partial pivoting on M' (last row replaced by ones), lanes on consecutive
//    columns, pivot by a group argmax taking the first maximum as the
//    reference's strict-greater scan, |pivot| < 1e-30 skipped, factors kept
//    below the diagonal and the row interchanges in `prow` for the adjoint;
//  * excited-chain reduction (RED = true): K = A^T BR^T over the scaled rates
//    and its stationary vector by state reduction (the identity of
//    reduced.cuh), for molecules whose beams pump every ground state and
//    connect the excited chain.
#pragma once
#include "rate_core.cuh"

constexpr int kSmNB = MM_MAX_BEAMS;

// One molecule's tables in shared memory.
struct SmMol {
    const double *E, *zd;   // [n_s]
    const double *d2s;      // |d|^2 at [(e * 3 + q) * NGMAX + g]
    const double *BR;       // branching ratios at [g * NEMAX + e]
    const double *czd;      // zd_g Gamma / 2pi
    int n_g, n_e;
    double Gam;
};

// One parameter set's beams in shared memory.
struct SmBeam {
    const double *freq, *ck, *hk, *s0, *c1;  // c1 = (Gamma/2) s0
    const int *pol;
    int n_b;
    double Bg;  // the set's B'
};

template <int NGMAX, int NEMAX>
struct SmMolLayout {
    static constexpr int doubles = 2 * (NGMAX + NEMAX) + NGMAX * NEMAX * 3 + NEMAX * NGMAX + NGMAX;
};
constexpr int kSmBeamDoubles = 5 * kSmNB;
constexpr int kSmBeamInts = kSmNB;

// Stage molecule data src (E[n_s], zd[n_s], d2[n_g][n_e][3], BR[n_e][n_g], the
// pack's and the bank's layout) into sm (SmMolLayout::doubles); all threads
// of the CTA take part, the caller synchronises afterwards.
template <int NGMAX, int NEMAX>
__device__ void sm_stage_mol(const double *src, int n_g, int n_e, double Gam, double *sm, SmMol &M)
{
    const int n_s = n_g + n_e;
    double *E = sm, *zd = E + NGMAX + NEMAX, *d2s = zd + NGMAX + NEMAX;
    double *BR = d2s + NGMAX * NEMAX * 3, *czd = BR + NEMAX * NGMAX;
    for (int i = threadIdx.x; i < n_s; i += blockDim.x) { E[i] = src[i]; zd[i] = src[n_s + i]; }
    // |d|^2 transposed to [e][q][g]: the lanes of a group own consecutive
    // ground states, so their reads of one (e, q) are consecutive doubles
    for (int i = threadIdx.x; i < n_g * n_e * 3; i += blockDim.x) {
        const int k = i / (n_e * 3), r = i - k * (n_e * 3);
        d2s[r * NGMAX + k] = src[2 * n_s + i];  // r = e * 3 + q
    }
    // branching ratios transposed to [g][e]: the chain build's lanes read
    // consecutive excited states of one ground state
    for (int i = threadIdx.x; i < n_e * n_g; i += blockDim.x) {
        const int e = i / n_g, g = i - e * n_g;
        BR[g * NEMAX + e] = src[2 * n_s + n_g * n_e * 3 + i];
    }
    for (int i = threadIdx.x; i < n_g; i += blockDim.x) czd[i] = src[n_s + i] * Gam / MM_TWO_PI;
    M.E = E; M.zd = zd; M.d2s = d2s; M.BR = BR; M.czd = czd;
    M.n_g = n_g; M.n_e = n_e; M.Gam = Gam;
}

// Stage one parameter set's beams (device arrays of the set) into smd
// (kSmBeamDoubles) and smi (kSmBeamInts).
__device__ __forceinline__ void sm_stage_beams(const double *kdir, const double *freq, const double *s0,
                                               const int32_t *pol, int n_b, double Bg, double kw,
                                               double hbar, double Gam, double *smd, int *smi,
                                               SmBeam &Bm)
{
    double *fr = smd, *ck = fr + kSmNB, *hk = ck + kSmNB, *s = hk + kSmNB, *c1 = s + kSmNB;
    const double gh = Gam / 2.0;
    for (int b = threadIdx.x; b < n_b; b += blockDim.x) {
        fr[b] = freq[b];
        ck[b] = __dmul_rn(-kw, kdir[b]);
        hk[b] = __dmul_rn(__dmul_rn(hbar, kw), kdir[b]);
        s[b] = s0[b];
        c1[b] = __dmul_rn(gh, s0[b]);
        smi[b] = pol[b];
    }
    Bm.freq = fr; Bm.ck = ck; Bm.hk = hk; Bm.s0 = s; Bm.c1 = c1; Bm.pol = smi;
    Bm.n_b = n_b; Bm.Bg = Bg;
}

// Per-group workspace (doubles, then ints) of sm_point.
template <int NGMAX, int NEMAX, bool RED, bool ADJ = false>
struct SmWorkLayout {
    static constexpr int LDA = NGMAX + 1;
    static constexpr int LDK = NEMAX + 1;
    // row stride of the rates Rm[g][e]: lanes own consecutive ground states,
    // so an odd stride keeps their row accesses in distinct banks
    static constexpr int LDR = NEMAX + 1;
    // elimination: A, Rm, bv, xv, invU, Fk, Rk, Esg, fd, Ese (+ adjoint: sat, gacc, nu)
    // reduced:     Rm (scaled rates), K, Fk, Rk, Esg, w, phi, fd, Ese, cw, cf, rs, pi
    static constexpr int raw = RED ? NGMAX * LDR + NEMAX * LDK + 5 * NGMAX + kSmNB + 5 * NEMAX
                                   : NGMAX * LDA + NGMAX * LDR + 6 * NGMAX + kSmNB + NEMAX +
                                         (ADJ ? NGMAX + 2 * kSmNB + NEMAX : 0);
    // two 16-lane groups of a warp read the same offsets of their own region:
    // a stride of 16 banks past a multiple of 128 bytes keeps those reads
    // conflict-free (a multiple of 128 bytes would put both in the same banks)
    static constexpr int doubles = (raw + 15) / 16 * 16 + 8;
    static constexpr int ints = ADJ ? NGMAX : 0;  // row interchanges of the elimination
};

struct SmWork {
    double *A, *Rm, *bv, *xv, *invU, *Fk, *Rk, *Esg, *fd, *Ese;
    double *Kc, *wg, *ph, *cw, *cf, *rsv, *piv;
    double *satk, *gacc, *nu;  // adjoint
    int *prow;                 // adjoint
};

template <int NGMAX, int NEMAX, bool RED, bool ADJ = false>
__device__ __forceinline__ SmWork sm_work(double *W, int *Wi)
{
    using L = SmWorkLayout<NGMAX, NEMAX, RED, ADJ>;
    SmWork w = {};
    if constexpr (RED) {
        w.Rm = W; w.Kc = w.Rm + NGMAX * L::LDR; w.Fk = w.Kc + NEMAX * L::LDK; w.Rk = w.Fk + NGMAX;
        w.Esg = w.Rk + NGMAX; w.wg = w.Esg + NGMAX; w.ph = w.wg + NGMAX; w.fd = w.ph + NGMAX;
        w.Ese = w.fd + kSmNB; w.cw = w.Ese + NEMAX; w.cf = w.cw + NEMAX; w.rsv = w.cf + NEMAX;
        w.piv = w.rsv + NEMAX;
    } else {
        w.A = W; w.Rm = w.A + NGMAX * L::LDA; w.bv = w.Rm + NGMAX * L::LDR; w.xv = w.bv + NGMAX;
        w.invU = w.xv + NGMAX; w.Fk = w.invU + NGMAX; w.Rk = w.Fk + NGMAX; w.Esg = w.Rk + NGMAX;
        w.fd = w.Esg + NGMAX; w.Ese = w.fd + kSmNB;
        if constexpr (ADJ) {
            w.satk = w.Ese + NEMAX; w.gacc = w.satk + NGMAX; w.nu = w.gacc + 2 * kSmNB;
            w.prow = Wi;
        }
    }
    return w;
}

struct SmOut {
    double F, R;
    int status;
    double gB;  // adjoint: dF/dB' (per T/m)
};

__device__ __forceinline__ double sm_gsum(double x, int G)
{
    for (int o = G >> 1; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    return x;
}

// One point (v, z) by the group whose lanes are t = 0 .. G-1 (G consecutive
// lanes of a warp; every lane of the warp must call it, since it uses
// full-warp shuffles).  Returns F, R and the status word on every lane of the
// group.  pop (nullable, device): the n_g populations of the point; it may
// differ between the groups of a warp (no shuffle depends on it).
// ADJ (elimination only): also dF/d(freq_b) and dF/d(s0_b) in W.gacc[0 .. 2 n_b)
// (the caller reads them after a __syncwarp) and dF/dB' in the result:
// implicit differentiation through M' p = e_last with the elimination's own
// factors, as solve_point<ADJ = true> of rate_core.cuh.
template <int NGMAX, int NEMAX, int G, bool RED, bool ADJ = false>
__device__ SmOut sm_point(const SmMol &M, const SmBeam &Bm, const SmWork &W, int t, double v, double z,
                          double Bgrad, double geff, int uniform_fb, double *pop)
{
    using L = SmWorkLayout<NGMAX, NEMAX, RED, ADJ>;
    constexpr int LDA = L::LDA, LDK = L::LDK, LDR = L::LDR;
    const int n_g = M.n_g, n_e = M.n_e, n_b = Bm.n_b;
    const double Gam = M.Gam, gh = Gam / 2.0, gh2 = gh * gh;
    const double *E = M.E, *zd = M.zd, *d2s = M.d2s, *BR = M.BR, *czd = M.czd;
    double *Rm = W.Rm, *Fk = W.Fk, *Rk = W.Rk, *Esg = W.Esg, *fd = W.fd, *Ese = W.Ese;
    int stat = 0;
    const double B = __dmul_rn(__dmul_rn(Bgrad, z), 1e4);
    __syncwarp();
    for (int b = t; b < n_b; b += G)
        fd[b] = __dadd_rn(Bm.freq[b], __ddiv_rn(__dmul_rn(Bm.ck[b], v), MM_TWO_PI));
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
            const int q = Bm.pol[b];
            const double fdb = fd[b], c1b = Bm.c1[b], hkb = Bm.hk[b], s0b = Bm.s0[b];
#pragma unroll
            for (int e = 0; e < NEMAX; e++) {
                if (e >= n_e) break;
                const double d2 = d2s[(e * 3 + q) * NGMAX + k];
                if (d2 < 1e-15) continue;
                const double om = __dsub_rn(Ese[e], Eg);
                const double de = __dmul_rn(__dsub_rn(fdb, om), MM_TWO_PI);
                const double Lz = gh2 * mm_rcp(fma(de, de, gh2));
                const double ru = c1b * d2 * geff * Lz;
                Racc[e] += ru;
                f = fma(hkb, ru, f);
                s = fma(s0b * d2, Lz, s);
            }
        }
        const double sat = mm_rcp(1.0 + s);
        if constexpr (ADJ) W.satk[k] = sat;
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
    SmOut out;
    out.gB = 0.0;
    if constexpr (RED) {
        double *Kc = W.Kc, *wg = W.wg, *ph = W.ph, *cw = W.cw, *cf = W.cf, *rsv = W.rsv, *piv = W.piv;
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
        double Fo = 0.0, Ro = 0.0, in = 0.0;
        int st = 0;
        if (t == 0) {
            double nrm = 0.0, fn = 0.0, rn = 0.0;
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
            in = mm_rcp(nrm);
            Fo = fn * in;
            Ro = rn * in;
            if (!ok || !isfinite(Fo)) st |= MM_ST_NONFINITE;
        }
        // lane 0 of the group holds the result: broadcast it within the group
        const int src = (threadIdx.x & 31) - t;
        out.F = __shfl_sync(0xffffffffu, Fo, src);
        out.R = __shfl_sync(0xffffffffu, Ro, src);
        out.status = __shfl_sync(0xffffffffu, st, src);
        in = __shfl_sync(0xffffffffu, in, src);
        __syncwarp();  // piv written by lane 0
        if (pop) {
            // p_g = w_g sum_e BR[e,g] pi_e / norm
            for (int g = t; g < n_g; g += G) {
                double a = 0.0;
                for (int e = 0; e < n_e; e++) a = fma(BR[g * NEMAX + e], piv[e], a);
                pop[g] = a * wg[g] * in;
            }
        }
        __syncwarp();
        return out;
    } else {
        double *A = W.A, *bv = W.bv, *xv = W.xv, *invU = W.invU;
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
            // brow stays n_g only when no entry compares (NaN rates): keep the row
            const int prow = brow < n_g ? brow : col;
            if constexpr (ADJ) {
                if (t == 0) W.prow[col] = prow;
            }
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
            part = sm_gsum(part, G);
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
        tot = sm_gsum(tot, G);
        Fs = sm_gsum(Fs, G);
        Rs = sm_gsum(Rs, G);
        fu = sm_gsum(fu, G);
        ru = sm_gsum(ru, G);
        double Fo, Ro, it = 0.0;
        if (tot > 0.0) {
            it = mm_rcp(tot);
            Fo = Fs * it;
            Ro = Rs * it;
        } else {
            stat |= MM_ST_ZERO_POP;
            Fo = uniform_fb ? fu / n_g : 0.0;
            Ro = uniform_fb ? ru / n_g : 0.0;
        }
        if (!isfinite(Fo)) stat |= MM_ST_NONFINITE;
        for (int o = G >> 1; o > 0; o >>= 1) stat |= __shfl_xor_sync(0xffffffffu, stat, o);
        // normalised populations (the reference's clamp and normalisation)
        const bool fb = !(tot > 0.0);
        if (pop || ADJ) {
            for (int i = t; i < n_g; i += G) {
                const double p = xv[i] > 0.0 ? xv[i] : 0.0;
                const double pn = fb ? (uniform_fb ? 1.0 / (double)n_g : 0.0) : p * it;
                if (pop) pop[i] = pn;
                if constexpr (ADJ) xv[i] = pn;
            }
        }
        out.F = Fo;
        out.R = Ro;
        out.status = stat;
        if constexpr (ADJ) {
            // lambda solves M'^T lambda = dF/dp = F_k with P M' = L U:
            // U^T w = F, L^T u = w, lambda = P^T u (in bv), on the fixed active set
            double *lam = bv, *nu = W.nu, *gacc = W.gacc;
            __syncwarp();
            if (t == 0) {
                for (int i = 0; i < n_g; i++) {
                    double a = Fk[i];
                    for (int j = 0; j < i; j++) a = fma(-A[j * LDA + i], lam[j], a);  // U[j][i]
                    lam[i] = a * invU[i];
                }
                for (int i = n_g - 1; i >= 0; i--) {
                    double a = lam[i];
                    for (int j = i + 1; j < n_g; j++) a = fma(-A[j * LDA + i], lam[j], a);  // L[j][i]
                    lam[i] = a;
                }
                for (int col = n_g - 1; col >= 0; col--) {
                    const int pr = W.prow[col];
                    if (pr != col) { const double tmp = lam[col]; lam[col] = lam[pr]; lam[pr] = tmp; }
                }
            }
            __syncwarp();
            // nu_e = sum_{g < n-1} lambda_g BR[e, g]
            for (int e = t; e < n_e; e += G) {
                double a = 0.0;
                for (int g = 0; g < n_g - 1; g++) a = fma(lam[g], BR[g * NEMAX + e], a);
                nu[e] = a;
            }
            for (int i = t; i < 2 * n_b; i += G) gacc[i] = 0.0;
            __syncwarp();
            // dF/dtheta = sum_{b,g,e} (p_g hk_b - mu[g,e]) d rate_bge / dtheta with
            // mu[g,e] = p_g (nu_e - lambda_g [g < n-1]); the saturation enters through a
            // second pass (C = sum (w rate) sat)
            double gB = 0.0;
            for (int k = t; k < n_g; k += G) {
                const double pk = xv[k], sat = W.satk[k], lamk = (k < n_g - 1) ? lam[k] : 0.0;
                const double Eg = Esg[k];
                double T = 0.0;
                for (int pass = 0; pass < 2; pass++) {
                    const double C = T * sat;
                    for (int b = 0; b < n_b; b++) {
                        const int q = Bm.pol[b];
                        const double fdb = fd[b], c1b = Bm.c1[b], hkb = Bm.hk[b], s0b = Bm.s0[b];
                        for (int e = 0; e < n_e; e++) {
                            const double d2 = d2s[(e * 3 + q) * NGMAX + k];
                            if (d2 < 1e-15) continue;
                            const double om = __dsub_rn(Ese[e], Eg);
                            const double de = __dmul_rn(__dsub_rn(fdb, om), MM_TWO_PI);
                            const double Lz = gh2 * mm_rcp(fma(de, de, gh2));
                            const double rate = c1b * d2 * geff * Lz * sat;
                            const double w = pk * hkb - pk * (nu[e] - lamk);
                            if (pass == 0) {
                                T = fma(w, rate, T);
                            } else {
                                const double Q = w * rate - C * (s0b * d2) * Lz;
                                const double dLL = -2.0 * de * Lz / gh2;  // (dL/d delta) / L
                                atomicAdd(&gacc[b], Q * dLL * MM_TWO_PI);
                                atomicAdd(&gacc[n_b + b], d2 * Lz * (w * gh * geff * sat - C));
                                const double ddB = -z * 1e4 * (zd[n_g + e] - zd[k]) * Gam;
                                gB = fma(Q * dLL, ddB, gB);
                            }
                        }
                    }
                }
            }
            out.gB = sm_gsum(gB, G);
            __syncwarp();
        }
        return out;
    }
}
