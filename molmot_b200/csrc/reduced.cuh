// reduced.cuh -- the FP32-bulk steady-state force, one point per thread,
// with the population system solved exactly on the excited manifold.
//
// Model (molmot/obe/rate_equations_jit.py:18-145): rates R[g,e] (saturated),
// r_g = sum_e R[g,e], M[g,k] = sum_e R[k,e] BR[e,g] - delta_gk r_k, the last
// row replaced by ones, M' p = e_last, clamp, normalise, F = sum_g p_g F_g.
//
// Reduction.  Every column of M sums to zero (sum_g BR[e,g] = 1), so M' p =
// e_last is M p = 0 with sum p = 1.  Row g of M p = 0 reads
//     r_g p_g = sum_e BR[e,g] n_e,   n_e = sum_k R[k,e] p_k  (excitation flux),
// hence p_g = (sum_e BR[e,g] n_e) / r_g and n = K n with the column-stochastic
//     K[e,e'] = sum_g R[g,e] BR[e',g] / r_g   (n_e x n_e).
// n is the stationary vector of the excited-state chain, computed by the
// Grassmann-Taksar-Heyman state reduction (Gaussian elimination on I - K^T
// written without subtractions, so every step adds non-negative numbers).
// Then, with w_g = 1/r_g and phi_g = F_g / r_g,
//     norm = sum_e n_e sum_g BR[e,g] w_g,   F = sum_e n_e sum_g BR[e,g] phi_g / norm,
//     R    = sum_e n_e sum_g BR[e,g] / norm.
// The per-ground-state sums are folded into K and two n_e-vectors while the
// rates of g are computed, so a point keeps n_e^2 + 2 n_e FP64 accumulators.
// The saturation factor 1/(1+s_g) cancels in R[g,e]/r_g and F_g/r_g and enters
// only through w_g = (1+s_g)/sum_e R_unsat[g,e].
//
// Precision.  The Lorentzian of each (g, beam, e) triple runs in FP32 from
// u = delta/(Gamma/2) = u0 + uv v - uB B (u0 rounded once from FP64); the
// rate terms are summed in FP64 (the force sum cancels between
// counter-propagating beams, and FP32 sums of those terms alone exceed 1e-6
// of max|F| on some parameter sets).  Everything after the rates is FP64.
//
// Degenerate sets: a ground state with no active triple (r_g = 0), or an
// excited-state chain that is not strongly connected.  Both are properties of the parameter set (which triples exist), so
// the CTA decides once per set and then solves every point with
// dense_point(), the reference's own elimination in FP64 on the same rates.
#pragma once
#include "rate_core.cuh"

// Lists of the triples of one (ground, excited) pair may be padded with
// zero-weight triples to a multiple of kRedPad, so the loop over a list runs
// whole groups of kRedPad independent Lorentzians with no remainder.  The
// host picks the granule per launch (kRedPad when padding adds at most a
// quarter to the batch's triples, else 1); it is a template parameter of
// the kernel, which then holds one loop form only.
constexpr int kRedPad = 4;

// Slots per ground state of reduced_adjoint_point's KEEP buffer: the rate sums
// (R[g,e] for e < NEMAX, f_g, s_g), later alpha_ge, beta_g, gamma_g, then the
// transition offsets omega_ge = E_e(B) - E_g(B).
template <int NEMAX>
constexpr int kKeepSlots = 2 * NEMAX + 2;

// One active (ground g, beam b, excited e) triple: 32 bytes.
struct TripR {
    float u0;    // (freq_b - (E_e - E_g)) 2pi/(Gamma/2)  (FP64, rounded once)
    float uv;    // (-k kdir_b / 2pi) 2pi/(Gamma/2)      per m/s
    float uB;    // ((zd_e - zd_g) Gamma/2pi) 2pi/(Gamma/2) per G
    float c2;    // s0_b d2
    double c1;   // (Gamma/2) s0_b d2 Geff
    double hc1;  // hbar k kdir_b c1
};

// The same triple for the FP64 form (MM_PREC_FP64_REDUCED): the Lorentzian
// follows the reference's detuning chain from the point's Doppler-shifted
// beam frequency fd[b] and Zeeman-shifted energies.
struct TripD {
    double c1;   // ((Gamma/2) s0_b) d2 Geff
    double c2;   // s0_b d2
    double hk;   // (hbar k) kdir_b
    int b, pad;
};
static_assert(sizeof(TripR) == 32 && sizeof(TripD) == 32, "triple records are 32 bytes");

// Per-point inputs of the rate loop.  FP32 form: v and B (Gauss) in FP32.
// FP64 form: B, the Doppler-shifted beam frequencies fd[b * stride] (this
// thread's slots of a shared-memory scratch) and the excited energies.
template <int NEMAX>
struct RateCtx {
    float vf, Bf;
    double B;
    const double *fd;
    int stride;
    double Ese[NEMAX];
};

template <int NGMAX, int NEMAX>
struct RedLayout {
    // offs[g*NEMAX + e] .. offs[g*NEMAX + e + 1]: triples of (g, e), beams ascending
    static constexpr int n_offs = NGMAX * NEMAX + 1;
    size_t offs, brt, rsum, flags, E, czd, zde, freq, ck, trip, d2t, total;
    __host__ __device__ static size_t al(size_t x) { return (x + 15) & ~size_t(15); }
    // with_d2: also |d|^2 of every triple slot (the adjoints' d/ds0 terms)
    __host__ __device__ void build(int n_b, bool with_d2 = false)
    {
        size_t o = 0;
        offs = o;  o = al(o + sizeof(int) * n_offs);
        brt = o;   o = al(o + sizeof(double) * NGMAX * NEMAX);   // BR[e,g] at [g][e]
        rsum = o;  o = al(o + sizeof(double) * NEMAX);           // sum_g BR[e,g]
        flags = o; o = al(o + sizeof(int) * 4);
        E = o;     o = al(o + sizeof(double) * (NGMAX + NEMAX));  // FP64 form: energies,
        czd = o;   o = al(o + sizeof(double) * NGMAX);            // zd_g Gamma / 2pi,
        zde = o;   o = al(o + sizeof(double) * NEMAX);            // zd_e,
        freq = o;  o = al(o + sizeof(double) * n_b);              // beam frequencies,
        ck = o;    o = al(o + sizeof(double) * n_b);              // -k kdir_b
        const size_t slots = (size_t)NGMAX * NEMAX * (size_t)((n_b + kRedPad - 1) / kRedPad * kRedPad);
        trip = o;  o = al(o + sizeof(TripR) * slots);
        d2t = with_d2 ? o : 0;
        if (with_d2) o = al(o + sizeof(double) * slots);
        total = o;
    }
};

struct RedView {
    const int *offs;
    const double *brt, *rsum;
    const double *E, *czd, *zde, *freq, *ck;
    const void *trip;  // TripR (FP32 form) or TripD (FP64 form)
    const double *d2t; // |d|^2 per triple slot (layouts built with_d2), else null
    int valid;
};

// Parameter-set tables for the reduced kernel (all threads of the CTA);
// lists padded to multiples of PAD.
template <int NGMAX, int NEMAX, int PAD, bool F64>
__device__ void build_reduced_tables(const ForceParams &P, int set, unsigned char *sm,
                                     const RedLayout<NGMAX, NEMAX> &Ly, RedView &S)
{
    const int n_g = P.n_g, n_e = P.n_e, n_b = P.n_b;
    int *offs = (int *)(sm + Ly.offs), *flags = (int *)(sm + Ly.flags);
    double *brt = (double *)(sm + Ly.brt), *rsum = (double *)(sm + Ly.rsum);
    TripR *trip = (TripR *)(sm + Ly.trip);
    TripD *tripd = (TripD *)(sm + Ly.trip);
    double *Es = (double *)(sm + Ly.E), *czd = (double *)(sm + Ly.czd), *zde = (double *)(sm + Ly.zde);
    double *frq = (double *)(sm + Ly.freq), *ck = (double *)(sm + Ly.ck);
    const int tid = threadIdx.x, nt = blockDim.x;
    const int32_t *pol = P.pol + (size_t)set * n_b;
    const double *kdir = P.kdir + (size_t)set * n_b, *fr = P.freq + (size_t)set * n_b;
    const double *s0 = P.s0 + (size_t)set * n_b;

    // triple counts per (g, e) (d2 >= 1e-15, rate_equations_jit.py:67-69), BR transposed
    for (int i = tid; i < NGMAX * NEMAX; i += nt) {
        const int g = i / NEMAX, e = i % NEMAX;
        int c = 0;
        double br = 0.0;
        if (g < n_g && e < n_e) {
            for (int b = 0; b < n_b; b++)
                if (P.d2[(g * n_e + e) * 3 + pol[b]] >= 1e-15) c++;
            br = P.BR[e * n_g + g];
        }
        offs[i + 1] = c;
        brt[i] = br;
    }
    __syncthreads();
    if (tid == 0) {
        offs[0] = 0;
        for (int i = 1; i <= NGMAX * NEMAX; i++) offs[i] = offs[i - 1] + (offs[i] + PAD - 1) / PAD * PAD;
        // structural checks: every ground state pumped, and the excited-state
        // chain (e' -> e when e' decays to a ground state that a beam excites
        // to e) strongly connected, so its stationary vector is unique and
        // the state reduction never meets a zero outflow
        int valid = 1;
        for (int g = 0; g < n_g; g++)
            if (offs[g * NEMAX + NEMAX] == offs[g * NEMAX]) valid = 0;
        unsigned T[NEMAX];
        for (int i = 0; i < n_e; i++) {
            unsigned ti = 1u << i;
            for (int g = 0; g < n_g; g++)
                if (brt[g * NEMAX + i] > 0.0)
                    for (int j = 0; j < n_e; j++)
                        if (offs[g * NEMAX + j + 1] > offs[g * NEMAX + j]) ti |= 1u << j;
            T[i] = ti;
        }
        for (int k = 0; k < n_e; k++)
            for (int i = 0; i < n_e; i++)
                if (T[i] >> k & 1u) T[i] |= T[k];
        const unsigned all = (1u << n_e) - 1u;
        for (int i = 0; i < n_e; i++)
            if ((T[i] & all) != all) valid = 0;
        for (int e = 0; e < NEMAX; e++) {
            double a = 0.0;
            for (int g = 0; g < n_g; g++) a += brt[g * NEMAX + e];
            rsum[e] = a;
        }
        flags[0] = valid;
    }
    __syncthreads();
    for (int i = tid; i < n_g + n_e; i += nt) Es[i] = P.E[i];
    for (int i = tid; i < n_g; i += nt) czd[i] = P.zd[i] * P.Gamma / MM_TWO_PI;
    for (int i = tid; i < n_e; i += nt) zde[i] = P.zd[n_g + i];
    for (int b = tid; b < n_b; b += nt) {
        frq[b] = fr[b];
        ck[b] = __dmul_rn(-P.k, kdir[b]);
    }
    const double cu = MM_TWO_PI / (P.Gamma / 2.0);
    const double gh = P.Gamma / 2.0;
    for (int i = tid; i < NGMAX * NEMAX; i += nt) {
        const int g = i / NEMAX, e = i % NEMAX;
        if (g >= n_g || e >= n_e) continue;
        int o = offs[i];
        for (int b = 0; b < n_b; b++) {
            const double d2 = P.d2[(g * n_e + e) * 3 + pol[b]];
            if (d2 < 1e-15) continue;
            if constexpr (F64) {  // the plain form's products, in its order
                if (Ly.d2t) ((double *)(sm + Ly.d2t))[o] = d2;
                TripD tr;
                tr.c1 = __dmul_rn(__dmul_rn(gh, s0[b]), d2) * P.geff;
                tr.c2 = __dmul_rn(s0[b], d2);
                tr.hk = __dmul_rn(__dmul_rn(P.hbar, P.k), kdir[b]);
                tr.b = b;
                tr.pad = 0;
                tripd[o++] = tr;
            } else {
                TripR tr;
                tr.u0 = (float)((fr[b] - (P.E[n_g + e] - P.E[g])) * cu);
                tr.uv = (float)((-P.k * kdir[b]) / MM_TWO_PI * cu);
                tr.uB = (float)((P.zd[n_g + e] - P.zd[g]) * P.Gamma / MM_TWO_PI * cu);
                tr.c2 = (float)(s0[b] * d2);
                tr.c1 = gh * s0[b] * d2 * P.geff;
                tr.hc1 = P.hbar * P.k * kdir[b] * tr.c1;
                trip[o++] = tr;
            }
        }
        for (; o < offs[i + 1]; o++) {  // zero-weight padding: every term 0
            if constexpr (F64) {
                if (Ly.d2t) ((double *)(sm + Ly.d2t))[o] = 0.0;
                TripD tr = {};
                tr.pad = 1;  // marks list padding for the adjoint
                tripd[o] = tr;
            } else {
                TripR tr = {};
                trip[o] = tr;
            }
        }
    }
    __syncthreads();
    S.offs = offs; S.brt = brt; S.rsum = rsum; S.trip = trip; S.valid = flags[0];
    S.d2t = Ly.d2t ? (const double *)(sm + Ly.d2t) : nullptr;
    S.E = Es; S.czd = czd; S.zde = zde; S.freq = frq; S.ck = ck;
}

struct RedOut {
    double F, R;
    int status;
};

// One triple's Lorentzian (FP32) and its FP64 contributions.
__device__ __forceinline__ void reduced_triple(const TripR &tr, float vf, float Bf, double &acc,
                                               double &f, float &s)
{
    float u = fmaf(tr.uv, vf, tr.u0);
    u = fmaf(-Bf, tr.uB, u);
    const float L = mm_rcpf(fmaf(u, u, 1.0f));
    s = fmaf(tr.c2, L, s);
    // FP32 -> FP64 on the bits (ALU) instead of a conversion on the XU pipe,
    // which the reciprocal above already loads: for a positive normal float,
    // shift the exponent and mantissa into place and rebias the exponent
    // (+ (1023 - 127) << 52), exactly (double)L.  L lies in [2^-126, 1] or is
    // 0 (u^2 overflowed; this gives 2^-127, far below the FP64 rounding of the
    // sums) or NaN (non-finite parameters; the FP32 saturation sum s still
    // carries the NaN into F).  The force maps took 5.75 ms instead of 6.26 ms
    // (1024 SrOH sets x 256 x 256), with the same bits.
    const unsigned lb = __float_as_uint(L);
    const double Ld = __hiloint2double((int)((lb >> 3) + 0x38000000u), (int)(lb << 29));
    acc = fma(tr.c1, Ld, acc);
    f = fma(tr.hc1, Ld, f);
}

// One triple of the FP64 form: the plain form's detuning and Lorentzian
// (rate_equations_jit.py:58-83 operation order).
__device__ __forceinline__ void reduced_triple64(const TripD &tr, double fdb, double Ese, double Esg,
                                                 double gh2, double &acc, double &f, double &s)
{
    const double om = __dsub_rn(Ese, Esg);
    const double de = __dmul_rn(__dsub_rn(fdb, om), MM_TWO_PI);
    const double L = gh2 * mm_rcp(fma(de, de, gh2));
    const double ru = tr.c1 * L;
    acc += ru;
    f = fma(tr.hk, ru, f);
    s = fma(tr.c2, L, s);
}

// Rates of ground state g at one point: unsaturated FP64 sums over the
// triples of each excited state, the force sum, and the saturation sum
// (FP32 in the FP32 form).  PAD: the list granule (kRedPad or 1).
template <int NEMAX, int PAD, bool F64>
__device__ __forceinline__ void reduced_rates(const RedView &S, int g, const RateCtx<NEMAX> &C,
                                              double gh2, double (&Re)[NEMAX], double &f,
                                              std::conditional_t<F64, double, float> &s)
{
    f = 0.0;
    s = 0;
    double Esg = 0.0;
    if constexpr (F64) Esg = fma(C.B, S.czd[g], S.E[g]);  // |error| <= 1 ulp of E_g
#pragma unroll
    for (int e = 0; e < NEMAX; e++) {
        double acc = 0.0;
        const int i1 = S.offs[g * NEMAX + e + 1];
        auto one = [&](int i) {
            if constexpr (F64) {
                const TripD tr = ((const TripD *)S.trip)[i];
                reduced_triple64(tr, C.fd[tr.b * C.stride], C.Ese[e], Esg, gh2, acc, f, s);
            } else {
                reduced_triple(((const TripR *)S.trip)[i], C.vf, C.Bf, acc, f, s);
            }
        };
        if constexpr (PAD > 1) {
#pragma unroll 1
            for (int i = S.offs[g * NEMAX + e]; i < i1; i += PAD) {
#pragma unroll
                for (int j = 0; j < PAD; j++) one(i + j);
            }
        } else {
#pragma unroll 4
            for (int i = S.offs[g * NEMAX + e]; i < i1; i++) one(i);
        }
        Re[e] = acc;
    }
}

// Stationary vector of the column-stochastic K (K[to][from]) by state
// reduction; returns false if a reduction step has no outflow.
template <int NEMAX>
__device__ __forceinline__ bool gth_stationary(double (&K)[NEMAX][NEMAX], int n_e, double (&pi)[NEMAX])
{
    bool ok = true;
    // Q[i][j] = K[j][i]: probability i -> j
#pragma unroll
    for (int k = NEMAX - 1; k >= 1; k--) {
        if (k < n_e) {
            double S = 0.0;
#pragma unroll
            for (int j = 0; j < k; j++) S += K[j][k];
            ok = ok && (S > 0.0);
            const double inv = mm_rcp(S > 0.0 ? S : 1.0);
#pragma unroll
            for (int i = 0; i < k; i++) K[k][i] *= inv;            // Q[i][k] /= S
#pragma unroll
            for (int i = 0; i < k; i++)
#pragma unroll
                for (int j = 0; j < k; j++) K[j][i] = fma(K[k][i], K[j][k], K[j][i]);  // Q[i][j] += Q[i][k] Q[k][j]
        }
    }
    pi[0] = 1.0;
#pragma unroll
    for (int k = 1; k < NEMAX; k++) {
        double a = 0.0;
        if (k < n_e) {
#pragma unroll
            for (int i = 0; i < k; i++) a = fma(pi[i], K[k][i], a);  // pi[i] Q[i][k]
        }
        pi[k] = a;
    }
    return ok;
}

// Dense fallback: the reference's elimination (rate_equations_jit.py:92-136)
// in FP64 on the same FP32-bulk rates, one point per thread (local memory).
template <int NGMAX, int NEMAX, int PAD, bool F64>
__device__ __noinline__ RedOut dense_point(const ForceParams &P, const RedView &S,
                                           const RateCtx<NEMAX> &C, double *pop_out)
{
    const int n_g = P.n_g, n_e = P.n_e;
    double R[NGMAX][NEMAX], Fk[NGMAX], Rk[NGMAX];
    for (int g = 0; g < n_g; g++) {
        double Re[NEMAX], f;
        std::conditional_t<F64, double, float> s;
        reduced_rates<NEMAX, PAD, F64>(S, g, C, (P.Gamma / 2.0) * (P.Gamma / 2.0), Re, f, s);
        const double sat = 1.0 / (1.0 + (double)s);
        double rs = 0.0;
        for (int e = 0; e < NEMAX; e++) { R[g][e] = Re[e] * sat; rs += R[g][e]; }
        Rk[g] = rs;
        Fk[g] = f * sat;
    }
    double A[NGMAX][NGMAX + 1];
    for (int gg = 0; gg < n_g; gg++) {
        for (int k = 0; k < n_g; k++) {
            double a = (gg == k) ? -Rk[gg] : 0.0;
            for (int e = 0; e < n_e; e++) a += R[k][e] * S.brt[gg * NEMAX + e];
            A[gg][k] = a;
        }
        A[gg][n_g] = 0.0;
    }
    for (int k = 0; k < n_g; k++) A[n_g - 1][k] = 1.0;
    A[n_g - 1][n_g] = 1.0;
    int status = 0;
    for (int col = 0; col < n_g; col++) {
        int prow = col;
        double mx = fabs(A[col][col]);
        for (int r = col + 1; r < n_g; r++)
            if (fabs(A[r][col]) > mx) { mx = fabs(A[r][col]); prow = r; }
        if (prow != col)
            for (int j = 0; j <= n_g; j++) { const double t = A[col][j]; A[col][j] = A[prow][j]; A[prow][j] = t; }
        const double pv = A[col][col];
        if (fabs(pv) < 1e-30) { status |= MM_ST_PIVOT; continue; }
        for (int r = col + 1; r < n_g; r++) {
            const double fct = A[r][col] / pv;
            for (int j = col; j <= n_g; j++) A[r][j] -= fct * A[col][j];
        }
    }
    double p[NGMAX];
    for (int i = n_g - 1; i >= 0; i--) {
        double sacc = A[i][n_g];
        for (int j = i + 1; j < n_g; j++) sacc -= A[i][j] * p[j];
        p[i] = (fabs(A[i][i]) > 1e-30) ? sacc / A[i][i] : 0.0;
    }
    double tot = 0.0;
    for (int g = 0; g < n_g; g++) { if (p[g] < 0.0) p[g] = 0.0; tot += p[g]; }
    if (tot > 0.0) {
        for (int g = 0; g < n_g; g++) p[g] /= tot;
    } else {
        status |= MM_ST_ZERO_POP;
        if (P.uniform_fb)
            for (int g = 0; g < n_g; g++) p[g] = 1.0 / (double)n_g;
    }
    RedOut o;
    o.F = 0.0;
    o.R = 0.0;
    for (int g = 0; g < n_g; g++) {
        o.F += p[g] * Fk[g];
        o.R += p[g] * Rk[g];
        if (pop_out) pop_out[g] = p[g];
    }
    o.status = status;
    return o;
}

// One point by the reduced solve.  pop_out (nullable): n_g populations.
// fd (FP64 form only): this thread's first slot of a shared scratch of n_b
// doubles at the given stride, for the point's Doppler-shifted frequencies.
template <int NGMAX, int NEMAX, bool EXACT, int PAD, bool F64 = false>
__device__ __forceinline__ RedOut reduced_point(const ForceParams &P, const RedView &S, double v,
                                                double z, double Bgrad, double *pop_out,
                                                double *fd = nullptr, int stride = 0)
{
    const int n_g = EXACT ? NGMAX : P.n_g;
    const int n_e = EXACT ? NEMAX : P.n_e;
    RateCtx<NEMAX> C;
    C.B = __dmul_rn(__dmul_rn(Bgrad, z), 1e4);
    C.vf = (float)v;
    C.Bf = (float)C.B;
    C.fd = fd;
    C.stride = stride;
    if constexpr (F64) {
        // laser frequency seen by the moving molecule and Zeeman-shifted
        // excited energies, in the reference's order (exact roundings)
        for (int b = 0; b < P.n_b; b++)
            fd[b * stride] = __dadd_rn(S.freq[b], __ddiv_rn(__dmul_rn(S.ck[b], v), MM_TWO_PI));
#pragma unroll
        for (int e = 0; e < NEMAX; e++)
            C.Ese[e] = (e < n_e) ? __dadd_rn(S.E[n_g + e], __ddiv_rn(__dmul_rn(__dmul_rn(C.B, S.zde[e]), P.Gamma),
                                                                      MM_TWO_PI))
                                 : 0.0;
    }
    if (!(isfinite(v) && isfinite(z))) {  // the rate chain assumes finite, normal Lorentzians
        RedOut o;
        o.F = o.R = __longlong_as_double(0x7ff8000000000000ll);
        o.status = MM_ST_NONFINITE;
        if (pop_out)
            for (int g = 0; g < n_g; g++) pop_out[g] = o.F;
        return o;
    }
    if (!S.valid) return dense_point<NGMAX, NEMAX, PAD, F64>(P, S, C, pop_out);
    const double gh2 = (P.Gamma / 2.0) * (P.Gamma / 2.0);

    double K[NEMAX][NEMAX], cw[NEMAX], cf[NEMAX];
#pragma unroll
    for (int e = 0; e < NEMAX; e++) {
        cw[e] = 0.0;
        cf[e] = 0.0;
#pragma unroll
        for (int e2 = 0; e2 < NEMAX; e2++) K[e][e2] = 0.0;
    }
    for (int g = 0; g < n_g; g++) {
        double Re[NEMAX], f;
        std::conditional_t<F64, double, float> s;
        reduced_rates<NEMAX, PAD, F64>(S, g, C, gh2, Re, f, s);
        double rt = 0.0;
#pragma unroll
        for (int e = 0; e < NEMAX; e++) rt += Re[e];
        const double inv = mm_rcp(rt);             // rt > 0: every ground state is pumped
        const double phi = f * inv;                // F_g / r_g
        const double w = (1.0 + (double)s) * inv;  // 1 / r_g
        double br[NEMAX];
#pragma unroll
        for (int e = 0; e < NEMAX; e++) br[e] = S.brt[g * NEMAX + e];
#pragma unroll
        for (int e = 0; e < NEMAX; e++) {
            const double a = Re[e] * inv;          // R[g,e] / r_g
#pragma unroll
            for (int e2 = 0; e2 < NEMAX; e2++) K[e][e2] = fma(a, br[e2], K[e][e2]);
        }
#pragma unroll
        for (int e = 0; e < NEMAX; e++) {
            cw[e] = fma(br[e], w, cw[e]);
            cf[e] = fma(br[e], phi, cf[e]);
        }
        if (pop_out) pop_out[g] = w;
    }
    double pi[NEMAX];
    const bool ok = gth_stationary<NEMAX>(K, n_e, pi);
    double nrm = 0.0, fn = 0.0, rn = 0.0;
#pragma unroll
    for (int e = 0; e < NEMAX; e++) {
        nrm = fma(cw[e], pi[e], nrm);
        fn = fma(cf[e], pi[e], fn);
        rn = fma(S.rsum[e], pi[e], rn);
    }
    const double in = mm_rcp(nrm);
    RedOut o;
    o.F = fn * in;
    o.R = rn * in;
    o.status = 0;
    if (pop_out) {
        for (int g = 0; g < n_g; g++) {
            double a = 0.0;
#pragma unroll
            for (int e = 0; e < NEMAX; e++) a = fma(S.brt[g * NEMAX + e], pi[e], a);
            pop_out[g] = a * pop_out[g] * in;
        }
    }
    if (!ok || !isfinite(o.F)) o.status |= MM_ST_NONFINITE;
    return o;
}

// Two points of the FP32 form at once (finite inputs, valid set): each triple
// record is read once for both, and the two points' Lorentzian chains give
// the scheduler independent work; per point the operations are those of
// reduced_point, so the results are the same bits.
template <int NGMAX, int NEMAX, bool EXACT, int PAD>
__device__ __forceinline__ void reduced_point2(const ForceParams &P, const RedView &S, const double *v,
                                               const double *z, double Bgrad, RedOut *o)
{
    const int n_g = EXACT ? NGMAX : P.n_g;
    const int n_e = EXACT ? NEMAX : P.n_e;
    float vf[2], Bf[2];
#pragma unroll
    for (int h = 0; h < 2; h++) {
        const double B = __dmul_rn(__dmul_rn(Bgrad, z[h]), 1e4);
        vf[h] = (float)v[h];
        Bf[h] = (float)B;
    }
    double K[2][NEMAX][NEMAX], cw[2][NEMAX], cf[2][NEMAX];
#pragma unroll
    for (int h = 0; h < 2; h++)
#pragma unroll
        for (int e = 0; e < NEMAX; e++) {
            cw[h][e] = 0.0;
            cf[h][e] = 0.0;
#pragma unroll
            for (int e2 = 0; e2 < NEMAX; e2++) K[h][e][e2] = 0.0;
        }
    for (int g = 0; g < n_g; g++) {
        double Re[2][NEMAX], f[2] = {0.0, 0.0};
        float sat[2] = {0.0f, 0.0f};
#pragma unroll
        for (int e = 0; e < NEMAX; e++) {
            double acc[2] = {0.0, 0.0};
            const int i1 = S.offs[g * NEMAX + e + 1];
#pragma unroll 1
            for (int i = S.offs[g * NEMAX + e]; i < i1; i += PAD) {
#pragma unroll
                for (int j = 0; j < PAD; j++) {
                    const TripR tr = ((const TripR *)S.trip)[i + j];
                    reduced_triple(tr, vf[0], Bf[0], acc[0], f[0], sat[0]);
                    reduced_triple(tr, vf[1], Bf[1], acc[1], f[1], sat[1]);
                }
            }
            Re[0][e] = acc[0];
            Re[1][e] = acc[1];
        }
        double br[NEMAX];
#pragma unroll
        for (int e = 0; e < NEMAX; e++) br[e] = S.brt[g * NEMAX + e];
#pragma unroll
        for (int h = 0; h < 2; h++) {
            double rt = 0.0;
#pragma unroll
            for (int e = 0; e < NEMAX; e++) rt += Re[h][e];
            const double inv = mm_rcp(rt);
            const double phi = f[h] * inv;
            const double w = (1.0 + (double)sat[h]) * inv;
#pragma unroll
            for (int e = 0; e < NEMAX; e++) {
                const double a = Re[h][e] * inv;
#pragma unroll
                for (int e2 = 0; e2 < NEMAX; e2++) K[h][e][e2] = fma(a, br[e2], K[h][e][e2]);
            }
#pragma unroll
            for (int e = 0; e < NEMAX; e++) {
                cw[h][e] = fma(br[e], w, cw[h][e]);
                cf[h][e] = fma(br[e], phi, cf[h][e]);
            }
        }
    }
#pragma unroll
    for (int h = 0; h < 2; h++) {
        double pi[NEMAX];
        const bool ok = gth_stationary<NEMAX>(K[h], n_e, pi);
        double nrm = 0.0, fn = 0.0, rn = 0.0;
#pragma unroll
        for (int e = 0; e < NEMAX; e++) {
            nrm = fma(cw[h][e], pi[e], nrm);
            fn = fma(cf[h][e], pi[e], fn);
            rn = fma(S.rsum[e], pi[e], rn);
        }
        const double in = mm_rcp(nrm);
        o[h].F = fn * in;
        o[h].R = rn * in;
        o[h].status = (!ok || !isfinite(o[h].F)) ? MM_ST_NONFINITE : 0;
    }
}

// ---------------------------------------------------------------------------
// Adjoint of the FP64-reduced form: F and dF/d(freq_b, s0_b, B) at one point
// (one thread; B the field in Gauss, B = B' z 1e4).  With
// u = dF/dpi = (cf - F cw) / norm (u . pi = 0) and lambda solving
// (I - K)^T lambda = u (lambda_0 = 0: K's columns sum to one, so lambda is
// defined up to a multiple of the ones vector, which dK annihilates),
//     dF = sum_g [ y_g sum_e lambda_e d a_ge + (y_g / norm) d phi_g
//                  - (F y_g / norm) d w_g ],   y_g = sum_e BR[e,g] pi_e,
// and a_ge, phi_g, w_g are functions of the unsaturated rate sums R_ge, the
// force sum f_g and the saturation sum s_g.  Each triple (g, b, e) enters
// those sums through c1 L, hk c1 L and c2 L, so its contribution is
//     q = alpha_ge c1 + beta_g hk c1 + gamma_g c2   times dL,
// with dL/dfreq_b = L'(delta) 2 pi, dL/dB = L'(delta) (-(zd_e - zd_g) Gamma)
// and d(c1, c2)/ds0_b = (c1, c2) / s0_b written with d2 (s0_b may be 0).
// gf[b * stride], gs[b * stride]: this thread's per-beam accumulators
// (shared memory); the caller zeroes them.  pol: the set's polarisations.
// Valid sets only (S.valid); finite v and z.
// NL > 1: the point is shared by NL consecutive lanes (sub-lane j), each
// taking the ground states g = j (mod NL) in both passes; the partial sums
// (K, cw, cf after the first pass, the per-beam accumulators and dF/dB after
// the second) are added over the NL lanes with shuffles, so every lane ends
// with the whole result.  All lanes of the warp must call it together.
template <int NL>
__device__ __forceinline__ double red_lane_sum(double x)
{
#pragma unroll
    for (int o = 1; o < NL; o <<= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    return x;
}

template <int NGMAX, int NEMAX, bool EXACT, int PAD, int NL = 1, bool KEEP = false>
__device__ __forceinline__ RedOut reduced_adjoint_point(const ForceParams &P, const RedView &S,
                                                        const int32_t *pol, double v, double z,
                                                        double Bgrad, double *fd, int stride,
                                                        double *gf, double *gs, double &gBG, int j = 0,
                                                        double *keep = nullptr, const int *bofs = nullptr,
                                                        const int *bidx = nullptr)
{
    // KEEP: the first pass stores each ground state's sums (R[g,e] for e <
    // NEMAX, f_g, s_g) in this thread's slots keep[(g kKeepSlots + i) stride],
    // and the second pass reads them instead of recomputing the rates (the
    // same operations on the same inputs).  Its coefficients (alpha_ge, beta_g,
    // gamma_g) then replace them, and the triples run beam by beam through
    // the beam-major index (bofs[b] .. bofs[b + 1] into bidx, each entry
    // i | g << 16 | e << 24): each beam's dF/dfreq_b and dF/ds0_b add up in
    // registers and are stored once.  Ground-major, the shared-memory
    // accumulators indexed by each triple's beam kept the compiler from
    // overlapping consecutive triples (a store may alias the next load).
    const int n_g = EXACT ? NGMAX : P.n_g;
    const int n_e = EXACT ? NEMAX : P.n_e;
    RateCtx<NEMAX> C;
    C.B = __dmul_rn(__dmul_rn(Bgrad, z), 1e4);
    C.fd = fd;
    C.stride = stride;
    for (int b = 0; b < P.n_b; b++)
        fd[b * stride] = __dadd_rn(S.freq[b], __ddiv_rn(__dmul_rn(S.ck[b], v), MM_TWO_PI));
#pragma unroll
    for (int e = 0; e < NEMAX; e++)
        C.Ese[e] = (e < n_e) ? __dadd_rn(S.E[n_g + e], __ddiv_rn(__dmul_rn(__dmul_rn(C.B, S.zde[e]), P.Gamma),
                                                                  MM_TWO_PI))
                             : 0.0;
    const double gh = P.Gamma / 2.0, gh2 = gh * gh;

    // forward: K, cw, cf and the stationary vector
    double K[NEMAX][NEMAX], K0[NEMAX][NEMAX], cw[NEMAX], cf[NEMAX];
#pragma unroll
    for (int e = 0; e < NEMAX; e++) {
        cw[e] = 0.0;
        cf[e] = 0.0;
#pragma unroll
        for (int e2 = 0; e2 < NEMAX; e2++) K[e][e2] = 0.0;
    }
    for (int g = j; g < n_g; g += NL) {
        double Re[NEMAX], f, s;
        reduced_rates<NEMAX, PAD, true>(S, g, C, gh2, Re, f, s);
        if constexpr (KEEP) {
            double *kg = keep + (size_t)g * kKeepSlots<NEMAX> * stride;
#pragma unroll
            for (int e = 0; e < NEMAX; e++) kg[e * stride] = Re[e];
            kg[NEMAX * stride] = f;
            kg[(NEMAX + 1) * stride] = s;
        }
        double rt = 0.0;
#pragma unroll
        for (int e = 0; e < NEMAX; e++) rt += Re[e];
        const double inv = mm_rcp(rt);
        const double phi = f * inv, w = (1.0 + s) * inv;
#pragma unroll
        for (int e = 0; e < NEMAX; e++) {
            const double br = S.brt[g * NEMAX + e];
            cw[e] = fma(br, w, cw[e]);
            cf[e] = fma(br, phi, cf[e]);
#pragma unroll
            for (int e2 = 0; e2 < NEMAX; e2++) K[e2][e] = fma(Re[e2] * inv, br, K[e2][e]);
        }
    }
    if constexpr (NL > 1) {
#pragma unroll
        for (int e = 0; e < NEMAX; e++) {
            cw[e] = red_lane_sum<NL>(cw[e]);
            cf[e] = red_lane_sum<NL>(cf[e]);
#pragma unroll
            for (int e2 = 0; e2 < NEMAX; e2++) K[e][e2] = red_lane_sum<NL>(K[e][e2]);
        }
    }
#pragma unroll
    for (int i = 0; i < NEMAX; i++)
#pragma unroll
        for (int jj = 0; jj < NEMAX; jj++) K0[i][jj] = K[i][jj];
    double pi[NEMAX];
    const bool ok = gth_stationary<NEMAX>(K, n_e, pi);
    double nrm = 0.0, fn = 0.0, rn = 0.0;
#pragma unroll
    for (int e = 0; e < NEMAX; e++) {
        nrm = fma(cw[e], pi[e], nrm);
        fn = fma(cf[e], pi[e], fn);
        rn = fma(S.rsum[e], pi[e], rn);
    }
    const double in = mm_rcp(nrm);
    const double F = fn * in;

    // adjoint of the chain: lambda_0 = 0, (delta_kj - K0[j][k]) lambda_j = u_k for k, j >= 1
    double lam[NEMAX], A[NEMAX][NEMAX];
#pragma unroll
    for (int k = 0; k < NEMAX; k++) {
        lam[k] = (k >= 1 && k < n_e) ? (cf[k] - F * cw[k]) * in : 0.0;
#pragma unroll
        for (int j = 0; j < NEMAX; j++) A[k][j] = ((k == j) ? 1.0 : 0.0) - ((k < n_e && j < n_e) ? K0[j][k] : 0.0);
    }
    // elimination without pivoting on rows/columns 1..n_e-1 (an M-matrix for a
    // strongly connected chain), then back substitution
#pragma unroll
    for (int c = 1; c < NEMAX; c++) {
        if (c < n_e) {
            const double ip = mm_rcp(A[c][c]);
#pragma unroll
            for (int r = c + 1; r < NEMAX; r++) {
                if (r < n_e) {
                    const double m = A[r][c] * ip;
#pragma unroll
                    for (int j = c + 1; j < NEMAX; j++) A[r][j] = fma(-m, A[c][j], A[r][j]);
                    lam[r] = fma(-m, lam[c], lam[r]);
                }
            }
        }
    }
#pragma unroll
    for (int c = NEMAX - 1; c >= 1; c--) {
        if (c < n_e) {
            double a = lam[c];
#pragma unroll
            for (int j = c + 1; j < NEMAX; j++)
                if (j < n_e) a = fma(-A[c][j], lam[j], a);
            lam[c] = a * mm_rcp(A[c][c]);
        }
    }
    lam[0] = 0.0;

    // second pass: per ground state coefficients, then the triples once more
    gBG = 0.0;
    const double inrm = in, Fin = F * in;
    if constexpr (KEEP) {
        for (int g = j; g < n_g; g += NL) {
            double *kg = keep + (size_t)g * kKeepSlots<NEMAX> * stride;
            double Re[NEMAX];
#pragma unroll
            for (int e = 0; e < NEMAX; e++) Re[e] = kg[e * stride];
            const double f = kg[NEMAX * stride], s = kg[(NEMAX + 1) * stride];
            double rt = 0.0, yg = 0.0;
#pragma unroll
            for (int e = 0; e < NEMAX; e++) {
                rt += Re[e];
                yg = fma(S.brt[g * NEMAX + e], pi[e], yg);
            }
            const double inv = mm_rcp(rt);
            const double phi = f * inv, w = (1.0 + s) * inv;
            double Lam = 0.0;
#pragma unroll
            for (int e = 0; e < NEMAX; e++) Lam = fma(lam[e], Re[e] * inv, Lam);
            const double yi = yg * inv;
            const double common = -Lam - phi * inrm + w * Fin;
#pragma unroll
            for (int e = 0; e < NEMAX; e++) kg[e * stride] = yi * (lam[e] + common);  // alpha_ge
            kg[NEMAX * stride] = yi * inrm;                                            // beta_g
            kg[(NEMAX + 1) * stride] = -yi * Fin;                                      // gamma_g
            const double Esg = fma(C.B, S.czd[g], S.E[g]);
#pragma unroll
            for (int e = 0; e < NEMAX; e++) kg[(NEMAX + 2 + e) * stride] = __dsub_rn(C.Ese[e], Esg);  // omega_ge
        }
        const double ggh = gh * P.geff;
        for (int b = 0; b < P.n_b; b++) {
            const double fdb = fd[b * stride];
            double gfb = 0.0, gsb = 0.0;
            for (int k = bofs[b]; k < bofs[b + 1]; k++) {
                const int code = bidx[k];
                const int i = code & 0xffff, g = (code >> 16) & 0xff, e = code >> 24;
                if (NL > 1 && g % NL != j) continue;
                const TripD tr = ((const TripD *)S.trip)[i];
                const double *kg = keep + (size_t)g * kKeepSlots<NEMAX> * stride;
                const double alpha = kg[e * stride], om = kg[(NEMAX + 2 + e) * stride];
                const double beta = kg[NEMAX * stride], gamma = kg[(NEMAX + 1) * stride];
                const double de = __dmul_rn(__dsub_rn(fdb, om), MM_TWO_PI);
                const double iden = mm_rcp1(fma(de, de, gh2));  // feeds the gradient only
                const double L = gh2 * iden;
                const double dLd = -2.0 * de * L * iden;  // dL / d delta
                const double ab = alpha + beta * tr.hk;
                const double q = fma(ab, tr.c1, gamma * tr.c2);
                gfb = fma(q * dLd, MM_TWO_PI, gfb);
                // d(c1, c2)/ds0_b with d2 = c2 / s0_b written out: c1 = ((Gamma/2) s0 d2) Geff
                const double d2 = S.d2t[i];
                gsb = fma(fma(ab * ggh, d2, gamma * d2), L, gsb);
                const double dBde = -(S.zde[e] - P.zd[g]) * P.Gamma;  // d delta / dB
                gBG = fma(q * dLd, dBde, gBG);
            }
            gf[b * stride] += gfb;
            gs[b * stride] += gsb;
        }
    } else {
        for (int g = j; g < n_g; g += NL) {
            double Re[NEMAX], f, s;
            reduced_rates<NEMAX, PAD, true>(S, g, C, gh2, Re, f, s);
            double rt = 0.0, yg = 0.0;
#pragma unroll
            for (int e = 0; e < NEMAX; e++) {
                rt += Re[e];
                yg = fma(S.brt[g * NEMAX + e], pi[e], yg);
            }
            const double inv = mm_rcp(rt);
            const double phi = f * inv, w = (1.0 + s) * inv;
            double Lam = 0.0;
#pragma unroll
            for (int e = 0; e < NEMAX; e++) Lam = fma(lam[e], Re[e] * inv, Lam);
            const double yi = yg * inv;
            const double beta = yi * inrm, gamma = -yi * Fin;
            const double common = -Lam - phi * inrm + w * Fin;
            const double Esg = fma(C.B, S.czd[g], S.E[g]);
#pragma unroll
            for (int e = 0; e < NEMAX; e++) {
                const double alpha = yi * (lam[e] + common);
                const int i0 = S.offs[g * NEMAX + e], i1 = S.offs[g * NEMAX + e + 1];
                const double om = __dsub_rn(C.Ese[e], Esg);
                const double dBde = -(S.zde[e] - P.zd[g]) * P.Gamma;  // d delta / dB
                for (int i = i0; i < i1; i++) {
                    const TripD tr = ((const TripD *)S.trip)[i];
                    if (tr.pad) continue;  // list padding
                    const int b = tr.b;
                    const double de = __dmul_rn(__dsub_rn(fd[b * stride], om), MM_TWO_PI);
                    const double iden = mm_rcp1(fma(de, de, gh2));  // feeds the gradient only
                    const double L = gh2 * iden;
                    const double dLd = -2.0 * de * L * iden;  // dL / d delta
                    const double q = fma(alpha + beta * tr.hk, tr.c1, gamma * tr.c2);
                    gf[b * stride] = fma(q * dLd, MM_TWO_PI, gf[b * stride]);
                    // d(c1, c2)/ds0_b with d2 = c2 / s0_b written out: c1 = ((Gamma/2) s0 d2) Geff
                    const double d2 = S.d2t[i];
                    const double qs = fma((alpha + beta * tr.hk) * gh * P.geff, d2, gamma * d2);
                    gs[b * stride] = fma(qs, L, gs[b * stride]);
                    gBG = fma(q * dLd, dBde, gBG);
                }
            }
        }
    }
    if constexpr (NL > 1) {
        gBG = red_lane_sum<NL>(gBG);
        for (int b = 0; b < P.n_b; b++) {
            gf[b * stride] = red_lane_sum<NL>(gf[b * stride]);
            gs[b * stride] = red_lane_sum<NL>(gs[b * stride]);
        }
    }
    RedOut o;
    o.F = F;
    o.R = rn * in;
    o.status = (!ok || !isfinite(F)) ? MM_ST_NONFINITE : 0;
    return o;
}
