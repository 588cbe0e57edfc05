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
// (slot c = 0 .. CPL-1): it computes their rates and holds column k of M in
// registers.  The right-hand side b is replicated in every lane.  Pivot
// search is lane-local (the owner of the pivot column); the pivot row and
// the elimination factors are broadcast with shuffles.  Row swaps are
// predicated register moves, taken only when some group of the warp pivots
// (warp-uniform branch).  Every register-array index is a compile-time
// constant (static_for), so the matrix never leaves the register file.
//
// Exactness: the detuning chain (doppler, excited-state Zeeman shift,
// omega, delta) uses the reference's operations in its order with explicit
// round-to-nearest intrinsics and IEEE division (no FMA contraction): with
// E_e ~ 4.3e14 Hz, delta is a difference of nearly equal numbers and one
// rounding flip of an absolute frequency moves F by ~1e-8.  The ground-state
// Zeeman shift, Lorentzian, saturation, matrix build, elimination and
// reductions use FMA and Newton-refined reciprocals; they agree with the
// reference to rounding (~1e-15 of max|F|).
#pragma once
#include "common.cuh"
#include <type_traits>

// Compile-time loop: f(std::integral_constant<int, I>) for I in [B, E).
template <int B, int E, class Fn>
__device__ __forceinline__ void static_for(Fn &&f)
{
    if constexpr (B < E) {
        f(std::integral_constant<int, B>{});
        static_for<B + 1, E>(f);
    }
}

// Reciprocal by Newton-Raphson iteration y <- y (2 - d y), written as
// e = 1 - d y, y <- y + y e, started from the PTX hardware approximation
// rcp.approx.ftz.f64; two steps reach double precision (within an ulp).
// d must be a normal, finite, non-zero number.
__device__ __forceinline__ double mm_rcp(double d)
{
    double y;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(d));
    double e = fma(-d, y, 1.0);
    y = fma(y, e, y);
    e = fma(-d, y, 1.0);
    return fma(y, e, y);
}

// Reciprocal by one Newton-Raphson step from rcp.approx.ftz.f64: relative
// error about the square of the approximation's, well below 1e-12; for
// quantities that only feed derivatives (checked at 1e-8), never forces.
__device__ __forceinline__ double mm_rcp1(double d)
{
    double y;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(d));
    const double e = fma(-d, y, 1.0);
    return fma(y, e, y);
}

// Reciprocal square root by Newton-Raphson iteration y <- y (3 - x y^2) / 2,
// written as e = 1/2 - (x/2) y y, y <- y + y e, started from the PTX hardware
// approximation rsqrt.approx.ftz.f64; two steps reach double precision.
// x must be a normal, finite, positive number.
__device__ __forceinline__ double mm_rsqrt(double x)
{
    double y;
    asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
    const double h = 0.5 * x;
    double e = fma(-h * y, y, 0.5);
    y = fma(y, e, y);
    e = fma(-h * y, y, 0.5);
    return fma(y, e, y);
}

// Single-precision reciprocal: the PTX hardware approximation
// rcp.approx.ftz.f32 alone (within an ulp).  A Newton step on top of it
// changed the FP32 form's worst per-set error against FP64 by 3e-9 of
// max|F| (5.18e-7 -> 5.21e-7, the error being set by the rounding of the
// detuning u in FP32) and cost 2% of the force-map time.
__device__ __forceinline__ float mm_rcpf(float d)
{
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(d));
    return y;
}

// Active (ground k, beam b, excited e) triple of one parameter set (32 B).
struct Trip64 {
    double c1g;  // ((Gamma/2 s0_b) d2) Geff   -> rate = c1g * L
    double c2;   // s0_b d2                    -> saturation term c2 * L
    double hk;   // hbar k kdir_b              -> force term hk * rate
    int be;      // b | e << 8
    int pad;
};

// Shared-memory view of one parameter set's tables.
struct SetView {
    const double *E, *zd, *czd, *BR;  // czd[i] = zd[i] Gamma / (2 pi)
    const double *freq, *ck;          // per beam: freq, (-k) kdir
    const int *cnt, *off, *maxcnt;    // per ground state / per slot
    const Trip64 *t64;
};

// Byte layout of the dynamic shared memory of the 1D force kernels.
struct SmemLayout {
    size_t E, zd, czd, BR, freq, ck, cnt, off, maxcnt, trip, scratch, total;
    int ntrip_max, scratch_per_group;  // doubles per group

    __host__ __device__ static size_t al(size_t x) { return (x + 15) & ~size_t(15); }

    __host__ __device__ void build(int n_g, int n_e, int n_b, int cpl, int ngroups)
    {
        const int n_s = n_g + n_e;
        size_t o = 0;
        E = o;   o = al(o + sizeof(double) * n_s);
        zd = o;  o = al(o + sizeof(double) * n_s);
        czd = o; o = al(o + sizeof(double) * n_s);
        BR = o;  o = al(o + sizeof(double) * n_e * n_g);
        freq = o; o = al(o + sizeof(double) * n_b);
        ck = o;  o = al(o + sizeof(double) * n_b);
        cnt = o; o = al(o + sizeof(int) * n_g);
        off = o; o = al(o + sizeof(int) * n_g);
        maxcnt = o; o = al(o + sizeof(int) * cpl);
        // + 3 n_g: each ground state's list starts at an offset = k (mod 4), so
        // the 4 lanes of a group read records in different banks
        ntrip_max = n_g * n_b * n_e + 3 * n_g;
        trip = o; o = al(o + sizeof(Trip64) * (size_t)ntrip_max);
        // per group: doppler-shifted frequencies and excited energies;
        // a stride of 2 (mod 4) doubles puts the 8 groups of a warp in distinct banks
        scratch_per_group = ((n_b + n_e + 3) / 4) * 4 + 2;
        scratch = o; o = al(o + sizeof(double) * (size_t)scratch_per_group * ngroups);
        total = o;
    }
};

// Build the parameter-set tables (all threads of the CTA participate).
template <int G, int CPL>
__device__ void build_set_tables(const ForceParams &P, int set, unsigned char *sm,
                                 const SmemLayout &Ly, SetView &S)
{
    const int n_g = P.n_g, n_e = P.n_e, n_b = P.n_b, n_s = n_g + n_e;
    double *E = (double *)(sm + Ly.E), *zd = (double *)(sm + Ly.zd), *czd = (double *)(sm + Ly.czd);
    double *BR = (double *)(sm + Ly.BR);
    double *freq = (double *)(sm + Ly.freq), *ck = (double *)(sm + Ly.ck);
    int *cnt = (int *)(sm + Ly.cnt), *off = (int *)(sm + Ly.off), *maxcnt = (int *)(sm + Ly.maxcnt);
    Trip64 *t64 = (Trip64 *)(sm + Ly.trip);
    const int tid = threadIdx.x, nt = blockDim.x;
    const double *kdir = P.kdir + (size_t)set * n_b, *fr = P.freq + (size_t)set * n_b;
    const double *s0 = P.s0 + (size_t)set * n_b;
    const int32_t *pol = P.pol + (size_t)set * n_b;

    for (int i = tid; i < n_s; i += nt) {
        E[i] = P.E[i];
        zd[i] = P.zd[i];
        czd[i] = P.zd[i] * P.Gamma / MM_TWO_PI;
    }
    for (int i = tid; i < n_e * n_g; i += nt) BR[i] = P.BR[i];
    for (int b = tid; b < n_b; b += nt) {
        freq[b] = fr[b];
        ck[b] = __dmul_rn(-P.k, kdir[b]);  // -k_wave * kdir
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
        for (int k = 0; k < n_g; k++) {
            o += (k - o) & 3;  // o = k (mod 4): the lanes of a group read different banks
            off[k] = o;
            o += cnt[k];
        }
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
        // excited-state major, beams ascending: R[g,e] sums over b in the
        // reference's order, and the force and saturation sums of g follow the
        // order of the plain force maps (force_plain_kernel), so every plain-form
        // kernel gives the same bits for the same point
        for (int e = 0; e < n_e; e++)
            for (int b = 0; b < n_b; b++) {
                const double d2 = P.d2[(k * n_e + e) * 3 + pol[b]];
                if (d2 < 1e-15) continue;
                const double c1 = __dmul_rn(__dmul_rn(gh, s0[b]), d2);
                const double hk = __dmul_rn(__dmul_rn(P.hbar, P.k), kdir[b]);
                Trip64 tr;
                tr.c1g = c1 * P.geff;
                tr.c2 = __dmul_rn(s0[b], d2);
                tr.hk = hk;
                tr.be = b | (e << 8);
                tr.pad = 0;
                t64[o++] = tr;
            }
    }
    __syncthreads();
    S.E = E; S.zd = zd; S.czd = czd; S.BR = BR; S.freq = freq; S.ck = ck;
    S.cnt = cnt; S.off = off; S.maxcnt = maxcnt; S.t64 = t64;
}

// Result of one point, identical in every lane of the group.
struct PointOut {
    double F, R;
    int status;
    double gB;  // dF/dB' (adjoint variant only)
};

template <int NGMAX, int NEMAX, int G>
struct GroupShape {
    static constexpr int CPL = (NGMAX + G - 1) / G;  // column slots per lane
};

// One element of M' (lane t's column slot c holds column j = c*G + t): the
// same operations wherever the matrix is built, so every caller gets the same
// bits.  br[e] = BR[e, r].
template <int NGMAX, int NEMAX, int G, bool EXACT>
__device__ __forceinline__ double mprime_entry(int n_g, int r, int j, const double (&Rc)[NEMAX], double Rkc,
                                               const double (&br)[NEMAX])
{
    double a;
    if (EXACT || j < n_g) {
        a = (r == j) ? -Rkc : 0.0;
#pragma unroll
        for (int e = 0; e < NEMAX; e++) a = fma(Rc[e], br[e], a);
        if (r == n_g - 1) a = 1.0;           // normalisation row
        if (!EXACT && r >= n_g) a = 0.0;
    } else {
        a = (r == j) ? 1.0 : 0.0;            // identity padding beyond n_g
    }
    return a;
}

// Columns of M' for the group's lanes from the saturated rates (row-major
// pass; BR[e,r] read at BR[e * se + r * sr]).
template <int NGMAX, int NEMAX, int G, bool EXACT>
__device__ __forceinline__ void group_build(const ForceParams &P, const double *BR, int se, int sr, int t,
                                            const double (&R)[GroupShape<NGMAX, NEMAX, G>::CPL][NEMAX],
                                            const double (&Rk)[GroupShape<NGMAX, NEMAX, G>::CPL],
                                            double (&A)[GroupShape<NGMAX, NEMAX, G>::CPL][NGMAX])
{
    constexpr int CPL = GroupShape<NGMAX, NEMAX, G>::CPL;
    const int n_g = EXACT ? NGMAX : P.n_g;
    const int n_e = EXACT ? NEMAX : P.n_e;
#pragma unroll
    for (int r = 0; r < NGMAX; r++) {
        double br[NEMAX];
#pragma unroll
        for (int e = 0; e < NEMAX; e++) br[e] = (r < n_g && e < n_e) ? BR[e * se + r * sr] : 0.0;
#pragma unroll
        for (int c = 0; c < CPL; c++) A[c][r] = mprime_entry<NGMAX, NEMAX, G, EXACT>(n_g, r, c * G + t, R[c], Rk[c], br);
    }
}

// Population system of one point from its saturated rates (the part of the
// solve after the rates; rate_equations_jit.py:92-136), cooperatively on the
// group's G lanes: lane t owns column k = c*G + t (slot c) of
//   M'[r][k] = sum_e R[k,e] BR[e,r] - delta_rk Rk[k],  row n_g - 1 := 1
// (group_build), eliminates with partial pivoting and back-substitutes
// M' x = e_last (group_factor).  On return A holds the factors (L
// below the diagonal, U on and above it), invU the reciprocal pivots of the
// owned columns (0 below 1e-30), prows the row interchanges (also in
// `swapped` whether any was taken) and xs the unnormalised populations.
// Pivot search: partial pivoting takes row col unless some row below holds a
// strictly larger |A[r][col]|, so the owner of column col first only tests
// for such a row; the search and interchange run when some group of the warp
// found one (a warp-uniform branch).  The rows chosen are those of the plain
// search in every case.  KEEP_L = false (force without adjoint): the L factors
// are not kept, and every lane updates all of its column slots below the
// pivot row, including columns at or left of the pivot, whose entries there
// are never read again (back substitution reads U only); the elimination then
// runs without per-lane predicates.
template <int NGMAX, int NEMAX, int G, bool EXACT, bool KEEP_L = true>
__device__ __forceinline__ void group_factor(const ForceParams &P, int t, int gbase,
                                             double (&A)[GroupShape<NGMAX, NEMAX, G>::CPL][NGMAX],
                                             double (&invU)[GroupShape<NGMAX, NEMAX, G>::CPL],
                                             int (&prows)[NGMAX], bool &swapped,
                                             double (&xs)[GroupShape<NGMAX, NEMAX, G>::CPL], int &stat)
{
    constexpr int CPL = GroupShape<NGMAX, NEMAX, G>::CPL;
    constexpr unsigned FULL = 0xffffffffu;
    const int n_g = EXACT ? NGMAX : P.n_g;
    // right-hand side e_last, distributed like the columns: bs[c] = b[c*G + t]
    double bs[CPL];
#pragma unroll
    for (int c = 0; c < CPL; c++) bs[c] = (c * G + t == n_g - 1) ? 1.0 : 0.0;

    // ---------------- LU with partial pivoting ----------------
#pragma unroll
    for (int c = 0; c < CPL; c++) invU[c] = 0.0;
    swapped = false;
    static_for<0, NGMAX>([&](auto colc) {
        constexpr int col = decltype(colc)::value;
        constexpr int own = col % G, lc = col / G;
        prows[col] = col;
        if (EXACT || col < n_g) {
            bool larger = false;  // some row below holds a strictly larger |A[r][col]|
            if (t == own) {
                const double ad = fabs(A[lc][col]);
#pragma unroll
                for (int r = col + 1; r < NGMAX; r++)
                    if (EXACT || r < n_g) larger = larger || (fabs(A[lc][r]) > ad);
            }
            if (__any_sync(FULL, larger)) {
                int prow = col;
                if (t == own) {
                    double mx = fabs(A[lc][col]);
#pragma unroll
                    for (int r = col + 1; r < NGMAX; r++) {
                        const double av = fabs(A[lc][r]);
                        if ((EXACT || r < n_g) && av > mx) { mx = av; prow = r; }
                    }
                }
                prow = __shfl_sync(FULL, prow, gbase + own);
                prows[col] = prow;
                if (prow != col) swapped = true;
                if (prow != col) {
                    // rows col <-> prow through a local copy indexed at run time
                    // (rare: predicated register moves for every candidate row
                    // raised the register pressure of the whole elimination)
                    double Al[CPL][NGMAX];
#pragma unroll
                    for (int c = 0; c < CPL; c++)
#pragma unroll
                        for (int r = col; r < NGMAX; r++) Al[c][r] = A[c][r];
#pragma unroll
                    for (int c = 0; c < CPL; c++) {
                        const double tmp = Al[c][col]; Al[c][col] = Al[c][prow]; Al[c][prow] = tmp;
                    }
#pragma unroll
                    for (int c = 0; c < CPL; c++)
#pragma unroll
                        for (int r = col; r < NGMAX; r++) A[c][r] = Al[c][r];
                }
                // b[col] <-> b[prow]: b[col] sits on lane own (slot lc), b[prow] on lane prow % G
                double bp = 0.0;
#pragma unroll
                for (int c = 0; c < CPL; c++)
                    if (c * G + t == prow) bp = bs[c];
                bp = __shfl_sync(FULL, bp, gbase + prow % G);
                const double bc = __shfl_sync(FULL, bs[lc], gbase + own);
                if (prow != col) {
                    if (t == own) bs[lc] = bp;
#pragma unroll
                    for (int c = 0; c < CPL; c++)
                        if (c * G + t == prow) bs[c] = bc;
                }
            }
            double inv_e = 0.0;
            if (t == own) {
                const double pv = A[lc][col];
                const double ap = fabs(pv);
                const double y = mm_rcp(ap >= 1e-30 ? pv : 1.0);
                // elimination is skipped below 1e-30, back-substitution needs > 1e-30
                inv_e = (ap < 1e-30) ? 0.0 : y;
                invU[lc] = (ap > 1e-30) ? y : 0.0;
                if (ap < 1e-30) stat |= MM_ST_PIVOT;
            }
            const double bcol = __shfl_sync(FULL, bs[lc], gbase + own);  // b[col], final from here on
#pragma unroll
            for (int r = col + 1; r < NGMAX; r++) {
                if (EXACT || r < n_g) {
                    double f;
                    if constexpr (KEEP_L) {
                        f = 0.0;
                        if (t == own) { f = A[lc][r] * inv_e; A[lc][r] = f; }  // keep the L factor
                    } else {
                        f = A[lc][r] * inv_e;  // inv_e = 0 off the owner; only the owner's f is used
                    }
                    f = __shfl_sync(FULL, f, gbase + own);
                    static_for<0, CPL>([&](auto cc) {
                        constexpr int c = decltype(cc)::value;
                        if constexpr (c * G > col) {
                            A[c][r] = fma(-f, A[c][col], A[c][r]);
                        } else if constexpr (c * G + G - 1 > col) {
                            if constexpr (KEEP_L) {
                                if (c * G + t > col) A[c][r] = fma(-f, A[c][col], A[c][r]);
                            } else {
                                A[c][r] = fma(-f, A[c][col], A[c][r]);
                            }
                        }
                    });
                    if (r % G == t) bs[r / G] = fma(-f, bcol, bs[r / G]);
                }
            }
        }
    });

    // ---------------- back substitution ----------------
#pragma unroll
    for (int c = 0; c < CPL; c++) xs[c] = 0.0;
    static_for<0, NGMAX>([&](auto iic) {
        constexpr int i = NGMAX - 1 - decltype(iic)::value;
        constexpr int own = i % G, li = i / G;
        if (EXACT || i < n_g) {
            double part = 0.0;
            static_for<0, CPL>([&](auto cc) {
                constexpr int c = decltype(cc)::value;
                if constexpr (c * G > i) {
                    part = fma(A[c][i], xs[c], part);
                } else if constexpr (c * G + G - 1 > i) {
                    if (c * G + t > i) part = fma(A[c][i], xs[c], part);
                }
            });
            part = mm_group_sum(part, G);
            if (t == own) xs[li] = (bs[li] - part) * invU[li];
        }
    });
}

// Clamp, normalise (uniform populations when all clamp, if asked), and the
// point's force and scattering rate, identical in every lane of the group.
template <int NGMAX, int NEMAX, int G, bool EXACT>
__device__ __forceinline__ PointOut group_finish(const ForceParams &P, int t,
                                                 double (&xs)[GroupShape<NGMAX, NEMAX, G>::CPL],
                                                 const double (&Fk)[GroupShape<NGMAX, NEMAX, G>::CPL],
                                                 const double (&Rk)[GroupShape<NGMAX, NEMAX, G>::CPL],
                                                 int &stat)
{
    constexpr int CPL = GroupShape<NGMAX, NEMAX, G>::CPL;
    const int n_g = EXACT ? NGMAX : P.n_g;
    double tot = 0.0;
#pragma unroll
    for (int c = 0; c < CPL; c++) {
        const int j = c * G + t;
        if (EXACT ? (j < NGMAX) : (j < n_g)) { if (xs[c] < 0.0) xs[c] = 0.0; }
        else xs[c] = 0.0;
        tot += xs[c];
    }
    tot = mm_group_sum(tot, G);
    if (tot > 0.0) {
        const double it = mm_rcp(tot);
#pragma unroll
        for (int c = 0; c < CPL; c++) xs[c] *= it;
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
        if (EXACT ? (c * G + t < NGMAX) : (c * G + t < n_g)) {
            F = fma(xs[c], Fk[c], F);
            Rs = fma(xs[c], Rk[c], Rs);
        }
    }
    PointOut out;
    out.F = mm_group_sum(F, G);
    out.R = mm_group_sum(Rs, G);
    out.gB = 0.0;
    out.status = 0;
    return out;
}

// Multipliers of the adjoint: lambda solving M'^T lambda = F_g (the ground
// states' force terms) with the factors of group_factor<KEEP_L = true>,
// P M' = L U:  U^T w = F, L^T u = w, lambda = P^T u (replicated in every lane
// of the group), and nu[e] = sum_{g < n_g - 1} lambda_g BR[e,g].
template <int NGMAX, int NEMAX, int G, bool EXACT>
__device__ __forceinline__ void group_lambda(const ForceParams &P, const double *BR, int se, int sr, int t,
                                             int gbase,
                                             const double (&A)[GroupShape<NGMAX, NEMAX, G>::CPL][NGMAX],
                                             const double (&invU)[GroupShape<NGMAX, NEMAX, G>::CPL],
                                             const int (&prows)[NGMAX], bool swapped,
                                             const double (&Fk)[GroupShape<NGMAX, NEMAX, G>::CPL],
                                             double (&wv)[NGMAX], double (&nu)[NEMAX])
{
    constexpr unsigned FULL = 0xffffffffu;
    const int n_g = EXACT ? NGMAX : P.n_g;
    const int n_e = EXACT ? NEMAX : P.n_e;
    static_for<0, NGMAX>([&](auto ic) {
        constexpr int i = decltype(ic)::value;
        constexpr int own = i % G, li = i / G;
        double wi = 0.0;
        if (EXACT || i < n_g) {
            if (t == own) {
                double sacc = Fk[li];
#pragma unroll
                for (int j = 0; j < i; j++) sacc = fma(-A[li][j], wv[j], sacc);  // U[j][i]
                wi = sacc * invU[li];
            }
            wi = __shfl_sync(FULL, wi, gbase + own);
        }
        wv[i] = wi;
    });
    static_for<0, NGMAX>([&](auto iic) {
        constexpr int i = NGMAX - 1 - decltype(iic)::value;
        constexpr int own = i % G, li = i / G;
        if (EXACT || i < n_g) {
            double ui = 0.0;
            if (t == own) {
                double sacc = wv[i];
#pragma unroll
                for (int j = i + 1; j < NGMAX; j++)
                    if (EXACT || j < n_g) sacc = fma(-A[li][j], wv[j], sacc);  // L[j][i]
                ui = sacc;
            }
            wv[i] = __shfl_sync(FULL, ui, gbase + own);
        }
    });
    if (__any_sync(FULL, swapped)) {
#pragma unroll
        for (int col = NGMAX - 1; col >= 0; col--) {
#pragma unroll
            for (int r = col + 1; r < NGMAX; r++)
                if (r == prows[col]) { const double tmp = wv[col]; wv[col] = wv[r]; wv[r] = tmp; }
        }
    }
#pragma unroll
    for (int e = 0; e < NEMAX; e++) {
        double a = 0.0;
#pragma unroll
        for (int g = 0; g < NGMAX; g++)
            if (g < n_g - 1 && e < n_e) a = fma(wv[g], BR[e * se + g * sr], a);
        nu[e] = a;
    }
}

// Solve one point.  xs[c] receives p[c*G + t] for the owned columns.
// fd / Ese: this group's scratch (n_b + n_e doubles) in shared memory
// (FP64 form only).  EXACT: the molecule has exactly NGMAX ground and NEMAX
// excited states (size predicates vanish at compile time).
template <int NGMAX, int NEMAX, int G, bool EXACT>
__device__ __forceinline__ PointOut solve_point(const ForceParams &P, const SetView &S, double *fd,
                                                double *Ese, int t, int gbase, double v, double z,
                                                double Bgrad,
                                                double (&xs)[GroupShape<NGMAX, NEMAX, G>::CPL])
{
    constexpr int CPL = GroupShape<NGMAX, NEMAX, G>::CPL;
    const int n_g = EXACT ? NGMAX : P.n_g;
    const int n_e = EXACT ? NEMAX : P.n_e;
    const double gh = P.Gamma / 2.0;
    const double gh2 = gh * gh;
    int stat = 0;

    // ---------------- rates of the owned ground states ----------------
    double R[CPL][NEMAX];
    double Fk[CPL], Rk[CPL];
    const double B_gauss = __dmul_rn(__dmul_rn(Bgrad, z), 1e4);
    __syncwarp();
    // laser frequency seen by the moving molecule, per beam (exact order)
    for (int b = t; b < P.n_b; b += G)
        fd[b] = __dadd_rn(S.freq[b], __ddiv_rn(__dmul_rn(S.ck[b], v), MM_TWO_PI));
    // Zeeman-shifted excited energies (exact order)
    for (int e = t; e < n_e; e += G)
        Ese[e] = __dadd_rn(S.E[n_g + e], __ddiv_rn(__dmul_rn(__dmul_rn(B_gauss, S.zd[n_g + e]),
                                                             P.Gamma), MM_TWO_PI));
    __syncwarp();

#pragma unroll
    for (int c = 0; c < CPL; c++) {
        const int k = c * G + t;
        const bool own = EXACT ? (k < NGMAX) : (k < n_g);
        const int kk = own ? k : 0;
        const int cntk = own ? S.cnt[kk] : 0;
        const int o = S.off[kk];
        const int mc = S.maxcnt[c];
        double Rr[NEMAX];
#pragma unroll
        for (int e = 0; e < NEMAX; e++) Rr[e] = 0.0;
        // ground-state shift: |error| <= 1 ulp of E_g (1.5e10 Hz), i.e. 2e-6 Hz
        const double Esg = fma(B_gauss, S.czd[kk], S.E[kk]);
        double s = 0.0, f = 0.0;
#pragma unroll 2
        for (int i = 0; i < mc; i++) {
            if (i < cntk) {
                const Trip64 tr = S.t64[o + i];
                const int b = tr.be & 0xff, e = tr.be >> 8;
                const double om = __dsub_rn(Ese[e], Esg);
                const double de = __dmul_rn(__dsub_rn(fd[b], om), MM_TWO_PI);
                const double L = gh2 * mm_rcp(fma(de, de, gh2));
                const double ru = tr.c1g * L;
#pragma unroll
                for (int ee = 0; ee < NEMAX; ee++)
                    if (ee == e) Rr[ee] += ru;
                f = fma(tr.hk, ru, f);
                s = fma(tr.c2, L, s);
            }
        }
        // saturation correction 1/(1 + s_total[g]) (rate_equations_jit.py:85-90)
        const double sat = mm_rcp(1.0 + s);
        double rs = 0.0;
#pragma unroll
        for (int e = 0; e < NEMAX; e++) {
            R[c][e] = Rr[e] * sat;
            rs += R[c][e];
        }
        Rk[c] = rs;
        Fk[c] = f * sat;
    }

    double A[CPL][NGMAX], invU[CPL];
    int prows[NGMAX];
    bool swapped;
    group_build<NGMAX, NEMAX, G, EXACT>(P, S.BR, n_g, 1, t, R, Rk, A);
    group_factor<NGMAX, NEMAX, G, EXACT>(P, t, gbase, A, invU, prows, swapped, xs, stat);
    PointOut out = group_finish<NGMAX, NEMAX, G, EXACT>(P, t, xs, Fk, Rk, stat);
    if (!isfinite(out.F)) stat |= MM_ST_NONFINITE;
    out.status = mm_group_or(stat, G);
    return out;
}
