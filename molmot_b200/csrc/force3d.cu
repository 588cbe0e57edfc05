// force3d.cu -- 3D rate-equation force (quadrupole field, ground Zeeman
// eigenbasis, per-beam polarisation weights, Gaussian beams) and the fused
// 3D leapfrog ensemble with photon-recoil kicks; C-ABI entry points
// mm_force3d_batch and mm_traj3d_run.
//
// Reference: molmot/mot/simulator_3d.py:168-365 (rate_eq_force_3d, the CPU
// path with numpy eigh -- the only correct 3D reference; the reference's own
// GPU kernel, molmot_cuda/simulator_3d_cuda.py:53-562, converges to wrong
// eigenvalues) and :443-504 (simulate_trajectory_3d, leapfrog).
//
// One point per group of 16 lanes (two per warp).  Per point:
//  1. B = B'(-x/2, -y/2, z) 1e4 G;  H = B.Z (ground block), Hermitianised.
//  2. Eigen-decomposition of the complex Hermitian H in shared memory
//     (hermitian_eigen): Householder reduction to tridiagonal form (a lane per
//     row), a phase change to a real tridiagonal matrix and implicit QL
//     iterations whose scalar recurrences every lane runs on shuffled values,
//     rotating its own row of the eigenvector matrix.  Eigenvalues are sorted ascending with their
//     vectors, as numpy.linalg.eigh returns them; Es_g[i] = E_g[i] + lambda_i.
//  3. |U^H |tdm||^2 per (eigenstate, e, q); branching ratios.
//  4. Lane g accumulates, over beams and excited states, the unsaturated rates,
//     s_total[g] and the per-state force vector in one pass (the saturation
//     factor 1/(1+s_total[g]) is common to all of a state's terms).
//  5. Population matrix, Gaussian elimination with partial pivoting (lane k
//     holds column k), clamp, normalise (uniform populations if all clamp).
//  6. F = hbar k sum_b khat_b rate_b p, R = sum rate p.
#include <stdio.h>
#include <algorithm>
#include "rate_core.cuh"
#include "kicks.cuh"

namespace {

constexpr int kG3 = 16;        // lanes per point
constexpr int NBM = 32;        // max beams

// Size classes of the 3D kernels: NGM ground and NEM excited states at most,
// THREADS per CTA (8 points per CTA for SrOH-sized molecules, 4 for the
// larger class, whose per-point tables are twice as large).
template <int NGM_, int NEM_, int THREADS_>
struct C3 {
    static constexpr int NGM = NGM_, NEM = NEM_, THREADS = THREADS_;
};
using C3Small = C3<12, 4, 128>;
using C3Large = C3<16, 8, 64>;

struct Force3Params {
    int n_g, n_e, n_b, n_sets;
    double Gamma, k, hbar, geff, mass;
    const double *E, *Zre, *Zim, *Ze, *tdm;  // pack arrays
    const double *khat, *freq, *s0, *radius, *bgrad;
    const int32_t *pol;
    long long n_points, pps;
    const double *r, *v;                       // [n][3]
    double *F, *R, *pop;                       // [n][3], [n], [n][n_g]
    int32_t *status;
    int uniform_fb;
};

struct Traj3Params {
    double dt, r_escape;
    long long n_particles, n_steps, step0;
    int kicks;
    unsigned long long seed;
    const double *r0, *v0;          // [N][3]; v0 is the half-step velocity when step0 > 0
    double *r_out, *vh_out, *v_out; // [N][3]: position, half-step velocity, synchronised velocity
    int32_t *n_actual;              // [N] steps completed (escape step or n_steps)
    double *r_traj, *v_traj;        // [N][n_steps][3] or null
    double *ke_sum;                 // [N] or null: final 0.5 m |v|^2
    int32_t *n_events;              // [N] or null: scattering events drawn
};

// Per-CTA constants (molecule + one beam set) and per-group work arrays.
// The two 16-lane groups of a warp read the same offsets of their own
// Group (rotation coefficients, beam terms, ...).  Groups that sit 16 banks
// apart (sizeof % 128 == 64) make those pairs of reads conflict-free; a
// multiple of 128 bytes would put both in the same banks.
template <int NGM, int NEM, int THREADS>
struct Smem3 {
    static constexpr int LDH = NGM + 1;  // padded row length of the matrices
    double Zre[3][NGM * NGM], Zim[3][NGM * NGM];
    double tdm[NGM * NEM * 3];
    double E[NGM + NEM], Ze[NEM];
    double khat[NBM][3], freq[NBM], s0[NBM], radius[NBM];
    int pol[NBM];
    struct GroupBody {
        double Hre[NGM * LDH], Him[NGM * LDH];
        double Vre[NGM * LDH], Vim[NGM * LDH];
        double lam[NGM];
        int perm[NGM];
        double dsq[NEM * 3 * NGM];   // |U^H d|^2 at [(e * 3 + q) * NGM + a]: lanes a read consecutive doubles
        double BR[NEM * NGM];
        double Esg[NGM], Ese[NEM];
        double bm[NBM][5];           // doppler, s_eff, w0, w1, w2
    };
    static constexpr size_t kPad = (64 + 128 - sizeof(GroupBody) % 128) % 128;
    struct Group : GroupBody {
        unsigned char pad_[kPad == 0 ? 128 : kPad];
    };
    static_assert(sizeof(Group) % 128 == 64, "Group stride must be 16 banks off a 128-byte multiple");
    Group grp[THREADS / kG3];
};

__device__ __forceinline__ double gsum16(double x)
{
#pragma unroll
    for (int o = 8; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    return x;
}


// 1/sqrt(x) for x >= 0: the Newton-refined hardware approximation
// (mm_rsqrt, within an ulp) for normal x, IEEE sqrt and division otherwise
// (0, subnormal, inf).  The eigensolver's rotations and norms use it in place
// of a square root and one or two divisions.
__device__ __forceinline__ double rsqrt_any(double x)
{
    if (x >= 2.2250738585072014e-308 && x <= 1.0e300) return mm_rsqrt(x);
    return 1.0 / sqrt(x);
}

template <int NGM, int NEM, int TH>
__device__ void load_consts3(const Force3Params &P, int set, Smem3<NGM, NEM, TH> &S)
{
    const int n_g = P.n_g, n_e = P.n_e, n_b = P.n_b, tid = threadIdx.x, nt = blockDim.x;
    for (int i = tid; i < 3 * n_g * n_g; i += nt) {
        const int a = i / (n_g * n_g), rc = i % (n_g * n_g);
        S.Zre[a][rc] = P.Zre[i];
        S.Zim[a][rc] = P.Zim[i];
    }
    for (int i = tid; i < n_g * n_e * 3; i += nt) S.tdm[i] = P.tdm[i];
    for (int i = tid; i < n_g + n_e; i += nt) S.E[i] = P.E[i];
    for (int i = tid; i < n_e; i += nt) S.Ze[i] = P.Ze[i];
    const size_t o = (size_t)set * n_b;
    for (int b = tid; b < n_b; b += nt) {
        for (int c = 0; c < 3; c++) S.khat[b][c] = P.khat[(o + b) * 3 + c];
        S.freq[b] = P.freq[o + b];
        S.s0[b] = P.s0[o + b];
        S.radius[b] = P.radius ? P.radius[o + b] : 0.0;
        S.pol[b] = P.pol[o + b];
    }
}

struct Out3 {
    double F[3], R;
    int status;
};

// Lane-local values of one point kept for the tangent pass (lane t = sorted
// ground eigenstate t): unsaturated and saturated rates per excited state,
// the saturation sum and factor, the unsaturated force vector, the total rate,
// the population before the clamp, the population and the population sum.
template <int NGM, int NEM>
struct Keep3 {
    double Ru[NEM], Rs[NEM], sg, cg, Fv[3], Rk, xraw, x, tot;
    double A[NGM], invd;  // this lane's column of the eliminated population matrix, 1/pivot
    int prow[NGM];        // row interchanges of the elimination (same on every lane)
};


// Eigen-decomposition of the Hermitian H held in W.Hre / W.Him (rows and
// columns < n; lane t owns row t), by the standard route of Householder
// reduction to a Hermitian tridiagonal matrix, a diagonal phase change to a
// real symmetric tridiagonal one, and implicit QL iterations with Wilkinson
// shifts (Golub & Van Loan, Matrix Computations, 4th ed., sections 8.3.1
// and 8.3.5).  On entry W.Vre / W.Vim hold the identity; on exit column j of
// V is the unit eigenvector of eigenvalue lam_j (V = Q D Z: Q the product of
// the reflections, D the phases, Z the QL rotations), and the eigenvalues are
// sorted ascending (ties by index) into W.lam with W.perm[rank] = column, as
// numpy.linalg.eigh returns the spectrum.  Returns false when an eigenvalue
// needed more than 60 QL iterations.
//  * Reduction: lane i < n holds row i.  For column k the reflection
//    P = I - 2 v v^H (|v| = 1) maps H[k+1 .., k] to (alpha, 0, ..),
//    alpha = -e^{i arg H[k+1][k]} |H[k+1 .., k]|; the trailing block becomes
//    H - 2 v w^H - 2 w v^H with w = p - (v^H p) v, p = H v, and Q <- Q P.
//  * QL: lane i holds d_i and e_i; every lane runs the same scalar
//    recurrences on values fetched by shuffles and applies each rotation to
//    its own row of Z (in shared memory).
template <int NGM, class GroupT>
__device__ bool hermitian_eigen(GroupT &W, int t, int n)
{
    constexpr int LDH = NGM + 1;
    const bool row = t < n;
    // the Householder vector v and w = H v - (v^H H v) v live in W.dsq, which
    // is filled only after the decomposition (4 NGM <= NEM 3 NGM doubles)
    static_assert(sizeof(W.dsq) >= 4 * NGM * sizeof(double), "scratch for v and w");
    double *hvr = W.dsq, *hvi = hvr + NGM, *hwr = hvi + NGM, *hwi = hwr + NGM;
    // every step runs on every lane of the warp: the two 16-lane groups of a
    // warp hold different points and reach the shuffles and __syncwarp()
    // below together whatever their matrices; a column that is already
    // tridiagonal gets v = 0, a no-op reflection
    for (int k = 0; k + 2 < n; k++) {
        double xr = 0.0, xi = 0.0;
        if (t > k && row) { xr = W.Hre[t * LDH + k]; xi = W.Him[t * LDH + k]; }
        const double rest = gsum16((t > k + 1) ? xr * xr + xi * xi : 0.0);
        const bool act = rest > 0.0;  // the same on the 16 lanes of a group
        const double x0r = W.Hre[(k + 1) * LDH + k], x0i = W.Him[(k + 1) * LDH + k];
        const double a0s = x0r * x0r + x0i * x0i;
        const double ia0 = rsqrt_any(a0s);
        const double a0 = (a0s > 0.0) ? a0s * ia0 : 0.0;  // |x0|
        const double nxs = fma(a0, a0, rest);
        const double nx = (nxs > 0.0) ? nxs * rsqrt_any(nxs) : 0.0;
        const double phr = (a0 > 0.0) ? x0r * ia0 : 1.0, phi = (a0 > 0.0) ? x0i * ia0 : 0.0;
        // v = x - alpha e1 = x + ph nx e1, normalised: |v|^2 = rest + (a0 + nx)^2
        const double iv = act ? rsqrt_any(fma(a0 + nx, a0 + nx, rest)) : 0.0;
        if (t > k && row) {
            double vr = xr, vi = xi;
            if (t == k + 1) { vr = phr * (a0 + nx); vi = phi * (a0 + nx); }
            hvr[t] = vr * iv;
            hvi[t] = vi * iv;
        }
        __syncwarp();
        // p = H v over the trailing block (lane i: row i), K = v^H p
        double pr = 0.0, pi = 0.0;
        if (t > k && row) {
            for (int j = k + 1; j < n; j++) {
                const double hr = W.Hre[t * LDH + j], hi = W.Him[t * LDH + j];
                pr += hr * hvr[j] - hi * hvi[j];
                pi += hr * hvi[j] + hi * hvr[j];
            }
        }
        const double vtr = (t > k && row) ? hvr[t] : 0.0, vti = (t > k && row) ? hvi[t] : 0.0;
        const double Kv = gsum16(vtr * pr + vti * pi);  // Re(conj(v) p); the imaginary part is zero
        const double wr = pr - Kv * vtr, wi = pi - Kv * vti;
        if (t > k && row) { hwr[t] = wr; hwi[t] = wi; }
        __syncwarp();
        // trailing block: H[i][j] -= 2 (v_i conj(w_j) + w_i conj(v_j)); column k: (alpha, 0, ..)
        if (t > k && row) {
            for (int j = k + 1; j < n; j++) {
                const double ar = vtr * hwr[j] + vti * hwi[j], ai = vti * hwr[j] - vtr * hwi[j];
                const double br = wr * hvr[j] + wi * hvi[j], bi = wi * hvr[j] - wr * hvi[j];
                W.Hre[t * LDH + j] -= 2.0 * (ar + br);
                W.Him[t * LDH + j] -= 2.0 * (ai + bi);
            }
            if (act) {
                const double alr = -phr * nx, ali = -phi * nx;
                const double cr = (t == k + 1) ? alr : 0.0, ci = (t == k + 1) ? ali : 0.0;
                W.Hre[t * LDH + k] = cr; W.Him[t * LDH + k] = ci;
                W.Hre[k * LDH + t] = cr; W.Him[k * LDH + t] = -ci;
            }
        }
        // Q <- Q P on every row r < n: Q[r][j] -= 2 (Q v)_r conj(v_j)
        if (row) {
            double qr = 0.0, qi = 0.0;
            for (int j = k + 1; j < n; j++) {
                const double ur = W.Vre[t * LDH + j], ui = W.Vim[t * LDH + j];
                qr += ur * hvr[j] - ui * hvi[j];
                qi += ur * hvi[j] + ui * hvr[j];
            }
            for (int j = k + 1; j < n; j++) {
                W.Vre[t * LDH + j] -= 2.0 * (qr * hvr[j] + qi * hvi[j]);
                W.Vim[t * LDH + j] -= 2.0 * (qi * hvr[j] - qr * hvi[j]);
            }
        }
        __syncwarp();
    }
    // real symmetric tridiagonal: lane i holds d_i = H[i][i] and
    // e_i = |H[i+1][i]| in registers; phases delta_0 = 1,
    // delta_{i+1} = delta_i H[i+1][i] / |H[i+1][i]|
    double dr[NGM], di[NGM];
    double dl = (row) ? W.Hre[t * LDH + t] : 0.0, el = 0.0;
    double cr = 1.0, ci = 0.0;
#pragma unroll
    for (int i = 0; i < NGM; i++) {
        dr[i] = cr;
        di[i] = ci;
        if (i + 1 < n) {
            const double hr = W.Hre[(i + 1) * LDH + i], hi = W.Him[(i + 1) * LDH + i];
            const double as = hr * hr + hi * hi;
            const double ia = rsqrt_any(as);
            const double a = (as > 0.0) ? as * ia : 0.0;
            if (i == t) el = a;
            if (a > 0.0) {
                const double ur = hr * ia, ui = hi * ia;
                const double nr = cr * ur - ci * ui;
                ci = cr * ui + ci * ur;
                cr = nr;
            }
        }
    }
    __syncwarp();
    // row t of the rotation product Z, kept in row t of Hre (H is no longer needed)
    double *z = W.Hre + (row ? t : 0) * LDH;
    if (row)
        for (int j = 0; j < n; j++) z[j] = (j == t) ? 1.0 : 0.0;
    // implicit QL with Wilkinson shifts.  The recurrences run on every lane of
    // the group with d_i, e_i fetched from lane i by shuffles (an index of a
    // register array that is only known at run time would put the array in
    // local memory); lane i + 1 updates its own d, e; lane t applies each
    // rotation to its row of Z.  All control flow is uniform over the group
    // (it depends only on shuffled values), and the two groups of a warp may
    // take different paths: the shuffles name this group's 16 lanes only.
    const unsigned gmask = 0xffffu << (threadIdx.x & 16);
    bool ok = true;
    for (int l = 0; l < n; l++) {
        for (int iter = 0;; iter++) {
            // m = the first index >= l with a negligible e_m (n - 1 if none)
            const double dn = __shfl_down_sync(gmask, dl, 1, 16);
            const bool small = (t + 1 < n) && t >= l &&
                               fabs(el) <= 2.220446049250313e-16 * (fabs(dl) + fabs(dn));
            const unsigned bal = (__ballot_sync(gmask, small) >> (threadIdx.x & 16)) & 0xffffu;
            const int m = bal ? __ffs(bal) - 1 : n - 1;
            if (m == l) break;
            if (iter == 60) { ok = false; break; }
            const double d_l = __shfl_sync(gmask, dl, l, 16), d_l1 = __shfl_sync(gmask, dl, l + 1, 16);
            const double e_l = __shfl_sync(gmask, el, l, 16), d_m = __shfl_sync(gmask, dl, m, 16);
            double g = (d_l1 - d_l) / (2.0 * e_l);
            double r = sqrt(fma(g, g, 1.0));
            g = d_m - d_l + e_l / (g + copysign(r, g));
            double s = 1.0, c = 1.0, p = 0.0;
            double dnext = d_m;  // d_{i+1} before this sweep
            bool defl = false;
            for (int i = m - 1; i >= l; i--) {
                const double ei = __shfl_sync(gmask, el, i, 16), dii = __shfl_sync(gmask, dl, i, 16);
                const double f = s * ei, b = c * ei;
                const double rs = fma(f, f, g * g);
                if (rs == 0.0) {  // deflation: the rotation vanished
                    if (t == i + 1) { el = 0.0; dl -= p; }
                    if (t == m) el = 0.0;
                    defl = true;
                    break;
                }
                const double ir = rsqrt_any(rs);
                r = rs * ir;
                if (t == i + 1) el = r;
                s = f * ir;
                c = g * ir;
                g = dnext - p;
                r = (dii - g) * s + 2.0 * c * b;
                p = s * r;
                if (t == i + 1) dl = g + p;
                g = c * r - b;
                if (row) {
                    const double z1 = z[i + 1], z0 = z[i];
                    z[i + 1] = fma(s, z0, c * z1);
                    z[i] = fma(c, z0, -s * z1);
                }
                dnext = dii;
            }
            if (defl) continue;
            if (t == l) { dl -= p; el = g; }
            if (t == m) el = 0.0;
        }
    }
    __syncwarp();
    // V <- Q D Z (Z rows in Hre)
    if (row) {
        double qr[NGM], qi[NGM];
#pragma unroll
        for (int k = 0; k < NGM; k++) {  // Q[t][k] delta_k
            const double ur = (k < n) ? W.Vre[t * LDH + k] : 0.0, ui = (k < n) ? W.Vim[t * LDH + k] : 0.0;
            qr[k] = ur * dr[k] - ui * di[k];
            qi[k] = ur * di[k] + ui * dr[k];
        }
        for (int j = 0; j < n; j++) {
            double ar = 0.0, ai = 0.0;
#pragma unroll
            for (int k = 0; k < NGM; k++)
                if (k < n) {
                    const double zk = W.Hre[k * LDH + j];
                    ar = fma(qr[k], zk, ar);
                    ai = fma(qi[k], zk, ai);
                }
            W.Vre[t * LDH + j] = ar;
            W.Vim[t * LDH + j] = ai;
        }
    }
    // ascending order (ties by index); n is the same on both groups of the warp
    int rank = 0;
    for (int j = 0; j < n; j++) {
        const double dj = __shfl_sync(0xffffffffu, dl, j, 16);
        rank += (dj < dl || (dj == dl && j < t)) ? 1 : 0;
    }
    if (row) {
        W.perm[rank] = t;
        W.lam[rank] = dl;
    }
    __syncwarp();
    return ok;
}

// The 3D force at (r, v) for the group of 16 lanes (lane t, base gbase).
// pl receives the population of ground state t (t < n_g).
template <int NGM, int NEM, int TH>
__device__ Out3 force3d_point(const Force3Params &P, Smem3<NGM, NEM, TH> &S,
                              typename Smem3<NGM, NEM, TH>::Group &W, int t, int gbase,
                              const double r[3], const double v[3], double Bg, double &pl,
                              Keep3<NGM, NEM> *kp = nullptr)
{
    constexpr int LDH = NGM + 1;
    constexpr unsigned FULL = 0xffffffffu;
    const int n_g = P.n_g, n_e = P.n_e, n_b = P.n_b;
    const double G = P.Gamma;
    int stat = 0;

    // 1. field and Hermitian Zeeman matrix, padded to NGM x NGM with zero rows
    //    and columns beyond n_g (a padded state couples to nothing, so no
    //    rotation ever touches it, and it is left out of the spectrum)
    const double B0 = ((-Bg * r[0]) / 2.0) * 1e4;
    const double B1 = ((-Bg * r[1]) / 2.0) * 1e4;
    const double B2 = (Bg * r[2]) * 1e4;
    const double Bm = sqrt(B0 * B0 + B1 * B1 + B2 * B2);
    // only the z component of B_hat enters the polarisation weights (cos theta)
    const double bh2 = (Bm > 1e-10) ? B2 / Bm : 1.0;
    __syncwarp();
    if (t < NGM) {  // lane t writes column t
#pragma unroll
        for (int i = 0; i < NGM; i++) {
            double hr = 0.0, hi = 0.0;
            if (i < n_g && t < n_g) {
                const int ij = i * n_g + t, ji = t * n_g + i;
                const double ar = (B0 * S.Zre[0][ij] + B1 * S.Zre[1][ij]) + B2 * S.Zre[2][ij];
                const double ai = (B0 * S.Zim[0][ij] + B1 * S.Zim[1][ij]) + B2 * S.Zim[2][ij];
                const double br = (B0 * S.Zre[0][ji] + B1 * S.Zre[1][ji]) + B2 * S.Zre[2][ji];
                const double bi = (B0 * S.Zim[0][ji] + B1 * S.Zim[1][ji]) + B2 * S.Zim[2][ji];
                hr = 0.5 * (ar + br);  // 0.5 (H + H^H)
                hi = 0.5 * (ai - bi);
            }
            W.Hre[i * LDH + t] = hr;
            W.Him[i * LDH + t] = hi;
            W.Vre[i * LDH + t] = (i == t) ? 1.0 : 0.0;
            W.Vim[i * LDH + t] = 0.0;
        }
    }
    __syncwarp();

    // 2. eigenvalues (ascending) and eigenvectors of the ground Zeeman block
    if (!hermitian_eigen<NGM>(W, t, n_g)) stat |= MM_ST_NONFINITE;
    // 3. energies and |U^H d|^2 in the eigenbasis (lane a = sorted eigenstate)
    if (t < n_g) W.Esg[t] = S.E[t] + W.lam[t] * G / (2 * MM_PI);
    if (t < n_e)  // exact order of simulator_3d.py:241-243
        W.Ese[t] = __dadd_rn(S.E[n_g + t], __ddiv_rn(__dmul_rn(__dmul_rn(B2, S.Ze[t]), G), MM_TWO_PI));
    double rowsum[NEM];
#pragma unroll
    for (int e = 0; e < NEM; e++) rowsum[e] = 0.0;
    if (t < n_g) {
        const int col = W.perm[t];
#pragma unroll
        for (int e = 0; e < NEM; e++) {
            if (e >= n_e) continue;
            for (int q = 0; q < 3; q++) {
                double ar = 0.0, ai = 0.0;
                for (int g = 0; g < n_g; g++) {
                    const double d = S.tdm[(g * n_e + e) * 3 + q];
                    ar += W.Vre[g * LDH + col] * d;   // conj(U[g, col]) d
                    ai -= W.Vim[g * LDH + col] * d;
                }
                const double d2 = ar * ar + ai * ai;
                W.dsq[(e * 3 + q) * NGM + t] = d2;
                rowsum[e] += d2;
            }
        }
    }
    // branching ratios BR[e][a] = sum_q dsq[a,e,q] / sum_{a,q} dsq[a,e,q]
#pragma unroll
    for (int e = 0; e < NEM; e++) {
        const double tot = gsum16(rowsum[e]);
        if (t < n_g && e < n_e) W.BR[e * n_g + t] = tot > 1e-30 ? rowsum[e] / tot : 0.0;
    }
    // per-beam doppler, Gaussian-weighted s0 and local polarisation weights
    const double ct = fmin(fmax(bh2, -1.0), 1.0);
    const double st = sin(acos(ct));
    const double wd = ((1 + ct) / 2) * ((1 + ct) / 2), wo = ((1 - ct) / 2) * ((1 - ct) / 2);
    const double wm = (st / sqrt(2.0)) * (st / sqrt(2.0)), wc = ct * ct;
    for (int b = t; b < n_b; b += kG3) {
        // doppler -k (khat . v) / 2pi in the reference's uncontracted order
        const double kv = __dadd_rn(__dadd_rn(__dmul_rn(S.khat[b][0], v[0]), __dmul_rn(S.khat[b][1], v[1])),
                                    __dmul_rn(S.khat[b][2], v[2]));
        W.bm[b][0] = __ddiv_rn(__dmul_rn(-P.k, kv), MM_TWO_PI);
        double gf = 1.0;
        if (S.radius[b] > 0.0) {
            const double rp = r[0] * S.khat[b][0] + r[1] * S.khat[b][1] + r[2] * S.khat[b][2];
            const double rps = fmax((r[0] * r[0] + r[1] * r[1] + r[2] * r[2]) - rp * rp, 0.0);
            gf = exp(-2.0 * rps / (S.radius[b] * S.radius[b]));
        }
        W.bm[b][1] = S.s0[b] * gf;
        // column q of |d^1(theta)|^2 (rows m_local = -1, 0, +1), normalised
        const int q = S.pol[b];
        double w0, w1, w2;
        if (q == 0) { w0 = wd; w1 = wm; w2 = wo; }
        else if (q == 1) { w0 = wm; w1 = wc; w2 = wm; }
        else { w0 = wo; w1 = wm; w2 = wd; }
        const double ws = w0 + w1 + w2;
        if (ws > 1e-15) { w0 /= ws; w1 /= ws; w2 /= ws; }
        W.bm[b][2] = w0; W.bm[b][3] = w1; W.bm[b][4] = w2;
    }
    __syncwarp();

    // 4. rates of ground eigenstate g = t, one pass over beams and excited states
    const double gh = G / 2.0, gh2 = gh * gh;
    double Racc[NEM], Fv[3] = {0.0, 0.0, 0.0}, sg = 0.0;
#pragma unroll
    for (int e = 0; e < NEM; e++) Racc[e] = 0.0;
    if (t < n_g) {
        const double Eg = W.Esg[t];
        // per-state constants of the beam loop, in registers: the transition
        // frequencies and |x|^2 (0 below the 1e-15 cut, which adds an exact 0)
        double om[NEM], d2m[NEM][3];
#pragma unroll
        for (int e = 0; e < NEM; e++) {
            om[e] = (e < n_e) ? __dsub_rn(W.Ese[e], Eg) : 0.0;
#pragma unroll
            for (int q = 0; q < 3; q++) {
                const double d2 = (e < n_e) ? W.dsq[(e * 3 + q) * NGM + t] : 0.0;
                d2m[e][q] = (d2 >= 1e-15) ? d2 : 0.0;
            }
        }
        for (int b = 0; b < n_b; b++) {
            const double fd = __dadd_rn(S.freq[b], W.bm[b][0]);
            const double se = W.bm[b][1];
            const double w0 = W.bm[b][2], w1 = W.bm[b][3], w2 = W.bm[b][4];
            double Qb = 0.0;
#pragma unroll
            for (int e = 0; e < NEM; e++) {
                if (e < n_e) {
                    const double de = __dmul_rn(__dsub_rn(fd, om[e]), MM_TWO_PI);
                    const double L = gh2 * mm_rcp(fma(de, de, gh2));
                    double ws = 0.0;
                    ws = fma(w0, d2m[e][0], ws);
                    ws = fma(w1, d2m[e][1], ws);
                    ws = fma(w2, d2m[e][2], ws);
                    const double rb = ws * L * se;
                    Racc[e] += rb;
                    Qb += rb;
                }
            }
            sg += Qb;
            Fv[0] = fma(S.khat[b][0], Qb, Fv[0]);
            Fv[1] = fma(S.khat[b][1], Qb, Fv[1]);
            Fv[2] = fma(S.khat[b][2], Qb, Fv[2]);
        }
    }
    const double cg = gh * P.geff * mm_rcp(1.0 + sg);  // rate = cg * unsaturated sum
    if (kp) {
#pragma unroll
        for (int e = 0; e < NEM; e++) kp->Ru[e] = Racc[e];
        kp->sg = sg;
        kp->cg = cg;
        for (int c = 0; c < 3; c++) kp->Fv[c] = Fv[c];
    }
    double Rk = 0.0;
#pragma unroll
    for (int e = 0; e < NEM; e++) { Racc[e] *= cg; Rk += Racc[e]; }
    if (kp) {
#pragma unroll
        for (int e = 0; e < NEM; e++) kp->Rs[e] = Racc[e];
        kp->Rk = Rk;
    }

    // 5. population matrix (lane k owns column k), elimination, back substitution
    double A[NGM], bv[NGM];
#pragma unroll
    for (int i = 0; i < NGM; i++) {
        double a = 0.0;
        if (t < n_g && i < n_g) {
            a = (i == t) ? -Rk : 0.0;
#pragma unroll
            for (int e = 0; e < NEM; e++)
                if (e < n_e) a = fma(Racc[e], W.BR[e * n_g + i], a);
            if (i == n_g - 1) a = 1.0;
        } else if (i == t) {
            a = 1.0;  // identity padding
        }
        A[i] = a;
        bv[i] = (i == n_g - 1) ? 1.0 : 0.0;
    }
    double invd = 0.0;
    // static_for keeps every index of A and bv a compile-time constant (a
    // plain unrolled loop left them in local memory in one size class)
    static_for<0, NGM>([&](auto colc) {
        constexpr int col = decltype(colc)::value;
        if (col < n_g) {
            int prow = col;
            if (t == col) {
                double mx = fabs(A[col]);
#pragma unroll
                for (int rr = col + 1; rr < NGM; rr++)
                    if (rr < n_g && fabs(A[rr]) > mx) { mx = fabs(A[rr]); prow = rr; }
            }
            prow = __shfl_sync(FULL, prow, gbase + col);
            if (kp) kp->prow[col] = prow;
            if (__any_sync(FULL, prow != col)) {
#pragma unroll
                for (int rr = col + 1; rr < NGM; rr++)
                    if (rr == prow) {
                        double x = A[col]; A[col] = A[rr]; A[rr] = x;
                        x = bv[col]; bv[col] = bv[rr]; bv[rr] = x;
                    }
            }
            double inv_e = 0.0;
            if (t == col) {
                const double ap = fabs(A[col]);
                const double y = mm_rcp(ap >= 1e-30 ? A[col] : 1.0);
                inv_e = ap < 1e-30 ? 0.0 : y;
                invd = ap > 1e-30 ? y : 0.0;
                if (ap < 1e-30) stat |= MM_ST_PIVOT;
            }
#pragma unroll
            for (int rr = col + 1; rr < NGM; rr++) {
                if (rr < n_g) {
                    double f = (t == col) ? A[rr] * inv_e : 0.0;
                    f = __shfl_sync(FULL, f, gbase + col);
                    if (t > col) A[rr] = fma(-f, A[col], A[rr]);
                    bv[rr] = fma(-f, bv[col], bv[rr]);
                }
            }
        }
    });
    double x = 0.0;
    static_for<0, NGM>([&](auto iic) {
        constexpr int i = NGM - 1 - decltype(iic)::value;
        if (i < n_g) {
            double part = (t > i && t < n_g) ? A[i] * x : 0.0;
            part = gsum16(part);
            if (t == i) x = (bv[i] - part) * invd;
        }
    });
    if (kp) {
        kp->xraw = (t < n_g) ? x : 0.0;
#pragma unroll
        for (int i = 0; i < NGM; i++) kp->A[i] = A[i];
        kp->invd = invd;
    }
    if (t >= n_g || x < 0.0) x = 0.0;
    const double tot = gsum16(x);
    if (tot > 0.0) x *= mm_rcp(tot);
    else {
        stat |= MM_ST_ZERO_POP;
        if (P.uniform_fb) x = (t < n_g) ? 1.0 / n_g : 0.0;
    }
    pl = x;
    if (kp) { kp->x = x; kp->tot = tot; }
    // 6. force and scattering rate
    const double hk = P.hbar * P.k;
    Out3 o;
    const double wgt = (t < n_g) ? x * cg : 0.0;
    o.F[0] = hk * gsum16(wgt * Fv[0]);
    o.F[1] = hk * gsum16(wgt * Fv[1]);
    o.F[2] = hk * gsum16(wgt * Fv[2]);
    o.R = gsum16((t < n_g) ? x * Rk : 0.0);
    if (!isfinite(o.F[0]) || !isfinite(o.F[1]) || !isfinite(o.F[2])) stat |= MM_ST_NONFINITE;
    o.status = stat;
    for (int off = 8; off > 0; off >>= 1) o.status |= __shfl_xor_sync(FULL, o.status, off);
    return o;
}

template <int NGM, int NEM, int TH>
__global__ void __launch_bounds__(TH)
force3d_kernel(Force3Params P)
{
    extern __shared__ __align__(16) unsigned char smraw[];
    auto &S = *reinterpret_cast<Smem3<NGM, NEM, TH> *>(smraw);
    const int lane = threadIdx.x & 31, t = lane % kG3, gbase = lane - t;
    const int group = threadIdx.x / kG3, ngroups = TH / kG3;
    for (int set = blockIdx.y; set < P.n_sets; set += gridDim.y) {
        const long long first = (long long)set * P.pps;
        long long count = P.pps;
        if (first + count > P.n_points) count = P.n_points - first;
        if (count <= 0) continue;
        __syncthreads();
        load_consts3(P, set, S);
        __syncthreads();
        const double Bg = P.bgrad[set];
        for (long long base = (long long)blockIdx.x * ngroups; base < count;
             base += (long long)gridDim.x * ngroups) {
            const long long ip = base + group;
            const bool valid = ip < count;
            const long long gi = first + (valid ? ip : 0);
            double r[3], v[3], pl;
            for (int c = 0; c < 3; c++) { r[c] = P.r[gi * 3 + c]; v[c] = P.v[gi * 3 + c]; }
            const Out3 o = force3d_point(P, S, S.grp[group], t, gbase, r, v, Bg, pl);
            if (valid) {
                if (t == 0) {
                    for (int c = 0; c < 3; c++) P.F[gi * 3 + c] = o.F[c];
                    if (P.R) P.R[gi] = o.R;
                    if (P.status) P.status[gi] = o.status;
                }
                if (P.pop && t < P.n_g) P.pop[gi * P.n_g + t] = pl;
            }
        }
    }
}

// Leapfrog ensemble (simulator_3d.py:443-504):
//   v_1/2 = v_0 + (0.5 dt) F(r_0, v_0)/m;  r_j = r_{j-1} + dt v_half;
//   escape when |r_j| > r_escape (position and half-step velocity freeze);
//   F = F(r_j, v_half); v_new = v_half + dt F/m (+ recoil kick); v_j = (v_half + v_new)/2.
template <int NGM, int NEM, int TH>
__global__ void __launch_bounds__(TH)
traj3d_kernel(Force3Params P, Traj3Params T)
{
    extern __shared__ __align__(16) unsigned char smraw[];
    auto &S = *reinterpret_cast<Smem3<NGM, NEM, TH> *>(smraw);
    const int lane = threadIdx.x & 31, t = lane % kG3, gbase = lane - t;
    const int group = threadIdx.x / kG3, ngroups = TH / kG3;
    load_consts3(P, 0, S);
    __syncthreads();
    const double Bg = P.bgrad[0];
    const double m = P.mass, dt = T.dt;
    const double v_rec = P.hbar * P.k / m;
    const long long ip = (long long)blockIdx.x * ngroups + group;
    const bool valid = ip < T.n_particles;
    const long long ipc = valid ? ip : 0;
    double r[3], vh[3], vs[3], pl;
    for (int c = 0; c < 3; c++) { r[c] = T.r0[ipc * 3 + c]; vh[c] = T.v0[ipc * 3 + c]; vs[c] = vh[c]; }
    bool done = !valid;
    long long na = T.step0 + T.n_steps;
    long long nev = 0;
    const long long row = ipc * T.n_steps * 3;
    if (T.step0 == 0 && valid && T.r_traj && t == 0)
        for (int c = 0; c < 3; c++) { T.r_traj[row + c] = r[c]; T.v_traj[row + c] = vh[c]; }
    // iteration j = 0 (a run from step 0) is the first half kick at (r0, v0);
    // it shares the loop's single inlined force evaluation (two call sites
    // doubled the kernel's code and its instruction-cache misses)
    const long long j0 = (T.step0 == 0) ? 0 : T.step0;
    const long long j1 = T.step0 + T.n_steps;
    for (long long j = j0; j < j1; j++) {
        if (__all_sync(0xffffffffu, done)) break;
        const bool kick0 = j == 0;  // the same on every lane
        double rn[3];
        for (int c = 0; c < 3; c++) rn[c] = kick0 ? r[c] : __dadd_rn(r[c], __dmul_rn(dt, vh[c]));  // r + dt v_half
        const double rr = sqrt(rn[0] * rn[0] + rn[1] * rn[1] + rn[2] * rn[2]);
        const bool esc = !done && !kick0 && rr > T.r_escape;
        const Out3 o = force3d_point(P, S, S.grp[group], t, gbase, rn, vh, Bg, pl);
        if (kick0) {
            for (int c = 0; c < 3; c++) vh[c] = vh[c] + 0.5 * dt * o.F[c] / m;
            continue;
        }
        if (!done) {
            for (int c = 0; c < 3; c++) r[c] = rn[c];
            const long long out_j = j - T.step0;
            if (esc) {
                na = j;
                done = true;
                for (int c = 0; c < 3; c++) vs[c] = vh[c];
                if (T.r_traj && t == 0)
                    for (long long s = out_j; s < T.n_steps; s++)
                        for (int c = 0; c < 3; c++) {
                            T.r_traj[row + s * 3 + c] = r[c];
                            T.v_traj[row + s * 3 + c] = vh[c];
                        }
            } else {
                double vn[3];
                for (int c = 0; c < 3; c++) vn[c] = vh[c] + dt * o.F[c] / m;
                if (T.kicks) {
                    double kick[3];
                    nev += recoil_kick(T.seed, (unsigned)ip, (unsigned)j, o.R * dt, v_rec, kick);
                    for (int c = 0; c < 3; c++) vn[c] += kick[c];
                }
                for (int c = 0; c < 3; c++) { vs[c] = 0.5 * (vh[c] + vn[c]); vh[c] = vn[c]; }
                if (T.r_traj && t == 0)
                    for (int c = 0; c < 3; c++) {
                        T.r_traj[row + out_j * 3 + c] = r[c];
                        T.v_traj[row + out_j * 3 + c] = vs[c];
                    }
            }
        }
    }
    if (valid && t == 0) {
        for (int c = 0; c < 3; c++) {
            T.r_out[ip * 3 + c] = r[c];
            T.vh_out[ip * 3 + c] = vh[c];
            if (T.v_out) T.v_out[ip * 3 + c] = vs[c];
        }
        T.n_actual[ip] = (int32_t)na;
        if (T.ke_sum) T.ke_sum[ip] = 0.5 * m * (vs[0] * vs[0] + vs[1] * vs[1] + vs[2] * vs[2]);
        if (T.n_events) T.n_events[ip] = (int32_t)nev;
    }
}

// ---------------------------------------------------------------------------
// Trajectory tangents of the 3D leapfrog (forward mode): d(r, v)/d theta_k for
// parameters theta_k that add to beam frequencies (freq_par), saturation
// parameters (s0_par) and B' (bprime_par), through the 24-beam force
// including the field dependence of the ground Zeeman eigenbasis.  With H =
// B.Zh (Zh = Hermitian part of the Zeeman blocks) and a non-degenerate
// spectrum, first-order perturbation theory gives, in the sorted eigenbasis,
//   d lambda_a = Re Y[a][a],   d x_{a,j} = sum_{b != a} conj(Y[b][a]) / (lambda_a - lambda_b) x_{b,j},
// Y = V^H dH V, x_{a,j} = v_a^H |tdm_j| (j = (e, q)); |x|^2 and the branching
// ratios follow.  The rates, saturation, population solve (the forward's own
// LU factors, M dx = -dM x) and the force are differentiated term by term.
// A gap |lambda_a - lambda_b| below gap_tol max|lambda| makes the eigenbasis
// (and dF/dr) undefined: the step's terms through that pair are dropped and
// the particle's status gets MM_ST_DEGENERATE.

struct Tg3Params {
    double dt, r_escape, mass, v_rec, gap_tol;
    long long n_particles, n_steps, step0, ckpt_every;
    int n_par, kicks, bprime_par;
    unsigned long long seed;
    signed char freq_par[NBM], s0_par[NBM];
    double *state;      // [N][6 + 6 n_par]: r, vh, dr[3][n_par], dvh[3][n_par] (in/out)
    double *vsync;      // [N][3 + 3 n_par]: synchronised velocity and its tangent (out)
    int32_t *n_actual;  // [N] in/out
    int32_t *status;    // [N] out
    int32_t *n_events;  // [N] out or null
    double *ckpt;       // [n_steps / ckpt_every][N][6 + 6 n_par] or null
};

constexpr int kT3MaxPar = MM_TGRAD_MAX_PAR;
constexpr int kT3Threads = 64;  // 4 particles per CTA (the tangent workspace is large)

// Per-group workspace of the tangent pass.
template <int NGM, int NEM>
struct Tan3Work {
    double Yre[NGM][3][NGM], Yim[NGM][3][NGM];  // lane a: column a of V^H Zh_c V (sorted basis)
    double xr[NGM][NEM * 3], xi[NGM][NEM * 3];  // x_{a, e*3+q}
    double LU[NGM][NGM];                         // the forward's factors, row i, column j
    double invd[NGM];
    double dBR[NEM][NGM];
    double dbm[NBM][5];                          // per beam: d doppler, d s_eff, d w0..w2
    double dr[kT3MaxPar][3], dv[kT3MaxPar][3];   // the direction of each parameter's tangent
    double dF[kT3MaxPar][3];
    double Tr[3][kT3MaxPar], Tv[3][kT3MaxPar], Tvs[3][kT3MaxPar];
    double pad_[2];
};

// dF/d theta_k (k < n_par) at (r, v) along the directions TW.dr[k], TW.dv[k]
// (the tangents of the force's position and velocity arguments), written to
// TW.dF[k] by lane 0.  Runs after force3d_point(..., kp) on the same point
// (its shared tables W and lane values kp).  Every lane of the warp calls it.
template <int NGM, int NEM, int TH>
__device__ void force3d_tangent(const Force3Params &P, const Tg3Params &T, Smem3<NGM, NEM, TH> &S,
                                typename Smem3<NGM, NEM, TH>::Group &W, Tan3Work<NGM, NEM> &TW, int t,
                                const double r[3], const double v[3], double Bg,
                                const Keep3<NGM, NEM> &kp, int &stat)
{
    constexpr int LDH = NGM + 1;
    const int n_g = P.n_g, n_e = P.n_e, n_b = P.n_b;
    const double G = P.Gamma, gh = G / 2.0, gh2 = gh * gh;
    const bool lane = t < n_g;
    const int ca = lane ? W.perm[t] : 0;
    // field and its direction
    const double Bd[3] = {((-r[0]) / 2.0) * 1e4, ((-r[1]) / 2.0) * 1e4, r[2] * 1e4};  // dB/dB'
    const double B[3] = {Bg * Bd[0], Bg * Bd[1], Bg * Bd[2]};
    const double Bm = sqrt(B[0] * B[0] + B[1] * B[1] + B[2] * B[2]);
    const double bh2 = (Bm > 1e-10) ? B[2] / Bm : 1.0;
    const double ct = fmin(fmax(bh2, -1.0), 1.0);
    // 1. x_{a,j} and column a of Y_c = V^H Zh_c V, once per point
    if (lane) {
        for (int e = 0; e < n_e; e++)
            for (int q = 0; q < 3; q++) {
                double ar = 0.0, ai = 0.0;
                for (int g = 0; g < n_g; g++) {
                    const double d = S.tdm[(g * n_e + e) * 3 + q];
                    ar += W.Vre[g * LDH + ca] * d;
                    ai -= W.Vim[g * LDH + ca] * d;
                }
                TW.xr[t][e * 3 + q] = ar;
                TW.xi[t][e * 3 + q] = ai;
            }
        for (int c = 0; c < 3; c++) {
            double wr[NGM], wi[NGM];
#pragma unroll
            for (int g = 0; g < NGM; g++) {
                double ar = 0.0, ai = 0.0;
                if (g < n_g) {
                    for (int h = 0; h < n_g; h++) {
                        // Zh[g][h] = (Z[g][h] + conj(Z[h][g])) / 2
                        const double zr = 0.5 * (S.Zre[c][g * n_g + h] + S.Zre[c][h * n_g + g]);
                        const double zi = 0.5 * (S.Zim[c][g * n_g + h] - S.Zim[c][h * n_g + g]);
                        const double vr = W.Vre[h * LDH + ca], vi = W.Vim[h * LDH + ca];
                        ar += zr * vr - zi * vi;
                        ai += zr * vi + zi * vr;
                    }
                }
                wr[g] = ar;
                wi[g] = ai;
            }
            for (int b = 0; b < n_g; b++) {
                const int cb = W.perm[b];
                double yr = 0.0, yi = 0.0;
#pragma unroll
                for (int g = 0; g < NGM; g++) {
                    if (g < n_g) {  // conj(V[g][cb]) w[g]
                        const double vr = W.Vre[g * LDH + cb], vi = W.Vim[g * LDH + cb];
                        yr += vr * wr[g] + vi * wi[g];
                        yi += vr * wi[g] - vi * wr[g];
                    }
                }
                TW.Yre[t][c][b] = yr;
                TW.Yim[t][c][b] = yi;
            }
        }
        // the forward's population factors, column t
#pragma unroll
        for (int i = 0; i < NGM; i++)  // compile-time indices keep kp in registers
            if (i < n_g) TW.LU[i][t] = kp.A[i];
        TW.invd[t] = kp.invd;
    }
    __syncwarp();
    double lmax = 0.0;
    for (int a = 0; a < n_g; a++) lmax = fmax(lmax, fabs(W.lam[a]));
    const double gap_min = T.gap_tol * lmax;
    // excited-state totals of |x|^2 (the branching ratios' denominators)
    double tot_e[NEM];
#pragma unroll
    for (int e = 0; e < NEM; e++) {
        double a = 0.0;
        if (e < n_e && lane)
            for (int q = 0; q < 3; q++) a += W.dsq[(e * 3 + q) * NGM + t];
        tot_e[e] = gsum16(a);
    }
    const double hk = P.hbar * P.k;
    for (int k = 0; k < T.n_par; k++) {
        const double *dr = TW.dr[k], *dv = TW.dv[k];
        const double dBg = (k == T.bprime_par) ? 1.0 : 0.0;
        const double dB[3] = {dBg * Bd[0] + Bg * (((-dr[0]) / 2.0) * 1e4), dBg * Bd[1] + Bg * (((-dr[1]) / 2.0) * 1e4),
                              dBg * Bd[2] + Bg * (dr[2] * 1e4)};
        double dct = 0.0;
        if (Bm > 1e-10 && bh2 > -1.0 && bh2 < 1.0) {
            const double dBm = (B[0] * dB[0] + B[1] * dB[1] + B[2] * dB[2]) / Bm;
            dct = (dB[2] - bh2 * dBm) / Bm;
        }
        // 2. eigenvalue and |x|^2 tangents of lane a = t
        double dlam = 0.0, ddsq[NEM * 3];
#pragma unroll
        for (int j = 0; j < NEM * 3; j++) ddsq[j] = 0.0;
        if (lane) {
            dlam = dB[0] * TW.Yre[t][0][t] + dB[1] * TW.Yre[t][1][t] + dB[2] * TW.Yre[t][2][t];
            double dxr[NEM * 3], dxi[NEM * 3];
#pragma unroll
            for (int j = 0; j < NEM * 3; j++) { dxr[j] = 0.0; dxi[j] = 0.0; }
            for (int b = 0; b < n_g; b++) {
                if (b == t) continue;
                const double gap = W.lam[t] - W.lam[b];
                if (!(fabs(gap) > gap_min)) { stat |= MM_ST_DEGENERATE; continue; }
                const double ig = 1.0 / gap;
                // conj(Y_k[b][a]) / gap
                const double yr = (dB[0] * TW.Yre[t][0][b] + dB[1] * TW.Yre[t][1][b] + dB[2] * TW.Yre[t][2][b]) * ig;
                const double yi = -(dB[0] * TW.Yim[t][0][b] + dB[1] * TW.Yim[t][1][b] + dB[2] * TW.Yim[t][2][b]) * ig;
#pragma unroll
                for (int j = 0; j < NEM * 3; j++) {
                    if (j < n_e * 3) {
                        const double xr = TW.xr[b][j], xi = TW.xi[b][j];
                        dxr[j] += yr * xr - yi * xi;
                        dxi[j] += yr * xi + yi * xr;
                    }
                }
            }
#pragma unroll
            for (int j = 0; j < NEM * 3; j++)
                if (j < n_e * 3) ddsq[j] = 2.0 * (TW.xr[t][j] * dxr[j] + TW.xi[t][j] * dxi[j]);
        }
        // branching-ratio tangents dBR[e][a] = (d row_ea - BR[e][a] d tot_e) / tot_e
#pragma unroll
        for (int e = 0; e < NEM; e++) {
            double drow = 0.0;
            if (e < n_e && lane) drow = ddsq[e * 3] + ddsq[e * 3 + 1] + ddsq[e * 3 + 2];
            const double dtot = gsum16(drow);
            if (e < n_e && lane)
                TW.dBR[e][t] = tot_e[e] > 1e-30 ? (drow - W.BR[e * n_g + t] * dtot) / tot_e[e] : 0.0;
        }
        // 3. per-beam tangents: doppler, Gaussian profile, polarisation weights
        for (int b = t; b < n_b; b += kG3) {
            const double *kh = S.khat[b];
            TW.dbm[b][0] = -P.k * (kh[0] * dv[0] + kh[1] * dv[1] + kh[2] * dv[2]) / MM_TWO_PI;
            double gf = 1.0, dgf = 0.0;
            if (S.radius[b] > 0.0) {
                const double rp = r[0] * kh[0] + r[1] * kh[1] + r[2] * kh[2];
                const double rps0 = (r[0] * r[0] + r[1] * r[1] + r[2] * r[2]) - rp * rp;
                const double w2 = S.radius[b] * S.radius[b];
                gf = exp(-2.0 * fmax(rps0, 0.0) / w2);
                if (rps0 > 0.0) {
                    const double drp = dr[0] * kh[0] + dr[1] * kh[1] + dr[2] * kh[2];
                    const double drps = 2.0 * (r[0] * dr[0] + r[1] * dr[1] + r[2] * dr[2]) - 2.0 * rp * drp;
                    dgf = gf * (-2.0 / w2) * drps;
                }
            }
            const double ds0 = (T.s0_par[b] == k) ? 1.0 : 0.0;
            TW.dbm[b][1] = ds0 * gf + S.s0[b] * dgf;
            const double dd = 0.5 * (1.0 + ct) * dct, dm = -ct * dct, dov = -0.5 * (1.0 - ct) * dct,
                         dc = 2.0 * ct * dct;
            const int q = S.pol[b];
            double w0, w1, w2;
            if (q == 0) { w0 = dd; w1 = dm; w2 = dov; }
            else if (q == 1) { w0 = dm; w1 = dc; w2 = dm; }
            else { w0 = dov; w1 = dm; w2 = dd; }
            TW.dbm[b][2] = w0; TW.dbm[b][3] = w1; TW.dbm[b][4] = w2;
        }
        __syncwarp();
        // 4. rate tangents of lane a = t (the forward's rate loop, differentiated)
        double dRu[NEM], dFv[3] = {0.0, 0.0, 0.0}, dsg = 0.0;
#pragma unroll
        for (int e = 0; e < NEM; e++) dRu[e] = 0.0;
        if (lane) {
            // 1/(Gamma/2)^2 and 1/2pi once: a division in this loop ran for every
            // (parameter, beam, excited state)
            const double igh2 = 1.0 / gh2, kInv2Pi = 1.0 / MM_TWO_PI;
            const double Eg = W.Esg[t], dEg = dlam * G / (2 * MM_PI);
            for (int b = 0; b < n_b; b++) {
                const double fd = __dadd_rn(S.freq[b], W.bm[b][0]);
                const double se = W.bm[b][1];
                const double dfd = ((T.freq_par[b] == k) ? 1.0 : 0.0) + TW.dbm[b][0];
                const double dse = TW.dbm[b][1];
                double dQ = 0.0;
#pragma unroll
                for (int e = 0; e < NEM; e++) {
                    if (e < n_e) {
                        const double om = __dsub_rn(W.Ese[e], Eg);
                        const double de = __dmul_rn(__dsub_rn(fd, om), MM_TWO_PI);
                        const double L = gh2 * mm_rcp(fma(de, de, gh2));
                        const double dEe = dB[2] * S.Ze[e] * G * kInv2Pi;
                        const double dde = (dfd - (dEe - dEg)) * MM_TWO_PI;
                        const double dL = -2.0 * de * L * L * igh2 * dde;
                        double ws = 0.0, dws = 0.0;
#pragma unroll
                        for (int q = 0; q < 3; q++) {
                            const double d2 = W.dsq[(e * 3 + q) * NGM + t];
                            if (d2 >= 1e-15) {
                                ws = fma(W.bm[b][2 + q], d2, ws);
                                dws += TW.dbm[b][2 + q] * d2 + W.bm[b][2 + q] * ddsq[e * 3 + q];
                            }
                        }
                        const double drb = (dws * L + ws * dL) * se + ws * L * dse;
                        dRu[e] += drb;
                        dQ += drb;
                    }
                }
                dsg += dQ;
                dFv[0] = fma(S.khat[b][0], dQ, dFv[0]);
                dFv[1] = fma(S.khat[b][1], dQ, dFv[1]);
                dFv[2] = fma(S.khat[b][2], dQ, dFv[2]);
            }
        }
        const double dcg = -kp.cg * dsg / (1.0 + kp.sg);
        double dRs[NEM], dRk = 0.0;
#pragma unroll
        for (int e = 0; e < NEM; e++) { dRs[e] = dRu[e] * kp.cg + kp.Ru[e] * dcg; dRk += dRs[e]; }
        __syncwarp();
        // 5. population tangent: M dx = -dM x (column t of dM on lane t; row n_g - 1 is constant)
        double rhs[NGM];
#pragma unroll
        for (int i = 0; i < NGM; i++) {
            double c = 0.0;
            if (lane && i < n_g - 1) {
                double a = (i == t) ? -dRk : 0.0;
#pragma unroll
                for (int e = 0; e < NEM; e++)
                    if (e < n_e) a += dRs[e] * W.BR[e * n_g + i] + kp.Rs[e] * TW.dBR[e][i];
                c = a * kp.xraw;
            }
            rhs[i] = -gsum16(c);
        }
        // P M = L U with the forward's interchanges and factors (later interchanges
        // were applied to the stored L columns, so all of P goes first); static_for
        // keeps the indices of rhs and xs compile-time constants (registers)
        static_for<0, NGM>([&](auto colc) {
            constexpr int col = decltype(colc)::value;
            if (col < n_g) {
                const int pr = kp.prow[col];
#pragma unroll
                for (int rr = col + 1; rr < NGM; rr++)
                    if (rr == pr) { const double x = rhs[col]; rhs[col] = rhs[rr]; rhs[rr] = x; }
            }
        });
        static_for<0, NGM>([&](auto colc) {
            constexpr int col = decltype(colc)::value;
            if (col < n_g) {
                const double iv = TW.invd[col];
#pragma unroll
                for (int rr = col + 1; rr < NGM; rr++)
                    if (rr < n_g) rhs[rr] = fma(-(TW.LU[rr][col] * iv), rhs[col], rhs[rr]);
            }
        });
        double dx = 0.0, xs[NGM];
        static_for<0, NGM>([&](auto iic) {
            constexpr int i = NGM - 1 - decltype(iic)::value;
            double xi = 0.0;
            if (i < n_g) {
                double part = 0.0;
#pragma unroll
                for (int j = i + 1; j < NGM; j++)
                    if (j < n_g) part = fma(TW.LU[i][j], xs[j], part);
                xi = (rhs[i] - part) * TW.invd[i];
            }
            xs[i] = xi;
            if (i == t) dx = xi;
        });
        // clamp and normalisation
        double dxc = (lane && kp.xraw > 0.0) ? dx : 0.0;
        const double dtot = gsum16(dxc);
        const double dp = (kp.tot > 0.0 && lane) ? (dxc - kp.x * dtot) / kp.tot : 0.0;
        // 6. force tangent: F = hbar k sum_a p_a cg_a Fv_a
        double f[3];
        for (int c = 0; c < 3; c++) {
            const double a = lane ? (dp * kp.cg * kp.Fv[c] + kp.x * (dcg * kp.Fv[c] + kp.cg * dFv[c])) : 0.0;
            f[c] = hk * gsum16(a);
        }
        if (t == 0)
            for (int c = 0; c < 3; c++) TW.dF[k][c] = f[c];
        __syncwarp();
    }
}

// Leapfrog ensemble with tangents, one particle per group: the trajectory of
// traj3d_kernel (bit for bit, kicks included) plus d(r, vh, v)/d theta_k.
template <int NGM, int NEM, int TH>
__global__ void __launch_bounds__(TH)
traj3d_grad_kernel(Force3Params P, Tg3Params T)
{
    extern __shared__ __align__(16) unsigned char smraw[];
    auto &S = *reinterpret_cast<Smem3<NGM, NEM, TH> *>(smraw);
    const int lane = threadIdx.x & 31, t = lane % kG3, gbase = lane - t;
    const int group = threadIdx.x / kG3, ngroups = TH / kG3;
    auto &TW = reinterpret_cast<Tan3Work<NGM, NEM> *>(smraw + (sizeof(Smem3<NGM, NEM, TH>) + 15) / 16 * 16)[group];
    load_consts3(P, 0, S);
    __syncthreads();
    const double Bg = P.bgrad[0];
    const double m = P.mass, dt = T.dt;
    const int np = T.n_par, Wd = 6 + 6 * np;
    const long long ip = (long long)blockIdx.x * ngroups + group;
    const bool valid = ip < T.n_particles;
    const long long ipc = valid ? ip : 0;
    double *row = T.state + ipc * Wd;
    double r[3], vh[3], vs[3], pl;
    for (int c = 0; c < 3; c++) { r[c] = row[c]; vh[c] = row[3 + c]; vs[c] = vh[c]; }
    for (int i = t; i < 3 * kT3MaxPar; i += kG3) {
        const int c = i / kT3MaxPar, k = i % kT3MaxPar;
        TW.Tr[c][k] = (k < np) ? row[6 + c * np + k] : 0.0;
        TW.Tv[c][k] = (k < np) ? row[6 + 3 * np + c * np + k] : 0.0;
        TW.Tvs[c][k] = TW.Tv[c][k];
    }
    __syncwarp();
    int stat = 0, nev = 0;
    Keep3<NGM, NEM> kp;
    // a particle already beyond r_escape stopped in an earlier call
    const bool stopped = !valid || sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]) > T.r_escape;
    bool done = stopped;
    long long na = -1, n_ck = 0;
    auto set_dirs = [&]() {  // the force's argument tangents: TW.dr = Tr, TW.dv = Tv
        for (int i = t; i < 3 * kT3MaxPar; i += kG3) {
            const int c = i % 3, k = i / 3;
            TW.dr[k][c] = TW.Tr[c][k];
            TW.dv[k][c] = TW.Tv[c][k];
        }
        __syncwarp();
    };
    auto write_state = [&](double *dst) {
        if (valid && t == 0) {
            for (int c = 0; c < 3; c++) { dst[c] = r[c]; dst[3 + c] = vh[c]; }
            for (int c = 0; c < 3; c++)
                for (int k = 0; k < np; k++) {
                    dst[6 + c * np + k] = TW.Tr[c][k];
                    dst[6 + 3 * np + c * np + k] = TW.Tv[c][k];
                }
        }
    };
    // iteration j = 0 (a run from step 0) is the first half kick at (r0, v0),
    // as traj3d_kernel; it shares the loop's single inlined force and tangent
    // evaluation, and runs for every particle, stopped ones included
    const long long j0 = (T.step0 == 0) ? 0 : T.step0;
    const long long j1 = T.step0 + T.n_steps;
    long long j = j0;
    for (; j < j1; j++) {
        const bool kick0 = j == 0;  // the same on every lane
        if (!kick0 && __all_sync(0xffffffffu, done)) break;
        double rn[3];
        for (int c = 0; c < 3; c++) rn[c] = kick0 ? r[c] : __dadd_rn(r[c], __dmul_rn(dt, vh[c]));  // r + dt v_half
        const double rr = sqrt(rn[0] * rn[0] + rn[1] * rn[1] + rn[2] * rn[2]);
        const bool esc = !done && !kick0 && rr > T.r_escape;
        // position tangent first: the force is evaluated at (r_j, v_half)
        if (!kick0 && !done && t < 3)
            for (int k = 0; k < np; k++) TW.Tr[t][k] = fma(dt, TW.Tv[t][k], TW.Tr[t][k]);
        __syncwarp();
        set_dirs();
        const Out3 o = force3d_point(P, S, S.grp[group], t, gbase, rn, vh, Bg, pl, &kp);
        int st = 0;
        force3d_tangent(P, T, S, S.grp[group], TW, t, rn, vh, Bg, kp, st);
        if (kick0) {
            stat |= st;
            for (int c = 0; c < 3; c++) vh[c] = vh[c] + 0.5 * dt * o.F[c] / m;
            if (t < 3)
                for (int k = 0; k < np; k++) TW.Tv[t][k] = fma(0.5 * dt / m, TW.dF[k][t], TW.Tv[t][k]);
            __syncwarp();
            continue;
        }
        if (!done) {
            stat |= st;
            for (int c = 0; c < 3; c++) r[c] = rn[c];
            if (esc) {
                na = j;
                done = true;
                for (int c = 0; c < 3; c++) vs[c] = vh[c];
                if (t < 3)
                    for (int k = 0; k < np; k++) TW.Tvs[t][k] = TW.Tv[t][k];
            } else {
                double vn[3];
                for (int c = 0; c < 3; c++) vn[c] = vh[c] + dt * o.F[c] / m;
                if (T.kicks) {
                    double kick[3];
                    nev += recoil_kick(T.seed, (unsigned)ip, (unsigned)j, o.R * dt, T.v_rec, kick);
                    for (int c = 0; c < 3; c++) vn[c] += kick[c];
                }
                for (int c = 0; c < 3; c++) { vs[c] = 0.5 * (vh[c] + vn[c]); vh[c] = vn[c]; }
                if (t < 3)
                    for (int k = 0; k < np; k++) {
                        const double tvn = fma(dt / m, TW.dF[k][t], TW.Tv[t][k]);
                        TW.Tvs[t][k] = 0.5 * (TW.Tv[t][k] + tvn);
                        TW.Tv[t][k] = tvn;
                    }
            }
        }
        __syncwarp();
        if (T.ckpt && j % T.ckpt_every == 0) {
            write_state(T.ckpt + ((size_t)n_ck * T.n_particles + ipc) * Wd);
            n_ck++;
        }
    }
    // checkpoints after the whole warp stopped: the frozen state
    if (T.ckpt)
        for (; j < j1; j++)
            if (j % T.ckpt_every == 0) {
                write_state(T.ckpt + ((size_t)n_ck * T.n_particles + ipc) * Wd);
                n_ck++;
            }
    write_state(row);
    if (valid && t == 0) {
        double *vo = T.vsync + ipc * (3 + 3 * np);
        for (int c = 0; c < 3; c++) {
            vo[c] = vs[c];
            for (int k = 0; k < np; k++) vo[3 + c * np + k] = TW.Tvs[c][k];
        }
        if (na >= 0) T.n_actual[ip] = (int32_t)na;
        else if (!stopped) T.n_actual[ip] = (int32_t)j1;
        T.status[ip] = stat;
        if (T.n_events) T.n_events[ip] = nev;
    }
}

int fill3(const mm_pack *pack, const mm_beams *beams, double hbar, int uniform_fb, Force3Params &P)
{
    if (!pack || !beams) { mm_set_error("null pack or beams handle"); return -1; }
    if (!pack->has3d) { mm_set_error("the molecule pack has no 3D data (Zeeman blocks, |tdm|)"); return -1; }
    if (!beams->has3d) { mm_set_error("the beam sets have no 3D data (khat)"); return -1; }
    if (pack->n_g > C3Large::NGM || pack->n_e > C3Large::NEM) {
        mm_set_error("3D kernel supports n_ground <= %d, n_excited <= %d (got %d, %d)", C3Large::NGM,
                     C3Large::NEM, pack->n_g, pack->n_e);
        return -1;
    }
    if (beams->n_b > NBM) { mm_set_error("3D kernel supports <= %d beams", NBM); return -1; }
    P.n_g = pack->n_g; P.n_e = pack->n_e; P.n_b = beams->n_b; P.n_sets = beams->n_sets;
    P.Gamma = pack->Gamma; P.k = pack->k; P.mass = pack->mass;
    P.hbar = hbar > 0 ? hbar : 1.054571817e-34;
    P.geff = beams->gamma_eff;
    P.E = pack->buf + pack->oE; P.Zre = pack->buf + pack->oZre; P.Zim = pack->buf + pack->oZim;
    P.Ze = pack->buf + pack->oZe; P.tdm = pack->buf + pack->oTdm;
    P.khat = beams->khat; P.freq = beams->freq; P.s0 = beams->s0; P.radius = beams->radius;
    P.bgrad = beams->bgrad; P.pol = beams->pol;
    P.uniform_fb = uniform_fb;
    return 0;
}

template <class K>
int prep_smem(K kern, size_t sb)
{
    return mm_cuda_check(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sb),
                         "cudaFuncSetAttribute") ? -3 : 0;
}

// The 3D size class of a molecule: SrOH-sized (12 + 4) or the larger one (16 + 8).
template <class F>
int dispatch3(int n_g, int n_e, F &&f)
{
    if (n_g <= C3Small::NGM && n_e <= C3Small::NEM) return f(C3Small{});
    return f(C3Large{});
}

template <class C>
int launch_force3d(const Force3Params &P, long long n_points, long long pps, cudaStream_t st)
{
    auto kern = force3d_kernel<C::NGM, C::NEM, C::THREADS>;
    const size_t sb = sizeof(Smem3<C::NGM, C::NEM, C::THREADS>);
    if (prep_smem(kern, sb)) return -3;
    int dev = 0, nsm = 148, per_sm = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, C::THREADS, sb);
    const int ngroups = C::THREADS / kG3;
    const int n_sets_used = (int)((n_points + pps - 1) / pps);
    long long gx = std::max<long long>(1, (long long)nsm * std::max(per_sm, 1) * 2 / n_sets_used);
    gx = std::min<long long>(gx, (pps + ngroups - 1) / ngroups);
    dim3 grid((unsigned)gx, (unsigned)std::min(n_sets_used, 65535));
    kern<<<grid, C::THREADS, sb, st>>>(P);
    return mm_cuda_check(cudaGetLastError(), "force3d_kernel launch") ? -3 : 0;
}

template <class C>
int launch_traj3d(const Force3Params &P, const Traj3Params &T, cudaStream_t st)
{
    auto kern = traj3d_kernel<C::NGM, C::NEM, C::THREADS>;
    const size_t sb = sizeof(Smem3<C::NGM, C::NEM, C::THREADS>);
    if (prep_smem(kern, sb)) return -3;
    const int ngroups = C::THREADS / kG3;
    const long long gx = (T.n_particles + ngroups - 1) / ngroups;
    kern<<<(unsigned)gx, C::THREADS, sb, st>>>(P, T);
    return mm_cuda_check(cudaGetLastError(), "traj3d_kernel launch") ? -3 : 0;
}

}  // namespace

extern "C" int mm_force3d_batch(const mm_pack *pack, const mm_beams *beams, const double *r,
                                const double *v, int64_t n_points, int64_t points_per_set,
                                double hbar, double *F, double *R, double *pop, int32_t *status,
                                void *stream)
{
    Force3Params P;
    if (fill3(pack, beams, hbar, 1, P)) return -1;
    if (n_points < 0) { mm_set_error("n_points < 0"); return -1; }
    if (n_points == 0) return 0;  // an empty batch may pass null arrays
    if (!r || !v || !F) { mm_set_error("r, v and F must be non-null"); return -1; }
    const long long pps = points_per_set > 0 ? points_per_set : n_points;
    if ((n_points + pps - 1) / pps > beams->n_sets) {
        mm_set_error("%lld points at %lld per set need more than %d sets", (long long)n_points, pps,
                     beams->n_sets);
        return -1;
    }
    P.n_points = n_points; P.pps = pps; P.r = r; P.v = v; P.F = F; P.R = R; P.pop = pop;
    P.status = status;
    return dispatch3(P.n_g, P.n_e, [&](auto C) -> int {
        return launch_force3d<decltype(C)>(P, n_points, pps, (cudaStream_t)stream);
    });
}

extern "C" int mm_traj3d_run(const mm_pack *pack, const mm_beams *beams, const double *r0,
                             const double *v0, int64_t n_particles, int64_t step0, int64_t n_steps,
                             double dt, double r_escape, int32_t kicks, uint64_t seed, double hbar,
                             double *r_out, double *vh_out, double *v_out, int32_t *n_actual,
                             double *r_traj, double *v_traj, double *ke, int32_t *n_events,
                             void *stream)
{
    Force3Params P;
    if (fill3(pack, beams, hbar, 1, P)) return -1;
    if (n_particles > 0 && (!r0 || !v0 || !r_out || !vh_out || !n_actual)) {
        mm_set_error("r0, v0, r_out, vh_out and n_actual must be non-null");
        return -1;
    }
    if ((r_traj == nullptr) != (v_traj == nullptr)) { mm_set_error("r_traj and v_traj go together"); return -1; }
    if (n_particles < 0 || n_steps < 1 || step0 < 0) {
        mm_set_error("n_particles >= 0, n_steps >= 1, step0 >= 0 required");
        return -1;
    }
    if (n_particles > 0xffffffffLL || step0 + n_steps > 0xffffffffLL) {
        mm_set_error("particle and step indices must fit the 32-bit RNG counter words");
        return -1;
    }
    if (n_particles == 0) return 0;
    P.n_points = 0; P.pps = 1; P.r = P.v = nullptr; P.F = P.R = P.pop = nullptr; P.status = nullptr;
    Traj3Params T;
    T.dt = dt; T.r_escape = r_escape; T.n_particles = n_particles; T.n_steps = n_steps;
    T.step0 = step0; T.kicks = kicks; T.seed = seed;
    T.r0 = r0; T.v0 = v0; T.r_out = r_out; T.vh_out = vh_out; T.v_out = v_out;
    T.n_actual = n_actual; T.r_traj = r_traj; T.v_traj = v_traj; T.ke_sum = ke;
    T.n_events = n_events;
    return dispatch3(P.n_g, P.n_e, [&](auto C) -> int {
        return launch_traj3d<decltype(C)>(P, T, (cudaStream_t)stream);
    });
}

namespace {

// Checkpoints of one mm_traj3d_grad_run call: updates j in [j0, j1) with j % every == 0.
long long t3_checkpoints(long long step0, long long n_steps, long long every)
{
    const long long j0 = (step0 == 0) ? 1 : step0, j1 = step0 + n_steps;
    if (every < 1 || j1 <= j0) return 0;
    return (j1 - 1) / every - (j0 - 1) / every;
}

template <class C>
int launch_traj3d_grad(const Force3Params &P, const Tg3Params &T, cudaStream_t st)
{
    constexpr int TH = kT3Threads;
    auto kern = traj3d_grad_kernel<C::NGM, C::NEM, TH>;
    const size_t sb = (sizeof(Smem3<C::NGM, C::NEM, TH>) + 15) / 16 * 16 +
                      sizeof(Tan3Work<C::NGM, C::NEM>) * (TH / kG3);
    int dev = 0, smax = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&smax, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (sb > (size_t)smax) {
        mm_set_error("the 3D tangent kernel needs %zu bytes of shared memory (limit %d)", sb, smax);
        return -1;
    }
    if (prep_smem(kern, sb)) return -3;
    const int ngroups = TH / kG3;
    const long long gx = (T.n_particles + ngroups - 1) / ngroups;
    kern<<<(unsigned)gx, TH, sb, st>>>(P, T);
    return mm_cuda_check(cudaGetLastError(), "traj3d_grad_kernel launch") ? -3 : 0;
}

}  // namespace

extern "C" int mm_traj3d_grad_run(const mm_pack *pack, const mm_beams *beams, const mm_t3grad_opts *opts,
                                  int64_t n_particles, double *state, double *vsync, int32_t *n_actual,
                                  int32_t *status, int32_t *n_events, double *ckpt, void *stream)
{
    if (!opts) { mm_set_error("3D trajectory-gradient options are required"); return -1; }
    Force3Params P;
    if (fill3(pack, beams, opts->hbar, 1, P)) return -1;
    if (n_particles < 0 || opts->n_steps < 1 || opts->step0 < 0) {
        mm_set_error("n_particles >= 0, n_steps >= 1, step0 >= 0 required");
        return -1;
    }
    if (n_particles > 0xffffffffLL || opts->step0 + opts->n_steps > 0x7fffffffLL) {
        mm_set_error("particle and step indices must fit the 32-bit RNG counter words");
        return -1;
    }
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
    if (n_particles == 0) return 0;
    if (!state || !vsync || !n_actual || !status) {
        mm_set_error("state, vsync, n_actual and status must be non-null");
        return -1;
    }
    P.n_points = 0; P.pps = 1; P.r = P.v = nullptr; P.F = P.R = P.pop = nullptr; P.status = nullptr;
    Tg3Params T;
    T.dt = opts->dt; T.r_escape = opts->r_escape; T.mass = pack->mass;
    T.v_rec = P.hbar * P.k / pack->mass;
    T.gap_tol = opts->gap_tol > 0 ? opts->gap_tol : 1e-9;
    T.n_particles = n_particles; T.n_steps = opts->n_steps; T.step0 = opts->step0;
    T.ckpt_every = ckpt ? opts->ckpt_every : 1;
    T.n_par = opts->n_par; T.kicks = opts->kicks ? 1 : 0; T.bprime_par = opts->bprime_par;
    T.seed = opts->seed;
    for (int b = 0; b < NBM; b++) {
        T.freq_par[b] = (signed char)(b < beams->n_b ? opts->freq_par[b] : -1);
        T.s0_par[b] = (signed char)(b < beams->n_b ? opts->s0_par[b] : -1);
    }
    T.state = state; T.vsync = vsync; T.n_actual = n_actual; T.status = status; T.n_events = n_events;
    T.ckpt = ckpt;
    return dispatch3(P.n_g, P.n_e, [&](auto C) -> int {
        return launch_traj3d_grad<decltype(C)>(P, T, (cudaStream_t)stream);
    });
}

extern "C" int64_t mm_traj3d_grad_checkpoints(int64_t step0, int64_t n_steps, int64_t ckpt_every)
{
    return t3_checkpoints(step0, n_steps, ckpt_every);
}
