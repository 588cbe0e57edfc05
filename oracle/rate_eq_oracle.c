/*
 * rate_eq_oracle.c -- TEST INFRASTRUCTURE ONLY (the oracle).
 *
 * A plain-C, FP64, CPU restatement of molmot's rate-equation steady-state
 * force and of the 1D trajectory integrator that calls it.  It is the
 * checker for the CUDA product path: only tests/, __graft_entry__.smoke()
 * and bench.py's cpu_baseline / --impl reference legs load it.  Nothing in
 * molmot_b200/ may import or call it.
 *
 * Reference algorithm followed (paths relative to the molmot project root):
 *   molmot/obe/rate_equations_jit.py:18-145   _rate_eq_core      (default)
 *   molmot/obe/rate_equations.py:24-191       solve_rate_equations
 *       (ORC_TWO_PASS: saturation applied per rate, uniform fallback; the
 *        scipy LAPACK solve is replaced by the same partial-pivoting
 *        elimination, so this variant agrees with it to rounding only)
 *   molmot/propagation/trajectories_jit.py:18-58  _trajectory_1d_jit
 *
 * Every floating-point operation is written in the reference's order
 * (left-to-right evaluation of each Python expression) and the file must be
 * compiled with -ffp-contract=off and without -ffast-math, so that the
 * results are bit-identical to numba's compilation of _rate_eq_core (numba
 * does not contract a*b+c into an FMA unless fastmath is requested).
 * Pinned against the reference's JIT on random inputs and against the
 * golden arrays of validation/three_way_results.npz (tests/golden/).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <pthread.h>
#include <unistd.h>

#define ORC_MAX_G 64
#define ORC_MAX_E 64
#define ORC_MAX_B 64

/* flags */
#define ORC_UNIFORM_FALLBACK 1 /* p = 1/n_g when all clamped populations are 0 */
#define ORC_TWO_PASS 2         /* rate_equations.py: rate/(1+s_total) per rate */

/* 2.0 * np.pi: doubling is exact, so this equals 2*(double)pi bit for bit. */
static const double ORC_PI = 3.141592653589793;

typedef struct {
    int n_g, n_e;
    const double *E;   /* [n_g + n_e]   Hz                          */
    const double *d2;  /* [n_g][n_e][3] |TDM|^2                     */
    const double *zd;  /* [n_g + n_e]   Zeeman diag, Gamma/2pi per G */
    double Gamma, k, Geff, hbar;
} orc_mol;

typedef struct {
    int n_b;
    const double *kdir, *freq, *pol, *s0; /* [n_b] each; pol as float like the JIT */
} orc_beams;

/* Branching ratios BR[e][g], summed in rate_equations_jit.py:38-49 order. */
static void orc_branching(const orc_mol *m, double *BR)
{
    const int n_g = m->n_g, n_e = m->n_e;
    for (int ie = 0; ie < n_e; ie++) {
        double total = 0.0;
        for (int ig = 0; ig < n_g; ig++)
            for (int q = 0; q < 3; q++)
                total += m->d2[(ig * n_e + ie) * 3 + q];
        for (int ig = 0; ig < n_g; ig++) BR[ie * n_g + ig] = 0.0;
        if (total > 1e-30) {
            for (int ig = 0; ig < n_g; ig++) {
                double s = 0.0;
                for (int q = 0; q < 3; q++) s += m->d2[(ig * n_e + ie) * 3 + q];
                BR[ie * n_g + ig] = s / total;
            }
        }
    }
}

/*
 * One steady-state point.  Returns 0, or a status bit set:
 *   1 = a pivot with |pivot| < 1e-30 was skipped (elimination or back-subst)
 *   2 = non-finite force
 *   4 = all populations clamped to zero (sum p == 0)
 */
static int orc_point(const orc_mol *m, const orc_beams *bm, const double *BR,
                     double v, double z, double Bgrad, int flags,
                     double *F_out, double *pop_out, double *R_out)
{
    const int n_g = m->n_g, n_e = m->n_e, n_s = n_g + n_e;
    const double Gamma = m->Gamma, k_wave = m->k, Geff = m->Geff, hbar_val = m->hbar;
    double Es[ORC_MAX_G + ORC_MAX_E];
    double R_sum[ORC_MAX_G * ORC_MAX_E], F_tot[ORC_MAX_G * ORC_MAX_E];
    double s_total[ORC_MAX_G];
    static __thread double A[ORC_MAX_G * ORC_MAX_G];
    double b[ORC_MAX_G], p[ORC_MAX_G];
    int status = 0;

    const double B_gauss = Bgrad * z * 1e4;
    const double gamma_half = Gamma / 2.0;
    const double gamma_half_sq = gamma_half * gamma_half;
    for (int i = 0; i < n_s; i++)
        Es[i] = m->E[i] + B_gauss * m->zd[i] * Gamma / (2.0 * ORC_PI);

    for (int i = 0; i < n_g * n_e; i++) { R_sum[i] = 0.0; F_tot[i] = 0.0; }
    for (int i = 0; i < n_g; i++) s_total[i] = 0.0;

    if (!(flags & ORC_TWO_PASS)) {
        /* rate_equations_jit.py:58-83 -- one pass, saturation applied after */
        for (int ib = 0; ib < bm->n_b; ib++) {
            const double kdir = bm->kdir[ib], freq = bm->freq[ib], s0 = bm->s0[ib];
            const int pol = (int)bm->pol[ib];
            const double doppler = -k_wave * kdir * v / (2.0 * ORC_PI);
            for (int ig = 0; ig < n_g; ig++) {
                for (int ie = 0; ie < n_e; ie++) {
                    const double d2 = m->d2[(ig * n_e + ie) * 3 + pol];
                    if (d2 < 1e-15) continue;
                    const double omega_trans = Es[n_g + ie] - Es[ig];
                    const double delta_eff = (freq + doppler - omega_trans) * 2.0 * ORC_PI;
                    const double L = gamma_half_sq / (delta_eff * delta_eff + gamma_half_sq);
                    const double rate_unsat = gamma_half * s0 * d2 * L * Geff;
                    R_sum[ig * n_e + ie] += rate_unsat;
                    F_tot[ig * n_e + ie] += hbar_val * k_wave * kdir * rate_unsat;
                    s_total[ig] += s0 * d2 * L;
                }
            }
        }
        for (int ig = 0; ig < n_g; ig++) {
            const double sat_corr = 1.0 / (1.0 + s_total[ig]);
            for (int ie = 0; ie < n_e; ie++) {
                R_sum[ig * n_e + ie] *= sat_corr;
                F_tot[ig * n_e + ie] *= sat_corr;
            }
        }
    } else {
        /* rate_equations.py:105-154 -- two passes, rate/(1+s_total) per rate */
        for (int ib = 0; ib < bm->n_b; ib++) {
            const double kdir = bm->kdir[ib], freq = bm->freq[ib], s0 = bm->s0[ib];
            const int pol = (int)bm->pol[ib];
            const double doppler = -k_wave * kdir * v / (2.0 * ORC_PI);
            for (int ig = 0; ig < n_g; ig++)
                for (int ie = 0; ie < n_e; ie++) {
                    const double d2 = m->d2[(ig * n_e + ie) * 3 + pol];
                    if (d2 < 1e-15) continue;
                    const double omega_trans = Es[n_g + ie] - Es[ig];
                    const double delta_eff = (freq + doppler - omega_trans) * 2.0 * ORC_PI;
                    const double L = gamma_half_sq / (delta_eff * delta_eff + gamma_half_sq);
                    s_total[ig] += s0 * d2 * L;
                }
        }
        for (int ib = 0; ib < bm->n_b; ib++) {
            const double kdir = bm->kdir[ib], freq = bm->freq[ib], s0 = bm->s0[ib];
            const int pol = (int)bm->pol[ib];
            const double doppler = -k_wave * kdir * v / (2.0 * ORC_PI);
            for (int ig = 0; ig < n_g; ig++)
                for (int ie = 0; ie < n_e; ie++) {
                    const double d2 = m->d2[(ig * n_e + ie) * 3 + pol];
                    if (d2 < 1e-15) continue;
                    const double omega_trans = Es[n_g + ie] - Es[ig];
                    const double delta_eff = (freq + doppler - omega_trans) * 2.0 * ORC_PI;
                    const double L = gamma_half_sq / (delta_eff * delta_eff + gamma_half_sq);
                    const double rate = gamma_half * s0 * d2 * L * Geff / (1.0 + s_total[ig]);
                    R_sum[ig * n_e + ie] += rate;
                    F_tot[ig * n_e + ie] += hbar_val * k_wave * kdir * rate;
                }
        }
    }

    /* population matrix, rate_equations_jit.py:86-97 */
    const int n = n_g;
    for (int i = 0; i < n * n; i++) A[i] = 0.0;
    for (int ig = 0; ig < n_g; ig++) {
        for (int ie = 0; ie < n_e; ie++) A[ig * n + ig] -= R_sum[ig * n_e + ie];
        for (int ik = 0; ik < n_g; ik++)
            for (int ie = 0; ie < n_e; ie++)
                A[ig * n + ik] += R_sum[ik * n_e + ie] * BR[ie * n_g + ig];
    }
    for (int j = 0; j < n; j++) A[(n - 1) * n + j] = 1.0;
    for (int i = 0; i < n; i++) b[i] = 0.0;
    b[n - 1] = 1.0;

    /* Gaussian elimination with partial pivoting, rate_equations_jit.py:99-118 */
    for (int col = 0; col < n; col++) {
        double max_val = fabs(A[col * n + col]);
        int max_row = col;
        for (int row = col + 1; row < n; row++) {
            if (fabs(A[row * n + col]) > max_val) {
                max_val = fabs(A[row * n + col]);
                max_row = row;
            }
        }
        if (max_row != col) {
            for (int j = 0; j < n; j++) {
                double t = A[col * n + j];
                A[col * n + j] = A[max_row * n + j];
                A[max_row * n + j] = t;
            }
            double t = b[col]; b[col] = b[max_row]; b[max_row] = t;
        }
        for (int row = col + 1; row < n; row++) {
            if (fabs(A[col * n + col]) < 1e-30) { status |= 1; continue; }
            const double factor = A[row * n + col] / A[col * n + col];
            for (int j = col; j < n; j++) A[row * n + j] -= factor * A[col * n + j];
            b[row] -= factor * b[col];
        }
    }
    /* back substitution, rate_equations_jit.py:120-126 */
    for (int i = 0; i < n; i++) p[i] = 0.0;
    for (int i = n - 1; i >= 0; i--) {
        double s = b[i];
        for (int j = i + 1; j < n; j++) s -= A[i * n + j] * p[j];
        if (fabs(A[i * n + i]) > 1e-30) p[i] = s / A[i * n + i];
        else status |= 1;
    }
    /* clamp and normalise, rate_equations_jit.py:128-136 */
    for (int i = 0; i < n; i++) if (p[i] < 0) p[i] = 0.0;
    double total_p = 0.0;
    for (int i = 0; i < n; i++) total_p += p[i];
    if (total_p > 0) {
        for (int i = 0; i < n; i++) p[i] /= total_p;
    } else {
        status |= 4;
        if (flags & ORC_UNIFORM_FALLBACK)
            for (int i = 0; i < n; i++) p[i] = 1.0 / (double)n;
    }
    /* force and scattering rate, rate_equations_jit.py:138-145 */
    double force = 0.0, R_scatter = 0.0;
    for (int ig = 0; ig < n_g; ig++)
        for (int ie = 0; ie < n_e; ie++) {
            force += p[ig] * F_tot[ig * n_e + ie];
            R_scatter += p[ig] * R_sum[ig * n_e + ie];
        }
    if (!isfinite(force)) status |= 2;
    *F_out = force;
    if (R_out) *R_out = R_scatter;
    if (pop_out) for (int i = 0; i < n; i++) pop_out[i] = p[i];
    return status;
}


/* Minimal static-partition parallel for over [0, n) with pthreads. */
typedef struct {
    void (*body)(void *ctx, int64_t i);
    void *ctx;
    int64_t lo, hi;
} orc_chunk;

static void *orc_chunk_run(void *arg)
{
    orc_chunk *c = (orc_chunk *)arg;
    for (int64_t i = c->lo; i < c->hi; i++) c->body(c->ctx, i);
    return NULL;
}

int orc_max_threads(void)
{
    long n = sysconf(_SC_NPROCESSORS_ONLN);
    return n > 0 ? (int)n : 1;
}

static void orc_parallel_for(int64_t n, int n_threads, void (*body)(void *, int64_t), void *ctx)
{
    if (n_threads <= 0) n_threads = orc_max_threads();
    if (n_threads > 256) n_threads = 256;
    if ((int64_t)n_threads > n) n_threads = (int)(n > 0 ? n : 1);
    if (n_threads == 1) {
        for (int64_t i = 0; i < n; i++) body(ctx, i);
        return;
    }
    pthread_t th[256];
    orc_chunk ch[256];
    for (int t = 0; t < n_threads; t++) {
        ch[t].body = body;
        ch[t].ctx = ctx;
        ch[t].lo = n * t / n_threads;
        ch[t].hi = n * (t + 1) / n_threads;
        pthread_create(&th[t], NULL, orc_chunk_run, &ch[t]);
    }
    for (int t = 0; t < n_threads; t++) pthread_join(th[t], NULL);
}

static int orc_check(int n_g, int n_e, int n_b)
{
    if (n_g < 1 || n_g > ORC_MAX_G || n_e < 0 || n_e > ORC_MAX_E || n_b < 0 || n_b > ORC_MAX_B)
        return -1;
    return 0;
}

/* Single point: the _rate_eq_core call signature plus hbar and flags. */
int orc_rate_eq_point(int n_g, int n_e, const double *E, const double *d2, const double *zd,
                      int n_b, const double *kdir, const double *freq, const double *pol,
                      const double *s0, double v, double z, double Bgrad, double Gamma,
                      double k, double Geff, double hbar, int flags,
                      double *F, double *pop, double *R)
{
    if (orc_check(n_g, n_e, n_b)) return -1;
    orc_mol m = {n_g, n_e, E, d2, zd, Gamma, k, Geff, hbar};
    orc_beams bm = {n_b, kdir, freq, pol, s0};
    double BR[ORC_MAX_E * ORC_MAX_G];
    orc_branching(&m, BR);
    return orc_point(&m, &bm, BR, v, z, Bgrad, flags, F, pop, R);
}

/*
 * Batch of points over parameter sets.  Beam arrays are [n_sets][n_b];
 * Bgrad is [n_sets].  Point i uses set i / points_per_set and (v[i], z[i]),
 * or, with grid_nv > 0, the grid point (set, iv, iz) with
 * i = (set * grid_nv + iv) * grid_nz + iz and v = v[iv], z = z[iz]
 * (molmot_cuda/rate_equations_cuda.py:448-544 layout, per set).
 * n_threads <= 0 uses every online core.
 */
typedef struct {
    orc_mol m;
    double BR[ORC_MAX_E * ORC_MAX_G];
    int flags, n_b, n_sets;
    const double *kdir, *freq, *pol, *s0, *Bgrad, *v, *z;
    int64_t points_per_set, grid_nv, grid_nz;
    double *F, *pop, *R;
    int32_t *status;
} orc_batch_ctx;

static void orc_batch_body(void *vctx, int64_t i)
{
    const orc_batch_ctx *c = (const orc_batch_ctx *)vctx;
    int64_t set;
    double vi, zi;
    if (c->grid_nv > 0) {
        const int64_t per = c->grid_nv * c->grid_nz;
        set = i / per;
        const int64_t r = i - set * per;
        vi = c->v[r / c->grid_nz];
        zi = c->z[r % c->grid_nz];
    } else {
        set = i / c->points_per_set;
        vi = c->v[i];
        zi = c->z[i];
    }
    if (set >= c->n_sets) set = c->n_sets - 1;
    const int n_b = c->n_b;
    orc_beams bm = {n_b, c->kdir + set * n_b, c->freq + set * n_b, c->pol + set * n_b,
                    c->s0 + set * n_b};
    double Rv;
    int st = orc_point(&c->m, &bm, c->BR, vi, zi, c->Bgrad[set], c->flags, &c->F[i],
                       c->pop ? c->pop + i * c->m.n_g : NULL, &Rv);
    if (c->R) c->R[i] = Rv;
    if (c->status) c->status[i] = st;
}

int orc_force_batch(int n_g, int n_e, const double *E, const double *d2, const double *zd,
                    double Gamma, double k, double Geff, double hbar, int flags,
                    int n_b, int n_sets, const double *kdir, const double *freq,
                    const double *pol, const double *s0, const double *Bgrad,
                    int64_t n_points, int64_t points_per_set, int64_t grid_nv, int64_t grid_nz,
                    const double *v, const double *z, int n_threads,
                    double *F, double *pop, double *R, int32_t *status)
{
    if (orc_check(n_g, n_e, n_b) || n_sets < 1) return -1;
    if (grid_nv <= 0 && points_per_set <= 0) return -1;
    orc_batch_ctx *c = (orc_batch_ctx *)calloc(1, sizeof(orc_batch_ctx));
    if (!c) return -2;
    orc_mol m = {n_g, n_e, E, d2, zd, Gamma, k, Geff, hbar};
    c->m = m;
    orc_branching(&c->m, c->BR);
    c->flags = flags; c->n_b = n_b; c->n_sets = n_sets;
    c->kdir = kdir; c->freq = freq; c->pol = pol; c->s0 = s0; c->Bgrad = Bgrad;
    c->v = v; c->z = z;
    c->points_per_set = points_per_set; c->grid_nv = grid_nv; c->grid_nz = grid_nz;
    c->F = F; c->pop = pop; c->R = R; c->status = status;
    orc_parallel_for(n_points, n_threads, orc_batch_body, c);
    free(c);
    return 0;
}

/*
 * N independent 1D trajectories (trajectories_jit.py:18-58): symplectic
 * Euler, force at (v_{j-1}, z_{j-1}), truncated when |z| > z_escape.
 * z_traj / v_traj are [N][n_steps] or NULL.
 */
typedef struct {
    orc_mol m;
    orc_beams bm;
    double BR[ORC_MAX_E * ORC_MAX_G];
    int flags;
    double Bgrad, mass, dt, z_escape;
    int64_t n_steps;
    const double *z0, *v0;
    double *z_final, *v_final, *z_traj, *v_traj;
    int32_t *n_actual;
} orc_traj_ctx;

static void orc_traj_body(void *vctx, int64_t ip)
{
    const orc_traj_ctx *c = (const orc_traj_ctx *)vctx;
    const int64_t n_steps = c->n_steps;
    double z = c->z0[ip], v = c->v0[ip];
    int64_t na = n_steps;
    double *zt = c->z_traj ? c->z_traj + ip * n_steps : NULL;
    double *vt = c->v_traj ? c->v_traj + ip * n_steps : NULL;
    if (zt) { zt[0] = z; vt[0] = v; }
    for (int64_t j = 1; j < n_steps; j++) {
        double force;
        orc_point(&c->m, &c->bm, c->BR, v, z, c->Bgrad, c->flags, &force, NULL, NULL);
        const double a = force / c->mass;
        v = v + a * c->dt;
        z = z + v * c->dt;
        if (zt) { zt[j] = z; vt[j] = v; }
        if (fabs(z) > c->z_escape) {
            na = j;
            if (zt)
                for (int64_t s = j + 1; s < n_steps; s++) { zt[s] = z; vt[s] = v; }
            break;
        }
    }
    c->z_final[ip] = z;
    c->v_final[ip] = v;
    c->n_actual[ip] = (int32_t)na;
}

int orc_traj1d(int n_g, int n_e, const double *E, const double *d2, const double *zd,
               double Gamma, double k, double Geff, double hbar, int flags,
               int n_b, const double *kdir, const double *freq, const double *pol,
               const double *s0, double Bgrad, double mass, double dt, int64_t n_steps,
               double z_escape, int64_t n_part, const double *z0, const double *v0,
               int n_threads, double *z_final, double *v_final, int32_t *n_actual,
               double *z_traj, double *v_traj)
{
    if (orc_check(n_g, n_e, n_b) || n_steps < 1) return -1;
    orc_traj_ctx *c = (orc_traj_ctx *)calloc(1, sizeof(orc_traj_ctx));
    if (!c) return -2;
    orc_mol m = {n_g, n_e, E, d2, zd, Gamma, k, Geff, hbar};
    orc_beams bm = {n_b, kdir, freq, pol, s0};
    c->m = m; c->bm = bm;
    orc_branching(&c->m, c->BR);
    c->flags = flags; c->Bgrad = Bgrad; c->mass = mass; c->dt = dt; c->z_escape = z_escape;
    c->n_steps = n_steps; c->z0 = z0; c->v0 = v0;
    c->z_final = z_final; c->v_final = v_final; c->n_actual = n_actual;
    c->z_traj = z_traj; c->v_traj = v_traj;
    orc_parallel_for(n_part, n_threads, orc_traj_body, c);
    free(c);
    return 0;
}
