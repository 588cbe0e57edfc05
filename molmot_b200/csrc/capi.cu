// capi.cu -- handles (molecule packs, beam sets), error reporting, version.
#include <stdarg.h>
#include <stdio.h>
#include <string.h>
#include <vector>
#include "common.cuh"

static thread_local char g_err[512] = "";

void mm_set_error(const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof g_err, fmt, ap);
    va_end(ap);
}

int mm_cuda_check(cudaError_t e, const char *what)
{
    if (e == cudaSuccess) return 0;
    mm_set_error("%s: %s", what, cudaGetErrorString(e));
    // the error is reported here; clear the runtime's pending copy of it so a
    // later, unrelated check in this thread does not return it again
    (void)cudaGetLastError();
    return 1;
}

extern "C" const char *mm_last_error(void) { return g_err; }

extern "C" const char *mm_version(void) { return "molmot_b200 0.1.0 (sm_100a)"; }

template <class T>
static int upload(T **dst, const T *src, size_t n)
{
    *dst = nullptr;
    if (n == 0) return 0;
    if (mm_cuda_check(cudaMalloc((void **)dst, n * sizeof(T)), "cudaMalloc")) return -3;
    if (mm_cuda_check(cudaMemcpy(*dst, src, n * sizeof(T), cudaMemcpyHostToDevice), "cudaMemcpy")) {
        cudaFree(*dst);
        *dst = nullptr;
        return -3;
    }
    return 0;
}

// Branching ratios BR[e][g] in the order of molmot/obe/rate_equations_jit.py:38-49.
static void branching(int n_g, int n_e, const double *d2, double *BR)
{
    for (int ie = 0; ie < n_e; ie++) {
        double total = 0.0;
        for (int ig = 0; ig < n_g; ig++)
            for (int q = 0; q < 3; q++) total += d2[(ig * n_e + ie) * 3 + q];
        for (int ig = 0; ig < n_g; ig++) {
            double s = 0.0;
            for (int q = 0; q < 3; q++) s += d2[(ig * n_e + ie) * 3 + q];
            BR[ie * n_g + ig] = total > 1e-30 ? s / total : 0.0;
        }
    }
}

extern "C" int mm_pack_create(const mm_mol_desc *d, mm_pack **out)
{
    if (!out) { mm_set_error("out is null"); return -1; }
    *out = nullptr;
    if (!d || !d->energies || !d->d_squared || !d->zeeman_z_diag) {
        mm_set_error("molecule description incomplete (energies, d_squared, zeeman_z_diag)");
        return -1;
    }
    const int n_g = d->n_ground, n_e = d->n_excited;
    if (n_g < 2 || n_g > MM_MAX_GROUND || n_e < 1 || n_e > MM_MAX_EXCITED) {
        mm_set_error("n_ground=%d (2..%d) / n_excited=%d (1..%d) out of range", n_g, MM_MAX_GROUND,
                     n_e, MM_MAX_EXCITED);
        return -1;
    }
    if (!(d->Gamma > 0) || !(d->k > 0) || !(d->mass > 0)) {
        mm_set_error("Gamma, k and mass must be positive");
        return -1;
    }
    const int n_s = n_g + n_e;
    const bool has3d = d->zeeman_ground_re && d->zeeman_ground_im && d->tdm_abs && d->zeeman_excited_z;
    mm_pack *p = new mm_pack();
    p->n_g = n_g; p->n_e = n_e; p->n_s = n_s;
    p->Gamma = d->Gamma; p->k = d->k; p->mass = d->mass;
    p->has3d = has3d ? 1 : 0;
    cudaGetDevice(&p->device);
    size_t o = 0;
    p->oE = o; o += n_s;
    p->ozd = o; o += n_s;
    p->od2 = o; o += (size_t)n_g * n_e * 3;
    p->oBR = o; o += (size_t)n_e * n_g;
    p->oZre = o; o += has3d ? 3 * (size_t)n_g * n_g : 0;
    p->oZim = o; o += has3d ? 3 * (size_t)n_g * n_g : 0;
    p->oZe = o; o += has3d ? n_e : 0;
    p->oTdm = o; o += has3d ? (size_t)n_g * n_e * 3 : 0;
    p->n_buf = o;
    std::vector<double> h(o, 0.0);
    memcpy(&h[p->oE], d->energies, sizeof(double) * n_s);
    memcpy(&h[p->ozd], d->zeeman_z_diag, sizeof(double) * n_s);
    memcpy(&h[p->od2], d->d_squared, sizeof(double) * n_g * n_e * 3);
    branching(n_g, n_e, d->d_squared, &h[p->oBR]);
    if (has3d) {
        memcpy(&h[p->oZre], d->zeeman_ground_re, sizeof(double) * 3 * n_g * n_g);
        memcpy(&h[p->oZim], d->zeeman_ground_im, sizeof(double) * 3 * n_g * n_g);
        memcpy(&h[p->oZe], d->zeeman_excited_z, sizeof(double) * n_e);
        memcpy(&h[p->oTdm], d->tdm_abs, sizeof(double) * n_g * n_e * 3);
    }
    for (size_t i = 0; i < o; i++)
        if (!isfinite(h[i])) { mm_set_error("molecule data contains a non-finite value"); delete p; return -1; }
    p->act.resize((size_t)n_g * n_e * 3);
    for (size_t i = 0; i < p->act.size(); i++) p->act[i] = d->d_squared[i] >= 1e-15 ? 1 : 0;
    p->h_br.assign(h.begin() + p->oBR, h.begin() + p->oBR + (size_t)n_e * n_g);
    if (upload(&p->buf, h.data(), o)) { delete p; return -3; }
    *out = p;
    return 0;
}

extern "C" int mm_pack_destroy(mm_pack *p)
{
    if (!p) return 0;
    if (p->buf) cudaFree(p->buf);
    delete p;
    return 0;
}

extern "C" int mm_beams_create(const mm_beam_desc *d, int32_t n_sets, mm_beams **out)
{
    if (!out) { mm_set_error("out is null"); return -1; }
    *out = nullptr;
    if (!d || !d->kdir || !d->freq || !d->pol || !d->s0 || !d->b_gradient) {
        mm_set_error("beam description incomplete (kdir, freq, pol, s0, b_gradient)");
        return -1;
    }
    const int n_b = d->n_beams;
    if (n_b < 1 || n_b > MM_MAX_BEAMS || n_sets < 1) {
        mm_set_error("n_beams=%d (1..%d) or n_sets=%d (>= 1) out of range", n_b, MM_MAX_BEAMS, n_sets);
        return -1;
    }
    const size_t nb = (size_t)n_b * n_sets;
    for (size_t i = 0; i < nb; i++) {
        if (d->pol[i] < 0 || d->pol[i] > 2) { mm_set_error("polarization index %d not in {0,1,2}", d->pol[i]); return -1; }
        if (!isfinite(d->kdir[i]) || !isfinite(d->freq[i]) || !isfinite(d->s0[i])) {
            mm_set_error("beam %zu has a non-finite parameter", i);
            return -1;
        }
    }
    for (int s = 0; s < n_sets; s++)
        if (!isfinite(d->b_gradient[s])) { mm_set_error("set %d has a non-finite B gradient", s); return -1; }
    mm_beams *b = new mm_beams();
    b->n_sets = n_sets; b->n_b = n_b; b->gamma_eff = d->gamma_eff;
    b->h_pol_store = std::make_shared<std::vector<int32_t>>(d->pol, d->pol + nb);
    b->h_pol = b->h_pol_store->data();
    b->has3d = (d->khat != nullptr) ? 1 : 0;
    cudaGetDevice(&b->device);
    int rc = 0;
    rc |= upload(&b->kdir, d->kdir, nb);
    rc |= upload(&b->freq, d->freq, nb);
    rc |= upload(&b->s0, d->s0, nb);
    rc |= upload(&b->pol, d->pol, nb);
    rc |= upload(&b->bgrad, d->b_gradient, (size_t)n_sets);
    if (d->khat) rc |= upload(&b->khat, d->khat, nb * 3);
    if (d->radius) rc |= upload(&b->radius, d->radius, nb);
    if (rc) { mm_beams_destroy(b); return -3; }
    *out = b;
    return 0;
}

extern "C" int mm_beams_destroy(mm_beams *b)
{
    if (!b) return 0;
    if (!b->view) {
        cudaFree(b->kdir); cudaFree(b->freq); cudaFree(b->s0); cudaFree(b->pol);
        cudaFree(b->bgrad); cudaFree(b->khat); cudaFree(b->radius);
    }
    delete b;
    return 0;
}

extern "C" int mm_beams_view(const mm_beams *parent, int32_t first_set, int32_t n_sets, mm_beams **out)
{
    if (!out) { mm_set_error("out is null"); return -1; }
    *out = nullptr;
    if (!parent) { mm_set_error("parent is null"); return -1; }
    if (first_set < 0 || n_sets < 1 || first_set + (long long)n_sets > parent->n_sets) {
        mm_set_error("sets [%d, %d) outside the parent's %d", first_set, first_set + n_sets, parent->n_sets);
        return -1;
    }
    mm_beams *b = new mm_beams(*parent);
    const size_t o = (size_t)first_set * parent->n_b;
    b->n_sets = n_sets;
    b->kdir += o; b->freq += o; b->s0 += o; b->pol += o;
    b->h_pol += o;
    b->bgrad += first_set;
    if (b->khat) b->khat += 3 * o;
    if (b->radius) b->radius += o;
    b->view = 1;
    *out = b;
    return 0;
}
