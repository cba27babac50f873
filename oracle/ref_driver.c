/*
 * Test-oracle driver around the UNMODIFIED reference sources (compiled from the
 * C files under simulation/ by oracle/Makefile into oracle/_ref/libephref.so).
 *
 * This file is test infrastructure: only tests/, __graft_entry__.smoke() and
 * bench.py's CPU-baseline / reference arm load the resulting library, and only
 * as the checker or as the timed CPU reference, never as the product path.
 *
 * It exposes flat C entry points (plain pointers, no FILE*, no fftw_plan) so
 * Python's ctypes can drive the reference functions:
 *   - seeding: the reference seeds MT19937-64 with time(NULL)
 *     (simulation/organic_hmc.c:314, organic_trans_loc.c:97); the Makefile
 *     compiles those files with -Dtime=ephref_time so the seed is settable;
 *   - one force+logdet evaluation = construct_M_hat + logDetM_and_inv_M_hat +
 *     force, exactly the body of leap_frog (simulation/organic_hmc.c:177-180);
 *   - the Fourier-acceleration routines bound to plans over [x|p] and [xc|pc]
 *     exactly as run_hmc lays them out (simulation/organic_hmc.c:307-322);
 *   - organic_main's main() renamed to ref_organic_main (-Dmain=...).
 */
#define _GNU_SOURCE
#include <complex.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#include <omp.h>

#include "mt19937-64.h"
#include "organic_random.h"
#include "organic_flags.h"
#include "organic_aux.h"
#include "organic_lattice.h"
#include "organic_dense_matrix.h"
#include "organic_bosons.h"
#include "organic_hmc.h"
#include "organic_trans_loc.h"

/* ------------------------------------------------------------------ seeding */
static unsigned long g_seed_time = 1;

time_t ephref_time(time_t *t) {
    if (t) *t = (time_t)g_seed_time;
    return (time_t)g_seed_time;
}

void ref_set_seed_time(unsigned long s) { g_seed_time = s; }

void ref_init(void) { set_taylor_pair_order(); }

extern void openblas_set_num_threads(int);

void ref_set_threads(int n) {
    if (n < 1) n = 1;
    omp_set_num_threads(n);
    openblas_set_num_threads(n);
}

int ref_max_threads(void) { return omp_get_max_threads(); }

/* ------------------------------------------------------------------ RNG */
void ref_init_genrand64(unsigned long seed) { init_genrand64(seed); }
double ref_genrand64_real2(void) { return genrand64_real2(); }
void ref_random_vector_only(double *x, unsigned n) { random_vector(x, n); }

void ref_random_vector(unsigned long seed, double *x, unsigned n) {
    init_genrand64(seed);
    random_vector(x, n);
}

/* ------------------------------------------------------------------ lattice */
void ref_lattice(unsigned l1, unsigned l2, unsigned *out, unsigned *ns, unsigned *nn) {
    unsigned *nnt = construct_triangular(l1, l2, ns, nn);
    memcpy(out, nnt, sizeof(unsigned) * 2 * (*nn) * (*ns));
    free(nnt);
}

static void fill_flags(organic_flags *m, const int *f) {
    memset(m, 0, sizeof(*m));
    if (!f) return;
    m->schur_form_inv = f[0];
    m->zero_filling = f[1];
    m->static_disorder = f[2];
    m->single_particle = f[3];
    m->constant_force = f[4];
    m->no_fourier_acc = f[5];
    m->classical_fourier_acc = f[6];
    m->cfa_steps = 1;
    m->cfa_mass = 0;
}

/* ------------------------------------------------------------------ eval context */
typedef struct {
    unsigned l1, l2, nt, ns, nn;
    unsigned *nnt;
    double t[3], kappa[3], mu, omega;
    unsigned flavors;
    organic_flags mode;
    double *M_hat, *QM1P, *w;
    int *perm;
    double last_time_s;
} ref_ctx;

ref_ctx *ref_ctx_new(unsigned l1, unsigned l2, unsigned nt, const double *t,
                     const double *kappa, double mu, double omega,
                     unsigned flavors, const int *flags) {
    ref_ctx *c = calloc(1, sizeof(*c));
    c->l1 = l1; c->l2 = l2; c->nt = nt;
    c->nnt = construct_triangular(l1, l2, &c->ns, &c->nn);
    for (int k = 0; k < 3; k++) { c->t[k] = t[k]; c->kappa[k] = kappa[k]; }
    c->mu = mu; c->omega = omega; c->flavors = flavors;
    fill_flags(&c->mode, flags);
    const size_t md = (size_t)c->ns * c->ns;
    c->M_hat = malloc(sizeof(double) * md);
    c->QM1P = malloc(sizeof(double) * md * nt);
    c->w = malloc(sizeof(double) * md * 5);
    const unsigned np = c->ns > 2 * nt ? c->ns : 2 * nt;
    c->perm = malloc(sizeof(int) * np);
    set_taylor_pair_order();
    return c;
}

void ref_ctx_free(ref_ctx *c) {
    if (!c) return;
    free(c->nnt); free(c->M_hat); free(c->QM1P); free(c->w); free(c->perm);
    free(c);
}

static double now_s(void) {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

/* One evaluation as in leap_frog (simulation/organic_hmc.c:177-180).
 * x is read-only for the caller (copied).  Outputs (optional, may be NULL):
 *   p_dot[dim], M_hat_pre[V*V] (before LU), M_inv[V*V] (after dgetri).
 * Returns log|det M|; the wall time of the three calls is kept in the ctx. */
double ref_ctx_eval(ref_ctx *c, const double *x_in, double *p_dot, double *M_hat_pre, double *M_inv) {
    const unsigned dim = c->nt * c->ns * c->nn / 2;
    double *x = malloc(sizeof(double) * dim);
    double *pd = malloc(sizeof(double) * dim);
    memcpy(x, x_in, sizeof(double) * dim);
    const size_t md = (size_t)c->ns * c->ns;

    const double t0 = now_s();
    construct_M_hat(x, c->M_hat, c->w, c->t, c->kappa, c->mu, c->nnt, c->ns, c->nn, c->nt, &c->mode);
    if (M_hat_pre) memcpy(M_hat_pre, c->M_hat, sizeof(double) * md);
    const double t1 = now_s();
    const double logdet = logDetM_and_inv_M_hat(c->M_hat, c->w, c->perm, c->ns, c->flavors, &c->mode);
    force(x, pd, c->M_hat, c->QM1P, c->w, c->perm, c->t, c->kappa, c->mu, c->omega, c->flavors, c->nnt, c->ns, c->nn, c->nt, logdet, &c->mode);
    const double t2 = now_s();
    c->last_time_s = (t2 - t1) + (t1 - t0);

    if (p_dot) memcpy(p_dot, pd, sizeof(double) * dim);
    if (M_inv) memcpy(M_inv, c->M_hat, sizeof(double) * md);
    free(x); free(pd);
    return logdet;
}

double ref_ctx_last_time(const ref_ctx *c) { return c->last_time_s; }

/* construct_M_hat alone (simulation/organic_dense_matrix.c:251-265). */
void ref_ctx_construct_M_hat(ref_ctx *c, const double *x_in, double *M_hat_out) {
    const unsigned dim = c->nt * c->ns * c->nn / 2;
    double *x = malloc(sizeof(double) * dim);
    memcpy(x, x_in, sizeof(double) * dim);
    construct_M_hat(x, M_hat_out, c->w, c->t, c->kappa, c->mu, c->nnt, c->ns, c->nn, c->nt, &c->mode);
    free(x);
}

/* apply_exp_mu_K_to_M for one slice on a caller matrix (in place). */
void ref_ctx_apply_exp(ref_ctx *c, const double *x_slice, double *M, int revert, int stop) {
    const unsigned ld = c->ns * c->nn / 2;
    double *x = malloc(sizeof(double) * ld);
    memcpy(x, x_slice, sizeof(double) * ld);
    apply_exp_mu_K_to_M(x, M, c->w, c->t, c->kappa, c->mu, c->nnt, c->ns, c->nn, revert, stop);
    free(x);
}

/* apply_mu_K_to_v on one vector (simulation/organic_dense_matrix.c:96-120). */
void ref_ctx_apply_mu_K_v(ref_ctx *c, const double *x_slice, const double *v, double *w_out) {
    const unsigned ld = c->ns * c->nn / 2;
    double *x = malloc(sizeof(double) * ld);
    double *vv = malloc(sizeof(double) * c->ns);
    memcpy(x, x_slice, sizeof(double) * ld);
    memcpy(vv, v, sizeof(double) * c->ns);
    apply_mu_K_to_v(x, vv, w_out, c->t, c->kappa, c->mu, c->nnt, c->ns, c->nn);
    free(x); free(vv);
}

/* construct_all_QM1P from a given M_inv (G_t before refinement, all t). */
void ref_ctx_all_QM1P(ref_ctx *c, const double *x_in, const double *M_inv, double *G_out) {
    const unsigned dim = c->nt * c->ns * c->nn / 2;
    const size_t md = (size_t)c->ns * c->ns;
    double *x = malloc(sizeof(double) * dim);
    double *Mi = malloc(sizeof(double) * md);
    memcpy(x, x_in, sizeof(double) * dim);
    memcpy(Mi, M_inv, sizeof(double) * md);
    construct_all_QM1P(x, Mi, c->QM1P, c->w, c->perm, c->t, c->kappa, c->mu, c->nnt, c->ns, c->nn, c->nt, &c->mode);
    memcpy(G_out, c->QM1P, sizeof(double) * md * c->nt);
    free(x); free(Mi);
}

/* refine_QM1P for one slice, in place on G (simulation/organic_dense_matrix.c:383-442). */
void ref_ctx_refine(ref_ctx *c, const double *x_in, double *G, int time) {
    const unsigned dim = c->nt * c->ns * c->nn / 2;
    double *x = malloc(sizeof(double) * dim);
    memcpy(x, x_in, sizeof(double) * dim);
    refine_QM1P(x, G, c->w, c->t, c->kappa, c->mu, c->nnt, c->ns, c->nn, time);
    free(x);
}

/* LU log-det + inverse alone (simulation/organic_dense_matrix.c:547-607). */
double ref_ctx_logdet_inv(ref_ctx *c, double *M_inout) {
    return logDetM_and_inv_M_hat(M_inout, c->w, c->perm, c->ns, c->flavors, &c->mode);
}

/* hamilton (simulation/organic_hmc.c:67-84). */
double ref_hamilton(const double *x_in, double logDetM, double energyP, double omega,
                    unsigned flavors, unsigned ns, unsigned nt) {
    const unsigned dim = nt * ns * 3;
    double *x = malloc(sizeof(double) * dim);
    memcpy(x, x_in, sizeof(double) * dim);
    const double h = hamilton(x, NULL, logDetM, energyP, omega, flavors, ns, 6, nt);
    free(x);
    return h;
}

/* check_force (simulation/organic_hmc.c:20-54): p_dot supplied by the caller. */
double ref_ctx_check_force(ref_ctx *c, const double *x_in, const double *p_dot) {
    const unsigned dim = c->nt * c->ns * c->nn / 2;
    double *x = malloc(sizeof(double) * dim);
    double *pd = malloc(sizeof(double) * dim);
    memcpy(x, x_in, sizeof(double) * dim);
    memcpy(pd, p_dot, sizeof(double) * dim);
    const double r = check_force(x, NULL, pd, c->M_hat, c->w, c->perm, c->t, c->kappa, c->mu, c->omega, c->flavors, c->nnt, c->ns, c->nn, c->nt, &c->mode);
    free(x); free(pd);
    return r;
}

/* ------------------------------------------------------------------ Fourier acceleration */
typedef struct {
    unsigned ns, nt, loc_dim, dim, compl_dim;
    double *xp;            /* [x | p], dim each */
    double complex *xc;    /* [xc | pc], compl_dim each */
    fftw_plan fft[4];
} ref_fa;

ref_fa *ref_fa_new(unsigned ns, unsigned nt) {
    ref_fa *f = calloc(1, sizeof(*f));
    f->ns = ns; f->nt = nt;
    f->loc_dim = ns * 3;
    f->dim = nt * f->loc_dim;
    f->compl_dim = f->loc_dim * (nt / 2 + 1);
    f->xp = malloc(sizeof(double) * 2 * f->dim);
    f->xc = malloc(sizeof(double complex) * 2 * f->compl_dim);
    int fft_dim[1] = {(int)nt};
    const int ld = (int)f->loc_dim;
    double *x = f->xp;
    double complex *xc = f->xc;
    /* same four plans as simulation/organic_hmc.c:319-322 */
    f->fft[0] = fftw_plan_many_dft_r2c(1, fft_dim, ld, x, NULL, ld, 1, xc, NULL, ld, 1, FFTW_MEASURE);
    f->fft[1] = fftw_plan_many_dft_r2c(1, fft_dim, ld, x + f->dim, NULL, ld, 1, xc + f->compl_dim, NULL, ld, 1, FFTW_MEASURE);
    f->fft[2] = fftw_plan_many_dft_c2r(1, fft_dim, ld, xc, NULL, ld, 1, x, NULL, ld, 1, FFTW_MEASURE);
    f->fft[3] = fftw_plan_many_dft_c2r(1, fft_dim, ld, xc + f->compl_dim, NULL, ld, 1, x + f->dim, NULL, ld, 1, FFTW_MEASURE);
    return f;
}

void ref_fa_free(ref_fa *f) {
    if (!f) return;
    for (int i = 0; i < 4; i++) fftw_destroy_plan(f->fft[i]);
    free(f->xp); free(f->xc); free(f);
}

void ref_fa_set(ref_fa *f, const double *x, const double *p) {
    if (x) memcpy(f->xp, x, sizeof(double) * f->dim);
    if (p) memcpy(f->xp + f->dim, p, sizeof(double) * f->dim);
}

void ref_fa_get(const ref_fa *f, double *x, double *p) {
    if (x) memcpy(x, f->xp, sizeof(double) * f->dim);
    if (p) memcpy(p, f->xp + f->dim, sizeof(double) * f->dim);
}

/* evolve_bosons (simulation/organic_bosons.c:126-150) */
void ref_fa_evolve(ref_fa *f, double omega, double h) {
    evolve_bosons(f->xc, omega, f->ns, 6, f->nt, f->fft, h);
}

/* sample_fourier_momenta (simulation/organic_bosons.c:76-100); uses the
 * current MT stream state (seed it with ref_init_genrand64). */
void ref_fa_sample_momenta(ref_fa *f, double omega, const int *flags) {
    organic_flags m;
    fill_flags(&m, flags);
    sample_fourier_momenta(f->xp + f->dim, f->xc + f->compl_dim, omega, f->ns, 6, f->nt, f->fft, &m);
}

/* energy_fourier_momenta (simulation/organic_bosons.c:102-124) */
double ref_fa_energy(ref_fa *f, double omega) {
    return energy_fourier_momenta(f->xc + f->compl_dim, omega, f->ns, 6, f->nt, f->fft);
}

/* evolve_bosons_approx_step (simulation/organic_bosons.c:152-177) with
 * CLASSICAL_FOURIER_ACC set and the given mass */
void ref_fa_approx_step(ref_fa *f, double omega, double h, double cfa_mass) {
    organic_flags m;
    memset(&m, 0, sizeof(m));
    m.classical_fourier_acc = 1;
    m.cfa_steps = 1;
    m.cfa_mass = cfa_mass;
    evolve_bosons_approx_step(f->xc, omega, f->ns, 6, f->nt, f->fft, h, &m);
}

/* update_x (simulation/organic_hmc.c:136-165) on [x|p] with the given flags
 * (as fill_flags reads them) and classical acceleration parameters; p_dot is
 * caller scratch of dim doubles */
void ref_fa_update_x(ref_fa *f, double *p_dot, double omega, double h, double half, const int *flags,
                     unsigned cfa_steps, double cfa_mass) {
    organic_flags m;
    fill_flags(&m, flags);
    m.cfa_steps = cfa_steps;
    m.cfa_mass = cfa_mass;
    update_x(f->xp, f->xp + f->dim, p_dot, f->xc, omega, f->ns, 6, f->nt, f->fft, h, half, &m);
}

/* sample_free_bosons (simulation/organic_bosons.c:55-74) */
void ref_fa_sample_free(ref_fa *f, double omega) {
    sample_free_bosons(f->xp, f->xc, omega, f->ns, 6, f->nt, f->fft);
}

/* higher_Matsubaras_norm (simulation/organic_bosons.c:36-53) */
double ref_higher_matsubaras_norm(const double *x_in, unsigned ns, unsigned nt) {
    const unsigned dim = nt * ns * 3;
    double *x = malloc(sizeof(double) * dim);
    memcpy(x, x_in, sizeof(double) * dim);
    const double r = higher_Matsubaras_norm(x, NULL, ns, 6, nt);
    free(x);
    return r;
}

/* boson_force (simulation/organic_bosons.c:179-194) */
void ref_boson_force(const double *x_in, double *p_dot, double omega, unsigned ns, unsigned nt, int overwrite) {
    const unsigned dim = nt * ns * 3;
    double *x = malloc(sizeof(double) * dim);
    memcpy(x, x_in, sizeof(double) * dim);
    boson_force(x, p_dot, omega, ns, 6, nt, overwrite);
    free(x);
}

/* ------------------------------------------------------------------ whole programs */
int ref_organic_main(int argc, char **argv);

int ref_run_main(unsigned long seed, const char *input, const char *res, const char *corr) {
    g_seed_time = seed;
    char *argv[5];
    argv[0] = (char *)"organic_main";
    argv[1] = (char *)input;
    argv[2] = (char *)res;
    argv[3] = (char *)corr;
    argv[4] = NULL;
    return ref_organic_main(corr ? 4 : 3, argv);
}

/* correlator pieces (simulation/organic_dense_matrix.c:451-524) with M_inv given */
void ref_ctx_cc_correlator(ref_ctx *c, const double *x_in, const double *M_inv, double logDetM, double *greens) {
    const unsigned dim = c->nt * c->ns * c->nn / 2;
    const size_t md = (size_t)c->ns * c->ns;
    double *x = malloc(sizeof(double) * dim);
    double *Mi = malloc(sizeof(double) * md);
    double *R0t = malloc(sizeof(double) * md);
    memcpy(x, x_in, sizeof(double) * dim);
    memcpy(Mi, M_inv, sizeof(double) * md);
    cc_correlator(x, Mi, c->QM1P, R0t, c->w, c->t, c->kappa, c->mu, c->nnt, c->ns, c->nn, c->nt, greens, logDetM, &c->mode);
    free(x); free(Mi); free(R0t);
}

/* ------------------------------------------------------------------ static disorder (TL mode) */
/* hist_trans_loc (simulation/organic_trans_loc.c:25-83) for nsamples samples in
 * a row, the way run_trans_loc calls it (:102-103), on the MT19937-64 stream
 * seeded with `seed`.  greens[nbins] += the summed sample histograms (not
 * divided by nsamples); z[s] = results[0] of sample s; x_out[s*3ns ...] (may be
 * NULL) = the bond field drawn for sample s.  The histogram is laid out as in
 * organic_main (greens, then one result per sample) with room behind it for
 * bins past the end, which the reference writes there; returns 1 if any such
 * bin was written, else 0. */
int ref_trans_loc_samples(unsigned long seed, unsigned l1, unsigned l2, unsigned nbins, const double *t_in,
                          const double *kappa_in, double mu, const double *contr_in, double width,
                          unsigned nsamples, double *greens, double *z, double *x_out) {
    unsigned ns, nn;
    unsigned *nnt = construct_triangular(l1, l2, &ns, &nn);
    const unsigned nn2 = nn / 2, dim = ns * nn2, mat_dim = ns * ns;
    const size_t slack = 64 * (size_t)nbins + 4096;
    const size_t room = nbins + nsamples + slack;
    double *buf = calloc(room, sizeof(double));
    double *x = malloc((dim + 2 * mat_dim + ns + (nn2 + 1) * nn2) * sizeof(double));
    double t[3], kappa[3], contr[6];
    memcpy(t, t_in, sizeof t);
    memcpy(kappa, kappa_in, sizeof kappa);
    memcpy(contr, contr_in, sizeof contr);
    int overflow = 0;
    init_genrand64(seed);
    for (unsigned s = 0; s < nsamples; s++) {
        for (unsigned r = s; r < nsamples; r++) overflow |= buf[nbins + r] != 0;
        hist_trans_loc(x, t, kappa, mu, contr, nnt, ns, nn, nbins, width, buf + nbins + s, buf, NULL);
        z[s] = buf[nbins + s];
        if (x_out) memcpy(x_out + (size_t)s * dim, x, sizeof(double) * dim);
    }
    for (size_t b = nbins + nsamples; b < room; b++) overflow |= buf[b] != 0;
    for (unsigned b = 0; b < nbins; b++) greens[b] += buf[b];
    free(buf);
    free(x);
    free(nnt);
    return overflow;
}

/* run_trans_loc (simulation/organic_trans_loc.c:85-114) with time(NULL) = seed:
 * greens[nbins + meas] as organic_main allocates it; returns its length. */
unsigned ref_run_trans_loc(unsigned long seed, unsigned l1, unsigned l2, unsigned nbins, const double *t_in,
                           const double *kappa_in, double mu, const double *contr_in, unsigned meas,
                           const char *res_name, const char *corr_name, double *greens) {
    double t[3], kappa[3], contr[6];
    memcpy(t, t_in, sizeof t);
    memcpy(kappa, kappa_in, sizeof kappa);
    memcpy(contr, contr_in, sizeof contr);
    g_seed_time = seed;
    return run_trans_loc(greens, l1, l2, nbins, t, kappa, mu, contr, meas, res_name, corr_name);
}

/* ------------------------------------------------------------------ conductivity post-processing */
/* organic_conv's main (simulation/organic_conv.c:123-164), renamed by the Makefile */
int ref_conv_main(int argc, char **argv);

int ref_run_conv(const char *greens, const char *smear, const char *out_w, const char *out_t) {
    char *argv[6];
    argv[0] = (char *)"organic_conv";
    argv[1] = (char *)greens;
    argv[2] = (char *)smear;
    argv[3] = (char *)out_w;
    argv[4] = (char *)out_t;
    argv[5] = NULL;
    return ref_conv_main(out_t ? 5 : 4, argv);
}
