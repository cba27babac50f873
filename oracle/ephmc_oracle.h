/*
 * CPU restatement of the electron-phonon HMC hot path (TEST ORACLE ONLY).
 *
 * Plain C, double precision, written for this project from the reference's
 * algorithm (j-ostmeyer/electron-phonon-hmc, the C files under simulation/); each function
 * cites the reference file:line it restates.  Only tests/, the smoke check and
 * bench.py's CPU-baseline leg use it, as the checker.  It is pinned against the
 * reference itself, compiled unmodified into oracle/_ref (see oracle/Makefile).
 *
 * Conventions shared with the reference:
 *   V = L1*L2 sites, 6 neighbours, 3 links per site, Nt slices;
 *   x[(t*V + i)*3 + k]  phonon field of link k of site i at slice t;
 *   matrices are V*V doubles; "row" r is the contiguous segment r*V..r*V+V-1,
 *   the stencil acts on each row (LAPACK sees these as columns).
 */
#ifndef EPHMC_ORACLE_H
#define EPHMC_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    unsigned l1, l2, ns, nt, flavors;
    double t[3], kappa[3], mu, omega;
    /* flags in the order of organic_flags (simulation/organic_flags.h:4-11):
       schur_form_inv, zero_filling, static_disorder, single_particle,
       constant_force, no_fourier_acc, classical_fourier_acc */
    int flags[7];
    unsigned *nnt; /* 12*V, as construct_triangular */
} or_model;

/* MT19937-64 + Box-Muller normals */
void or_mt_seed(unsigned long long seed);
double or_mt_real2(void);
void or_normals(double *x, unsigned n);

/* lattice and parameters */
void or_lattice(unsigned l1, unsigned l2, unsigned *nnt);
void or_convert_params(double beta, unsigned nt, const double *J, const double *lam,
                       double mu0, double omega0, int static_disorder,
                       double *t, double *kappa, double *mu, double *omega);
void or_pair_coeffs(double *a_lin, double *a_quad, int *is_complex);

or_model *or_model_new(unsigned l1, unsigned l2, unsigned nt, const double *t,
                       const double *kappa, double mu, double omega,
                       unsigned flavors, const int *flags);
void or_model_free(or_model *m);

/* stencil and slice propagators */
void or_apply_mu_K_v(const or_model *m, const double *x_slice, const double *v, double *w);
void or_apply_exp_M(const or_model *m, const double *x_slice, double *M, int revert, int stop);
void or_construct_M_hat(const or_model *m, const double *x, double *M);

/* LU log-det and in-place inverse; returns log|det|, *sign_out = +-1 */
double or_logdet_inverse(double *M, unsigned n, int *sign_out);

/* force pieces (reference algorithm) */
void or_all_G(const or_model *m, const double *x, const double *M_inv, double *G);
void or_refine(const or_model *m, const double *x, double *G, unsigned t);
void or_contract(const or_model *m, const double *G_t, unsigned t, double logdet, double *p_dot);

/* one force+logdet evaluation, reference algorithm; M_inv_out optional */
double or_eval_reference(const or_model *m, const double *x, double *p_dot, double *M_inv_out, int *sign_out);
/* same quantities by the O(Nt) adjoint; single != 0 rounds the adjoint sweep
   (q storage, y chain, contraction) to float to model the mixed path */
double or_eval_adjoint(const or_model *m, const double *x, double *p_dot, int single);

double or_hamilton(const double *x, double logdet, double energyP, double omega,
                   unsigned flavors, unsigned ns, unsigned nt);
double or_check_force(const or_model *m, const double *x, const double *p_dot);

/* Fourier acceleration (FFTW conventions, series stride = 3V) */
void or_rdft_forward(const double *x, double *Xc, unsigned ld, unsigned nt);
void or_rdft_inverse(const double *Xc, double *x, unsigned ld, unsigned nt);
void or_evolve_bosons(double *x, double *p, double omega, unsigned ns, unsigned nt, double h);
void or_sample_fourier_momenta(double *p, double omega, unsigned ns, unsigned nt);
double or_energy_fourier_momenta(const double *p, double omega, unsigned ns, unsigned nt);
void or_sample_free_bosons(double *x, double omega, unsigned ns, unsigned nt);
double or_higher_matsubaras_norm(const double *x, unsigned ns, unsigned nt);

#ifdef __cplusplus
}
#endif
#endif
