/*
 * Drop-in surface of libephmc_cuda.so: the reference's own function names and
 * prototypes, so the reference's C host code (organic_main.c, organic_R.c)
 * links against this library in place of organic_dense_matrix.o,
 * organic_hmc.o, organic_bosons.o and organic_trans_loc.o.  Each declaration cites the reference
 * prototype it replaces.
 *
 * Pointers may be host memory (as the reference's own callers pass them) or
 * device memory (from ephmc_alloc, used in place).  Work arrays the reference
 * requires from its callers (w, perm, QM1P, xc) are accepted and may be used
 * as staging space; results go where the reference puts them.  Outcomes the
 * reference only prints are also reported through ephmc_last_status() and
 * ephmc_last_warnings() (ephmc.h).
 *
 * fftw_plan is an opaque handle made by ephmc_fftw_plan_many_dft_r2c/_c2r
 * (FFTW's argument lists); it records the buffers a plan binds, as
 * evolve_bosons & co. find x and p through the plans
 * (simulation/organic_hmc.c:317-322).
 */
#ifndef EPHMC_ORGANIC_H
#define EPHMC_ORGANIC_H

#include <stdio.h>

#include "ephmc.h"

#ifdef __cplusplus
typedef __complex__ double ephmc_dcomplex;
extern "C" {
#else
typedef double _Complex ephmc_dcomplex;
#endif

#ifndef ORGANIC_FLAGS
typedef ephmc_flags organic_flags; /* simulation/organic_flags.h:4-14, same layout */
#endif

typedef struct fftw_plan_s *fftw_plan; /* FFTW3's own spelling of the handle type */

/* ---- simulation/organic_dense_matrix.h:4-38 ---- */
EPHMC_API void mat_mul(double *m, double *x, double *y, unsigned n);                 /* :4 */
EPHMC_API void mat_mul_tr(double *m, double *x, double *y, unsigned n);              /* :5 */
EPHMC_API void mat_mat_mul(double *m1, double *m2, double *y, unsigned n);           /* :6 */
EPHMC_API void construct_id(double *m, unsigned n);                                  /* :8 */
EPHMC_API void transpose(double *m, unsigned n);                                     /* :9 */
EPHMC_API void transpose_rect(double *x, double *y, unsigned n1, unsigned n2);       /* :10 */
EPHMC_API double trace(double *m, unsigned n);                                       /* :12 */
EPHMC_API void apply_mu_K_to_v(double *x, double *v, double *w, double *t, double *kappa, double mu,
                               unsigned *nnt, unsigned ns, unsigned nn);            /* :14 */
EPHMC_API void apply_mu_K_to_M(double *x, double *M, double *w, double *t, double *kappa, double mu,
                               unsigned *nnt, unsigned ns, unsigned nn);            /* :15 */
EPHMC_API void set_taylor_pair_order(void);                                          /* :17 */
EPHMC_API void apply_K_plus_1_v(double *x, double *v, double *w, double *t, double *kappa, double mu,
                                unsigned *nnt, unsigned ns, unsigned nn);           /* :19 */
EPHMC_API void apply_2nd_order_mu_K_to_v(double *x, double *v, double *w, double *t, double *kappa, double mu,
                                         unsigned *nnt, unsigned ns, unsigned nn, ephmc_dcomplex a); /* :20 */
EPHMC_API void apply_pair_expansion_mu_K_to_v(double *x, double *v, double *w, double *t, double *kappa, double mu,
                                              unsigned *nnt, unsigned ns, unsigned nn, int revert, int stop); /* :21 */
EPHMC_API void apply_exp_mu_K_to_v(double *x, double *v, double *w, double *t, double *kappa, double mu,
                                   unsigned *nnt, unsigned ns, unsigned nn, int revert, int stop); /* :22 */
EPHMC_API void apply_exp_mu_K_to_M(double *x, double *M, double *w, double *t, double *kappa, double mu,
                                   unsigned *nnt, unsigned ns, unsigned nn, int revert, int stop); /* :23 */
EPHMC_API void construct_hamilton(double *x, double *ham, double *w, double *t, double *kappa, double mu,
                                  unsigned *nnt, unsigned ns, unsigned nn);         /* :25 */
EPHMC_API void apply_current_to_v(double *x, double *v, double *w, double *t, double *kappa, unsigned *nnt,
                                  unsigned ns, unsigned nn, unsigned k);            /* :27 */
EPHMC_API void construct_M_hat(double *x, double *M_hat, double *w, double *t, double *kappa, double mu,
                               unsigned *nnt, unsigned ns, unsigned nn, unsigned nt, organic_flags *mode); /* :29 */
EPHMC_API void construct_QM1P(double *x, double *M_hat, double *QM1P, double *w, double *t, double *kappa, double mu,
                              unsigned *nnt, unsigned ns, unsigned nn, unsigned nt, int time,
                              organic_flags *mode);                                 /* :30 */
EPHMC_API void construct_all_QM1P(double *x, double *M_hat, double *QM1P, double *w, int *perm, double *t,
                                  double *kappa, double mu, unsigned *nnt, unsigned ns, unsigned nn, unsigned nt,
                                  organic_flags *mode);                             /* :31 */
EPHMC_API void refine_QM1P(double *x, double *QM1P, double *w, double *t, double *kappa, double mu, unsigned *nnt,
                           unsigned ns, unsigned nn, int time);                     /* :32 */
EPHMC_API void refine_QM1P_approx(double *x, double *QM1P, double *w, double *t, double *kappa, double mu,
                                  unsigned *nnt, unsigned ns, unsigned nn, int time); /* :33 */
EPHMC_API void cc_correlator(double *x, double *M_hat, double *R_t0, double *R_0t, double *w, double *t,
                             double *kappa, double mu, unsigned *nnt, unsigned ns, unsigned nn, unsigned nt,
                             double *greens, double logDetM, organic_flags *mode);  /* :35 */
EPHMC_API void phonon_correlator(double *x, unsigned ns, unsigned nn, unsigned nt, double *greens); /* :36 */
EPHMC_API double logDetM_and_inv_M_hat(double *M_hat, double *w, int *p, unsigned ns, unsigned flavors,
                                       organic_flags *mode);                        /* :38 */

/* ---- simulation/organic_hmc.h:9-21 ---- */
EPHMC_API double check_force(double *x, double *p, double *p_dot, double *M_hat, double *w, int *perm, double *t,
                             double *kappa, double mu, double omega, unsigned flavors, unsigned *nnt, unsigned ns,
                             unsigned nn, unsigned nt, organic_flags *mode);       /* :9 */
EPHMC_API double energy_momenta(double *p, ephmc_dcomplex *pc, double omega, unsigned ns, unsigned nn, unsigned nt,
                                const fftw_plan *fft, organic_flags *mode);         /* :11 */
EPHMC_API double hamilton(double *x, double *p, double logDetM, double energyP, double omega, unsigned flavors,
                          unsigned ns, unsigned nn, unsigned nt);                  /* :12 */
EPHMC_API void force(double *x, double *p_dot, double *M_hat, double *QM1P, double *w, int *perm, double *t,
                     double *kappa, double mu, double omega, unsigned flavors, unsigned *nnt, unsigned ns, unsigned nn,
                     unsigned nt, double logDetM, organic_flags *mode);            /* :14 */
EPHMC_API void update_x(double *x, double *p, double *p_dot, ephmc_dcomplex *xc, double omega, unsigned ns,
                        unsigned nn, unsigned nt, const fftw_plan *fft, double h, double half,
                        organic_flags *mode);                                       /* :15 */
EPHMC_API void leap_frog(double *x, double *p, double *p_dot, ephmc_dcomplex *xc, double *M_hat, double *QM1P,
                         double *w, int *perm, double *t, double *kappa, double mu, double omega, unsigned flavors,
                         unsigned *nnt, unsigned ns, unsigned nn, unsigned nt, unsigned steps, double traj_length,
                         const fftw_plan *fft, organic_flags *mode);               /* :17 */
EPHMC_API short trajectory(double *x, ephmc_dcomplex *xc, int *perm, double *t, double *kappa, double mu,
                           double omega, unsigned flavors, double *contr_mat, unsigned *nnt, unsigned ns, unsigned nn,
                           unsigned nt, unsigned steps, double traj_length, double *results, double *greens,
                           int iteration, unsigned meas_freq, const fftw_plan *fft, double *old, FILE *res_out,
                           FILE *corr_out, organic_flags *mode);                   /* :19 */
EPHMC_API unsigned run_hmc(double *greens, unsigned l1, unsigned l2, unsigned nt, double *t, double *kappa, double mu,
                           double omega, unsigned flavors, double *contr_mat, unsigned steps, double traj_length,
                           unsigned therm, unsigned meas, unsigned meas_freq, const char *res_name,
                           const char *corr_name, organic_flags *mode);             /* :21 */

/* ---- simulation/organic_bosons.h:9-20 ---- */
EPHMC_API void hot_start(double *x, double omega, unsigned ns, unsigned nn, unsigned nt);               /* :9 */
EPHMC_API double higher_Matsubaras_norm(double *x, unsigned *nnt, unsigned ns, unsigned nn, unsigned nt); /* :11 */
EPHMC_API void sample_free_bosons(double *x, ephmc_dcomplex *xc, double omega, unsigned ns, unsigned nn, unsigned nt,
                                  const fftw_plan *fft);                            /* :13 */
EPHMC_API void sample_fourier_momenta(double *p, ephmc_dcomplex *pc, double omega, unsigned ns, unsigned nn,
                                      unsigned nt, const fftw_plan *fft, organic_flags *mode); /* :14 */
EPHMC_API double energy_fourier_momenta(ephmc_dcomplex *pc, double omega, unsigned ns, unsigned nn, unsigned nt,
                                        const fftw_plan *fft);                      /* :16 */
EPHMC_API void evolve_bosons(ephmc_dcomplex *xc, double omega, unsigned ns, unsigned nn, unsigned nt,
                             const fftw_plan *fft, double h);                       /* :18 */
EPHMC_API void evolve_bosons_approx_step(ephmc_dcomplex *xc, double omega, unsigned ns, unsigned nn, unsigned nt,
                                         const fftw_plan *fft, double h, organic_flags *mode); /* :19 */
EPHMC_API void boson_force(double *x, double *p_dot, double omega, unsigned ns, unsigned nn, unsigned nt,
                           int overwrite);                                          /* :20 */

/* ---- simulation/organic_trans_loc.h:4-6 (static disorder) ---- */
/* One sample on the GPU; greens[nt] += its histogram, results[0] = partition
 * sum / ns, the bond field in x[0 .. 3ns).  Bins at or beyond nt are dropped
 * (the reference writes them past the end of greens). */
EPHMC_API void hist_trans_loc(double *x, double *t, double *kappa, double mu, double *contr_mat, unsigned *nnt,
                              unsigned ns, unsigned nn, unsigned nt, double width, double *results, double *greens,
                              FILE *res_out);                                       /* :4 */
/* Seeded with time(NULL), or with the environment variable EPHMC_SEED when set;
 * the samples' bond fields are drawn in the reference's order and the samples
 * are diagonalised in batches, EPHMC_TL_LANES (1-16, default 2) at a time. */
EPHMC_API unsigned run_trans_loc(double *greens, unsigned l1, unsigned l2, unsigned nt, double *t, double *kappa,
                                 double mu, double *contr_mat, unsigned meas, const char *res_name,
                                 const char *corr_name);                            /* :6 */

/* ---- plan handles (FFTW3 argument lists, simulation/organic_hmc.c:319-322) ---- */
EPHMC_API fftw_plan ephmc_fftw_plan_many_dft_r2c(int rank, const int *n, int howmany, double *in, const int *inembed,
                                                 int istride, int idist, ephmc_dcomplex *out, const int *onembed,
                                                 int ostride, int odist, unsigned flags);
EPHMC_API fftw_plan ephmc_fftw_plan_many_dft_c2r(int rank, const int *n, int howmany, ephmc_dcomplex *in,
                                                 const int *inembed, int istride, int idist, double *out,
                                                 const int *onembed, int ostride, int odist, unsigned flags);
EPHMC_API void ephmc_fftw_destroy_plan(fftw_plan p);

/* ---- native helpers for callers that drive chains themselves ---- */
/* Seed of the MT19937-64 stream the drop-in uses when the host program does
 * not provide init_genrand64 / genrand64_real2 / random_vector itself. */
EPHMC_API void ephmc_rng_seed(unsigned long long seed);
EPHMC_API double ephmc_rng_real2(void);
EPHMC_API void ephmc_random_vector(double *x, unsigned n);
/* run_hmc with an explicit seed instead of time(NULL) (simulation/organic_hmc.c:314). */
EPHMC_API unsigned ephmc_run_hmc_seeded(unsigned long long seed, double *greens, unsigned l1, unsigned l2,
                                        unsigned nt, double *t, double *kappa, double mu, double omega,
                                        unsigned flavors, double *contr_mat, unsigned steps, double traj_length,
                                        unsigned therm, unsigned meas, unsigned meas_freq, const char *res_name,
                                        const char *corr_name, organic_flags *mode);
/* run_trans_loc with an explicit seed instead of time(NULL) (simulation/organic_trans_loc.c:97). */
EPHMC_API unsigned ephmc_run_trans_loc_seeded(unsigned long long seed, double *greens, unsigned l1, unsigned l2,
                                              unsigned nt, double *t, double *kappa, double mu, double *contr_mat,
                                              unsigned meas, const char *res_name, const char *corr_name);
/* Force algorithm used by the drop-in force() / leap_frog (default EPHMC_FORCE_REFERENCE). */
EPHMC_API void ephmc_set_dropin_force_mode(int force_mode);

#ifdef __cplusplus
}
#endif
#endif
