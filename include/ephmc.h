/*
 * ephmc -- B200-native (sm_100a) CUDA implementation of the Hybrid Monte Carlo
 * hot path of j-ostmeyer/electron-phonon-hmc, exposed as a C ABI.
 *
 * Two surfaces, both exported by libephmc_cuda.so:
 *
 *  1. The drop-in surface: the reference's own functions with identical names
 *     and prototypes (declared in ephmc_organic.h), so the reference's C host
 *     code links against this library in place of organic_dense_matrix.o,
 *     organic_hmc.o, organic_bosons.o and organic_trans_loc.o.
 *
 *  2. The native surface below (prefix ephmc_): a device context that keeps
 *     the lattice, parameters and every work buffer resident on one GPU and
 *     evaluates log det M and the fermion force in one call, in one of three
 *     algorithms; and a static-disorder handle (ephmc_tl_) that bins the
 *     current matrix elements of batches of disorder samples.
 *
 * Pointers: every double* argument of the native surface may be a device
 * pointer (used in place) or a host pointer (staged through the context's
 * device buffers, copies included in the call).  Sizes are plain unsigned.
 * No context call allocates device memory after ephmc_ctx_create, except:
 * the explicit ephmc_alloc; ephmc_ctx_set_checkpoint; the first call of the
 * reference algorithm (its Nt V^2 G_t buffers); the first call of the mixed
 * force (its segment buffers, about 3 Nt/C V^2 doubles, and a cuBLAS handle
 * with a 32 MiB workspace), and again when a new segment length needs more;
 * and ephmc_leapfrog when it meets more steps than before (its step log).  The static-disorder handle
 * grows its per-run buffers on demand, and ephmc_conv_* allocate per call.
 *
 * Errors: every ephmc_ function returns an ephmc_status; the most recent
 * status of the calling thread, including calls made through the drop-in
 * surface, is available from ephmc_last_status().
 */
#ifndef EPHMC_H
#define EPHMC_H

#include <stddef.h>

#if defined(__GNUC__)
#define EPHMC_API __attribute__((visibility("default")))
#else
#define EPHMC_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ status */
typedef enum {
    EPHMC_OK = 0,
    EPHMC_ERR_CUDA = 1,        /* a CUDA runtime call failed (message via ephmc_last_error_message) */
    EPHMC_ERR_ARG = 2,         /* invalid argument (size, pointer, mode) */
    EPHMC_ERR_LATTICE = 3,     /* neighbour table is not a periodic triangular lattice */
    EPHMC_ERR_SINGULAR = 4,    /* exact zero pivot in the LU factorisation */
    EPHMC_ERR_NONFINITE = 5,   /* log det or force is not finite */
    EPHMC_ERR_NOMEM = 6,       /* device allocation failed */
    EPHMC_ERR_UNSUPPORTED = 7, /* flag combination or size not implemented on the GPU path */
    EPHMC_ERR_TIMEOUT = 8,     /* a bounded device-side wait gave up */
    EPHMC_ERR_NO_DEVICE = 9    /* no CUDA device / extension not usable */
} ephmc_status;

/* warning bits reported alongside EPHMC_OK (ephmc_last_warnings) */
#define EPHMC_WARN_NEGATIVE_DET 0x1u /* "Negative determinant!" of
                                        simulation/organic_dense_matrix.c:589 */

EPHMC_API int ephmc_last_status(void);
EPHMC_API unsigned ephmc_last_warnings(void);
EPHMC_API const char *ephmc_status_string(int status);
EPHMC_API const char *ephmc_last_error_message(void);

/* ------------------------------------------------------------------ force algorithms */
typedef enum {
    /* The reference algorithm in FP64: M_hat by Nt slice propagations,
     * dgetrf/dgetri-equivalent LU, G_t = Q_t M^-1 P_t by the log-depth
     * sharing of construct_all_QM1P, refine_QM1P and the link contraction
     * (simulation/organic_dense_matrix.c:251-442, organic_hmc.c:86-134).
     * Stencil sums run in the reference's order, so M_hat is bit-identical
     * to the reference's. */
    EPHMC_FORCE_REFERENCE = 0,
    /* Reverse-mode (adjoint) accumulation of d log det / dx in FP64:
     * O(Nt) slice propagations instead of O(Nt log Nt), no G_t matrices. */
    EPHMC_FORCE_ADJOINT_FP64 = 1,
    /* Adjoint with FP64 M_hat, LU and log det, and FP32 propagation and
     * contraction of the force (the mixed-precision MD force), segmented:
     * each segment's outer factor in FP64, the in-segment products in FP32
     * (ephmc_ctx_set_segment). */
    EPHMC_FORCE_MIXED = 2
} ephmc_force_mode;

/* organic_flags (simulation/organic_flags.h:4-14), same layout */
typedef struct ephmc_flags {
    int schur_form_inv;
    int zero_filling;
    int static_disorder;
    int single_particle;
    int constant_force;
    int no_fourier_acc;
    int classical_fourier_acc;
    unsigned cfa_steps;
    double cfa_mass;
} ephmc_flags;

/* ------------------------------------------------------------------ context */
typedef struct ephmc_ctx ephmc_ctx;

/* Model in lattice units, as run_hmc receives it (simulation/organic_hmc.c:296):
 * L1 x L2 periodic triangular lattice, nt slices, hoppings t[3], couplings
 * kappa[3], chemical potential mu, phonon frequency omega, fermion flavours.
 * flags may be NULL (all off).  device: CUDA ordinal (-1 = current). */
EPHMC_API int ephmc_ctx_create(ephmc_ctx **out, unsigned l1, unsigned l2, unsigned nt,
                     const double t[3], const double kappa[3], double mu,
                     double omega, unsigned flavors, const ephmc_flags *flags,
                     int device);
EPHMC_API int ephmc_ctx_destroy(ephmc_ctx *ctx);

/* Change the couplings of an existing context (no reallocation). */
EPHMC_API int ephmc_ctx_set_params(ephmc_ctx *ctx, const double t[3], const double kappa[3],
                         double mu, double omega, unsigned flavors);

/* Neighbour table of the context, 12*V entries in the layout of
 * construct_triangular (simulation/organic_lattice.c:10-46); host pointer. */
EPHMC_API int ephmc_ctx_lattice(const ephmc_ctx *ctx, unsigned *nnt_out);

/* Bind the context to a CUDA stream (cudaStream_t passed as void*); 0 = legacy default. */
EPHMC_API int ephmc_ctx_set_stream(ephmc_ctx *ctx, void *stream);

/* One force+logdet evaluation, the body of leap_frog
 * (simulation/organic_hmc.c:177-180):
 *   x[nt*V*3]      phonon field, layout [t][site][link]       (in)
 *   p_dot[nt*V*3]  fermion force = flavors * d log det / dx    (out, may be NULL)
 *   logdet         log|det M_hat|                              (out, host, may be NULL)
 * The inverse M_hat^-1 stays in the context (ephmc_ctx_get_inverse). */
EPHMC_API int ephmc_eval(ephmc_ctx *ctx, const double *x, double *p_dot, double *logdet, int force_mode);

/* No counterpart in the reference.  ephmc_eval for n independent chains (one
 * context each, any lattice, Nt and couplings): the phases of all chains are
 * issued on their contexts' streams before any host wait, so small chains
 * overlap on the GPU.  x[i], p_dot[i]: as ephmc_eval (p_dot or p_dot[i] may
 * be NULL); logdet[n] (host, may be NULL).  Returns the first failure; the
 * other chains' outputs are valid. */
EPHMC_API int ephmc_batch_eval(ephmc_ctx *const *ctxs, const double *const *x, double *const *p_dot,
                               double *logdet, unsigned n, int force_mode);

/* M_hat = 1 + B_0...B_{Nt-1} only (construct_M_hat), out[V*V] row layout of the reference. */
EPHMC_API int ephmc_construct_M_hat(ephmc_ctx *ctx, const double *x, double *M_hat_out);

/* log|det| and in-place inverse of a V x V matrix (logDetM_and_inv_M_hat):
 * M is overwritten by its inverse; pivots (1-based, LAPACK convention) are
 * written to ipiv if not NULL (host).  Returns status; *logdet and *sign out. */
EPHMC_API int ephmc_logdet_inverse(ephmc_ctx *ctx, double *M, int *ipiv, double *logdet, int *sign);

/* No counterpart in the reference.  log|det| and in-place inverse of a device
 * matrix M (n x n, n <= 256) that allocates nothing: for callers whose device
 * memory is owned by a framework's caching allocator or by a pool sized at
 * start-up, or who must not allocate after initialisation.  The LU workspace
 * is a file-scope device array (about 0.5 MB, held by every GPU that loads the
 * library until exit), shared by all calls and left holding the last call's
 * data: calls that overlap on the GPU race and must be serialised by the
 * caller.  Every call looks up the array's address on the current device, and
 * M must be memory of that device (else EPHMC_ERR_ARG).  The call synchronizes
 * the stream before it returns.  n > 256 returns EPHMC_ERR_ARG; on any failure
 * *logdet and *sign are left unchanged.  ipiv (host, may be NULL) receives
 * 1-based pivots; stream may be NULL. */
EPHMC_API int ephmc_logdet_inverse_noalloc(double *M, unsigned n, double *logdet, int *sign, int *ipiv,
                                           void *stream);

/* Copy of the most recent M_hat^-1 (row layout of the reference). */
EPHMC_API int ephmc_ctx_get_inverse(ephmc_ctx *ctx, double *out);

/* Elapsed device milliseconds of the phases of the last ephmc_eval
 * (M_hat, LU, force), measured with CUDA events on the context stream. */
EPHMC_API int ephmc_ctx_last_timings(const ephmc_ctx *ctx, float *ms_mhat, float *ms_lu, float *ms_force);

/* Context over a caller-supplied neighbour table (12*ns entries in the layout
 * of construct_triangular); every site must be the forward neighbour of
 * exactly one site per link direction.  Used by the drop-in surface, whose
 * functions receive nnt rather than L1, L2. */
EPHMC_API int ephmc_ctx_create_nnt(ephmc_ctx **out, const unsigned *nnt, unsigned ns, unsigned nt,
                         const double t[3], const double kappa[3], double mu, double omega,
                         unsigned flavors, const ephmc_flags *flags, int device);
EPHMC_API int ephmc_ctx_set_flags(ephmc_ctx *ctx, const ephmc_flags *flags);

/* No counterpart in the reference.  Checkpointed adjoint sweeps: sweep 1
 * keeps the FP64 propagator states Q_t = B_t...B_{Nt-1} only every
 * `interval` slices, and sweep 2 recomputes each segment's states from its
 * checkpoint before using them, so the adjoint and mixed forces hold
 * ceil(Nt/interval) - 1 + interval matrices of V^2 doubles instead of Nt
 * (interval ~ sqrt(Nt) minimises it).  The force, log det and M_hat are
 * those of the whole-stack sweep (recomputation repeats the same arithmetic;
 * only the order of the force's atomic sums differs).  One extra propagation
 * of the V vectors through Nt - ceil(Nt/interval) slices per evaluation.
 * interval 0 restores the whole stack.  The reference algorithm's G_t
 * buffers (Nt V^2 doubles) are separate and allocated on first use. */
EPHMC_API int ephmc_ctx_set_checkpoint(ephmc_ctx *ctx, unsigned interval);
/* No counterpart in the reference.  Segment length of the mixed force
 * (EPHMC_FORCE_MIXED): the slice chain is cut into segments of `length`
 * slices; each segment's G_t = L_t Z R_t takes its outer factor
 * Z = Q_{t1-1} M^-1 P_{t0} in FP64 (sweep 1's state at the segment top, an
 * FP64 y chain and one GEMM per segment) and only the in-segment products
 * L_t, R_t in FP32, so the FP32 sums cancel over one segment's growth instead
 * of the whole chain's.  0 restores the built-in length, min(16, max(1, Nt/4)).
 * With checkpointing (ephmc_ctx_set_checkpoint) the checkpoint interval is the
 * segment length.  A stabilised context (ephmc_ctx_set_stabilize) cuts its
 * chain into segments of `length` slices, by default min(6, max(1, Nt/4)). */
EPHMC_API int ephmc_ctx_set_segment(ephmc_ctx *ctx, unsigned length);
/* No counterpart in the reference.  on != 0: the adjoint and mixed forces
 * (and their log det) come from an FP64 re-stabilised slice chain, for low
 * temperatures where the raw product 1 + B_0...B_{Nt-1} that the reference
 * factors (simulation/organic_dense_matrix.c:251-265, :547-607) loses log det
 * to rounding (at 48x48, Nt = 128, beta = 40 its LU resolves log det only to
 * about 4e-6).  The partial products over the segments (ephmc_ctx_set_segment)
 * are kept as U diag(d) T (QR with columns sorted by norm at every segment
 * boundary); log det comes from a well-conditioned matrix N_0 and the
 * segments' outer factors Z_k from N_k, and the segment sweeps run as in the
 * unstabilised segmented force.  Costs about 17 V^3 flops per segment
 * (cuSOLVER geqrf/orgqr/getrf/getrs, cuBLAS GEMM/trsm) on top of the sweeps.
 * No M_hat^-1 is formed (ephmc_ctx_get_inverse then reports none).  Ignored
 * by the reference force and by CONSTANT_FORCE, SINGLE_PARTICLE, ZERO_FILLING
 * and SCHUR_FORM_INV contexts.  ephmc_eval with p_dot NULL computes the log
 * det only (one chain of QR steps). */
EPHMC_API int ephmc_ctx_set_stabilize(ephmc_ctx *ctx, int on);
/* No counterpart in the reference.  Chooses the launch shapes of the
 * thread-per-site sweeps (sites per thread, vectors per CTA; the strip and
 * tile kernels of L1 = 8, 12, 16, 24, 32, 48 have fixed shapes and are not
 * tuned) and the dataflow LU's rows per thread (V <= 1024) for this context
 * by timing each candidate
 * over a few evaluations of x (host or device) with force_mode, and keeps
 * the fastest.  The sweeps sum in the same order for every shape (M_hat is
 * unchanged); the LU's pivots and inverse are unchanged, and its log det is
 * summed over terms grouped by the CTA size, so a new LU shape can move it
 * in the last bit.  ms_before / ms_after (may be NULL): median evaluation
 * time before and after.  Takes a few hundred evaluations. */
EPHMC_API int ephmc_ctx_autotune(ephmc_ctx *ctx, const double *x, int force_mode, float *ms_before,
                                 float *ms_after);
/* The shapes in use: out[0..1] sweep sites per thread and vectors per CTA,
 * out[2..3] the same for the adjoint sweep, out[4] LU rows per thread
 * (0: the built-in rule). */
EPHMC_API int ephmc_ctx_tuning(const ephmc_ctx *ctx, int out[5]);
/* Device bytes the context holds now (buffers allocated on first use included
 * once they exist). */
EPHMC_API int ephmc_ctx_memory(const ephmc_ctx *ctx, size_t *bytes);

/* force() given the inverse (simulation/organic_hmc.c:86-134): p_dot from x and
 * M_inv (the output of logDetM_and_inv_M_hat); flags as the reference
 * (CONSTANT_FORCE, SINGLE_PARTICLE with weight exp(-logdet), NO_FOURIER_ACC). */
EPHMC_API int ephmc_force(ephmc_ctx *ctx, const double *x, const double *M_inv, double logdet, double *p_dot,
                          int force_mode);
/* construct_all_QM1P (simulation/organic_dense_matrix.c:311-381): G_t for every
 * slice into G_out[nt*V*V]; perm_out[2*nt] (host, may be NULL) receives the
 * slices taken on the Q side, then on the P side, as the reference's perm. */
EPHMC_API int ephmc_all_G(ephmc_ctx *ctx, const double *x, const double *M_inv, double *G_out, int *perm_out);
/* refine_QM1P (:383-442) of one V x V matrix in place, slice t. */
EPHMC_API int ephmc_refine_G(ephmc_ctx *ctx, const double *x, double *G, unsigned t);
/* apply_exp_mu_K_to_M (:209-216) on nrows rows of length V; x_slice = 3V fields. */
EPHMC_API int ephmc_apply_exp_rows(ephmc_ctx *ctx, const double *x_slice, double *M, unsigned nrows, int revert,
                                   int stop);
/* out = (mu + K) in on nrows rows (apply_mu_K_to_v/_M, :96-131); add_in != 0
 * gives out = in + (mu + K) in (apply_K_plus_1_v, :162-166). */
EPHMC_API int ephmc_apply_stencil_rows(ephmc_ctx *ctx, const double *x_slice, const double *in, double *out,
                                       unsigned nrows, int add_in);
/* w = I_k v, current operator along link k (apply_current_to_v, :226-249). */
EPHMC_API int ephmc_apply_current(ephmc_ctx *ctx, const double *x_slice, const double *v, double *w, unsigned k);

/* ------------------------------------------------------------------ phonon side */
/* Exact harmonic flow of every Matsubara mode for time h, x and p in place
 * (evolve_bosons, simulation/organic_bosons.c:126-150). */
EPHMC_API int ephmc_fa_evolve(ephmc_ctx *ctx, double *x, double *p, double h);
/* p holds N(0,1) normals (drawn by the caller's MT19937-64 stream as
 * random_vector does); scaled per mode into Fourier-accelerated momenta
 * (sample_fourier_momenta, simulation/organic_bosons.c:76-100). */
EPHMC_API int ephmc_fa_scale_momenta(ephmc_ctx *ctx, double *p);
/* x holds N(0,1) normals; scaled into a free-phonon sample
 * (sample_free_bosons, simulation/organic_bosons.c:55-74). */
EPHMC_API int ephmc_fa_scale_free_bosons(ephmc_ctx *ctx, double *x);
/* Kinetic energy of p in Fourier space (energy_fourier_momenta, :102-124). */
EPHMC_API int ephmc_fa_energy(ephmc_ctx *ctx, const double *p, double *energy);
/* Kinetic step of classical Fourier acceleration: x += h * (p divided per
 * Matsubara mode by omega + (2 sin(pi k/Nt))^2/omega, at the accelerated
 * omega sqrt(cfa_mass^2 + omega^2) when the context's flags set
 * CLASSICAL_FOURIER_ACC); p is not changed (evolve_bosons_approx_step,
 * simulation/organic_bosons.c:152-177). */
EPHMC_API int ephmc_fa_approx_step(ephmc_ctx *ctx, double *x, const double *p, double h);
/* Action -flavors*logdet + energyP + (sum (dx_t)^2/omega + omega sum x^2)/2
 * (hamilton, simulation/organic_hmc.c:67-84). */
EPHMC_API int ephmc_hamilton(ephmc_ctx *ctx, const double *x, double logdet, double energyP, double *H);

/* The molecular-dynamics part of a trajectory, leap_frog
 * (simulation/organic_hmc.c:167-190), on device x and p (3 V Nt doubles
 * each): update_x by h/2, then per step one force+logdet evaluation,
 * p += h p_dot and update_x by h (by -h/2 after the last), h =
 * traj_length / steps (2 traj_length when steps = 0), with the context's
 * Fourier-acceleration flags.  Every step is issued before any host wait;
 * each step's log det, sign and status are read once at the end.  Afterwards
 * the context holds the last step's inverse (ephmc_ctx_get_inverse).
 * negative_steps (may be NULL): steps whose determinant was negative with an
 * odd number of flavours (the reference prints "Negative determinant!" for
 * each).  SINGLE_PARTICLE and SCHUR_FORM_INV contexts return
 * EPHMC_ERR_UNSUPPORTED. */
EPHMC_API int ephmc_leapfrog(ephmc_ctx *ctx, double *x, double *p, unsigned steps, double traj_length,
                             int force_mode, unsigned *negative_steps);
/* No counterpart in the reference.  ephmc_leapfrog as one CUDA graph: the
 * trajectory's launches are captured at the first call for a given (x, p,
 * steps, traj_length, force_mode) and replayed by later calls, on a stream of
 * the context's own that is ordered after the caller's stream.  A change of
 * couplings, flags or checkpointing makes the next call capture again.  Same
 * results as ephmc_leapfrog; fewer host launch costs per trajectory. */
EPHMC_API int ephmc_leapfrog_graph(ephmc_ctx *ctx, double *x, double *p, unsigned steps, double traj_length,
                                   int force_mode, unsigned *negative_steps);

/* ------------------------------------------------------------------ static disorder (TL mode) */
/* Transient-localisation histograms, the GPU form of hist_trans_loc
 * (simulation/organic_trans_loc.c:25-83); run_trans_loc (:85-114) is a loop
 * of ephmc_tl_run over batches of bond fields.  One handle per lattice and
 * bin count.  t, kappa, mu: the couplings as run_trans_loc receives them
 * (H = -mu + K(x), construct_hamilton with -mu); contr_mat[6]: the output of
 * construct_contraction_mat (simulation/organic_lattice.c:48-60), required.
 * lanes: samples processed concurrently, each lane from its own host thread
 * (each lane holds about 7 V^2 doubles of device memory; 0 or 1 = one at a
 * time, on the calling thread). */
typedef struct ephmc_tl ephmc_tl;
EPHMC_API int ephmc_tl_create(ephmc_tl **out, unsigned l1, unsigned l2, unsigned nbins, const double t[3],
                              const double kappa[3], double mu, const double contr_mat[6], unsigned lanes,
                              int device);
EPHMC_API int ephmc_tl_destroy(ephmc_tl *tl);
EPHMC_API int ephmc_tl_set_stream(ephmc_tl *tl, void *stream);
/* The bin width of run_trans_loc, (-2 mu + 8 sum_k |kappa_k|) / nbins. */
EPHMC_API int ephmc_tl_default_width(const ephmc_tl *tl, double *width);
/* nsamples bond fields x[nsamples][3V] (host or device, layout [site][link],
 * the reference's random_vector draw per sample):
 *   hist[nbins] += sum over samples of the sample histogram (not divided by
 *                  the number of samples; run_trans_loc divides at the end)
 *   z[nsamples]  = the partition sums / V, results[0] of each hist_trans_loc
 *                  call (may be NULL)
 * hist and z may be host or device memory.  Bins at or beyond nbins are
 * dropped (the reference writes them past the end of greens). */
EPHMC_API int ephmc_tl_run(ephmc_tl *tl, const double *x, unsigned nsamples, double width, double *hist, double *z);
/* Device milliseconds of the stages of the first sample that the last run
 * gave lane 0: ms[0] Hamiltonian, [1] eigensolver, [2] current operators,
 * [3] matrix-element products, [4] Boltzmann weights and binning.  With
 * several lanes the stages overlap other lanes' work. */
EPHMC_API int ephmc_tl_last_timings(const ephmc_tl *tl, float ms[5]);

/* ------------------------------------------------------------------ conductivity post-processing */
/* The computations of organic_conv (simulation/organic_conv.c:9-121) on a
 * histogram sigma[n] of bin width h (the contents of greens.bin), for n_smear
 * smearing widths (already multiplied by beta, as organic_conv's main does):
 *   out[i*n_smear + k] = smeared_sigma_w(i h, sigma, widths[k], h, n),  i < n
 * and for the Euclidean-time transform, t = i / nt, i <= nt/2:
 *   out[i*n_smear + k] = smeared_sigma_t(t, sigma, widths[k], h, n, nt_matsubara)
 * (organic_conv's main passes nt_matsubara = 0: tanh-sinh quadrature).
 * Pointers may be host or device memory. */
EPHMC_API int ephmc_conv_sigma_w(const double *sigma, unsigned n, double h, const double *widths, unsigned n_smear,
                                 double *out);
EPHMC_API int ephmc_conv_sigma_t(const double *sigma, unsigned n, double h, const double *widths, unsigned n_smear,
                                 unsigned nt, unsigned nt_matsubara, double *out);

/* ------------------------------------------------------------------ memory */
EPHMC_API void *ephmc_alloc(size_t bytes);   /* device memory on the current device */
EPHMC_API void ephmc_free(void *p);
EPHMC_API int ephmc_memcpy_h2d(void *dst, const void *src, size_t bytes);
EPHMC_API int ephmc_memcpy_d2h(void *dst, const void *src, size_t bytes);
EPHMC_API int ephmc_device_synchronize(void);

/* Cumulative number of kernel launches issued by this library (all contexts). */
EPHMC_API unsigned long long ephmc_launch_count(void);
/* CUDA-core FMA throughput of the current device in TFLOP/s (fp64 != 0: FP64,
 * else FP32), from a dependent-chain FMA probe; the roofline denominator for
 * the stencil kernels. */
EPHMC_API int ephmc_measure_fma_peak(int fp64, float *tflops);

/* No counterpart in the reference.  Test hook of the LU's failure path: the
 * next dataflow LU launch (V <= 2304) does not set the ready flag of panel
 * `panel`, so the CTAs that wait for it give up after their bounded wait (2 s)
 * and the call returns EPHMC_ERR_TIMEOUT, with the flags cleared for the next
 * call.  -1 cancels.  Affects one launch only. */
EPHMC_API void ephmc_test_lu_withhold_next(int panel);

/* Library version string. */
EPHMC_API const char *ephmc_version(void);

#ifdef __cplusplus
}
#endif
#endif
