// Internal declarations shared by the CUDA translation units of libephmc_cuda.so.
#pragma once

#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/ephmc.h"

namespace ephmc {

constexpr int kPairs = 2;  // Taylor-4 as two quadratic pairs (simulation/taylor-coeff_pairs.h:35-42)

// ---------------------------------------------------------------- status plumbing
void set_status(int status, const char *msg = nullptr);
int last_status();
unsigned last_warnings();
const char *last_message();
void add_warning(unsigned bits);
void clear_status();
int cuda_fail(cudaError_t e, const char *what);
void count_launch(unsigned n);  // kernel launches issued by this library (diag.cu)

#define EPHMC_CUDA(call)                                              \
    do {                                                              \
        cudaError_t _e = (call);                                      \
        if (_e != cudaSuccess) return ::ephmc::cuda_fail(_e, #call);  \
    } while (0)

// ---------------------------------------------------------------- model constants
// Lattice-unit couplings and the Taylor pair coefficients, passed by value to kernels.
struct Couplings {
    double t[3];
    double kappa[3];
    double mu;
    double a_lin[kPairs];   // 2 Re a_p,  a_p = c_p / (2P)
    double a_quad[kPairs];  // |a_p|^2
    int cplx[kPairs];       // Im a_p != 0
};

void pair_coefficients(double a_lin[kPairs], double a_quad[kPairs], int cplx[kPairs]);

// Device-resident lattice tables derived from the neighbour table nnt.
//   ev_src[e*V + j], ev_fac[e*V + j], e = 0..5: the six hopping terms that the
//   reference's scatter loop (simulation/organic_dense_matrix.c:103-119) adds
//   into w[j], in the order it adds them: operand site and coefficient index
//   (3*site + link) of the slice's hopping table.
//   nbr[k*V + i]: forward neighbour of site i along link k (nnt[6i+2k]).
struct LatticeDev {
    int V = 0;
    int l1 = 0, l2 = 0;
    int *ev_src = nullptr;
    int *ev_fac = nullptr;
    int *nbr = nullptr;
    int *rev = nullptr;  // rev[k*V + j]: the site whose link-k neighbour is j
    // launch shapes chosen by ephmc_ctx_autotune (0: the built-in rule):
    // sites per thread and vectors per CTA of k_slices and of k_adjoint
    int tune_slices_S = 0, tune_slices_R = 0, tune_adj_S = 0, tune_adj_R = 0;
    // every site's forward neighbours nbr[k][j] are three consecutive entries
    // of its event sources (true unless a self-link sorts inside the site's
    // own block, as on lattices of one row): the FP32 force sweep then keeps
    // only their offset (adjoint.cu)
    bool nb_in_events = false;
    // the packed FP32 force sweep's stencil coefficients, [nt][6][V] floats:
    // coef[t][e][j] = (float)(t_k - kappa_k x[t][f]), f = ev_fac[e][j],
    // k = f % 3, filled by the sweep's launcher for the slices it covers
    float *coef = nullptr;
    int coef_nt = 0;
};

// Host helper: build the event tables; returns EPHMC_OK or EPHMC_ERR_LATTICE.
int build_event_tables(const unsigned *nnt, int V, std::vector<int> &ev_src,
                       std::vector<int> &ev_fac, std::vector<int> &nbr);
void triangular_lattice(unsigned l1, unsigned l2, unsigned *nnt);
// LatticeDev::nb_in_events of the tables build_event_tables made
bool neighbours_in_events(const std::vector<int> &ev_src, const std::vector<int> &nbr, int V);

// what a captured trajectory (ephmc_leapfrog_graph) depends on besides the
// context's buffers: field pointers, steps, length, force mode and the
// context's parameter generation
struct LeapfrogKey {
    double *x, *p;
    unsigned steps;
    double traj;
    int mode;
    unsigned gen;
    bool operator==(const LeapfrogKey &o) const {
        return x == o.x && p == o.p && steps == o.steps && traj == o.traj && mode == o.mode && gen == o.gen;
    }
};
// while set on this thread, the upload caches copy every table (a stream
// capture must record all the uploads its replays need)
void uploads_uncached(bool on);
bool uploads_are_uncached();

// reference-algorithm buffers of a context, allocated on first use (context.cu)
int ensure_ref_buffers(ephmc_ctx *c);
// buffers and cuBLAS handle of the segmented mixed force, allocated on first use (context.cu)
int ensure_seg_buffers(ephmc_ctx *c);
// n slice jobs into the context's device job table at `slot`, on stream st.
// Entries the table already holds are not copied again: a copy from pageable
// host memory first waits for the stream to drain, so repeated evaluations
// would otherwise stall the host once per upload.
struct SliceJob;
int ctx_upload_jobs(ephmc_ctx *c, const SliceJob *jobs, int n, int slot, cudaStream_t st);
void ctx_forget_uploads(ephmc_ctx *c);
// sweep 1 + LU + force on the context stream, no host wait (context.cu)
int eval_async(ephmc_ctx *c, const double *xd, int mode);

// ---------------------------------------------------------------- SCHUR_FORM_INV (schur.cu)
struct SchurSolver;
void schur_free(SchurSolver *s);
// EPHMC_OK when the reference's Schur-factor regularisation does not apply to
// M (then the Schur-form inverse is M^-1); EPHMC_ERR_UNSUPPORTED when it does
int schur_check(SchurSolver **slot, const double *M, int V, double *scratch, cudaStream_t st);
int launch_one_minus(double *G, const double *M, int V, cudaStream_t st);
int launch_schur_clamp(double *force, size_t n, const double kappa[3], double f, cudaStream_t st);

// ---------------------------------------------------------------- stabilised chain (stabilize.cu)
struct StabWork;
void stab_free(StabWork *w);
size_t stab_bytes(const StabWork *w);
// UDT-stabilised chain of the field x over the segments b (top down): log det
// parts into stab_parts() (device: log|det M_hat|, sign), and with want_z each
// segment's y start Z_j (row-major, top-down j, contiguous from stab_ystart()).
// Uses 2m job slots from slot0 of the context's job table.
int stab_chain(ephmc_ctx *c, StabWork **slot, const double *x, const std::vector<int> &b, bool want_z,
               SliceJob *jobs_dev, int slot0);
double *stab_ystart(StabWork *w);
double *stab_parts(StabWork *w);
void *stab_stack(StabWork *w, size_t bytes);  // segment stacks, grown on demand

// ---------------------------------------------------------------- static disorder (trans_loc.cu)
int tl_create_nnt(ephmc_tl **out, const unsigned *nnt, unsigned V, unsigned nbins, const double t[3],
                  const double kappa[3], double mu, const double contr_mat[6], unsigned lanes, int device);
int tl_set_params(ephmc_tl *tl, const double t[3], const double kappa[3], double mu, const double contr_mat[6]);

// ---------------------------------------------------------------- slice propagation
// One job = one V x V matrix whose vectors (rows, or columns) get a sequence
// of slice propagators, optionally spilling the state after each slice.
// Slices [t0, t1) of an adjoint sweep 2 (checkpointed evaluation): q for
// slice t is stack entry t - t0, except slice t1 - 1, whose q is the FP64
// checkpoint q_top when given (and slice nt - 1, whose q is e_c); y starts
// from the rows of y_in (the previous segment's y_out, Real = the sweep's
// precision) or, when y_in is null, from M^-1; y_out (optional) receives y(t1).
struct AdjointRange {
    int t0, t1;
    const double *q_top;
    const void *y_in;
    void *y_out;
    bool zero_force;  // clear the force first (the first segment only)
    // Segment grid (seg_C > 0; t0, t1, q_top, y_in, y_out unused): segment
    // j = seg_j0 + blockIdx.y covers slices [max(0, nt - (j+1) C), nt - j C).
    // Its q at the top slice is e_c, its other q(t) are entry t - t0 of stack
    // region (seg_regions ? j : 0) (C entries of V^2 each), and its y starts
    // from the FP64 rows y_start + (seg_regions ? j : 0) V^2.  Segments are
    // independent: the segment's G_t = L_t Z_j R_t with Z_j = Q_top M^-1 P_t0
    // carried in its y start.
    int seg_C = 0, seg_j0 = 0;
    bool seg_regions = false;
    const double *y_start = nullptr;
    // set by the FP32 sweep's launcher: the slices' coefficient table
    // (LatticeDev::coef) of its packed instances
    const float *coef = nullptr;
};

struct SliceJob {
    const void *src;       // input matrix; nullptr = start from the identity
    void *dst;             // output matrix (may equal src); nullptr: the state after
                           // the last slice goes to the stack like the others
    void *stack;           // optional: state after slice s goes to stack[(s + stack_off) * V*V]
    int stack_off;
    int s_first, s_count, s_dir;  // slices s_first, s_first + s_dir, ...
    int p_begin, p_end, p_step;   // pairs p_begin, p_begin+p_step, ... != p_end
    int add_identity;             // dst[i][i] += 1 after the last slice
};

enum class Axis { Rows, Cols };

// Launch a batch of jobs on all vectors of every job matrix.
//   Real: arithmetic type; Store: element type of src/dst; StackT: of stack.
template <typename Real, typename Store, typename StackT>
int launch_slices(Axis axis, const double *x, const Couplings &c, const LatticeDev &lat,
                  const SliceJob *jobs_dev, int njobs, cudaStream_t st);

// Same jobs on rows (identity or src start, Rows axis only) with the lattice
// in registers: L1 = 32 (slices_strip.cu) and L1 = 8, 12, 16, 24, 48
// (register tiles, slices_tile.cu); sums in a different order from
// launch_slices, so results agree to rounding.
bool slices_strip32_supported(const LatticeDev &lat);
bool slices_tile_supported(const LatticeDev &lat);
bool slices_strip_supported(const LatticeDev &lat);  // either of the two
template <typename StackT>
int launch_slices_strip(const double *x, const Couplings &c, const LatticeDev &lat, const SliceJob *jobs_dev,
                        int njobs, cudaStream_t st);
template <typename StackT>
int launch_slices_tile(const double *x, const Couplings &c, const LatticeDev &lat, const SliceJob *jobs_dev,
                       int njobs, cudaStream_t st);
// jobs from the identity with FP32 stacks and no destination, in FP32
// arithmetic (the mixed force's segment stacks on the tile lattices)
int launch_slices_tile_identity_f32(const double *x, const Couplings &c, const LatticeDev &lat,
                                    const SliceJob *jobs_dev, int njobs, cudaStream_t st);
// FP32 (packed pairs) for jobs that start from the identity and spill every
// state, the last included, to an FP32 stack (dst null): the segmented mixed
// force's stacks (slices_strip.cu; L1 = 32).  max_ctas > 0 caps the grid (the work is
// taken grid-stride), so that the launch can run on the SMs the LU leaves free.
int launch_slices_strip_identity_f32(const double *x, const Couplings &c, const LatticeDev &lat,
                                     const SliceJob *jobs_dev, int njobs, cudaStream_t st, int max_ctas = 0);

// Reference-algorithm refinement + link contraction for slices t0..t0+nb-1:
//   A_t = pair 1 on columns of G_t, B_t = pair 0 on rows of G_t (already formed),
//   force[t][i][k] from the link entries of
//   D = a0 A + q0 (H A + A H) + a1 B + q1 (H B + B H)   (refine_QM1P, :383-442).
int launch_link_refine(const double *x, const Couplings &c, const LatticeDev &lat,
                       const double *A, const double *B, int t0, int nb, unsigned flavors,
                       int schur_clamp, int single_particle, double logdet, double *force,
                       cudaStream_t st);

// Adjoint sweep 2 (see adjoint.cu): y chain forward from M^-1, contraction with
// the stored q(t).  One thread per S sites, at most adjoint_max_threads(S)
// threads per CTA (the launch bounds of its instances; packed: the FP32
// sweep on a lattice with nb_in_events).
inline int adjoint_max_threads(int S, bool packed) { return S == 4 && packed ? 640 : 512; }
template <typename Real, typename QT>
int launch_adjoint_sweep(const double *x, const Couplings &c, const LatticeDev &lat,
                         const QT *qstack, const double *Minv, int nt, unsigned flavors,
                         int single_particle, double logdet, double *force, cudaStream_t st,
                         const AdjointRange *range = nullptr, int seg_count = 1);

// FP32 adjoint sweep 2 with the lattice in registers: L1 = 32 (adjoint_strip.cu)
// and the register-tile lattices L1 = 8, 12, 16, 24 (adjoint_tile.cu)
bool adjoint_strip32_supported(const LatticeDev &lat);
bool adjoint_tile_supported(const LatticeDev &lat);
bool adjoint_strip_supported(const LatticeDev &lat);  // either of the two
int launch_adjoint_tile(const double *x, const Couplings &c, const LatticeDev &lat, const float *qstack,
                        const double *Minv, int nt, unsigned flavors, int single_particle, double logdet,
                        double *force, cudaStream_t st, const AdjointRange *range = nullptr, int seg_count = 1);
int launch_adjoint_strip(const double *x, const Couplings &c, const LatticeDev &lat, const float *qstack,
                         const double *Minv, int nt, unsigned flavors, int single_particle, double logdet,
                         double *force, cudaStream_t st, const AdjointRange *range = nullptr,
                         int seg_count = 1);

// ---------------------------------------------------------------- drop-in helpers (helpers.cu)
// out = (mu + K) in on nvec rows (or columns) of V x V matrices, reference order;
// add_in: out = in + (mu + K) in (apply_K_plus_1_v)
int launch_stencil(const double *xs, const Couplings &c, const LatticeDev &lat, const double *in, double *out,
                   int nvec, bool cols, bool add_in, cudaStream_t st);
int launch_current(const double *xs, const Couplings &c, const LatticeDev &lat, const int *rev_k, const double *v,
                   double *w, int k, cudaStream_t st);
int launch_combine_refine(double *G, const double *X, const double *X1, const double *X2, size_t n, double al,
                          double aq, bool first, cudaStream_t st);
int launch_matvec(const double *m, const double *x, double *y, int n, bool tr, cudaStream_t st);
int launch_matmat_rows(const double *m1, const double *m2, double *out, int n, cudaStream_t st);
int launch_transpose_rect(const double *x, double *y, int n1, int n2, cudaStream_t st);
int launch_trace(const double *m, int n, double *out_dev, cudaStream_t st);
int launch_boson_force(const double *x, double *pd, double omega, int ld, int nt, bool overwrite, cudaStream_t st);
int device_moments(const double *x, size_t n, double *part_dev, double out[2], cudaStream_t st);
int device_matsubara_norm(const double *x, int ld, int nt, double *part_dev, double *out, cudaStream_t st);
int launch_phonon_corr(const double *x, int ns, int nt, double *g, cudaStream_t st);
int launch_add_diag(double *M, int V, double v, cudaStream_t st);
int launch_contract_full(const double *D, const Couplings &c, const LatticeDev &lat, int nt, unsigned flavors,
                         int schur, int sp, double spw, double *force, cudaStream_t st);
int launch_axpy(double *y, const double *x, double a, size_t n, cudaStream_t st);
// host bytes -> device, carried in kernel parameters (captured at launch), so
// the source may be a temporary and the stream may still be busy: a
// cudaMemcpyAsync from pageable memory can read its source after returning
int upload_small(void *dst, const void *src, size_t bytes, cudaStream_t st);
int launch_pair_combine(double *v, const double *w, const double *z, double al, double aq, size_t n, cudaStream_t st);

// ---------------------------------------------------------------- drop-in glue (organic_api.cu)
double dropin_contract_greens(const double *gr, const double *mat, unsigned nn, unsigned tau);
double dropin_rng_real2();
void dropin_rng_normals(double *x, unsigned n);
void dropin_rng_seed(unsigned long long s);
int dropin_force_mode();

// ---------------------------------------------------------------- measurement (correlator.cu)
// cc_correlator (simulation/organic_dense_matrix.c:451-524) on device buffers:
// Minv (V*V), R_t0 (nt*V*V), R_0t (V*V), greens (nt*9, device)
int cc_correlator_dev(ephmc_ctx *c, const double *x, const double *Minv, double *R_t0, double *R_0t, double *greens,
                      double logdet);

// ---------------------------------------------------------------- dense helpers
int launch_copy(double *dst, const double *src, size_t n, cudaStream_t st);
int launch_identity(double *M, int V, cudaStream_t st);
int launch_transpose(double *M, int V, cudaStream_t st);
int launch_fill(double *p, double v, size_t n, cudaStream_t st);

// ---------------------------------------------------------------- LU
struct LUWork {
    int V = 0;
    int *ipiv = nullptr;       // device, 0-based pivot rows
    double *diag = nullptr;    // device, U_ii
    int *info = nullptr;       // device: [0] first zero pivot (1-based), [1] dataflow wait timed out
    double *X = nullptr;       // device V*V: panels of the dataflow kernel, or the unpermuted inverse
    // device, zeroed once: the dataflow kernel's call counter (word 0, at the
    // same place for every V) and its ready flags; sync_words of them allocated
    unsigned *sync = nullptr;
    size_t sync_words = 0;
    int tune_rpt = 0;          // rows per thread of the dataflow kernel (ephmc_ctx_autotune; 0: built-in rule)
};
constexpr int kLuPanel = 8;  // columns per panel (and per CTA) of the dataflow kernel
constexpr size_t lu_sync_words(int V) { return 1 + (size_t)(V + kLuPanel - 1) / kLuPanel; }
int lu_alloc(LUWork &w, int V);
// rpt rows per thread is one of the dataflow kernel's shapes for V
bool lu_shape_ok(int V, int rpt);
// after a timed-out dataflow call: zero the counter, flags and messages (all
// sync_words), so that no stale word matches a later call's epoch
void lu_reset_sync(LUWork &w, cudaStream_t st);
void lu_free(LUWork &w);
// In-place LU with partial pivoting of the column-major matrix A(r,c) = M[c*V+r],
// followed by the in-place inverse; log|det| and sign into host outputs.
int lu_logdet_inverse(double *M, LUWork &w, double *logdet, int *sign, int *ipiv_host,
                      cudaStream_t st);
// Same without any host synchronisation: results stay on the device
// (w.ipiv, w.diag[V] = log|det|, w.diag[V+1] = sign, w.info[0] = first zero pivot).
int lu_logdet_inverse_async(double *M, LUWork &w, cudaStream_t st);

// ---------------------------------------------------------------- Fourier acceleration
// Mode tables of the Fourier-acceleration kernels are uploaded to the start of
// a scratch buffer; an upload whose contents the buffer already holds is
// skipped.  fa_forget_tables drops that knowledge (buffer freed, or its
// stream changed).
void fa_forget_tables(const double *scratch);
// scratch: device doubles, at least fa_scratch_doubles(ld, nt)
constexpr size_t kActionScratch = 2 * 64 + 8;  // k_action partial sums (fa_api.cu), after the FA tables
size_t fa_scratch_doubles(int ld, int nt);
int fa_evolve(double *x, double *p, int ld, int nt, double omega, double h, double *scratch, cudaStream_t st);
int fa_scale_modes(double *v, int ld, int nt, double omega, int mode, double *scratch, cudaStream_t st);
int fa_energy(const double *p, int ld, int nt, double omega, double *out_dev, double *scratch, cudaStream_t st);
int fa_approx_step(double *x, const double *p, int ld, int nt, double omega, double h, double *scratch,
                   cudaStream_t st);
// update_x of classical Fourier acceleration (simulation/organic_hmc.c:142-163)
// on device buffers of the context's shape; p_dot is scratch for the boson force
int classical_update_x(ephmc_ctx *c, double *x, double *p, double *p_dot, double h, double half);

}  // namespace ephmc

// ---------------------------------------------------------------- context
struct ephmc_ctx {
    int device = 0;
    unsigned l1 = 0, l2 = 0, V = 0, nt = 0, flavors = 1;
    double omega = 0;
    ephmc_flags flags{};
    ephmc::Couplings c{};
    ephmc::LatticeDev lat{};
    std::vector<unsigned> nnt;
    cudaStream_t stream = nullptr;

    // persistent device buffers
    double *x = nullptr;      // nt*V*3
    double *force = nullptr;  // nt*V*3
    double *M = nullptr;      // V*V  (M_hat, then its inverse)
    double *G = nullptr;      // nt*V*V (reference algorithm), allocated on first use
    double *A = nullptr;      // nb*V*V refine scratch, allocated on first use
    double *B = nullptr;      // nb*V*V refine scratch, allocated on first use
    int refine_batch = 0;
    void *qstack = nullptr;   // (nt)*V*V (adjoint), FP64 or FP32; checkpoints + one segment when ckpt > 0
    size_t qstack_bytes = 0;
    unsigned ckpt = 0;        // adjoint checkpoint interval in slices (0: whole stack)
    ephmc::SliceJob *jobs = nullptr;  // device job array
    int jobs_cap = 0;
    std::vector<ephmc::SliceJob> jobs_host;  // what the device job table holds (upload cache)
    std::vector<char> jobs_valid;
    ephmc::LUWork lu{};
    double last_logdet = 0;
    int last_sign = 1;
    bool have_inverse = false;
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    float t_mhat = 0, t_lu = 0, t_force = 0;
    double *work = nullptr;     // 4 V*V doubles: full-matrix refinement and drop-in staging
    double *cc_part = nullptr;  // nt * V * 9 doubles: correlator partial sums
    double *md_log = nullptr;   // ephmc_leapfrog: per MD step log det, sign, LU status (3 doubles each)
    unsigned md_cap = 0;        // steps md_log holds
    // ephmc_leapfrog_graph: the captured trajectory and what it was captured for
    cudaGraphExec_t lf_graph = nullptr;
    ephmc::LeapfrogKey lf_key{};
    unsigned param_gen = 0;     // advanced by every change of couplings, flags or buffers
    double *scratch = nullptr;  // small device scratch (Fourier mode tables, reductions)
    size_t scratch_n = 0;
    ephmc::SchurSolver *schur = nullptr;  // SCHUR_FORM_INV eigenvalue solver, created on first use
    // segmented mixed force (context.cu): FP64 segment-boundary states, the y
    // chain at the segment starts and the segments' y starts, allocated on
    // first use; the cuBLAS handle of its Z GEMMs and that handle's workspace
    unsigned seg_len = 0;       // ephmc_ctx_set_segment (0: the built-in rule)
    bool stabilize = false;     // ephmc_ctx_set_stabilize: UDT-stabilised chain (stabilize.cu)
    double *dropin_block = nullptr;  // the drop-in trajectory's device state block (host callers)
    size_t dropin_block_n = 0;
    ephmc::StabWork *stab = nullptr;
    double *seg = nullptr;
    size_t seg_bytes = 0;
    void *blas = nullptr;       // cublasHandle_t
    void *blas_ws = nullptr;
    // the segment stacks run on a side stream beside the LU, on the SMs it
    // leaves idle: fork after sweep 1, join before the force sweep
    cudaStream_t aux_stream = nullptr;
    cudaEvent_t aux_ev[2] = {nullptr, nullptr};
    bool aux_pending = false;
    int sm_count = 0;
    // ephmc_batch_eval: the context's own non-blocking stream, used in place of
    // the legacy default stream so that chains overlap; created on first use
    cudaStream_t batch_stream = nullptr;
    cudaEvent_t batch_ev[2] = {nullptr, nullptr};
};
