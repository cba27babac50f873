// Device context and the native C ABI (ephmc_*): lattice tables, persistent
// buffers and the three force+logdet algorithms.
#include "ephmc_internal.cuh"

#include <cublas_v2.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstring>
#include <new>

namespace ephmc {

// ---------------------------------------------------------------- status
namespace {
thread_local int g_status = EPHMC_OK;
thread_local unsigned g_warn = 0;
thread_local char g_msg[512] = {0};
}  // namespace

int last_status() { return g_status; }
unsigned last_warnings() { return g_warn; }
const char *last_message() { return g_msg; }

void set_status(int status, const char *msg) {
    g_status = status;
    if (msg) {
        std::snprintf(g_msg, sizeof(g_msg), "%s", msg);
    } else if (status == EPHMC_OK) {
        g_msg[0] = 0;
    }
}
void add_warning(unsigned bits) { g_warn |= bits; }
void clear_status() {
    g_status = EPHMC_OK;
    g_warn = 0;
    g_msg[0] = 0;
}
int cuda_fail(cudaError_t e, const char *what) {
    char buf[512];
    std::snprintf(buf, sizeof(buf), "%s: %s", what, cudaGetErrorString(e));
    set_status(EPHMC_ERR_CUDA, buf);
    return EPHMC_ERR_CUDA;
}

// ---------------------------------------------------------------- model constants
// a = 0.5 c_p / P, a_lin = 2 Re a, a_quad = |a|^2  (simulation/organic_dense_matrix.c:169,189,192;
// coefficients simulation/taylor-coeff_pairs.h:35-42, order {0,1} from set_taylor_pair_order :133-159)
void pair_coefficients(double a_lin[kPairs], double a_quad[kPairs], int cplx[kPairs]) {
    static const std::complex<double> coeff[kPairs] = {{1.8294933739891903, 0.9404019519941707},
                                                      {0.1705066260108097, 1.5785318126884535}};
    static const int order[kPairs] = {0, 1};
    for (int p = 0; p < kPairs; ++p) {
        const std::complex<double> a = 0.5 * coeff[order[p]] / (double)kPairs;
        a_lin[p] = 2 * a.real();
        a_quad[p] = std::pow(std::hypot(a.real(), a.imag()), 2);
        cplx[p] = a.imag() != 0;
    }
}

// Periodic L1 x L2 triangular lattice in the layout of construct_triangular
// (simulation/organic_lattice.c:10-46): 6 neighbour sites per site, then 6 link indices.
void triangular_lattice(unsigned l1, unsigned l2, unsigned *nnt) {
    const unsigned V = l1 * l2;
    for (unsigned i = 0; i < V; ++i) {
        const unsigned a = i % l1, b = i / l1;
        const unsigned right = b * l1 + (a + 1) % l1, left = b * l1 + (a + l1 - 1) % l1;
        const unsigned up = ((b + 1) % l2) * l1, down = ((b + l2 - 1) % l2) * l1;
        unsigned *s = nnt + 6 * i;
        s[0] = right;
        s[1] = left;
        s[2] = up + a;
        s[3] = down + a;
        s[4] = up + (a + l1 - 1) % l1;
        s[5] = down + (a + 1) % l1;
        unsigned *l = nnt + 6 * (V + i);
        l[0] = 3 * i;
        l[1] = 3 * s[1];
        l[2] = 3 * i + 1;
        l[3] = 3 * s[3] + 1;
        l[4] = 3 * i + 2;
        l[5] = 3 * s[5] + 2;
    }
}

// The reference's scatter loop (apply_mu_K_to_v, simulation/organic_dense_matrix.c:100-119)
// visits (i, k) in order and adds fac_ik v[n] into w[i] ("here") then fac_ik v[i] into
// w[n] ("there").  For the gather form, list for every site the six terms it
// receives, sorted by (i, k, here-before-there).  Only the forward entries
// nnt[6i+2k] are read, as in the reference.
int build_event_tables(const unsigned *nnt, int V, std::vector<int> &ev_src, std::vector<int> &ev_fac,
                       std::vector<int> &nbr) {
    struct Ev {
        long key;
        int src, fac;
    };
    std::vector<std::vector<Ev>> per(V);
    nbr.assign(3 * (size_t)V, 0);
    for (int i = 0; i < V; ++i) {
        for (int k = 0; k < 3; ++k) {
            const unsigned n = nnt[6 * (size_t)i + 2 * k];
            if (n >= (unsigned)V) return EPHMC_ERR_LATTICE;
            nbr[(size_t)k * V + i] = (int)n;
            const long base = ((long)i * 3 + k) * 2;
            per[i].push_back({base, (int)n, 3 * i + k});
            per[n].push_back({base + 1, i, 3 * i + k});
        }
    }
    ev_src.assign(6 * (size_t)V, 0);
    ev_fac.assign(6 * (size_t)V, 0);
    for (int j = 0; j < V; ++j) {
        if (per[j].size() != 6) return EPHMC_ERR_LATTICE;
        std::sort(per[j].begin(), per[j].end(), [](const Ev &a, const Ev &b) { return a.key < b.key; });
        for (int e = 0; e < 6; ++e) {
            ev_src[(size_t)e * V + j] = per[j][e].src;
            ev_fac[(size_t)e * V + j] = per[j][e].fac;
        }
    }
    return EPHMC_OK;
}

// Whether every site's forward neighbours nbr[k][j] are three consecutive
// entries of its event sources ev_src[e][j], e = p..p + 2 for some p in 0..3.
bool neighbours_in_events(const std::vector<int> &ev_src, const std::vector<int> &nbr, int V) {
    for (int j = 0; j < V; ++j) {
        bool found = false;
        for (int p = 0; p <= 3 && !found; ++p) {
            found = true;
            for (int k = 0; k < 3; ++k)
                found = found && ev_src[(size_t)(p + k) * V + j] == nbr[(size_t)k * V + j];
        }
        if (!found) return false;
    }
    return true;
}

}  // namespace ephmc

using namespace ephmc;

namespace {

bool is_device_ptr(const void *p) {
    if (!p) return false;
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

int ret(int status, const char *msg = nullptr) {
    if (status != EPHMC_OK) set_status(status, msg);
    return status;
}

unsigned ceil_half(unsigned n) { return n / 2 + n % 2; }  // simulation/organic_aux.c:11-13
unsigned ceil_log2(unsigned n) {                          // simulation/organic_aux.c:15-19
    unsigned l = 0;
    while (n > 1) {
        n = ceil_half(n);
        ++l;
    }
    return l;
}

void set_couplings(ephmc_ctx *c, const double t[3], const double kappa[3], double mu) {
    for (int k = 0; k < 3; ++k) {
        c->c.t[k] = t[k];
        c->c.kappa[k] = kappa[k];
    }
    c->c.mu = mu;
    pair_coefficients(c->c.a_lin, c->c.a_quad, c->c.cplx);
}

int ensure_jobs(ephmc_ctx *c, int n) {
    if (n <= c->jobs_cap) return EPHMC_OK;
    return ret(EPHMC_ERR_ARG, "job table too small");
}

int upload_jobs(ephmc_ctx *c, const std::vector<SliceJob> &jobs, SliceJob *dst) {
    if (jobs.empty()) return EPHMC_OK;
    return ctx_upload_jobs(c, jobs.data(), (int)jobs.size(), (int)(dst - c->jobs), c->stream);
}

SliceJob job(const void *src, void *dst, int s_first, int s_count, int s_dir, int pb, int pe, int ps) {
    SliceJob j{};
    j.src = src;
    j.dst = dst;
    j.stack = nullptr;
    j.stack_off = 0;
    j.s_first = s_first;
    j.s_count = s_count;
    j.s_dir = s_dir;
    j.p_begin = pb;
    j.p_end = pe;
    j.p_step = ps;
    j.add_identity = 0;
    return j;
}

// stage a caller pointer: device pointers are used in place, host ones copied
int stage_in(ephmc_ctx *c, const double *user, double *devbuf, size_t n, const double **out) {
    if (is_device_ptr(user)) {
        *out = user;
        return EPHMC_OK;
    }
    EPHMC_CUDA(cudaMemcpyAsync(devbuf, user, sizeof(double) * n, cudaMemcpyHostToDevice, c->stream));
    *out = devbuf;
    return EPHMC_OK;
}

int stage_out(ephmc_ctx *c, double *user, const double *devbuf, size_t n) {
    if (!user || user == devbuf) return EPHMC_OK;
    if (is_device_ptr(user)) {
        EPHMC_CUDA(cudaMemcpyAsync(user, devbuf, sizeof(double) * n, cudaMemcpyDeviceToDevice, c->stream));
    } else {
        EPHMC_CUDA(cudaMemcpyAsync(user, devbuf, sizeof(double) * n, cudaMemcpyDeviceToHost, c->stream));
    }
    return EPHMC_OK;
}

// The reference algorithm's G_t for every slice and its refinement scratch:
// allocated by the first call that needs them, so that contexts used only
// through the adjoint paths hold O(V^2) plus the q stack (or its checkpoints).
int ensure_ref(ephmc_ctx *c) {
    const size_t VV = (size_t)c->V * c->V;
    auto get = [&](double **p, size_t n) {
        if (*p) return true;
        if (cudaMalloc((void **)p, sizeof(double) * n) != cudaSuccess) {
            cudaGetLastError();
            *p = nullptr;
            return false;
        }
        return true;
    };
    if (!get(&c->G, VV * c->nt) || !get(&c->A, VV * c->refine_batch) || !get(&c->B, VV * c->refine_batch))
        return ret(EPHMC_ERR_NOMEM, "reference-algorithm buffers (G_t for every slice, refinement scratch)");
    return EPHMC_OK;
}

// ------------------------------------------------------------------ checkpointed adjoint
// Segments of the sweep, from the top: b_0 = nt > b_1 = nt - C > ... > b_m = 0.
// c->qstack holds the FP64 states Q_{b_j} = B_{b_j}...B_{nt-1}, j = 1..m-1
// (sweep 1's rows after slice b_j), then one segment's stack of C entries.
std::vector<int> ckpt_bounds(unsigned nt, unsigned C) {
    std::vector<int> b{(int)nt};
    while (b.back() > 0) b.push_back(std::max(0, b.back() - (int)C));
    return b;
}

size_t qstack_bytes_for(unsigned nt, unsigned C, size_t VV) {
    if (C == 0) return sizeof(double) * VV * nt;
    const size_t m = (nt + C - 1) / C;
    return sizeof(double) * VV * ((m - 1) + C);
}

double *ckpt_state(ephmc_ctx *c, int j) {
    return static_cast<double *>(c->qstack) + (size_t)(j - 1) * c->V * c->V;
}

void *ckpt_segment(ephmc_ctx *c, size_t m) { return static_cast<double *>(c->qstack) + (m - 1) * c->V * c->V; }

int launch_sweep1(ephmc_ctx *c, const double *x, const SliceJob *jobs_dev, bool stack_float, int n = 1) {
    if (slices_strip_supported(c->lat))
        return stack_float ? launch_slices_strip<float>(x, c->c, c->lat, jobs_dev, n, c->stream)
                           : launch_slices_strip<double>(x, c->c, c->lat, jobs_dev, n, c->stream);
    if (stack_float) return launch_slices<double, double, float>(Axis::Rows, x, c->c, c->lat, jobs_dev, n, c->stream);
    return launch_slices<double, double, double>(Axis::Rows, x, c->c, c->lat, jobs_dev, n, c->stream);
}

// sweep 1 keeping only the checkpoints: one launch per segment, the FP64 state
// passed through memory, so M_hat and every later recomputed q equal those of
// the uncheckpointed sweep bit for bit
int build_M_hat_ckpt(ephmc_ctx *c, const double *x, bool stack_float, double *dst) {
    const std::vector<int> b = ckpt_bounds(c->nt, c->ckpt);
    const int m = (int)b.size() - 1;
    std::vector<SliceJob> v;
    for (int j = 0; j < m; ++j) {
        SliceJob jb = job(j == 0 ? nullptr : ckpt_state(c, j), j == m - 1 ? dst : ckpt_state(c, j + 1), b[j] - 1,
                          b[j] - b[j + 1], -1, 0, kPairs, 1);
        jb.add_identity = (j == m - 1) && !(c->flags.zero_filling || c->flags.single_particle);
        v.push_back(jb);
    }
    int rc = upload_jobs(c, v, c->jobs);
    for (int j = 0; j < m && rc == EPHMC_OK; ++j) rc = launch_sweep1(c, x, c->jobs + j, stack_float);
    return rc;
}

// sweep 2 segment by segment, bottom up: recompute the segment's q(t) from its
// checkpoint into the segment stack, then run the adjoint over the segment
// with y carried between segments in c->work[2V^2, 3V^2)
int adjoint_ckpt(ephmc_ctx *c, const double *x, const double *y0, bool mixed, double logdet) {
    const std::vector<int> b = ckpt_bounds(c->nt, c->ckpt);
    const int m = (int)b.size() - 1;
    const size_t VV = (size_t)c->V * c->V;
    void *seg = ckpt_segment(c, m);
    double *junk = c->work + VV;       // final states of the recomputations (not needed)
    void *ybuf = c->work + 2 * VV;     // y between segments (FP64 or FP32 rows)
    std::vector<SliceJob> v;
    for (int j = m - 1; j >= 0; --j) {
        const int t0 = b[j + 1], t1 = b[j];
        SliceJob jb = job(j == 0 ? nullptr : ckpt_state(c, j), junk, t1 - 1, t1 - t0, -1, 0, kPairs, 1);
        jb.stack = seg;
        jb.stack_off = -1 - t0;
        v.push_back(jb);
    }
    int rc = upload_jobs(c, v, c->jobs + m);
    const ephmc_flags &f = c->flags;
    for (int k = 0; k < m && rc == EPHMC_OK; ++k) {
        const int j = m - 1 - k;
        const int t0 = b[j + 1], t1 = b[j];
        if (t1 - t0 > 1 && (rc = launch_sweep1(c, x, c->jobs + m + k, mixed))) break;
        AdjointRange rg{t0, t1, j == 0 ? nullptr : ckpt_state(c, j), j == m - 1 ? nullptr : ybuf,
                        j == 0 ? nullptr : ybuf, j == m - 1};
        if (!mixed)
            rc = launch_adjoint_sweep<double, double>(x, c->c, c->lat, static_cast<const double *>(seg), y0,
                                                      (int)c->nt, c->flavors, f.single_particle, logdet, c->force,
                                                      c->stream, &rg);
        else if (adjoint_strip_supported(c->lat))
            rc = launch_adjoint_strip(x, c->c, c->lat, static_cast<const float *>(seg), y0, (int)c->nt, c->flavors,
                                      f.single_particle, logdet, c->force, c->stream, &rg);
        else
            rc = launch_adjoint_sweep<float, float>(x, c->c, c->lat, static_cast<const float *>(seg), y0,
                                                    (int)c->nt, c->flavors, f.single_particle, logdet, c->force,
                                                    c->stream, &rg);
    }
    return rc;
}

// ------------------------------------------------------------------ segmented mixed force
// The mixed force splits the slice chain into segments of C slices (the
// checkpoint interval when one is set, else ephmc_ctx_set_segment's length,
// else min(16, max(1, Nt/4))): segment j covers [b_{j+1}, b_j),
// b_j = max(0, Nt - jC).
// For t in a segment [t0, t1) the reference's G_t = Q_t M^-1 P_t is
//   G_t = L_t Z R_t,  L_t = B_{t+1}...B_{t1-1},  R_t = B_{t0}...B_{t-1},
//   Z = Q_{t1-1} M^-1 P_{t0},
// so with q'_c(t) = L_t e_c and y'_c(t) = R_t^T Z^T e_c the sweep-2 kernels
// contract the same formulas over each segment independently.  Z is formed in
// FP64: Q_{t1-1} is sweep 1's FP64 state at b_j, the rows of M^-1 P_{t0} come
// from an FP64 y chain, and y'(t0) = Q_{t1-1}^T (M^-1 P_{t0}) is one GEMM per
// segment.  Only L_t and R_t run in FP32, so the terms of the FP32 sum over
// vectors grow over C slices of the chain instead of Nt, and the cancellation
// that bounded the unsegmented FP32 force (4e-3 at 32x32, Nt = 64) stays at
// the size of one segment's growth (6e-7 in an FP64/FP32 numpy model).
constexpr size_t kBlasWorkspace = (size_t)32 << 20;  // cuBLAS workspace of the Z GEMMs

struct SegPlan {
    int C = 0, m = 0;
    std::vector<int> b;   // b[0] = nt > b[1] > ... > b[m] = 0
    bool regions = true;  // one FP32 stack region per segment (else one, reused)
};

unsigned seg_length(const ephmc_ctx *c) {
    if (c->ckpt) return std::min(c->ckpt, c->nt);
    if (c->seg_len) return std::min(c->seg_len, c->nt);
    return std::min(16u, std::max(1u, c->nt / 4));
}

// segments of the stabilised chain: shorter, since the accuracy of each
// segment's Z_k falls with the conditioning of its middle product S_k (at
// dtau = 0.31: 6 slices give 3e-6 of the largest force entry at 48x48,
// beta = 40, against finite differences; 12 slices 3e-4)
unsigned stab_seg_length(const ephmc_ctx *c) {
    return std::min(c->seg_len ? c->seg_len : std::min(6u, std::max(1u, c->nt / 4)), c->nt);
}

SegPlan seg_plan(const ephmc_ctx *c, bool stab = false) {
    SegPlan p;
    p.C = (int)(stab ? stab_seg_length(c) : seg_length(c));
    p.b = ckpt_bounds(c->nt, (unsigned)p.C);
    p.m = (int)p.b.size() - 1;
    p.regions = c->ckpt == 0;
    return p;
}

// Buffers.  Regions: c->seg = [ck_1..ck_{m-1}][ys_1..ys_{m-1}][ys_0 = yst_0][yst_1..yst_{m-1}],
// the FP32 stack regions in c->qstack.  Checkpointed: ck_j are the context's
// checkpoints, one FP32 region after them, and the y chain and one segment's
// start rows live in c->work (no segment buffer).  ck_j: FP64 rows of
// Q_{b_j} = B_{b_j}...B_{Nt-1} (j = 1..m-1); ys_j: FP64 rows of
// M^-1 P_{b_{j+1}} (ys_{m-1}: M^-1 itself, transposed); yst_j: y'(b_{j+1}) of
// segment j.
size_t seg_doubles(const SegPlan &p, size_t VV) { return p.regions ? VV * (3 * (size_t)p.m - 2) : 0; }

double *seg_ck(ephmc_ctx *c, const SegPlan &p, int j) {
    const size_t VV = (size_t)c->V * c->V;
    return p.regions ? c->seg + (size_t)(j - 1) * VV : ckpt_state(c, j);
}
double *seg_ys(ephmc_ctx *c, const SegPlan &p, int j) {
    const size_t VV = (size_t)c->V * c->V;
    return c->seg + (size_t)(j == 0 ? 2 * p.m - 2 : p.m + j - 2) * VV;
}
double *seg_yst(ephmc_ctx *c, const SegPlan &p, int j) {
    const size_t VV = (size_t)c->V * c->V;
    return j == 0 ? seg_ys(c, p, 0) : c->seg + (size_t)(2 * p.m - 2 + j) * VV;
}
float *seg_region(ephmc_ctx *c, const SegPlan &p, int j) {
    const size_t VV = (size_t)c->V * c->V;
    if (p.regions) return static_cast<float *>(c->qstack) + (size_t)j * p.C * VV;
    return static_cast<float *>(ckpt_segment(c, (size_t)p.m));
}

int ensure_seg(ephmc_ctx *c, const SegPlan &p) {
    const size_t need = sizeof(double) * seg_doubles(p, (size_t)c->V * c->V);
    if (3 * p.m > c->jobs_cap) return ret(EPHMC_ERR_ARG, "segment length too small for Nt");
    if (c->seg_bytes != need) {
        cudaFree(c->seg);
        c->seg = nullptr;
        c->seg_bytes = 0;
        if (need && cudaMalloc((void **)&c->seg, need) != cudaSuccess) {
            cudaGetLastError();
            c->seg = nullptr;
            return ret(EPHMC_ERR_NOMEM, "segmented force buffers");
        }
        c->seg_bytes = need;
    }
    if (!c->blas) {
        cublasHandle_t h = nullptr;
        if (cublasCreate(&h) != CUBLAS_STATUS_SUCCESS) return ret(EPHMC_ERR_CUDA, "cublasCreate");
        c->blas = h;
        // an explicit workspace, so that no GEMM of a captured trajectory allocates
        if (cudaMalloc(&c->blas_ws, kBlasWorkspace) != cudaSuccess) {
            cudaGetLastError();
            c->blas_ws = nullptr;
            return ret(EPHMC_ERR_NOMEM, "cuBLAS workspace");
        }
    }
    if (!c->aux_stream) {
        if (cudaStreamCreateWithFlags(&c->aux_stream, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&c->aux_ev[0], cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&c->aux_ev[1], cudaEventDisableTiming) != cudaSuccess ||
            cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, c->device) != cudaSuccess) {
            cudaGetLastError();
            return ret(EPHMC_ERR_CUDA, "segmented force: side stream");
        }
    }
    cublasHandle_t h = static_cast<cublasHandle_t>(c->blas);
    if (cublasSetStream(h, c->stream) != CUBLAS_STATUS_SUCCESS ||
        cublasSetWorkspace(h, c->blas_ws, kBlasWorkspace) != CUBLAS_STATUS_SUCCESS)
        return ret(EPHMC_ERR_CUDA, "cublasSetStream / cublasSetWorkspace");
    return EPHMC_OK;
}

// FP32 stacks from the identity (jobs with no source and no destination):
// the packed FP32 strip kernel where it applies, else the FP64 slice kernel
// with an FP32 stack
int launch_identity_stacks(ephmc_ctx *c, const double *x, const SliceJob *jobs_dev, int n) {
    if (slices_strip32_supported(c->lat))
        return launch_slices_strip_identity_f32(x, c->c, c->lat, jobs_dev, n, c->stream);
    if (slices_tile_supported(c->lat)) return launch_slices_tile_identity_f32(x, c->c, c->lat, jobs_dev, n, c->stream);
    return launch_slices<double, double, float>(Axis::Rows, x, c->c, c->lat, jobs_dev, n, c->stream);
}

// rows of the jobs on the context's lattice: the register-strip kernel where it applies
int launch_rows(ephmc_ctx *c, const double *x, const SliceJob *jobs_dev, int n) {
    if (slices_strip_supported(c->lat)) return launch_slices_strip<double>(x, c->c, c->lat, jobs_dev, n, c->stream);
    return launch_slices<double, double, double>(Axis::Rows, x, c->c, c->lat, jobs_dev, n, c->stream);
}

// FP32 stack from the identity at the top of segment j:
// q'(t) = B_{t+1}...B_{t1-1} into its region
SliceJob seg_identity_job(ephmc_ctx *c, const SegPlan &p, int j) {
    const int t0 = p.b[j + 1], t1 = p.b[j];
    SliceJob jb = job(nullptr, nullptr, t1 - 1, t1 - t0 - 1, -1, 0, kPairs, 1);
    jb.stack = seg_region(c, p, j);
    jb.stack_off = -1 - t0;
    return jb;
}

// Sweep 1 of the segmented force: M_hat into dst in FP64, the FP64 states at
// the segment boundaries (one launch per segment, the state passed through
// memory, the same arithmetic as the whole chain), and (regions) every
// segment's FP32 stack from the identity in one more launch.
int sweep1_seg(ephmc_ctx *c, const double *x, double *dst) {
    const SegPlan p = seg_plan(c);
    int rc;
    if ((rc = ensure_seg(c, p))) return rc;
    std::vector<SliceJob> v;
    for (int j = 0; j < p.m; ++j) {
        SliceJob jb = job(j == 0 ? nullptr : seg_ck(c, p, j), j == p.m - 1 ? dst : seg_ck(c, p, j + 1), p.b[j] - 1,
                          p.b[j] - p.b[j + 1], -1, 0, kPairs, 1);
        jb.add_identity = (j == p.m - 1) && !(c->flags.zero_filling || c->flags.single_particle);
        v.push_back(jb);
    }
    if ((rc = upload_jobs(c, v, c->jobs))) return rc;
    for (int j = 0; j < p.m && rc == EPHMC_OK; ++j) rc = launch_sweep1(c, x, c->jobs + j, j == 0);
    if (rc || !p.regions) return rc;
    // every segment's stack from the identity in FP32 (segment 0 too, so that
    // the whole-stack and the checkpointed forces run the same arithmetic)
    std::vector<SliceJob> id;
    for (int j = 0; j < p.m; ++j)
        if (p.b[j] - p.b[j + 1] > 1) id.push_back(seg_identity_job(c, p, j));
    if (id.empty()) return EPHMC_OK;
    if ((rc = upload_jobs(c, id, c->jobs + p.m))) return rc;
    // Beside the LU: the dataflow LU (V <= 1024) holds one SM per 8 columns
    // and leaves the others idle; the FP32 stacks need nothing from sweep 1
    // or the LU, so they run on a side stream, forked here (after sweep 1, so
    // they do not slow it) with a grid that fits the idle SMs, and joined
    // before the force sweep reads them.
    const int lu_sms = c->V <= 1024 ? (int)((c->V + kLuPanel - 1) / kLuPanel) : c->sm_count;
    const int free_sms = c->sm_count - lu_sms;
    if (!slices_strip32_supported(c->lat) || free_sms < 8)
        return launch_identity_stacks(c, x, c->jobs + p.m, (int)id.size());
    EPHMC_CUDA(cudaEventRecord(c->aux_ev[0], c->stream));
    EPHMC_CUDA(cudaStreamWaitEvent(c->aux_stream, c->aux_ev[0], 0));
    // one CTA per SM (launch bound 512 threads, one block per SM) on at most
    // the idle SMs: the LU's cooperative grid always finds its SMs free
    if ((rc = launch_slices_strip_identity_f32(x, c->c, c->lat, c->jobs + p.m, (int)id.size(), c->aux_stream,
                                               free_sms)))
        return rc;
    EPHMC_CUDA(cudaEventRecord(c->aux_ev[1], c->aux_stream));
    c->aux_pending = true;
    return EPHMC_OK;
}

// y'(t0) of n segments: yst = ck^T ys (row-major V x V), the n operands and
// results each V^2 apart.  In cuBLAS's column-major view a row-major X is
// X^T, so yst^T = ys^T ck  <=>  C = A B^T with A = ys, B = ck as stored.
int seg_gemm(ephmc_ctx *c, const double *ys, const double *ck, double *yst, int n) {
    const int V = (int)c->V;
    const long long VV = (long long)V * V;
    const double one = 1.0, zero = 0.0;
    cublasHandle_t h = static_cast<cublasHandle_t>(c->blas);
    cublasStatus_t st;
    if (n == 1)
        st = cublasDgemm(h, CUBLAS_OP_N, CUBLAS_OP_T, V, V, V, &one, ys, V, ck, V, &zero, yst, V);
    else
        st = cublasDgemmStridedBatched(h, CUBLAS_OP_N, CUBLAS_OP_T, V, V, V, &one, ys, V, VV, ck, V, VV, &zero, yst,
                                       V, VV, n);
    count_launch((unsigned)n);
    if (st != CUBLAS_STATUS_SUCCESS) return ret(EPHMC_ERR_CUDA, "cublasDgemm (segment start rows)");
    return EPHMC_OK;
}

// Sweep 2 of the segmented force (after sweep1_seg and the LU): y0 is the
// FP64 matrix whose rows start the y chain (M^-1 as the inverse's array,
// or the identity for SINGLE_PARTICLE).
int force_mixed_seg(ephmc_ctx *c, const double *x, const double *y0, double logdet) {
    const SegPlan p = seg_plan(c);
    const int V = (int)c->V;
    const size_t VV = (size_t)V * V;
    const ephmc_flags &f = c->flags;
    int rc;
    if ((rc = ensure_seg(c, p))) return rc;
    AdjointRange rg{0, 0, nullptr, nullptr, nullptr, true};
    rg.seg_C = p.C;
    rg.seg_regions = p.regions;
    auto adjoint = [&](int count) {
        if (adjoint_strip_supported(c->lat))
            return launch_adjoint_strip(x, c->c, c->lat, seg_region(c, p, 0), y0, (int)c->nt, c->flavors,
                                        f.single_particle, logdet, c->force, c->stream, &rg, count);
        return launch_adjoint_sweep<float, float>(x, c->c, c->lat, seg_region(c, p, 0), y0, (int)c->nt, c->flavors,
                                                  f.single_particle, logdet, c->force, c->stream, &rg, count);
    };
    if (p.regions) {
        // FP64 y chain: ys_{m-1} = rows of M^-1, then forward through each
        // segment; all segments' start rows by one batched GEMM; one launch
        // for all segments
        if ((rc = launch_transpose_rect(y0, seg_ys(c, p, p.m - 1), V, V, c->stream))) return rc;
        std::vector<SliceJob> v;
        for (int j = p.m - 2; j >= 0; --j)
            v.push_back(job(seg_ys(c, p, j + 1), seg_ys(c, p, j), p.b[j + 2], p.b[j + 1] - p.b[j + 2], +1, 1, -1, -1));
        if ((rc = upload_jobs(c, v, c->jobs + 2 * p.m))) return rc;
        for (int k = 0; k < p.m - 1 && rc == EPHMC_OK; ++k) rc = launch_rows(c, x, c->jobs + 2 * p.m + k, 1);
        if (rc) return rc;
        if (p.m > 1 && (rc = seg_gemm(c, seg_ys(c, p, 1), seg_ck(c, p, 1), seg_yst(c, p, 1), p.m - 1))) return rc;
        if (c->aux_pending) {  // the stacks from the side stream
            EPHMC_CUDA(cudaStreamWaitEvent(c->stream, c->aux_ev[1], 0));
            c->aux_pending = false;
        }
        rg.seg_j0 = 0;
        rg.y_start = seg_yst(c, p, 0);
        return adjoint(p.m);
    }
    // checkpointed: one FP32 region, reused, segments bottom up; the y chain
    // advances in place in work[2V^2, 3V^2), a segment's start rows go to
    // work[3V^2, 4V^2), and every segment's stack is recomputed from the
    // identity just before its sweep
    double *Y = c->work + 2 * VV, *yst = c->work + 3 * VV;
    if ((rc = launch_transpose_rect(y0, Y, V, V, c->stream))) return rc;
    std::vector<SliceJob> v;
    for (int j = 0; j < p.m; ++j) v.push_back(seg_identity_job(c, p, j));
    for (int j = p.m - 2; j >= 0; --j) v.push_back(job(Y, Y, p.b[j + 2], p.b[j + 1] - p.b[j + 2], +1, 1, -1, -1));
    if ((rc = upload_jobs(c, v, c->jobs + p.m))) return rc;
    const SliceJob *id_jobs = c->jobs + p.m, *y_jobs = c->jobs + 2 * p.m;
    for (int j = p.m - 1; j >= 0 && rc == EPHMC_OK; --j) {
        if (j < p.m - 1 && (rc = launch_rows(c, x, y_jobs + (p.m - 2 - j), 1))) break;
        if (j > 0 && (rc = seg_gemm(c, Y, seg_ck(c, p, j), yst, 1))) break;
        if (p.b[j] - p.b[j + 1] > 1 && (rc = launch_identity_stacks(c, x, id_jobs + j, 1))) break;
        rg.seg_j0 = j;
        rg.zero_force = j == p.m - 1;
        rg.y_start = j > 0 ? yst : Y;
        rc = adjoint(1);
    }
    return rc;
}

// ------------------------------------------------------------------ stabilised evaluation
// ephmc_ctx_set_stabilize: log det and the segments' y starts from the
// UDT-stabilised chain (stabilize.cu), then the segment sweeps of the
// adjoint (FP64) or mixed (FP32) force over the same segments.  The stacks
// come from the identity at each segment's top (no sweep 1): all segments
// in one launch (regions) or one at a time in one region (checkpointed).
bool stab_applies(const ephmc_ctx *c, int mode) {
    const ephmc_flags &f = c->flags;
    return c->stabilize && mode != EPHMC_FORCE_REFERENCE && !f.constant_force && !f.single_particle &&
           !f.zero_filling && !f.schur_form_inv;
}

// Issues the stabilised evaluation on the context stream without a host
// wait: log|det| and its sign go to the LU's device words (c->lu.diag[V],
// [V+1], status 0 in c->lu.info), as the LU would leave them, so that
// ephmc_leapfrog collects them the same way; with want_force, the force.
int stab_issue(ephmc_ctx *c, const double *x, int mode, bool want_force) {
    const SegPlan p = seg_plan(c, true);
    const int V = (int)c->V;
    const size_t VV = (size_t)V * V;
    const bool mixed = mode == EPHMC_FORCE_MIXED;
    int rc;
    if (3 * p.m > c->jobs_cap) return ret(EPHMC_ERR_ARG, "segment length too small for Nt");
    if ((rc = stab_chain(c, &c->stab, x, p.b, want_force, c->jobs, 0))) return rc;
    EPHMC_CUDA(cudaMemcpyAsync(c->lu.diag + V, stab_parts(c->stab), 2 * sizeof(double), cudaMemcpyDeviceToDevice,
                               c->stream));
    EPHMC_CUDA(cudaMemsetAsync(c->lu.info, 0, 2 * sizeof(int), c->stream));
    c->have_inverse = false;  // the stabilised chain forms no M_hat^-1
    if (!want_force) return EPHMC_OK;
    // segment stacks: regions in the q stack when it holds them, else in the chain's own buffer
    const size_t esz = mixed ? sizeof(float) : sizeof(double);
    const size_t need = esz * VV * (size_t)p.C * (p.regions ? (size_t)p.m : 1);
    void *stack = c->qstack_bytes >= need ? c->qstack : stab_stack(c->stab, need);
    if (!stack) return ret(EPHMC_ERR_NOMEM, "stabilised force: segment stacks");
    std::vector<SliceJob> id;
    for (int j = 0; j < p.m; ++j) {
        const int t0 = p.b[j + 1], t1 = p.b[j];
        SliceJob jb = job(nullptr, nullptr, t1 - 1, t1 - t0 - 1, -1, 0, kPairs, 1);
        jb.stack = static_cast<char *>(stack) + (p.regions ? esz * VV * (size_t)j * p.C : 0);
        jb.stack_off = -1 - t0;
        id.push_back(jb);
    }
    if ((rc = upload_jobs(c, id, c->jobs + 2 * p.m))) return rc;
    AdjointRange rg{0, 0, nullptr, nullptr, nullptr, true};
    rg.seg_C = p.C;
    rg.seg_regions = p.regions;
    rg.y_start = stab_ystart(c->stab);
    const double *none = nullptr;
    auto adjoint = [&](int count) {
        if (!mixed)
            return launch_adjoint_sweep<double, double>(x, c->c, c->lat, static_cast<const double *>(stack), none,
                                                        (int)c->nt, c->flavors, 0, 0.0, c->force, c->stream, &rg,
                                                        count);
        if (adjoint_strip_supported(c->lat))
            return launch_adjoint_strip(x, c->c, c->lat, static_cast<const float *>(stack), none, (int)c->nt,
                                        c->flavors, 0, 0.0, c->force, c->stream, &rg, count);
        return launch_adjoint_sweep<float, float>(x, c->c, c->lat, static_cast<const float *>(stack), none, (int)c->nt,
                                                  c->flavors, 0, 0.0, c->force, c->stream, &rg, count);
    };
    auto launch_stacks = [&](const SliceJob *jd, int n) {
        return mixed ? launch_identity_stacks(c, x, jd, n) : launch_sweep1(c, x, jd, false, n);
    };
    auto stacks = [&](int j0, int n) {
        // segments of a single slice have no stack entries
        int rc2 = EPHMC_OK;
        for (int j = j0; j < j0 + n && rc2 == EPHMC_OK; ++j)
            if (p.b[j] - p.b[j + 1] > 1) rc2 = launch_stacks(c->jobs + 2 * p.m + j, 1);
        return rc2;
    };
    if (p.regions) {
        // all segments' stacks in one launch when every segment has entries
        bool all = true;
        for (int j = 0; j < p.m; ++j) all = all && p.b[j] - p.b[j + 1] > 1;
        rc = all ? launch_stacks(c->jobs + 2 * p.m, p.m) : stacks(0, p.m);
        rg.seg_j0 = 0;
        if (rc == EPHMC_OK) rc = adjoint(p.m);
    }
    for (int j = p.m - 1; !p.regions && j >= 0 && rc == EPHMC_OK; --j) {
        if ((rc = stacks(j, 1))) break;
        rg.seg_j0 = j;
        rg.zero_force = j == p.m - 1;
        rg.y_start = stab_ystart(c->stab) + (size_t)j * VV;
        rc = adjoint(1);
    }
    if (rc == EPHMC_OK && c->flags.no_fourier_acc)
        rc = launch_boson_force(x, c->force, c->omega, 3 * V, (int)c->nt, false, c->stream);
    return rc;
}

int stab_eval(ephmc_ctx *c, const double *x, int mode, bool want_force, double *logdet, int *sign) {
    int rc = stab_issue(c, x, mode, want_force);
    if (rc) return rc;
    double parts[2] = {0, 1};
    EPHMC_CUDA(cudaMemcpyAsync(parts, c->lu.diag + c->V, sizeof(parts), cudaMemcpyDeviceToHost, c->stream));
    EPHMC_CUDA(cudaStreamSynchronize(c->stream));
    *logdet = parts[0];
    *sign = parts[1] < 0 ? -1 : 1;
    c->last_logdet = parts[0];
    c->last_sign = *sign;
    if (*sign < 0 && (c->flavors % 2)) add_warning(EPHMC_WARN_NEGATIVE_DET);
    if (!std::isfinite(parts[0])) return ret(EPHMC_ERR_NONFINITE, "stabilised log det not finite");
    return EPHMC_OK;
}

// M_hat (or, with a stack, sweep 1 of the adjoint) into dst (default c->M)
int build_M_hat(ephmc_ctx *c, const double *x, void *stack, bool stack_float, double *dst = nullptr) {
    if (stack && stack_float) return sweep1_seg(c, x, dst ? dst : c->M);
    if (stack && c->ckpt) return build_M_hat_ckpt(c, x, stack_float, dst ? dst : c->M);
    SliceJob j = job(nullptr, dst ? dst : c->M, (int)c->nt - 1, (int)c->nt, -1, 0, kPairs, 1);
    j.add_identity = !(c->flags.zero_filling || c->flags.single_particle);
    j.stack = stack;
    j.stack_off = -1;
    std::vector<SliceJob> v{j};
    int rc = upload_jobs(c, v, c->jobs);
    if (rc) return rc;
    // the adjoint paths (those with a stack) take the register-strip kernel where
    // the lattice allows; the reference path keeps the reference's summation order
    if (stack && slices_strip_supported(c->lat))
        return stack_float ? launch_slices_strip<float>(x, c->c, c->lat, c->jobs, 1, c->stream)
                           : launch_slices_strip<double>(x, c->c, c->lat, c->jobs, 1, c->stream);
    if (stack && stack_float)
        return launch_slices<double, double, float>(Axis::Rows, x, c->c, c->lat, c->jobs, 1, c->stream);
    return launch_slices<double, double, double>(Axis::Rows, x, c->c, c->lat, c->jobs, 1, c->stream);
}

int factor(ephmc_ctx *c, double *logdet, int *ipiv_host) {
    int sign = 1;
    double ld = 0;
    int rc = lu_logdet_inverse(c->M, c->lu, &ld, &sign, ipiv_host, c->stream);
    c->last_logdet = ld;
    c->last_sign = sign;
    if (logdet) *logdet = ld;
    if (rc == EPHMC_OK && sign < 0 && (c->flavors % 2)) add_warning(EPHMC_WARN_NEGATIVE_DET);
    c->have_inverse = (rc == EPHMC_OK);
    return rc;
}

// construct_all_QM1P (simulation/organic_dense_matrix.c:311-381) as batched launches:
// per halving pass, every spawned copy (P side, on columns) in one launch, then
// every Q-side extension (on rows) in one launch.
int all_G(ephmc_ctx *c, const double *x, const double *Minv = nullptr, double *Gbase = nullptr,
          int *perm_out = nullptr) {
    const unsigned nt = c->nt;
    const size_t VV = (size_t)c->V * c->V;
    int rc;
    if ((rc = ensure_ref(c))) return rc;
    double *G = Gbase ? Gbase : c->G;
    if (!c->flags.single_particle) rc = launch_copy(G, Minv ? Minv : c->M, VV, c->stream);
    else rc = launch_identity(G, (int)c->V, c->stream);
    if (rc) return rc;
    std::vector<unsigned> from_q(nt, 0), from_p(nt, 0);
    unsigned left = nt - 1;
    const unsigned passes = ceil_log2(nt);
    for (unsigned r = 0; r < passes; ++r) {
        const unsigned chunk = ceil_half(left);
        std::vector<SliceJob> spawn, ext;
        for (int i = (int)nt - 1; i >= 0; --i) {
            if (!(i == 0 || from_q[i] || from_p[i])) continue;
            const unsigned j = (unsigned)i + chunk;
            double *Gi = G + (size_t)i * VV;
            if (j < nt && from_q[j] == 0 && from_p[j] == 0) {
                spawn.push_back(job(Gi, G + (size_t)j * VV, (int)from_p[i], (int)chunk, +1, 0, kPairs, 1));
                from_q[j] = from_q[i];
                from_p[j] = from_p[i] + chunk;
            }
            ext.push_back(job(Gi, Gi, (int)(nt - 1 - from_q[i]), (int)chunk, -1, 0, kPairs, 1));
            from_q[i] += chunk;
        }
        left -= chunk;
        if ((rc = ensure_jobs(c, (int)(spawn.size() + ext.size())))) return rc;
        if ((rc = upload_jobs(c, spawn, c->jobs))) return rc;
        if ((rc = upload_jobs(c, ext, c->jobs + spawn.size()))) return rc;
        if ((rc = launch_slices<double, double, double>(Axis::Cols, x, c->c, c->lat, c->jobs, (int)spawn.size(),
                                                        c->stream)))
            return rc;
        if ((rc = launch_slices<double, double, double>(Axis::Rows, x, c->c, c->lat, c->jobs + spawn.size(),
                                                        (int)ext.size(), c->stream)))
            return rc;
    }
    if (perm_out)
        for (unsigned i = 0; i < nt; ++i) {
            perm_out[i] = (int)from_q[i];
            perm_out[nt + i] = (int)from_p[i];
        }
    if (left != 0) return ret(EPHMC_ERR_UNSUPPORTED, "log-depth sharing left slices unaccounted");
    for (unsigned i = 0; i < nt; ++i)
        if (from_q[i] + from_p[i] != nt - 1) return ret(EPHMC_ERR_UNSUPPORTED, "G_t bookkeeping mismatch");
    return EPHMC_OK;
}

// refine_QM1P + force contraction for every slice, in batches of refine_batch slices
int refine_all(ephmc_ctx *c, const double *x, double logdet, const double *Gbase = nullptr) {
    if (int e = ensure_ref(c)) return e;
    const unsigned nt = c->nt;
    const size_t VV = (size_t)c->V * c->V;
    const int nb = c->refine_batch;
    const double *G = Gbase ? Gbase : c->G;
    int rc;
    for (unsigned t0 = 0; t0 < nt; t0 += nb) {
        const int cnt = (int)std::min<unsigned>(nb, nt - t0);
        std::vector<SliceJob> cols, rows;
        for (int b = 0; b < cnt; ++b) {
            const double *Gt = G + (size_t)(t0 + b) * VV;
            // pair 0: X_0 = G F_>0 -> pair 1 on columns (transpose, apply_exp revert, :410-413)
            cols.push_back(job(Gt, c->A + (size_t)b * VV, (int)(t0 + b), 1, 1, 1, 2, 1));
            // pair 1: X_1 = F_<1 G -> pair 0 on rows (apply_exp forward, :408)
            rows.push_back(job(Gt, c->B + (size_t)b * VV, (int)(t0 + b), 1, 1, 0, 1, 1));
        }
        if ((rc = upload_jobs(c, cols, c->jobs))) return rc;
        if ((rc = upload_jobs(c, rows, c->jobs + cnt))) return rc;
        if ((rc = launch_slices<double, double, double>(Axis::Cols, x, c->c, c->lat, c->jobs, cnt, c->stream)))
            return rc;
        if ((rc = launch_slices<double, double, double>(Axis::Rows, x, c->c, c->lat, c->jobs + cnt, cnt,
                                                        c->stream)))
            return rc;
        if ((rc = launch_link_refine(x, c->c, c->lat, c->A, c->B, (int)t0, cnt, c->flavors, c->flags.schur_form_inv,
                                     c->flags.single_particle, logdet, c->force, c->stream)))
            return rc;
    }
    return EPHMC_OK;
}

// Full-matrix refine_QM1P of one V x V matrix G (device) for slice t, in place
// (simulation/organic_dense_matrix.c:383-442), on the context's work buffers.
int refine_full(ephmc_ctx *c, const double *x, double *G, unsigned t) {
    const size_t VV = (size_t)c->V * c->V;
    const double *xs = x + (size_t)t * 3 * c->V;
    double *w0 = c->work, *w1 = w0 + VV, *w2 = w1 + VV, *w3 = w2 + VV;
    const int V = (int)c->V;
    int rc;
    for (int p = 0; p < kPairs; ++p) {
        // pair 0: X_0 = G with pair 1 on columns; pair 1: X_1 = G with pair 0 on rows
        SliceJob j = (p == 0) ? job(G, w0, 0, 1, 1, 1, 2, 1) : job(G, w0, 0, 1, 1, 0, 1, 1);
        std::vector<SliceJob> v{j};
        if ((rc = upload_jobs(c, v, c->jobs))) return rc;
        if ((rc = launch_slices<double, double, double>(p == 0 ? Axis::Cols : Axis::Rows, xs, c->c, c->lat,
                                                        c->jobs, 1, c->stream)))
            return rc;
        if ((rc = launch_stencil(xs, c->c, c->lat, w0, w1, V, true, false, c->stream))) return rc;   // X H
        if ((rc = launch_stencil(xs, c->c, c->lat, w0, w2, V, false, false, c->stream))) return rc;  // H X
        if ((rc = launch_combine_refine(w3, w0, w2, w1, VV, c->c.a_lin[p], c->c.a_quad[p], p == 0, c->stream)))
            return rc;
    }
    return launch_copy(G, w3, VV, c->stream);
}

// log det step of logDetM_and_inv_M_hat on c->M: single_particle takes log(trace M)
// (simulation/organic_dense_matrix.c:550-551), otherwise the LU.
int logdet_step(ephmc_ctx *c, double *ld, int *ipiv_host) {
    if (c->flags.schur_form_inv && !c->flags.single_particle) {
        const int rc = schur_check(&c->schur, c->M, (int)c->V, c->work, c->stream);
        if (rc) return rc;
    }
    if (c->flags.single_particle) {
        double *out = c->scratch + c->scratch_n - 8;
        int rc = launch_trace(c->M, (int)c->V, out, c->stream);
        if (rc) return rc;
        double tr = 0;
        EPHMC_CUDA(cudaMemcpyAsync(&tr, out, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        EPHMC_CUDA(cudaStreamSynchronize(c->stream));
        *ld = std::log(tr);
        c->last_logdet = *ld;
        c->have_inverse = false;
        return EPHMC_OK;
    }
    return factor(c, ld, ipiv_host);
}

// force() (simulation/organic_hmc.c:86-134) from the inverse Minv (device), into c->force.
// mode: reference algorithm or adjoint (FP64 / mixed); flags CONSTANT_FORCE,
// SINGLE_PARTICLE and NO_FOURIER_ACC as the reference.
int force_core(ephmc_ctx *c, const double *xd, const double *Minv, double logdet, int mode, bool have_qstack) {
    const ephmc_flags &f = c->flags;
    const size_t VV = (size_t)c->V * c->V;
    int rc;
    if (f.constant_force && (rc = ensure_ref(c))) return rc;
    if (f.constant_force && f.schur_form_inv) {
        // construct_QM1P's Schur branch (:270-279): 1 - M^-1 (M_hat itself with
        // SINGLE_PARTICLE), no slice products, no refinement
        double *G0 = c->G;
        rc = f.single_particle ? launch_copy(G0, Minv, VV, c->stream) : launch_one_minus(G0, Minv, (int)c->V, c->stream);
        if (rc) return rc;
        if ((rc = launch_contract_full(G0, c->c, c->lat, (int)c->nt, c->flavors, 1, f.single_particle,
                                       std::exp(-logdet), c->force, c->stream)))
            return rc;
    } else if (f.constant_force) {
        // construct_QM1P(time = 0): Q_0 M^-1, refined at slice 0, used for every slice (:92-105, :267-309)
        double *G0 = c->G;
        if (!f.single_particle) rc = launch_copy(G0, Minv, VV, c->stream);
        else rc = launch_identity(G0, (int)c->V, c->stream);
        if (rc) return rc;
        if (c->nt > 1) {
            std::vector<SliceJob> v{job(G0, G0, (int)c->nt - 1, (int)c->nt - 1, -1, 0, kPairs, 1)};
            if ((rc = upload_jobs(c, v, c->jobs))) return rc;
            if ((rc = launch_slices<double, double, double>(Axis::Rows, xd, c->c, c->lat, c->jobs, 1, c->stream)))
                return rc;
        }
        if ((rc = refine_full(c, xd, G0, 0))) return rc;
        if ((rc = launch_contract_full(G0, c->c, c->lat, (int)c->nt, c->flavors, f.schur_form_inv, f.single_particle,
                                       std::exp(-logdet), c->force, c->stream)))
            return rc;
    } else if (mode == EPHMC_FORCE_REFERENCE) {
        if ((rc = all_G(c, xd, Minv))) return rc;
        if ((rc = refine_all(c, xd, logdet))) return rc;
    } else {
        const bool mixed = mode == EPHMC_FORCE_MIXED;
        if (!have_qstack)
            if ((rc = build_M_hat(c, xd, c->qstack, mixed, c->work))) return rc;
        const double *y0 = Minv;
        if (f.single_particle) {  // G_t = Q_t P_t: y(0) rows are the identity
            if ((rc = launch_identity(c->work, (int)c->V, c->stream))) return rc;
            y0 = c->work;
        }
        if (mixed)
            rc = force_mixed_seg(c, xd, y0, logdet);
        else if (c->ckpt)
            rc = adjoint_ckpt(c, xd, y0, mixed, logdet);
        else if (!mixed)
            rc = launch_adjoint_sweep<double, double>(xd, c->c, c->lat, static_cast<const double *>(c->qstack), y0,
                                                      (int)c->nt, c->flavors, f.single_particle, logdet, c->force,
                                                      c->stream);
        else if (adjoint_strip_supported(c->lat))
            rc = launch_adjoint_strip(xd, c->c, c->lat, static_cast<const float *>(c->qstack), y0, (int)c->nt,
                                      c->flavors, f.single_particle, logdet, c->force, c->stream);
        else
            rc = launch_adjoint_sweep<float, float>(xd, c->c, c->lat, static_cast<const float *>(c->qstack), y0,
                                                    (int)c->nt, c->flavors, f.single_particle, logdet, c->force,
                                                    c->stream);
        if (rc) return rc;
        // the adjoint never forms G: the clamp of organic_hmc.c:116 on the finished projection
        if (f.schur_form_inv &&
            (rc = launch_schur_clamp(c->force, (size_t)c->nt * c->V * 3, c->c.kappa,
                                     c->flavors * (f.single_particle ? std::exp(-logdet) : 1.0), c->stream)))
            return rc;
    }
    if (f.no_fourier_acc)
        return launch_boson_force(xd, c->force, c->omega, 3 * (int)c->V, (int)c->nt, false, c->stream);
    return EPHMC_OK;
}

}  // namespace

int ephmc::ensure_ref_buffers(ephmc_ctx *c) { return ensure_ref(c); }
int ephmc::ensure_seg_buffers(ephmc_ctx *c) { return ensure_seg(c, seg_plan(c)); }

// One evaluation issued on the context stream without a host wait: sweep 1,
// LU (log det, sign and status stay in c->lu), force into c->force.  For the
// flags whose force needs no host-side log det (not SINGLE_PARTICLE, not
// SCHUR_FORM_INV).  xd: device field.
int ephmc::eval_async(ephmc_ctx *c, const double *xd, int mode) {
    if (c->flags.single_particle || c->flags.schur_form_inv)
        return ret(EPHMC_ERR_UNSUPPORTED, "eval_async: the force needs the log det on the host");
    if (stab_applies(c, mode)) return stab_issue(c, xd, mode, true);
    const bool adj = mode != EPHMC_FORCE_REFERENCE && !c->flags.constant_force;
    int rc;
    if ((rc = build_M_hat(c, xd, adj ? c->qstack : nullptr, mode == EPHMC_FORCE_MIXED))) return rc;
    if ((rc = lu_logdet_inverse_async(c->M, c->lu, c->stream))) return rc;
    return force_core(c, xd, c->M, 0.0, mode, adj);
}

static bool same_job(const SliceJob &a, const SliceJob &b) {
    return a.src == b.src && a.dst == b.dst && a.stack == b.stack && a.stack_off == b.stack_off &&
           a.s_first == b.s_first && a.s_count == b.s_count && a.s_dir == b.s_dir && a.p_begin == b.p_begin &&
           a.p_end == b.p_end && a.p_step == b.p_step && a.add_identity == b.add_identity;
}

int ephmc::ctx_upload_jobs(ephmc_ctx *c, const SliceJob *jobs, int n, int slot, cudaStream_t st) {
    if (n <= 0) return EPHMC_OK;
    if (slot < 0 || slot + n > c->jobs_cap) return ret(EPHMC_ERR_ARG, "job table too small");
    if ((int)c->jobs_host.size() < c->jobs_cap) {
        c->jobs_host.resize(c->jobs_cap);
        c->jobs_valid.assign(c->jobs_cap, 0);
    }
    bool same = !uploads_are_uncached();
    for (int i = 0; i < n && same; ++i) same = c->jobs_valid[slot + i] && same_job(c->jobs_host[slot + i], jobs[i]);
    if (same) return EPHMC_OK;
    if (int e = upload_small(c->jobs + slot, jobs, sizeof(SliceJob) * n, st)) return e;
    for (int i = 0; i < n; ++i) {
        c->jobs_host[slot + i] = jobs[i];
        c->jobs_valid[slot + i] = 1;
    }
    return EPHMC_OK;
}

void ephmc::ctx_forget_uploads(ephmc_ctx *c) {
    std::fill(c->jobs_valid.begin(), c->jobs_valid.end(), 0);
    fa_forget_tables(c->scratch);
}


extern "C" {

int ephmc_last_status(void) { return ephmc::last_status(); }
unsigned ephmc_last_warnings(void) { return ephmc::last_warnings(); }
const char *ephmc_last_error_message(void) { return ephmc::last_message(); }

const char *ephmc_status_string(int s) {
    switch (s) {
        case EPHMC_OK: return "ok";
        case EPHMC_ERR_CUDA: return "CUDA runtime error";
        case EPHMC_ERR_ARG: return "invalid argument";
        case EPHMC_ERR_LATTICE: return "neighbour table is not a periodic triangular lattice";
        case EPHMC_ERR_SINGULAR: return "singular fermion matrix (zero pivot)";
        case EPHMC_ERR_NONFINITE: return "non-finite log det or force";
        case EPHMC_ERR_NOMEM: return "device allocation failed";
        case EPHMC_ERR_UNSUPPORTED: return "unsupported on the GPU path";
        case EPHMC_ERR_TIMEOUT: return "bounded device wait gave up";
        case EPHMC_ERR_NO_DEVICE: return "no CUDA device";
        default: return "unknown status";
    }
}

const char *ephmc_version(void) { return "ephmc 0.1 (sm_100a)"; }

void *ephmc_alloc(size_t bytes) {
    void *p = nullptr;
    if (cudaMalloc(&p, bytes) != cudaSuccess) {
        cudaGetLastError();
        set_status(EPHMC_ERR_NOMEM, "ephmc_alloc");
        return nullptr;
    }
    return p;
}
void ephmc_free(void *p) {
    if (p) cudaFree(p);
}
int ephmc_memcpy_h2d(void *dst, const void *src, size_t bytes) {
    EPHMC_CUDA(cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice));
    return EPHMC_OK;
}
int ephmc_memcpy_d2h(void *dst, const void *src, size_t bytes) {
    EPHMC_CUDA(cudaMemcpy(dst, src, bytes, cudaMemcpyDeviceToHost));
    return EPHMC_OK;
}
int ephmc_device_synchronize(void) {
    EPHMC_CUDA(cudaDeviceSynchronize());
    return EPHMC_OK;
}

int ephmc_ctx_destroy(ephmc_ctx *c) {
    if (!c) return EPHMC_OK;
    int cur = 0;
    cudaGetDevice(&cur);
    cudaSetDevice(c->device);
    void *bufs[] = {c->x,         c->force,        c->M,          c->G,        c->A,
                    c->B,         c->qstack,       c->jobs,       c->lat.ev_src, c->lat.ev_fac,
                    c->lat.nbr,   c->lat.rev,      c->lat.coef,   c->scratch,  c->work,
                    c->cc_part};
    for (void *b : bufs)
        if (b) cudaFree(b);
    fa_forget_tables(c->scratch);
    if (c->lf_graph) cudaGraphExecDestroy(c->lf_graph);
    cudaFree(c->md_log);
    lu_free(c->lu);
    schur_free(c->schur);
    if (c->seg) cudaFree(c->seg);
    stab_free(c->stab);
    cudaFree(c->dropin_block);
    if (c->aux_stream) cudaStreamDestroy(c->aux_stream);
    for (cudaEvent_t e : c->aux_ev)
        if (e) cudaEventDestroy(e);
    if (c->blas) cublasDestroy(static_cast<cublasHandle_t>(c->blas));
    if (c->blas_ws) cudaFree(c->blas_ws);
    if (c->batch_stream) cudaStreamDestroy(c->batch_stream);
    for (cudaEvent_t e : c->batch_ev)
        if (e) cudaEventDestroy(e);
    for (auto &e : c->ev)
        if (e) cudaEventDestroy(e);
    cudaSetDevice(cur);
    delete c;
    return EPHMC_OK;
}

static int ctx_create_impl(ephmc_ctx **out, unsigned l1, unsigned l2, const unsigned *nnt_in, unsigned V,
                           unsigned nt, const double t[3], const double kappa[3], double mu, double omega,
                           unsigned flavors, const ephmc_flags *flags, int device) {
    clear_status();
    if (!out || V == 0 || nt == 0 || !t || !kappa) return ret(EPHMC_ERR_ARG, "ephmc_ctx_create arguments");
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return ret(EPHMC_ERR_NO_DEVICE, "no CUDA device");
    }
    if (device < 0) EPHMC_CUDA(cudaGetDevice(&device));
    EPHMC_CUDA(cudaSetDevice(device));
    ephmc_ctx *c = new (std::nothrow) ephmc_ctx();
    if (!c) return ret(EPHMC_ERR_NOMEM, "host allocation");
    c->device = device;
    c->l1 = l1;
    c->l2 = l2;
    c->V = V;
    c->nt = nt;
    c->flavors = flavors;
    c->omega = omega;
    if (flags) c->flags = *flags;
    set_couplings(c, t, kappa, mu);
    c->nnt.resize(12 * (size_t)V);
    if (nnt_in) std::memcpy(c->nnt.data(), nnt_in, sizeof(unsigned) * 12 * V);
    else triangular_lattice(l1, l2, c->nnt.data());
    std::vector<int> es, ef, nb;
    int rc = build_event_tables(c->nnt.data(), (int)V, es, ef, nb);
    if (rc) {
        delete c;
        return ret(rc, "neighbour table: every site must receive exactly three forward links");
    }
    c->lat.V = (int)V;
    c->lat.l1 = (int)l1;
    c->lat.l2 = (int)l2;
    const size_t VV = (size_t)V * V, dim = (size_t)nt * V * 3;
    c->refine_batch = (int)std::min<unsigned>(nt, 16);
    c->jobs_cap = (int)std::max<unsigned>(3 * nt, 2 * (unsigned)c->refine_batch) + 8;
    c->scratch_n = fa_scratch_doubles(3 * (int)V, (int)nt) + 16 + kActionScratch;
    auto fail = [&](cudaError_t e, const char *what) {
        cuda_fail(e, what);
        cudaGetLastError();
        ephmc_ctx_destroy(c);
        return (e == cudaErrorMemoryAllocation) ? ret(EPHMC_ERR_NOMEM, what) : EPHMC_ERR_CUDA;
    };
#define ALLOC(ptr, bytes)                                   \
    do {                                                    \
        cudaError_t _e = cudaMalloc((void **)&(ptr), bytes); \
        if (_e != cudaSuccess) return fail(_e, #ptr);       \
    } while (0)
    ALLOC(c->lat.ev_src, sizeof(int) * 6 * V);
    ALLOC(c->lat.ev_fac, sizeof(int) * 6 * V);
    ALLOC(c->lat.nbr, sizeof(int) * 3 * V);
    ALLOC(c->lat.rev, sizeof(int) * 3 * V);
    ALLOC(c->lat.coef, sizeof(float) * 6 * V * nt);
    c->lat.coef_nt = (int)nt;
    ALLOC(c->work, sizeof(double) * VV * 4);
    ALLOC(c->cc_part, sizeof(double) * (size_t)nt * V * 9);
    ALLOC(c->x, sizeof(double) * dim);
    ALLOC(c->force, sizeof(double) * dim);
    ALLOC(c->M, sizeof(double) * VV);
    c->qstack_bytes = sizeof(double) * VV * nt;
    ALLOC(c->qstack, c->qstack_bytes);
    ALLOC(c->jobs, sizeof(SliceJob) * c->jobs_cap);
    ALLOC(c->scratch, sizeof(double) * c->scratch_n);
#undef ALLOC
    if (lu_alloc(c->lu, (int)V) != EPHMC_OK) {
        ephmc_ctx_destroy(c);
        return ret(EPHMC_ERR_NOMEM, "LU workspace");
    }
    cudaMemcpy(c->lat.ev_src, es.data(), sizeof(int) * 6 * V, cudaMemcpyHostToDevice);
    cudaMemcpy(c->lat.ev_fac, ef.data(), sizeof(int) * 6 * V, cudaMemcpyHostToDevice);
    cudaMemcpy(c->lat.nbr, nb.data(), sizeof(int) * 3 * V, cudaMemcpyHostToDevice);
    c->lat.nb_in_events = neighbours_in_events(es, nb, (int)V);
    {
        std::vector<int> rv(3 * (size_t)V, 0);
        for (unsigned k = 0; k < 3; ++k)
            for (unsigned i = 0; i < V; ++i) rv[(size_t)k * V + nb[(size_t)k * V + i]] = (int)i;
        cudaMemcpy(c->lat.rev, rv.data(), sizeof(int) * 3 * V, cudaMemcpyHostToDevice);
    }
    for (auto &e : c->ev)
        if (cudaEventCreate(&e) != cudaSuccess) {
            ephmc_ctx_destroy(c);
            return ret(EPHMC_ERR_CUDA, "cudaEventCreate");
        }
    if (cudaGetLastError() != cudaSuccess) {
        ephmc_ctx_destroy(c);
        return ret(EPHMC_ERR_CUDA, "context upload");
    }
    *out = c;
    return EPHMC_OK;
}

int ephmc_ctx_create(ephmc_ctx **out, unsigned l1, unsigned l2, unsigned nt, const double t[3],
                     const double kappa[3], double mu, double omega, unsigned flavors, const ephmc_flags *flags,
                     int device) {
    if (l1 == 0 || l2 == 0) return ret(EPHMC_ERR_ARG, "lattice extent");
    return ctx_create_impl(out, l1, l2, nullptr, l1 * l2, nt, t, kappa, mu, omega, flavors, flags, device);
}

int ephmc_ctx_create_nnt(ephmc_ctx **out, const unsigned *nnt, unsigned ns, unsigned nt, const double t[3],
                         const double kappa[3], double mu, double omega, unsigned flavors, const ephmc_flags *flags,
                         int device) {
    if (!nnt) return ret(EPHMC_ERR_ARG, "nnt");
    return ctx_create_impl(out, 0, 0, nnt, ns, nt, t, kappa, mu, omega, flavors, flags, device);
}

int ephmc_ctx_set_params(ephmc_ctx *c, const double t[3], const double kappa[3], double mu, double omega,
                         unsigned flavors) {
    if (!c || !t || !kappa) return ret(EPHMC_ERR_ARG, "ephmc_ctx_set_params");
    ++c->param_gen;  // a captured trajectory baked the old values in
    set_couplings(c, t, kappa, mu);
    c->omega = omega;
    c->flavors = flavors;
    return EPHMC_OK;
}

int ephmc_ctx_set_checkpoint(ephmc_ctx *c, unsigned interval) {
    clear_status();
    if (!c) return ret(EPHMC_ERR_ARG, "ephmc_ctx_set_checkpoint");
    ++c->param_gen;  // a captured trajectory baked the old values in
    EPHMC_CUDA(cudaSetDevice(c->device));
    const size_t VV = (size_t)c->V * c->V;
    const size_t need = qstack_bytes_for(c->nt, interval, VV);
    const size_t m = interval ? (c->nt + interval - 1) / interval : 0;
    if (interval && 2 * m > (size_t)c->jobs_cap) return ret(EPHMC_ERR_ARG, "checkpoint interval too small for Nt");
    EPHMC_CUDA(cudaStreamSynchronize(c->stream));
    if (need != c->qstack_bytes) {
        cudaFree(c->qstack);
        c->qstack = nullptr;
        c->qstack_bytes = 0;
        if (cudaMalloc(&c->qstack, need) != cudaSuccess) {
            cudaGetLastError();
            c->qstack = nullptr;
            return ret(EPHMC_ERR_NOMEM, "q stack / checkpoints");
        }
        c->qstack_bytes = need;
    }
    c->ckpt = interval;
    return EPHMC_OK;
}

int ephmc_ctx_set_stabilize(ephmc_ctx *c, int on) {
    clear_status();
    if (!c) return ret(EPHMC_ERR_ARG, "ephmc_ctx_set_stabilize");
    ++c->param_gen;
    c->stabilize = on != 0;
    return EPHMC_OK;
}

int ephmc_ctx_set_segment(ephmc_ctx *c, unsigned length) {
    clear_status();
    if (!c) return ret(EPHMC_ERR_ARG, "ephmc_ctx_set_segment");
    const unsigned C = length ? std::min(length, c->nt) : 0;
    if (C && 3 * ((c->nt + C - 1) / C) > (unsigned)c->jobs_cap) return ret(EPHMC_ERR_ARG, "segment length too small for Nt");
    ++c->param_gen;  // a captured trajectory baked the old segments in
    c->seg_len = C;
    return EPHMC_OK;
}

// Launch shapes by measurement: each candidate is timed over a few
// evaluations of x with the context's own phase events, and the fastest per
// kernel stays in the context.  The candidates only change how threads and
// CTAs share the work: every entry is summed in the same order, so log det
// and M_hat do not change, and the force only by the order of its atomic sums.
int ephmc_ctx_autotune(ephmc_ctx *c, const double *x, int mode, float *ms_before, float *ms_after) {
    clear_status();
    if (!c || !x) return ret(EPHMC_ERR_ARG, "ephmc_ctx_autotune");
    if (mode < EPHMC_FORCE_REFERENCE || mode > EPHMC_FORCE_MIXED) return ret(EPHMC_ERR_ARG, "force mode");
    const int V = (int)c->V;
    // median over `reps` evaluations of the three phases
    auto phases = [&](float out[3]) -> int {
        const int reps = 3;
        std::vector<float> a(reps), b(reps), d(reps);
        double ld = 0;
        if (int rc = ephmc_eval(c, x, nullptr, &ld, mode); rc && rc != EPHMC_ERR_NONFINITE) return rc;
        for (int r = 0; r < reps; ++r) {
            if (int rc = ephmc_eval(c, x, nullptr, &ld, mode); rc && rc != EPHMC_ERR_NONFINITE) return rc;
            a[r] = c->t_mhat;
            b[r] = c->t_lu;
            d[r] = c->t_force;
        }
        for (auto *v : {&a, &b, &d}) std::sort(v->begin(), v->end());
        out[0] = a[reps / 2];
        out[1] = b[reps / 2];
        out[2] = d[reps / 2];
        return EPHMC_OK;
    };
    float t0[3];
    int rc = phases(t0);
    if (rc) return ret(rc);
    if (ms_before) *ms_before = t0[0] + t0[1] + t0[2];
    const bool adj = mode != EPHMC_FORCE_REFERENCE && !c->flags.constant_force;
    const bool mixed = mode == EPHMC_FORCE_MIXED;
    const int Ss[5] = {1, 2, 4, 8, 16}, Rs[6] = {1, 2, 3, 4, 6, 8};
    // k_slices: M_hat unless a strip or tile kernel builds it; the reference force's G_t passes
    const bool slices_mhat = !(adj && slices_strip_supported(c->lat));
    if (slices_mhat || !adj) {
        int bS = c->lat.tune_slices_S, bR = c->lat.tune_slices_R;
        float best = (slices_mhat ? t0[0] : 0.f) + (!adj ? t0[2] : 0.f);
        for (int S : Ss) {
            if ((V + S - 1) / S > 512) continue;
            for (int R : Rs) {
                if (((size_t)2 * R * V + 3 * (size_t)V) * sizeof(double) > 227 * 1024) continue;
                c->lat.tune_slices_S = S;
                c->lat.tune_slices_R = R;
                float t[3];
                if ((rc = phases(t))) return ret(rc);
                const float obj = (slices_mhat ? t[0] : 0.f) + (!adj ? t[2] : 0.f);
                if (obj < best) {
                    best = obj;
                    bS = S;
                    bR = R;
                }
            }
        }
        c->lat.tune_slices_S = bS;
        c->lat.tune_slices_R = bR;
    }
    // k_adjoint: the adjoint force unless a register-layout kernel runs it (mixed; L1 = 8, 12, 16, 24, 32)
    if (adj && !(mixed && adjoint_strip_supported(c->lat))) {
        float tb[3];
        if ((rc = phases(tb))) return ret(rc);
        int bS = c->lat.tune_adj_S, bR = c->lat.tune_adj_R;
        float best = tb[2];
        const size_t real = mixed ? sizeof(float) : sizeof(double);
        for (int S : Ss) {
            if ((V + S - 1) / S > adjoint_max_threads(S, mixed && c->lat.nb_in_events)) continue;
            for (int R = 1; R <= 4; ++R) {
                if (3 * (size_t)V * real + 9 * (size_t)V * real * R > 200 * 1024) continue;
                c->lat.tune_adj_S = S;
                c->lat.tune_adj_R = R;
                float t[3];
                if ((rc = phases(t))) return ret(rc);
                if (t[2] < best) {
                    best = t[2];
                    bS = S;
                    bR = R;
                }
            }
        }
        c->lat.tune_adj_S = bS;
        c->lat.tune_adj_R = bR;
    }
    // the dataflow LU's rows per thread
    if (V <= 1024) {
        float tb[3];
        if ((rc = phases(tb))) return ret(rc);
        int best_r = c->lu.tune_rpt;
        float best = tb[1];
        for (int r : {1, 2, 4}) {
            if (!lu_shape_ok((int)V, r)) continue;
            c->lu.tune_rpt = r;
            float t[3];
            if ((rc = phases(t))) return ret(rc);
            if (t[1] < best) {
                best = t[1];
                best_r = r;
            }
        }
        c->lu.tune_rpt = best_r;
    }
    ++c->param_gen;  // a captured trajectory used the old shapes
    float t1[3];
    if ((rc = phases(t1))) return ret(rc);
    if (ms_after) *ms_after = t1[0] + t1[1] + t1[2];
    return EPHMC_OK;
}

// the shapes in use: slices S, R; adjoint S, R; LU rows per thread (0 = the built-in rule)
int ephmc_ctx_tuning(const ephmc_ctx *c, int out[5]) {
    if (!c || !out) return ret(EPHMC_ERR_ARG, "ephmc_ctx_tuning");
    out[0] = c->lat.tune_slices_S;
    out[1] = c->lat.tune_slices_R;
    out[2] = c->lat.tune_adj_S;
    out[3] = c->lat.tune_adj_R;
    out[4] = c->lu.tune_rpt;
    return EPHMC_OK;
}

int ephmc_ctx_memory(const ephmc_ctx *c, size_t *bytes) {
    if (!c || !bytes) return ret(EPHMC_ERR_ARG, "ephmc_ctx_memory");
    const size_t VV = (size_t)c->V * c->V, dim = (size_t)c->nt * c->V * 3;
    size_t b = c->qstack_bytes + sizeof(double) * (2 * dim + VV + 4 * VV + (size_t)c->nt * c->V * 9 + c->scratch_n);
    if (c->G) b += sizeof(double) * VV * c->nt;
    if (c->A) b += 2 * sizeof(double) * VV * c->refine_batch;
    b += sizeof(double) * VV + sizeof(int) * ((size_t)c->V + lu_sync_words((int)c->V));  // LU panel store, pivots
    b += sizeof(float) * 6 * (size_t)c->V * c->nt;                                      // force sweep coefficients
    b += c->seg_bytes + (c->blas_ws ? kBlasWorkspace : 0);  // segmented mixed force
    b += stab_bytes(c->stab);                               // stabilised chain
    *bytes = b;
    return EPHMC_OK;
}

int ephmc_ctx_set_flags(ephmc_ctx *c, const ephmc_flags *flags) {
    if (!c) return ret(EPHMC_ERR_ARG, "ephmc_ctx_set_flags");
    ++c->param_gen;  // a captured trajectory baked the old values in
    c->flags = flags ? *flags : ephmc_flags{};
    return EPHMC_OK;
}

int ephmc_ctx_lattice(const ephmc_ctx *c, unsigned *nnt_out) {
    if (!c || !nnt_out) return ret(EPHMC_ERR_ARG, "ephmc_ctx_lattice");
    std::memcpy(nnt_out, c->nnt.data(), sizeof(unsigned) * c->nnt.size());
    return EPHMC_OK;
}

int ephmc_ctx_set_stream(ephmc_ctx *c, void *stream) {
    if (!c) return ret(EPHMC_ERR_ARG, "ephmc_ctx_set_stream");
    if (c->stream != static_cast<cudaStream_t>(stream)) ctx_forget_uploads(c);  // uploads queued on the old stream
    c->stream = static_cast<cudaStream_t>(stream);
    return EPHMC_OK;
}

int ephmc_construct_M_hat(ephmc_ctx *c, const double *x, double *M_hat_out) {
    clear_status();
    if (!c || !x) return ret(EPHMC_ERR_ARG, "ephmc_construct_M_hat");
    EPHMC_CUDA(cudaSetDevice(c->device));
    const size_t dim = (size_t)c->nt * c->V * 3;
    const double *xd = nullptr;
    int rc;
    if ((rc = stage_in(c, x, c->x, dim, &xd))) return ret(rc);
    if ((rc = build_M_hat(c, xd, nullptr, false))) return ret(rc);
    c->have_inverse = false;
    if ((rc = stage_out(c, M_hat_out, c->M, (size_t)c->V * c->V))) return ret(rc);
    EPHMC_CUDA(cudaStreamSynchronize(c->stream));
    return EPHMC_OK;
}

int ephmc_logdet_inverse(ephmc_ctx *c, double *M, int *ipiv, double *logdet, int *sign) {
    clear_status();
    if (!c || !M) return ret(EPHMC_ERR_ARG, "ephmc_logdet_inverse");
    EPHMC_CUDA(cudaSetDevice(c->device));
    const size_t VV = (size_t)c->V * c->V;
    const double *Md = nullptr;
    int rc;
    if ((rc = stage_in(c, M, c->M, VV, &Md))) return ret(rc);
    if (Md != c->M) EPHMC_CUDA(cudaMemcpyAsync(c->M, Md, sizeof(double) * VV, cudaMemcpyDeviceToDevice, c->stream));
    rc = factor(c, logdet, ipiv);
    if (sign) *sign = c->last_sign;
    if (rc) return ret(rc, rc == EPHMC_ERR_SINGULAR ? "zero pivot" : nullptr);
    if ((rc = stage_out(c, M, c->M, VV))) return ret(rc);
    EPHMC_CUDA(cudaStreamSynchronize(c->stream));
    return EPHMC_OK;
}

int ephmc_ctx_get_inverse(ephmc_ctx *c, double *out) {
    if (!c || !out) return ret(EPHMC_ERR_ARG, "ephmc_ctx_get_inverse");
    if (!c->have_inverse) return ret(EPHMC_ERR_ARG, "no inverse computed yet");
    int rc = stage_out(c, out, c->M, (size_t)c->V * c->V);
    if (rc) return ret(rc);
    EPHMC_CUDA(cudaStreamSynchronize(c->stream));
    return EPHMC_OK;
}

int ephmc_ctx_last_timings(const ephmc_ctx *c, float *a, float *b, float *d) {
    if (!c) return ret(EPHMC_ERR_ARG, "ephmc_ctx_last_timings");
    if (a) *a = c->t_mhat;
    if (b) *b = c->t_lu;
    if (d) *d = c->t_force;
    return EPHMC_OK;
}

int ephmc_eval(ephmc_ctx *c, const double *x, double *p_dot, double *logdet, int mode) {
    clear_status();
    if (!c || !x) return ret(EPHMC_ERR_ARG, "ephmc_eval");
    if (mode < EPHMC_FORCE_REFERENCE || mode > EPHMC_FORCE_MIXED) return ret(EPHMC_ERR_ARG, "force mode");
    const ephmc_flags &f = c->flags;
    EPHMC_CUDA(cudaSetDevice(c->device));
    const size_t dim = (size_t)c->nt * c->V * 3;
    const double *xd = nullptr;
    int rc;
    if ((rc = stage_in(c, x, c->x, dim, &xd))) return ret(rc);
    EPHMC_CUDA(cudaEventRecord(c->ev[0], c->stream));
    if (stab_applies(c, mode)) {
        double ld = 0;
        int sg = 1;
        rc = stab_eval(c, xd, mode, p_dot != nullptr, &ld, &sg);
        if (logdet) *logdet = ld;
        if (rc) return ret(rc);
        EPHMC_CUDA(cudaEventRecord(c->ev[3], c->stream));
        if ((rc = stage_out(c, p_dot, c->force, dim))) return ret(rc);
        EPHMC_CUDA(cudaStreamSynchronize(c->stream));
        cudaEventElapsedTime(&c->t_force, c->ev[0], c->ev[3]);
        c->t_mhat = c->t_lu = 0;
        return EPHMC_OK;
    }
    const bool adj = mode != EPHMC_FORCE_REFERENCE && !f.constant_force;
    const bool mixed = mode == EPHMC_FORCE_MIXED;
    if ((rc = build_M_hat(c, xd, adj ? c->qstack : nullptr, mixed))) return ret(rc);
    EPHMC_CUDA(cudaEventRecord(c->ev[1], c->stream));
    double ld = 0;
    rc = logdet_step(c, &ld, nullptr);
    if (rc) return ret(rc, rc == EPHMC_ERR_SINGULAR ? "zero pivot" : nullptr);
    EPHMC_CUDA(cudaEventRecord(c->ev[2], c->stream));
    if ((rc = force_core(c, xd, c->M, ld, mode, adj))) return ret(rc);
    EPHMC_CUDA(cudaEventRecord(c->ev[3], c->stream));
    if ((rc = stage_out(c, p_dot, c->force, dim))) return ret(rc);
    EPHMC_CUDA(cudaStreamSynchronize(c->stream));
    cudaEventElapsedTime(&c->t_mhat, c->ev[0], c->ev[1]);
    cudaEventElapsedTime(&c->t_lu, c->ev[1], c->ev[2]);
    cudaEventElapsedTime(&c->t_force, c->ev[2], c->ev[3]);
    if (logdet) *logdet = ld;
    if (!std::isfinite(ld)) return ret(EPHMC_ERR_NONFINITE, "log det not finite");
    return EPHMC_OK;
}

// Several chains' evaluations at once: every phase is issued for all chains
// (each on its context's stream) before the next, and nothing waits on the
// host until all forces are issued.  SINGLE_PARTICLE and SCHUR_FORM_INV
// chains, whose force needs the log det or a host-side eigenvalue check
// first, run through ephmc_eval after the others are issued.
int ephmc_batch_eval(ephmc_ctx *const *ctxs, const double *const *x, double *const *p_dot, double *logdet,
                     unsigned n, int mode) {
    clear_status();
    if (!ctxs || !x || n == 0) return ret(EPHMC_ERR_ARG, "ephmc_batch_eval");
    if (mode < EPHMC_FORCE_REFERENCE || mode > EPHMC_FORCE_MIXED) return ret(EPHMC_ERR_ARG, "force mode");
    for (unsigned i = 0; i < n; ++i) {
        if (!ctxs[i] || !x[i]) return ret(EPHMC_ERR_ARG, "ephmc_batch_eval: null context or field");
        for (unsigned j = 0; j < i; ++j)
            if (ctxs[j] == ctxs[i]) return ret(EPHMC_ERR_ARG, "ephmc_batch_eval: a context appears twice");
    }
    int cur = 0;
    cudaGetDevice(&cur);
    auto sync_fast = [&](const ephmc_ctx *c) { return !c->flags.single_particle && !c->flags.schur_form_inv; };
    // contexts on the legacy default stream run on their own stream for the
    // batch, ordered after the work already queued on the legacy stream
    std::vector<cudaStream_t> caller(n);
    for (unsigned i = 0; i < n; ++i) {
        ephmc_ctx *c = ctxs[i];
        caller[i] = c->stream;
        if (c->stream != nullptr || !sync_fast(c)) continue;
        if (cudaSetDevice(c->device) != cudaSuccess) return ret(EPHMC_ERR_CUDA, "cudaSetDevice");
        if (!c->batch_stream) {
            if (cudaStreamCreateWithFlags(&c->batch_stream, cudaStreamNonBlocking) != cudaSuccess ||
                cudaEventCreateWithFlags(&c->batch_ev[0], cudaEventDisableTiming) != cudaSuccess ||
                cudaEventCreateWithFlags(&c->batch_ev[1], cudaEventDisableTiming) != cudaSuccess) {
                cudaGetLastError();
                return ret(EPHMC_ERR_CUDA, "ephmc_batch_eval: stream creation");
            }
        }
        cudaEventRecord(c->batch_ev[0], nullptr);
        cudaStreamWaitEvent(c->batch_stream, c->batch_ev[0], 0);
        c->stream = c->batch_stream;
    }
    std::vector<const double *> xd(n, nullptr);
    int rc = EPHMC_OK;
    unsigned issued = 0;
    // sweep 1 (M_hat and, for the adjoint paths, the q stack or its checkpoints)
    for (unsigned i = 0; i < n && rc == EPHMC_OK; ++i, issued = i) {
        ephmc_ctx *c = ctxs[i];
        if (!sync_fast(c)) continue;
        if (cudaSetDevice(c->device) != cudaSuccess) { rc = ret(EPHMC_ERR_CUDA, "cudaSetDevice"); break; }
        const size_t dim = (size_t)c->nt * c->V * 3;
        const bool adj = mode != EPHMC_FORCE_REFERENCE && !c->flags.constant_force;
        if ((rc = stage_in(c, x[i], c->x, dim, &xd[i]))) break;
        rc = build_M_hat(c, xd[i], adj ? c->qstack : nullptr, mode == EPHMC_FORCE_MIXED);
    }
    // LU, inverse and log det, left on the device
    for (unsigned i = 0; i < issued && rc == EPHMC_OK; ++i) {
        ephmc_ctx *c = ctxs[i];
        if (!sync_fast(c)) continue;
        cudaSetDevice(c->device);
        rc = lu_logdet_inverse_async(c->M, c->lu, c->stream);
    }
    // forces
    for (unsigned i = 0; i < issued && rc == EPHMC_OK; ++i) {
        ephmc_ctx *c = ctxs[i];
        if (!sync_fast(c)) continue;
        cudaSetDevice(c->device);
        const bool adj = mode != EPHMC_FORCE_REFERENCE && !c->flags.constant_force;
        if ((rc = force_core(c, xd[i], c->M, 0.0, mode, adj))) break;
    }
    // collect: log det, sign, status of every issued chain
    for (unsigned i = 0; i < issued; ++i) {
        ephmc_ctx *c = ctxs[i];
        if (!sync_fast(c)) continue;
        cudaSetDevice(c->device);
        // (a copy to pageable host memory returns only when done: issued after every chain's force)
        if (rc == EPHMC_OK && p_dot && p_dot[i]) rc = stage_out(c, p_dot[i], c->force, (size_t)c->nt * c->V * 3);
        int info[2] = {0, 0};
        double ld[2] = {0, 1};
        cudaMemcpyAsync(info, c->lu.info, sizeof(info), cudaMemcpyDeviceToHost, c->stream);
        cudaMemcpyAsync(ld, c->lu.diag + c->V, sizeof(ld), cudaMemcpyDeviceToHost, c->stream);
        if (cudaStreamSynchronize(c->stream) != cudaSuccess && rc == EPHMC_OK)
            rc = ret(EPHMC_ERR_CUDA, "ephmc_batch_eval: stream synchronisation");
        if (rc != EPHMC_OK) continue;
        if (info[1] != 0) {
            lu_reset_sync(c->lu, c->stream);
            cudaStreamSynchronize(c->stream);
            rc = ret(EPHMC_ERR_TIMEOUT, "LU: a panel wait of the dataflow kernel ran out; the result is invalid");
            continue;
        }
        if (info[0] != 0) {
            rc = ret(EPHMC_ERR_SINGULAR, "zero pivot");
            continue;
        }
        c->last_logdet = ld[0];
        c->last_sign = ld[1] < 0 ? -1 : 1;
        c->have_inverse = true;
        if (c->last_sign < 0 && (c->flavors % 2)) add_warning(EPHMC_WARN_NEGATIVE_DET);
        if (logdet) logdet[i] = ld[0];
        if (!std::isfinite(ld[0])) rc = ret(EPHMC_ERR_NONFINITE, "log det not finite");
    }
    // back to the callers' streams (the legacy stream waits for the batch streams)
    for (unsigned i = 0; i < n; ++i) {
        ephmc_ctx *c = ctxs[i];
        if (c->stream == caller[i]) continue;
        cudaSetDevice(c->device);
        cudaEventRecord(c->batch_ev[1], c->stream);
        cudaStreamWaitEvent(caller[i], c->batch_ev[1], 0);
        c->stream = caller[i];
    }
    // chains whose force needs the log det first
    for (unsigned i = 0; i < n && rc == EPHMC_OK; ++i) {
        ephmc_ctx *c = ctxs[i];
        if (sync_fast(c)) continue;
        const unsigned warn = last_warnings();
        double ld = 0;
        rc = ephmc_eval(c, x[i], p_dot ? p_dot[i] : nullptr, &ld, mode);
        add_warning(warn);
        if (logdet) logdet[i] = ld;
    }
    cudaSetDevice(cur);
    return rc;
}

// force() given the inverse M_inv (simulation/organic_hmc.c:86-134)
int ephmc_force(ephmc_ctx *c, const double *x, const double *M_inv, double logdet, double *p_dot, int mode) {
    clear_status();
    if (!c || !x || !p_dot) return ret(EPHMC_ERR_ARG, "ephmc_force");
    if (mode < EPHMC_FORCE_REFERENCE || mode > EPHMC_FORCE_MIXED) return ret(EPHMC_ERR_ARG, "force mode");
    EPHMC_CUDA(cudaSetDevice(c->device));
    const size_t dim = (size_t)c->nt * c->V * 3, VV = (size_t)c->V * c->V;
    const double *xd = nullptr, *Mi = nullptr;
    int rc;
    if ((rc = stage_in(c, x, c->x, dim, &xd))) return ret(rc);
    if (!c->flags.single_particle && M_inv) {
        if ((rc = stage_in(c, M_inv, c->M, VV, &Mi))) return ret(rc);
    } else {
        Mi = c->M;
    }
    if ((rc = force_core(c, xd, Mi, logdet, mode, false))) return ret(rc);
    if ((rc = stage_out(c, p_dot, c->force, dim))) return ret(rc);
    EPHMC_CUDA(cudaStreamSynchronize(c->stream));
    return EPHMC_OK;
}

// construct_all_QM1P: G_t = Q_t M^-1 P_t for every t into G_out (nt*V*V), bookkeeping
// (slices taken on the Q side, then on the P side) into perm_out[2*nt] if given
int ephmc_all_G(ephmc_ctx *c, const double *x, const double *M_inv, double *G_out, int *perm_out) {
    clear_status();
    if (!c || !x || !G_out) return ret(EPHMC_ERR_ARG, "ephmc_all_G");
    EPHMC_CUDA(cudaSetDevice(c->device));
    const size_t dim = (size_t)c->nt * c->V * 3, VV = (size_t)c->V * c->V;
    const double *xd = nullptr, *Mi = c->M;
    int rc;
    if ((rc = stage_in(c, x, c->x, dim, &xd))) return ret(rc);
    if (M_inv && !c->flags.single_particle)
        if ((rc = stage_in(c, M_inv, c->M, VV, &Mi))) return ret(rc);
    const bool dev = is_device_ptr(G_out);
    if ((rc = ensure_ref(c))) return ret(rc);
    if ((rc = all_G(c, xd, Mi, dev ? G_out : c->G, perm_out))) return ret(rc);
    if (!dev) EPHMC_CUDA(cudaMemcpyAsync(G_out, c->G, sizeof(double) * VV * c->nt, cudaMemcpyDeviceToHost, c->stream));
    EPHMC_CUDA(cudaStreamSynchronize(c->stream));
    return EPHMC_OK;
}

// refine_QM1P on one matrix G (V*V, in place) for slice t
int ephmc_refine_G(ephmc_ctx *c, const double *x, double *G, unsigned t) {
    clear_status();
    if (!c || !x || !G || t >= c->nt) return ret(EPHMC_ERR_ARG, "ephmc_refine_G");
    EPHMC_CUDA(cudaSetDevice(c->device));
    const size_t dim = (size_t)c->nt * c->V * 3, VV = (size_t)c->V * c->V;
    const double *xd = nullptr, *Gd = nullptr;
    int rc;
    if ((rc = stage_in(c, x, c->x, dim, &xd))) return ret(rc);
    if ((rc = stage_in(c, G, c->M, VV, &Gd))) return ret(rc);
    if ((rc = refine_full(c, xd, const_cast<double *>(Gd), t))) return ret(rc);
    if ((rc = stage_out(c, G, Gd, VV))) return ret(rc);
    EPHMC_CUDA(cudaStreamSynchronize(c->stream));
    return EPHMC_OK;
}

// apply_exp_mu_K_to_M (simulation/organic_dense_matrix.c:209-216): nrows contiguous rows of
// length V in M get the pair product of one slice (x_slice: 3V fields); revert/stop as the reference
int ephmc_apply_exp_rows(ephmc_ctx *c, const double *x_slice, double *M, unsigned nrows, int revert, int stop) {
    clear_status();
    if (!c || !x_slice || !M || nrows == 0 || nrows > c->V) return ret(EPHMC_ERR_ARG, "ephmc_apply_exp_rows");
    EPHMC_CUDA(cudaSetDevice(c->device));
    const size_t n = (size_t)nrows * c->V;
    const double *xs = nullptr, *Md = nullptr;
    int rc;
    if ((rc = stage_in(c, x_slice, c->x, 3 * (size_t)c->V, &xs))) return ret(rc);
    if ((rc = stage_in(c, M, c->work, n, &Md))) return ret(rc);
    const int pb = revert ? kPairs - 1 : 0, pe = revert ? stop : stop, ps = revert ? -1 : 1;
    if ((revert && pb > pe) || (!revert && pe > pb)) {
        // the slice kernel propagates whole V x V matrices; nrows < V rows ride in a zero-padded copy
        double *tmp = c->work + 2 * (size_t)c->V * c->V;
        if (nrows < c->V) {
            EPHMC_CUDA(cudaMemsetAsync(tmp, 0, sizeof(double) * (size_t)c->V * c->V, c->stream));
            EPHMC_CUDA(cudaMemcpyAsync(tmp, Md, sizeof(double) * n, cudaMemcpyDeviceToDevice, c->stream));
        }
        double *target = (nrows < c->V) ? tmp : const_cast<double *>(Md);
        std::vector<SliceJob> v{job(target, target, 0, 1, 1, pb, pe, ps)};
        if ((rc = upload_jobs(c, v, c->jobs))) return ret(rc);
        if ((rc = launch_slices<double, double, double>(Axis::Rows, xs, c->c, c->lat, c->jobs, 1, c->stream)))
            return ret(rc);
        if (nrows < c->V)
            EPHMC_CUDA(cudaMemcpyAsync(const_cast<double *>(Md), tmp, sizeof(double) * n, cudaMemcpyDeviceToDevice,
                                       c->stream));
    }
    if ((rc = stage_out(c, M, Md, n))) return ret(rc);
    EPHMC_CUDA(cudaStreamSynchronize(c->stream));
    return EPHMC_OK;
}

// out = (mu + K) in on nrows rows (apply_mu_K_to_v / apply_mu_K_to_M, :96-131);
// add_in: out = in + (mu + K) in (apply_K_plus_1_v, :162-166)
int ephmc_apply_stencil_rows(ephmc_ctx *c, const double *x_slice, const double *in, double *out, unsigned nrows,
                             int add_in) {
    clear_status();
    if (!c || !x_slice || !in || !out || nrows == 0) return ret(EPHMC_ERR_ARG, "ephmc_apply_stencil_rows");
    EPHMC_CUDA(cudaSetDevice(c->device));
    const size_t n = (size_t)nrows * c->V;
    if (n > 2 * (size_t)c->V * c->V) return ret(EPHMC_ERR_ARG, "too many rows");
    const double *xs = nullptr, *ind = nullptr;
    int rc;
    if ((rc = stage_in(c, x_slice, c->x, 3 * (size_t)c->V, &xs))) return ret(rc);
    if ((rc = stage_in(c, in, c->work, n, &ind))) return ret(rc);
    double *od = is_device_ptr(out) ? out : c->work + 2 * (size_t)c->V * c->V;
    if ((rc = launch_stencil(xs, c->c, c->lat, ind, od, (int)nrows, false, add_in != 0, c->stream))) return ret(rc);
    if ((rc = stage_out(c, out, od, n))) return ret(rc);
    EPHMC_CUDA(cudaStreamSynchronize(c->stream));
    return EPHMC_OK;
}

// w = I_k v, the antisymmetric current along link k (apply_current_to_v, :226-249)
int ephmc_apply_current(ephmc_ctx *c, const double *x_slice, const double *v, double *w, unsigned k) {
    clear_status();
    if (!c || !x_slice || !v || !w || k > 2) return ret(EPHMC_ERR_ARG, "ephmc_apply_current");
    EPHMC_CUDA(cudaSetDevice(c->device));
    const size_t V = c->V;
    const double *xs = nullptr, *vd = nullptr;
    int rc;
    if ((rc = stage_in(c, x_slice, c->x, 3 * V, &xs))) return ret(rc);
    if ((rc = stage_in(c, v, c->work, V, &vd))) return ret(rc);
    double *wd = is_device_ptr(w) ? w : c->work + V;
    if ((rc = launch_current(xs, c->c, c->lat, c->lat.rev + (size_t)k * V, vd, wd, (int)k, c->stream))) return ret(rc);
    if ((rc = stage_out(c, w, wd, V))) return ret(rc);
    EPHMC_CUDA(cudaStreamSynchronize(c->stream));
    return EPHMC_OK;
}

}  // extern "C"
