// Transient-localisation (static disorder) mode: current-current matrix
// elements of disorder samples, Boltzmann-weighted and binned in frequency.
//
// Reference: hist_trans_loc / run_trans_loc (simulation/organic_trans_loc.c:25-114).
// Per sample, with H = -mu + K(x) the one-slice hopping matrix of a bond field
// x (construct_hamilton, simulation/organic_dense_matrix.c:218-224), its
// eigenpairs (E_i, psi_i), E ascending, and the current operators I_k
// (antisymmetric hopping along link k, apply_current_to_v :226-249):
//   P_k[i][j] = psi_j . I_k psi_i
//   for every pair with E_j >= E_i:
//     I = sum_c (sum_k mat[c][k] P_k[i][j])^2        (contr_gr_mat, organic_lattice.c:62-79)
//     hist[(unsigned)((E_j - E_i)/width + 0.5)] += (e^-E_i + e^-E_j) I / (width V)
//   Z = sum_i e^-E_i / V
//
// Device pipeline of one sample (one "lane": stream + solver + buffers):
//   k_tl_hamilton   H (V x V, FP64) and the contracted hopping factors
//   cuSOLVER dsyevd eigenvalues and eigenvectors (library)
//   k_tl_current    W_c = J_c psi for both Cartesian components c, where
//                   J_c = sum_k mat[c][k] I_k (the contraction moved inside
//                   the matrix element: two products instead of three)
//   cuBLAS dsyrkx   Q_c[i][j] = psi_j . W_c[i] on the triangle j >= i (library)
//   k_tl_boltzmann  e^-E_i and Z
//   k_tl_bin        the pairs j >= i: weight, bin, warp-segmented sums into a
//                   per-CTA shared-memory histogram, one global atomic per
//                   non-empty bin per CTA
// Independent samples run on several lanes at once.  Bins at or beyond nbins
// are dropped; the reference writes them past the end of its histogram.
#include "ephmc_internal.cuh"

#include <cublas_v2.h>
#include <cusolverDn.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <thread>
#include <vector>

namespace ephmc {

// Cartesian projection of the three link directions, contr_mat[c*3 + k]
// (construct_contraction_mat, simulation/organic_lattice.c:48-60)
struct TlMat {
    double m[6];
};

struct TlHop {
    double t[3], kappa[3];
};

namespace {

// H = mu_d 1 + sum_{i,k} fac_k(i) (e_i e_n^T + e_n e_i^T), n = nbr_k(i),
// fac_k(i) = t_k - kappa_k x[3i + k]; g[(c*3+k)*V + i] = mat[c][k] fac_k(i)
// and gr[(c*3+k)*V + n] = g[(c*3+k)*V + i] (the factor of the link that ends at n)
__global__ void k_tl_hamilton(const double *__restrict__ x, TlHop hp, TlMat mt, double mu_d,
                              const int *__restrict__ nbr, int V, double *__restrict__ g, double *__restrict__ gr,
                              double *__restrict__ H) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= V) return;
    atomicAdd(H + (size_t)i * V + i, mu_d);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const double f = hp.t[k] - hp.kappa[k] * x[3 * (size_t)i + k];
        const int n = nbr[k * V + i];
        atomicAdd(H + (size_t)i * V + n, f);
        atomicAdd(H + (size_t)n * V + i, f);
#pragma unroll
        for (int c = 0; c < 2; ++c) {
            const double gc = mt.m[c * 3 + k] * f;
            g[(c * 3 + k) * V + i] = gc;
            gr[(c * 3 + k) * V + n] = gc;
        }
    }
}

constexpr int kCurRows = 16;  // eigenvectors per CTA of k_tl_current

// W_c[v][s] = (J_c psi_v)[s] = sum_k g_ck(s) psi_v[nbr_k(s)] - gr_ck(s) psi_v[rev_k(s)]
__global__ void __launch_bounds__(256) k_tl_current(const double *__restrict__ psi, const double *__restrict__ g,
                                                    const double *__restrict__ gr, const int *__restrict__ nbr,
                                                    const int *__restrict__ rev, int V, double *__restrict__ W0,
                                                    double *__restrict__ W1) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= V) return;
    int n[3], r[3];
    double a0[3], a1[3], b0[3], b1[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        n[k] = nbr[k * V + s];
        r[k] = rev[k * V + s];
        a0[k] = g[k * V + s];
        a1[k] = g[(3 + k) * V + s];
        b0[k] = gr[k * V + s];
        b1[k] = gr[(3 + k) * V + s];
    }
    const int v0 = blockIdx.y * kCurRows, v1 = min(V, v0 + kCurRows);
    for (int v = v0; v < v1; ++v) {
        const double *p = psi + (size_t)v * V;
        double w0 = 0.0, w1 = 0.0;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const double pn = __ldg(p + n[k]), pr = __ldg(p + r[k]);
            w0 = fma(a0[k], pn, fma(-b0[k], pr, w0));
            w1 = fma(a1[k], pn, fma(-b1[k], pr, w1));
        }
        W0[(size_t)v * V + s] = w0;
        W1[(size_t)v * V + s] = w1;
    }
}

// zb[i] = e^-E_i and z = sum_i zb[i] / V (one CTA of 256 threads)
__global__ void k_tl_boltzmann(const double *__restrict__ ev, int V, double *__restrict__ zb, double *__restrict__ z) {
    __shared__ double red[256];
    double s = 0.0;
    for (int i = threadIdx.x; i < V; i += blockDim.x) {
        const double b = exp(-ev[i]);
        zb[i] = b;
        s += b;
    }
    red[threadIdx.x] = s;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) z[0] = red[0] / V;
}

constexpr int kBinWarps = 8;
constexpr size_t kBinShared = 64 * 1024;  // histograms up to 8192 bins stay in shared memory

// One warp per row i (rows dealt round-robin over the grid), 32 consecutive
// j per step from the aligned column at or below i.  E is ascending, so the
// bins of a warp's 32 pairs are non-decreasing in the lane: equal bins are
// contiguous and a segmented shuffle sum leaves one atomic per distinct bin.
// A pair with E_j == E_i, j > i, is also the reference's pair (j, i) and
// counts twice.  SHARED: per-CTA histogram in shared memory, else straight
// into global memory.
template <bool SHARED>
__global__ void __launch_bounds__(kBinWarps * 32) k_tl_bin(const double *__restrict__ Q0, const double *__restrict__ Q1,
                                                           const double *__restrict__ ev, const double *__restrict__ zb,
                                                           int V, int nbins, double inv_width, double scale,
                                                           double *__restrict__ hist) {
    extern __shared__ double sh[];  // [nbins] when SHARED
    double *acc = SHARED ? sh : hist;
    if (SHARED) {
        for (int b = threadIdx.x; b < nbins; b += blockDim.x) sh[b] = 0.0;
        __syncthreads();
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int i = blockIdx.x * kBinWarps + warp; i < V; i += gridDim.x * kBinWarps) {
        const double ei = ev[i], zi = zb[i];
        const double *q0 = Q0 + (size_t)i * V, *q1 = Q1 + (size_t)i * V;
        for (int j0 = i & ~31; j0 < V; j0 += 32) {
            const int j = j0 + lane;
            double val = 0.0;
            unsigned bin = 0;  // lanes j < i: bin 0 keeps the sequence non-decreasing
            if (j >= V) {
                bin = 0xFFFFFFFFu;
            } else if (j >= i) {
                const double ej = ev[j];
                const double c0 = q0[j], c1 = q1[j];
                val = (zi + zb[j]) * fma(c0, c0, c1 * c1) * scale;
                if (j > i && ej == ei) val *= 2.0;
                bin = (unsigned)((ej - ei) * inv_width + .5);
            }
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const double vu = __shfl_up_sync(0xFFFFFFFFu, val, o);
                const unsigned bu = __shfl_up_sync(0xFFFFFFFFu, bin, o);
                if (lane >= o && bu == bin) val += vu;
            }
            const unsigned bn = __shfl_down_sync(0xFFFFFFFFu, bin, 1);
            const bool last = lane == 31 || bn != bin;
            if (last && bin < (unsigned)nbins && val != 0.0) atomicAdd(acc + bin, val);
        }
    }
    if (SHARED) {
        __syncthreads();
        for (int b = threadIdx.x; b < nbins; b += blockDim.x)
            if (sh[b] != 0.0) atomicAdd(hist + b, sh[b]);
    }
}

}  // namespace

}  // namespace ephmc

using namespace ephmc;

namespace {

struct TlLane {
    cudaStream_t st = nullptr;
    cudaEvent_t done = nullptr;
    cusolverDnHandle_t solver = nullptr;
    cublasHandle_t blas = nullptr;
    double *g = nullptr, *gr = nullptr;  // 6V each
    double *H = nullptr, *ev = nullptr, *zb = nullptr, *W0 = nullptr, *W1 = nullptr, *Q0 = nullptr, *Q1 = nullptr;
    double *work = nullptr;
    int lwork = 0;
    cudaEvent_t stage[6] = {};  // stage boundaries of the first sample a run gives this lane
};

}  // namespace

struct ephmc_tl {
    int device = 0;
    int V = 0, nbins = 0;
    TlHop hop{};
    TlMat mat{};
    double mu_d = 0;
    unsigned max_lanes = 1;
    int nsm = 148;
    cudaStream_t stream = nullptr;  // caller's stream (nullptr = legacy default)
    cudaEvent_t start = nullptr;
    int *nbr = nullptr, *rev = nullptr;
    std::vector<TlLane> lanes;
    // per-run buffers, grown on demand
    double *xs = nullptr, *hist = nullptr, *z = nullptr;
    int *info = nullptr;
    size_t xs_cap = 0, z_cap = 0, info_cap = 0;
    bool timed_lane0 = false;  // lane 0's stage events hold a sample
};

namespace {

int tl_fail(int status, const char *msg) {
    set_status(status, msg);
    return status;
}

bool tl_is_device(const void *p) {
    if (!p) return false;
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

template <class T>
bool tl_malloc(T **p, size_t count) {
    if (cudaMalloc((void **)p, sizeof(T) * std::max<size_t>(count, 1)) != cudaSuccess) {
        cudaGetLastError();
        *p = nullptr;
        return false;
    }
    return true;
}

template <class T>
int grow(T **p, size_t *cap, size_t need) {
    if (need <= *cap) return EPHMC_OK;
    if (*p) cudaFree(*p);
    *p = nullptr;
    *cap = 0;
    if (!tl_malloc(p, need)) return tl_fail(EPHMC_ERR_NOMEM, "trans_loc: device allocation");
    *cap = need;
    return EPHMC_OK;
}

void lane_free(TlLane &l) {
    if (l.st) cudaStreamSynchronize(l.st);
    if (l.solver) cusolverDnDestroy(l.solver);
    if (l.blas) cublasDestroy(l.blas);
    double *bufs[] = {l.g, l.gr, l.H, l.ev, l.zb, l.W0, l.W1, l.Q0, l.Q1, l.work};
    for (double *b : bufs)
        if (b) cudaFree(b);
    if (l.done) cudaEventDestroy(l.done);
    for (cudaEvent_t &e : l.stage)
        if (e) cudaEventDestroy(e);
    if (l.st) cudaStreamDestroy(l.st);
    cudaGetLastError();
    l = TlLane{};
}

int lane_init(const ephmc_tl *tl, TlLane &l) {
    const int V = tl->V;
    const size_t VV = (size_t)V * V;
    if (cudaStreamCreateWithFlags(&l.st, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&l.done, cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        return tl_fail(EPHMC_ERR_CUDA, "trans_loc: stream creation");
    }
    for (cudaEvent_t &e : l.stage)
        if (cudaEventCreate(&e) != cudaSuccess) {
            cudaGetLastError();
            e = nullptr;
            return tl_fail(EPHMC_ERR_CUDA, "trans_loc: event creation");
        }
    if (!tl_malloc(&l.g, 6 * (size_t)V) || !tl_malloc(&l.gr, 6 * (size_t)V) || !tl_malloc(&l.H, VV) ||
        !tl_malloc(&l.ev, V) || !tl_malloc(&l.zb, V) || !tl_malloc(&l.W0, VV) || !tl_malloc(&l.W1, VV) ||
        !tl_malloc(&l.Q0, VV) || !tl_malloc(&l.Q1, VV))
        return tl_fail(EPHMC_ERR_NOMEM, "trans_loc: device allocation of a sample lane");
    if (cusolverDnCreate(&l.solver) != CUSOLVER_STATUS_SUCCESS) {
        l.solver = nullptr;
        return tl_fail(EPHMC_ERR_CUDA, "trans_loc: cusolverDnCreate");
    }
    if (cublasCreate(&l.blas) != CUBLAS_STATUS_SUCCESS) {
        l.blas = nullptr;
        return tl_fail(EPHMC_ERR_CUDA, "trans_loc: cublasCreate");
    }
    if (cusolverDnSetStream(l.solver, l.st) != CUSOLVER_STATUS_SUCCESS ||
        cublasSetStream(l.blas, l.st) != CUBLAS_STATUS_SUCCESS)
        return tl_fail(EPHMC_ERR_CUDA, "trans_loc: binding the lane stream");
    if (cusolverDnDsyevd_bufferSize(l.solver, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_UPPER, V, l.H, V, l.ev,
                                    &l.lwork) != CUSOLVER_STATUS_SUCCESS)
        return tl_fail(EPHMC_ERR_CUDA, "trans_loc: cusolverDnDsyevd_bufferSize");
    if (!tl_malloc(&l.work, (size_t)std::max(l.lwork, 1)))
        return tl_fail(EPHMC_ERR_NOMEM, "trans_loc: device allocation of the eigensolver workspace");
    return EPHMC_OK;
}

// one sample on lane l: x (3V, device) -> tl->hist (accumulated), z[0], info[0]
int tl_sample(ephmc_tl *tl, TlLane &l, const double *x, double inv_width, double scale, double *z, int *info,
              bool timed) {
    const int V = tl->V;
    const size_t VV = (size_t)V * V;
    cudaStream_t st = l.st;
    auto mark = [&](int k) {
        if (timed) cudaEventRecord(l.stage[k], st);
    };
    mark(0);
    EPHMC_CUDA(cudaMemsetAsync(l.H, 0, sizeof(double) * VV, st));
    k_tl_hamilton<<<(V + 127) / 128, 128, 0, st>>>(x, tl->hop, tl->mat, tl->mu_d, tl->nbr, V, l.g, l.gr, l.H);
    count_launch(1);
    EPHMC_CUDA(cudaGetLastError());
    mark(1);
    // H is symmetric: its row-major array is its column-major one.  On return
    // eigenvector v is column v, contiguous: psi[v*V + s] = l.H[v*V + s].
    if (cusolverDnDsyevd(l.solver, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_UPPER, V, l.H, V, l.ev, l.work, l.lwork,
                         info) != CUSOLVER_STATUS_SUCCESS)
        return tl_fail(EPHMC_ERR_CUDA, "trans_loc: cusolverDnDsyevd");
    mark(2);
    const double *psi = l.H;
    k_tl_current<<<dim3((V + 255) / 256, (V + kCurRows - 1) / kCurRows), 256, 0, st>>>(psi, l.g, l.gr, tl->nbr,
                                                                                      tl->rev, V, l.W0, l.W1);
    count_launch(1);
    EPHMC_CUDA(cudaGetLastError());
    mark(3);
    // column-major C = psi_cm^T W_cm = psi W_c^T: C_cm[j][i] = psi_j . W_c[i]
    // = Q_c[i][j], stored row-major at i*V + j; its lower triangle (j >= i) is
    // the set of pairs
    const double one = 1.0, zero = 0.0;
    if (cublasDsyrkx(l.blas, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_T, V, V, &one, psi, V, l.W0, V, &zero, l.Q0, V) !=
            CUBLAS_STATUS_SUCCESS ||
        cublasDsyrkx(l.blas, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_T, V, V, &one, psi, V, l.W1, V, &zero, l.Q1, V) !=
            CUBLAS_STATUS_SUCCESS)
        return tl_fail(EPHMC_ERR_CUDA, "trans_loc: cublasDsyrkx");
    mark(4);
    k_tl_boltzmann<<<1, 256, 0, st>>>(l.ev, V, l.zb, z);
    count_launch(1);
    EPHMC_CUDA(cudaGetLastError());
    const int grid = std::max(1, std::min((V + kBinWarps - 1) / kBinWarps, 4 * tl->nsm));
    const size_t sh = sizeof(double) * tl->nbins;
    if (sh <= kBinShared)
        k_tl_bin<true><<<grid, kBinWarps * 32, sh, st>>>(l.Q0, l.Q1, l.ev, l.zb, V, tl->nbins, inv_width, scale,
                                                         tl->hist);
    else
        k_tl_bin<false><<<grid, kBinWarps * 32, 0, st>>>(l.Q0, l.Q1, l.ev, l.zb, V, tl->nbins, inv_width, scale,
                                                          tl->hist);
    count_launch(1);
    EPHMC_CUDA(cudaGetLastError());
    mark(5);
    return EPHMC_OK;
}

// samples lane, lane + nl, ... of a run on lane `lane` (its own host thread when nl > 1)
int tl_lane_run(ephmc_tl *tl, unsigned lane, unsigned nl, const double *xd, unsigned nsamples, double inv_width,
                double scale) {
    if (nl > 1 && cudaSetDevice(tl->device) != cudaSuccess) return tl_fail(EPHMC_ERR_CUDA, "cudaSetDevice");
    const size_t dim = 3 * (size_t)tl->V;
    for (unsigned s = lane; s < nsamples; s += nl) {
        const int rc = tl_sample(tl, tl->lanes[lane], xd + dim * s, inv_width, scale, tl->z + s, tl->info + s,
                                 s == lane);
        if (rc != EPHMC_OK) return rc;
    }
    return EPHMC_OK;
}

}  // namespace

namespace ephmc {

int tl_create_nnt(ephmc_tl **out, const unsigned *nnt, unsigned V, unsigned nbins, const double t[3],
                  const double kappa[3], double mu, const double contr_mat[6], unsigned lanes, int device) {
    if (!out) return tl_fail(EPHMC_ERR_ARG, "ephmc_tl_create: out is NULL");
    *out = nullptr;
    if (!nnt || V == 0 || nbins == 0 || !t || !kappa)
        return tl_fail(EPHMC_ERR_ARG, "ephmc_tl_create: lattice, bins and couplings are required");
    if (!contr_mat)
        return tl_fail(EPHMC_ERR_ARG,
                       "ephmc_tl_create: the contraction matrix is required (input.txt unit vectors a and b)");
    if (V > 46340u) return tl_fail(EPHMC_ERR_ARG, "ephmc_tl_create: V x V exceeds the 32-bit eigensolver interface");
    std::vector<int> es, ef, nb;
    if (build_event_tables(nnt, (int)V, es, ef, nb) != EPHMC_OK)
        return tl_fail(EPHMC_ERR_LATTICE, "neighbour table: every site must receive exactly three forward links");
    std::vector<int> rv(3 * (size_t)V, 0);
    for (unsigned k = 0; k < 3; ++k)
        for (unsigned i = 0; i < V; ++i) rv[(size_t)k * V + nb[(size_t)k * V + i]] = (int)i;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return tl_fail(EPHMC_ERR_NO_DEVICE, "no CUDA device");
    }
    if (device < 0) EPHMC_CUDA(cudaGetDevice(&device));
    EPHMC_CUDA(cudaSetDevice(device));
    ephmc_tl *tl = new (std::nothrow) ephmc_tl();
    if (!tl) return tl_fail(EPHMC_ERR_NOMEM, "host allocation");
    tl->device = device;
    tl->V = (int)V;
    tl->nbins = (int)nbins;
    tl_set_params(tl, t, kappa, mu, contr_mat);
    tl->max_lanes = std::max(1u, std::min(lanes, 16u));
    cudaDeviceGetAttribute(&tl->nsm, cudaDevAttrMultiProcessorCount, device);
    int rc = EPHMC_OK;
    if (!tl_malloc(&tl->nbr, 3 * (size_t)V) || !tl_malloc(&tl->rev, 3 * (size_t)V) || !tl_malloc(&tl->hist, nbins))
        rc = tl_fail(EPHMC_ERR_NOMEM, "ephmc_tl_create: device allocation");
    if (rc == EPHMC_OK && cudaEventCreateWithFlags(&tl->start, cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        rc = tl_fail(EPHMC_ERR_CUDA, "ephmc_tl_create: event creation");
    }
    if (rc == EPHMC_OK &&
        (cudaMemcpy(tl->nbr, nb.data(), sizeof(int) * 3 * V, cudaMemcpyHostToDevice) != cudaSuccess ||
         cudaMemcpy(tl->rev, rv.data(), sizeof(int) * 3 * V, cudaMemcpyHostToDevice) != cudaSuccess)) {
        cudaGetLastError();
        rc = tl_fail(EPHMC_ERR_CUDA, "ephmc_tl_create: upload of the neighbour tables");
    }
    if (rc == EPHMC_OK && cudaFuncSetAttribute(k_tl_bin<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               (int)kBinShared) != cudaSuccess) {
        cudaGetLastError();
        rc = tl_fail(EPHMC_ERR_CUDA, "ephmc_tl_create: shared-memory attribute of the binning kernel");
    }
    if (rc == EPHMC_OK) {
        tl->lanes.emplace_back();
        rc = lane_init(tl, tl->lanes.back());
    }
    if (rc != EPHMC_OK) {
        const int keep = last_status();
        const std::string msg = last_message();
        ephmc_tl_destroy(tl);
        return tl_fail(keep, msg.c_str());
    }
    *out = tl;
    return EPHMC_OK;
}

int tl_set_params(ephmc_tl *tl, const double t[3], const double kappa[3], double mu, const double contr_mat[6]) {
    if (!tl || !t || !kappa || !contr_mat) return tl_fail(EPHMC_ERR_ARG, "trans_loc parameters");
    for (int k = 0; k < 3; ++k) {
        tl->hop.t[k] = t[k];
        tl->hop.kappa[k] = kappa[k];
    }
    tl->mu_d = -mu;  // construct_hamilton is called with -mu (organic_trans_loc.c:40)
    for (int e = 0; e < 6; ++e) tl->mat.m[e] = contr_mat[e];
    return EPHMC_OK;
}

}  // namespace ephmc

extern "C" {

EPHMC_API int ephmc_tl_create(ephmc_tl **out, unsigned l1, unsigned l2, unsigned nbins, const double t[3],
                              const double kappa[3], double mu, const double contr_mat[6], unsigned lanes,
                              int device) {
    clear_status();
    if (l1 == 0 || l2 == 0) return tl_fail(EPHMC_ERR_ARG, "ephmc_tl_create: lattice extent");
    std::vector<unsigned> nnt(12 * (size_t)l1 * l2);
    triangular_lattice(l1, l2, nnt.data());
    return tl_create_nnt(out, nnt.data(), l1 * l2, nbins, t, kappa, mu, contr_mat, lanes, device);
}

EPHMC_API int ephmc_tl_destroy(ephmc_tl *tl) {
    if (!tl) return EPHMC_OK;
    int cur = 0;
    cudaGetDevice(&cur);
    cudaSetDevice(tl->device);
    for (auto &l : tl->lanes) lane_free(l);
    void *bufs[] = {tl->nbr, tl->rev, tl->xs, tl->hist, tl->z, tl->info};
    for (void *b : bufs)
        if (b) cudaFree(b);
    if (tl->start) cudaEventDestroy(tl->start);
    cudaGetLastError();
    cudaSetDevice(cur);
    delete tl;
    return EPHMC_OK;
}

EPHMC_API int ephmc_tl_set_stream(ephmc_tl *tl, void *stream) {
    clear_status();
    if (!tl) return tl_fail(EPHMC_ERR_ARG, "ephmc_tl_set_stream: tl is NULL");
    tl->stream = static_cast<cudaStream_t>(stream);
    return EPHMC_OK;
}

EPHMC_API int ephmc_tl_default_width(const ephmc_tl *tl, double *width) {
    clear_status();
    if (!tl || !width) return tl_fail(EPHMC_ERR_ARG, "ephmc_tl_default_width arguments");
    // run_trans_loc (simulation/organic_trans_loc.c:99-100) with mu = -mu_d
    double w = 2 * tl->mu_d / tl->nbins;
    for (int k = 0; k < 3; ++k) w += 8 * std::fabs(tl->hop.kappa[k]) / tl->nbins;
    *width = w;
    return EPHMC_OK;
}

EPHMC_API int ephmc_tl_run(ephmc_tl *tl, const double *x, unsigned nsamples, double width, double *hist,
                           double *z) {
    clear_status();
    if (!tl || !x || !hist || nsamples == 0) return tl_fail(EPHMC_ERR_ARG, "ephmc_tl_run arguments");
    if (!(width > 0) || !std::isfinite(width)) return tl_fail(EPHMC_ERR_ARG, "ephmc_tl_run: width must be positive");
    EPHMC_CUDA(cudaSetDevice(tl->device));
    const int V = tl->V;
    const size_t dim = 3 * (size_t)V;
    cudaStream_t cs = tl->stream;
    // lanes: one per concurrently processed sample, created on first use; a
    // lane that does not fit in device memory caps the count
    const unsigned want = std::min<unsigned>(tl->max_lanes, nsamples);
    while (tl->lanes.size() < want) {
        tl->lanes.emplace_back();
        if (lane_init(tl, tl->lanes.back()) != EPHMC_OK) {
            lane_free(tl->lanes.back());
            tl->lanes.pop_back();
            tl->max_lanes = (unsigned)tl->lanes.size();
            clear_status();
            break;
        }
    }
    const unsigned nl = std::min<unsigned>((unsigned)tl->lanes.size(), nsamples);
    if (grow(&tl->z, &tl->z_cap, nsamples) != EPHMC_OK || grow(&tl->info, &tl->info_cap, nsamples) != EPHMC_OK)
        return last_status();
    const double *xd = x;
    if (!tl_is_device(x)) {
        if (grow(&tl->xs, &tl->xs_cap, dim * nsamples) != EPHMC_OK) return last_status();
        EPHMC_CUDA(cudaMemcpyAsync(tl->xs, x, sizeof(double) * dim * nsamples, cudaMemcpyHostToDevice, cs));
        xd = tl->xs;
    }
    const bool hist_dev = tl_is_device(hist);
    EPHMC_CUDA(cudaMemsetAsync(tl->hist, 0, sizeof(double) * tl->nbins, cs));
    EPHMC_CUDA(cudaMemsetAsync(tl->info, 0, sizeof(int) * nsamples, cs));
    EPHMC_CUDA(cudaEventRecord(tl->start, cs));
    for (unsigned l = 0; l < nl; ++l) EPHMC_CUDA(cudaStreamWaitEvent(tl->lanes[l].st, tl->start, 0));
    const double inv_width = 1.0 / width, scale = 1.0 / (width * V);
    // cuSOLVER's eigensolver returns to the host only when it is done, so each
    // lane gets its own host thread: the lanes' solver phases then overlap
    int rc = EPHMC_OK;
    if (nl == 1) {
        rc = tl_lane_run(tl, 0, 1, xd, nsamples, inv_width, scale);
    } else {
        std::vector<int> rcs(nl, EPHMC_OK);
        std::vector<std::string> msgs(nl);
        std::vector<std::thread> th;
        for (unsigned l = 0; l < nl; ++l)
            th.emplace_back([&, l] {
                rcs[l] = tl_lane_run(tl, l, nl, xd, nsamples, inv_width, scale);
                if (rcs[l] != EPHMC_OK) msgs[l] = last_message();
            });
        for (auto &t : th) t.join();
        for (unsigned l = 0; l < nl && rc == EPHMC_OK; ++l)
            if (rcs[l] != EPHMC_OK) rc = tl_fail(rcs[l], msgs[l].c_str());
    }
    tl->timed_lane0 = true;
    for (unsigned l = 0; l < nl; ++l) {
        cudaEventRecord(tl->lanes[l].done, tl->lanes[l].st);
        cudaStreamWaitEvent(cs, tl->lanes[l].done, 0);
    }
    if (rc != EPHMC_OK) {
        cudaStreamSynchronize(cs);
        return rc;
    }
    std::vector<int> info(nsamples);
    std::vector<double> hh;
    if (hist_dev) {
        if (launch_axpy(hist, tl->hist, 1.0, (size_t)tl->nbins, cs) != EPHMC_OK) return last_status();
    } else {
        hh.resize(tl->nbins);
        EPHMC_CUDA(cudaMemcpyAsync(hh.data(), tl->hist, sizeof(double) * tl->nbins, cudaMemcpyDeviceToHost, cs));
    }
    if (z)
        EPHMC_CUDA(cudaMemcpyAsync(z, tl->z, sizeof(double) * nsamples, cudaMemcpyDefault, cs));
    EPHMC_CUDA(cudaMemcpyAsync(info.data(), tl->info, sizeof(int) * nsamples, cudaMemcpyDeviceToHost, cs));
    EPHMC_CUDA(cudaStreamSynchronize(cs));
    if (!hist_dev)
        for (int b = 0; b < tl->nbins; ++b) hist[b] += hh[b];
    for (unsigned s = 0; s < nsamples; ++s)
        if (info[s] != 0) {
            char msg[128];
            std::snprintf(msg, sizeof msg, "trans_loc: dsyevd did not converge on sample %u (info %d)", s, info[s]);
            return tl_fail(EPHMC_ERR_CUDA, msg);
        }
    return EPHMC_OK;
}

EPHMC_API int ephmc_tl_last_timings(const ephmc_tl *tl, float ms[5]) {
    clear_status();
    if (!tl || !ms) return tl_fail(EPHMC_ERR_ARG, "ephmc_tl_last_timings arguments");
    if (!tl->timed_lane0 || tl->lanes.empty()) return tl_fail(EPHMC_ERR_ARG, "ephmc_tl_last_timings: no run yet");
    const TlLane &l = tl->lanes[0];
    EPHMC_CUDA(cudaEventSynchronize(l.stage[5]));
    for (int k = 0; k < 5; ++k) EPHMC_CUDA(cudaEventElapsedTime(ms + k, l.stage[k], l.stage[k + 1]));
    return EPHMC_OK;
}

}  // extern "C"
