// FP64 re-stabilisation of the slice chain for low temperatures: log det
// M_hat and the segments' outer factors Z_k from UDT decompositions of the
// partial products, instead of from the raw product.
//
// The reference forms M_hat = 1 + B_0...B_{Nt-1} as a raw product
// (simulation/organic_dense_matrix.c:251-265) and factors it
// (logDetM_and_inv_M_hat, :547-607).  The product's singular values span
// e^{+-beta |E|}: at 48x48, Nt = 128, beta = 40 from 5e9 down to 1e-71, and
// the LU of 1 + product resolves log det only to about 1e-16 cond(M) = 4e-6
// (the same for the reference), too coarse for a finite-difference check
// with step 1e-4 or for the segment factors Z_k of the force.
//
// Here the chain is cut into segments S_k = B_{s_k}...B_{e_k - 1} (the mixed
// force's segments, bottom up k = 0..m-1) and the partial products are kept
// in graded form (the UDT stratification of determinant quantum Monte Carlo,
// Loh and Gubernatis 1992; QR with columns pre-sorted by norm instead of
// column pivoting, as in C. Bauer, SciPost Phys. Core 2, 011 (2020)):
//   Qs_k   = S_{k+1}...S_{m-1}       = U_k  diag(d_k)  T_k
//   Ps_k^T = S_{k-1}^T...S_0^T       = U'_k diag(d'_k) T'_k
// with U orthogonal, d graded and T well conditioned (|det T| = 1).  Each
// step applies one segment to U (the slice kernels, on the columns), scales
// the columns by d, sorts them by norm, and takes a Householder QR:
//   (S U) diag(d) Pi = Q R,  U <- Q, d <- |diag R|, T^-1 <- T^-1 Pi R^-1 diag(d).
// With W = U'^T S_k U, X = T'^-T T^-1 and d = d_b d_s (d_b = max(d, 1),
// d_s = min(d, 1)):
//   M = 1 + Ps_k S_k Qs_k = T'^T (X + D' W D) T,
//   N_k = D'_b^-1 X D_b^-1 + D'_s W D_s              (well conditioned)
//   Z_k = Qs_k M^-1 Ps_k = U D_s N_k^-1 D'_s U'^T.
// The segment sweeps then take Z_k as their y start, as in the unstabilised
// segmented force.  log det takes one more step, through S_0, to the whole
// product U D T: 1 + U D T = U (U^T T^-1 D_b^-1 + D_s) D_b T, so
//   log|det M| = log|det(U^T T^-1 D_b^-1 + D_s)| + sum log d_b,
// with the sign from the LU, det U (its Householder reflectors) and det T
// (the signs of the R diagonals and the column permutations).
//
// Library calls: cuSOLVER geqrf, orgqr, getrf, getrs and cuBLAS GEMM and
// trsm (plain dense factorisations); the column norms, the sort, the
// gathers, scalings, N_k and the log det parts are this file's kernels.
#include "ephmc_internal.cuh"

#include <cublas_v2.h>
#include <cusolverDn.h>

#include <algorithm>
#include <cmath>
#include <vector>

namespace ephmc {

// The Q side and the P side of the chain are independent until the segment
// factors: the P side runs on a second stream (lane 1) with its own handles
// and temporaries.
struct StabLane {
    cudaStream_t st = nullptr;
    cusolverDnHandle_t sol = nullptr;
    cublasHandle_t blas = nullptr;
    double *ws = nullptr;    // cuSOLVER workspace (lwork doubles)
    int *info = nullptr;     // device: [0] solver info, [1] sign accumulator (+-1)
    double *tau = nullptr, *norms = nullptr;  // V each
    int *perm = nullptr;     // V
};

struct StabWork {
    int V = 0, m = 0;
    StabLane lane[2];        // lane 0 on the context's stream, lane 1 on its own
    cudaEvent_t ev[2] = {nullptr, nullptr};  // fork to and join from lane 1
    double *lane_buf = nullptr;  // lanes' workspaces, infos and vectors
    int lwork = 0;
    cusolverDnHandle_t sol = nullptr;  // = lane[0].sol
    cublasHandle_t blas = nullptr;     // = lane[0].blas
    double *ws = nullptr;
    int *info = nullptr;
    double *mats = nullptr;  // (6m + 3) V^2: U, Ti, SU, Up, Tpi, yst (m each), N, W, and lane 1's W
    double *vecs = nullptr;  // 2 m V (d, d') + 3 V (tau, norms: unused, whole-product d) + 8 (log det parts)
    int *ivecs = nullptr;    // 2 V: sort permutation, LU pivots
    void *stack = nullptr;   // segment stacks when the context's q stack is too small
    size_t stack_bytes = 0;
    size_t VV() const { return (size_t)V * V; }
    double *U(int k) const { return mats + (size_t)(0 * m + k) * VV(); }
    double *Ti(int k) const { return mats + (size_t)(1 * m + k) * VV(); }
    double *SU(int k) const { return mats + (size_t)(2 * m + k) * VV(); }
    double *Up(int k) const { return mats + (size_t)(3 * m + k) * VV(); }
    double *Tpi(int k) const { return mats + (size_t)(4 * m + k) * VV(); }
    double *yst(int j) const { return mats + (size_t)(5 * m + j) * VV(); }  // top-down segment index
    double *N() const { return mats + (size_t)(6 * m) * VV(); }
    double *W() const { return mats + (size_t)(6 * m + 1) * VV(); }
    double *W1() const { return mats + (size_t)(6 * m + 2) * VV(); }
    double *d(int k) const { return vecs + (size_t)k * V; }
    double *dp(int k) const { return vecs + (size_t)(m + k) * V; }
    double *tau() const { return vecs + (size_t)2 * m * V; }
    double *norms() const { return vecs + (size_t)(2 * m + 1) * V; }
    double *dwhole() const { return vecs + (size_t)(2 * m + 2) * V; }
    double *parts() const { return vecs + (size_t)(2 * m + 3) * V; }
    int *perm() const { return ivecs; }
    int *piv() const { return ivecs + V; }
};

namespace {

// norms[c] = scale[c] * ||A[:, c]|| (column-major, one warp per column)
__global__ void k_colnorm(const double *__restrict__ A, const double *__restrict__ scale, int V,
                          double *__restrict__ norms) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (warp >= V) return;
    const double *col = A + (size_t)warp * V;
    double s = 0;
    for (int i = lane; i < V; i += 32) s = fma(col[i], col[i], s);
#pragma unroll
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) norms[warp] = sqrt(s) * scale[warp];
}

// perm = indices sorted by decreasing key (ties: smaller index first), one
// CTA, bitonic sort of the keys padded to a power of two <= 4096 in shared memory
__global__ void k_argsort_desc(const double *__restrict__ key, int V, int *__restrict__ perm) {
    __shared__ double k[4096];
    __shared__ int ix[4096];
    int n = 1;
    while (n < V) n <<= 1;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        k[i] = i < V ? key[i] : -1.0;  // norms are >= 0: padding sorts last
        ix[i] = i;
    }
    __syncthreads();
    for (int size = 2; size <= n; size <<= 1) {
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            for (int i = threadIdx.x; i < n; i += blockDim.x) {
                const int j = i ^ stride;
                if (j > i) {
                    // "before(a, b)": a sorts ahead of b in decreasing order
                    const bool desc = (i & size) == 0;
                    const bool i_first = k[i] > k[j] || (k[i] == k[j] && ix[i] < ix[j]);
                    if (i_first != desc) {
                        const double tk = k[i];
                        k[i] = k[j];
                        k[j] = tk;
                        const int ti = ix[i];
                        ix[i] = ix[j];
                        ix[j] = ti;
                    }
                }
            }
            __syncthreads();
        }
    }
    for (int i = threadIdx.x; i < V; i += blockDim.x) perm[i] = ix[i];
}

// dst[:, i] = src[:, perm[i]] * (scale ? scale[perm[i]] : 1)
__global__ void k_gather_cols(const double *__restrict__ src, const double *__restrict__ scale,
                              const int *__restrict__ perm, int V, double *__restrict__ dst) {
    const size_t f = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (f >= (size_t)V * V) return;
    const int i = (int)(f / V), r = (int)(f % V);
    const int c = perm[i];
    dst[f] = src[(size_t)c * V + r] * (scale ? scale[c] : 1.0);
}

// d[i] = |R_ii|; acc[1] *= sign(prod R_ii) * parity(perm) (one CTA)
__global__ void k_qr_diag(const double *__restrict__ R, const int *__restrict__ perm, int V, double *__restrict__ d,
                          int *__restrict__ acc) {
    __shared__ int neg;
    __shared__ unsigned char seen[4096];
    if (threadIdx.x == 0) neg = 0;
    __syncthreads();
    int mine = 0;
    for (int i = threadIdx.x; i < V; i += blockDim.x) {
        const double r = R[(size_t)i * V + i];
        d[i] = fabs(r);
        mine += r < 0;
        seen[i] = 0;
    }
    atomicAdd(&neg, mine);
    __syncthreads();
    if (acc != nullptr && threadIdx.x == 0) {
        int cycles = 0;
        for (int i = 0; i < V; ++i) {
            if (seen[i]) continue;
            ++cycles;
            for (int j = i; !seen[j]; j = perm[j]) seen[j] = 1;
        }
        const int parity = (V - cycles) & 1;
        if ((neg + parity) & 1) acc[1] = -acc[1];
    }
}

__global__ void k_scale_cols(double *__restrict__ A, const double *__restrict__ s, int V) {
    const size_t f = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (f < (size_t)V * V) A[f] *= s[f / V];
}

// N = D'_b^-1 X D_b^-1 + D'_s W D_s, X given in N (column-major)
__global__ void k_form_N(double *__restrict__ N, const double *__restrict__ W, const double *__restrict__ d,
                         const double *__restrict__ dp, int V) {
    const size_t f = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (f >= (size_t)V * V) return;
    const int j = (int)(f / V), i = (int)(f % V);
    const double db = fmax(d[j], 1.0), ds = fmin(d[j], 1.0);
    const double dpb = fmax(dp[i], 1.0), dps = fmin(dp[i], 1.0);
    N[f] = N[f] / (dpb * db) + dps * W[f] * ds;
}

// B = D'_s U'^T (column-major): B[i + cV] = min(d'_i, 1) U'[c + iV]
__global__ void k_rhs(const double *__restrict__ Up, const double *__restrict__ dp, int V, double *__restrict__ B) {
    const size_t f = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (f >= (size_t)V * V) return;
    const int c = (int)(f / V), i = (int)(f % V);
    B[f] = fmin(dp[i], 1.0) * Up[(size_t)i * V + c];
}

// Y[i + cV] *= min(d_i, 1)
__global__ void k_scale_rows_small(double *__restrict__ Y, const double *__restrict__ d, int V) {
    const size_t f = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (f < (size_t)V * V) Y[f] *= fmin(d[f % V], 1.0);
}

// log det parts of the LU of N_0 and the scales of Qs_0:
// out[0] = sum log|N_ii| + sum log max(d_i, 1), out[1] = sign(det N_0) * acc[1]
__global__ void k_logdet_parts(const double *__restrict__ N, const int *__restrict__ piv, const double *__restrict__ d,
                               const int *__restrict__ acc, int V, double *__restrict__ out) {
    __shared__ double s_ld[32];
    __shared__ int s_neg[32];
    double ld = 0;
    int neg = 0;
    for (int i = threadIdx.x; i < V; i += blockDim.x) {
        const double u = N[(size_t)i * V + i];
        ld += log(fabs(u)) + log(fmax(d[i], 1.0));
        neg += (u < 0) + (piv[i] != i + 1);
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) {
        ld += __shfl_xor_sync(0xffffffffu, ld, o);
        neg += __shfl_xor_sync(0xffffffffu, neg, o);
    }
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) {
        s_ld[w] = ld;
        s_neg[w] = neg;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0;
        int n = 0;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) {
            a += s_ld[k];
            n += s_neg[k];
        }
        out[0] = a;
        out[1] = ((n & 1) ? -1.0 : 1.0) * (double)acc[1];
    }
}

// acc[1] *= (-1)^(number of Householder reflectors with tau != 0): the sign
// of det Q of a geqrf factorisation (one CTA)
__global__ void k_tau_sign(const double *__restrict__ tau, int V, int *__restrict__ acc) {
    __shared__ int cnt;
    if (threadIdx.x == 0) cnt = 0;
    __syncthreads();
    int mine = 0;
    for (int i = threadIdx.x; i < V; i += blockDim.x) mine += tau[i] != 0.0;
    atomicAdd(&cnt, mine);
    __syncthreads();
    if (threadIdx.x == 0 && (cnt & 1)) acc[1] = -acc[1];
}

// N = X D_b^-1 + D_s with X given in N (column-major): the well-conditioned
// factor of 1 + U D T = U (U^T T^-1 D_b^-1 + D_s) D_b T
__global__ void k_form_N_whole(double *__restrict__ N, const double *__restrict__ d, int V) {
    const size_t f = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (f >= (size_t)V * V) return;
    const int j = (int)(f / V), i = (int)(f % V);
    N[f] = N[f] / fmax(d[j], 1.0) + (i == j ? fmin(d[j], 1.0) : 0.0);
}

__global__ void k_eye(double *__restrict__ A, int V) {
    const size_t f = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (f < (size_t)V * V) A[f] = (f / V == f % V) ? 1.0 : 0.0;
}

__global__ void k_ones(double *__restrict__ a, int n, int *__restrict__ acc) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) a[i] = 1.0;
    if (acc != nullptr && i == 0) acc[1] = 1;
}

unsigned blocks(size_t n, unsigned t = 256) { return (unsigned)((n + t - 1) / t); }

int fail(int st, const char *msg) {
    set_status(st, msg);
    return st;
}

#define STAB_BLAS(call)                                                                \
    do {                                                                               \
        if ((call) != CUBLAS_STATUS_SUCCESS) return fail(EPHMC_ERR_CUDA, "stabilised chain: " #call); \
    } while (0)
#define STAB_SOLVER(call)                                                              \
    do {                                                                               \
        if ((call) != CUSOLVER_STATUS_SUCCESS) return fail(EPHMC_ERR_CUDA, "stabilised chain: " #call); \
    } while (0)

// One UDT step: (S U) diag(d_in) = U_out diag(d_out) R Pi^T; Ti_out = Ti_in Pi R^-1 diag(d_out).
// SU: the segment applied to U_in (column-major); acc: det T sign accumulator
// or null; q_sign: also multiply the accumulator by sign(det U_out).
int qr_step(StabWork &w, StabLane &ln, const double *SU, const double *d_in, const double *Ti_in, double *U_out,
            double *d_out, double *Ti_out, int *acc, bool q_sign = false) {
    const int V = w.V;
    const size_t VV = w.VV();
    cudaStream_t st = ln.st;
    k_colnorm<<<blocks((size_t)V * 32), 256, 0, st>>>(SU, d_in, V, ln.norms);
    k_argsort_desc<<<1, 1024, 0, st>>>(ln.norms, V, ln.perm);
    k_gather_cols<<<blocks(VV), 256, 0, st>>>(SU, d_in, ln.perm, V, U_out);
    k_gather_cols<<<blocks(VV), 256, 0, st>>>(Ti_in, nullptr, ln.perm, V, Ti_out);
    count_launch(4);
    STAB_SOLVER(cusolverDnDgeqrf(ln.sol, V, V, U_out, V, ln.tau, ln.ws, w.lwork, ln.info));
    k_qr_diag<<<1, 1024, 0, st>>>(U_out, ln.perm, V, d_out, acc);
    count_launch(1);
    const double one = 1.0;
    STAB_BLAS(cublasDtrsm(ln.blas, CUBLAS_SIDE_RIGHT, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_N, CUBLAS_DIAG_NON_UNIT, V, V,
                          &one, U_out, V, Ti_out, V));
    k_scale_cols<<<blocks(VV), 256, 0, st>>>(Ti_out, d_out, V);
    count_launch(1);
    STAB_SOLVER(cusolverDnDorgqr(ln.sol, V, V, V, U_out, V, ln.tau, ln.ws, w.lwork, ln.info));
    if (acc != nullptr && q_sign) {
        k_tau_sign<<<1, 1024, 0, st>>>(ln.tau, V, acc);  // det U_out: its Householder reflectors
        count_launch(1);
    }
    count_launch(3);
    EPHMC_CUDA(cudaGetLastError());
    return EPHMC_OK;
}

}  // namespace

void stab_free(StabWork *w) {
    if (!w) return;
    for (StabLane &ln : w->lane) {
        if (ln.sol) cusolverDnDestroy(ln.sol);
        if (ln.blas) cublasDestroy(ln.blas);
    }
    if (w->lane[1].st) cudaStreamDestroy(w->lane[1].st);
    for (cudaEvent_t e : w->ev)
        if (e) cudaEventDestroy(e);
    cudaFree(w->lane_buf);
    cudaFree(w->mats);
    cudaFree(w->vecs);
    cudaFree(w->ivecs);
    cudaFree(w->stack);
    delete w;
}

size_t stab_bytes(const StabWork *w) {
    if (!w || !w->mats) return 0;
    return sizeof(double) * ((6 * (size_t)w->m + 3) * w->VV() + (2 * (size_t)w->m + 3) * w->V + 8) +
           2 * (sizeof(double) * ((size_t)w->lwork + 2 * w->V + 1) + sizeof(int) * (size_t)w->V) +
           sizeof(int) * 2 * (size_t)w->V + w->stack_bytes;
}

// Buffers for m segments of a V-site lattice (reallocated when m changes).
static int stab_ensure(StabWork **slot, int V, int m, cudaStream_t st) {
    if (V > 4096) return fail(EPHMC_ERR_UNSUPPORTED, "stabilised chain: V > 4096 (the column sort is one CTA)");
    StabWork *w = *slot;
    if (!w) {
        w = new StabWork();
        *slot = w;
        for (StabLane &ln : w->lane)
            if (cusolverDnCreate(&ln.sol) != CUSOLVER_STATUS_SUCCESS || cublasCreate(&ln.blas) != CUBLAS_STATUS_SUCCESS)
                return fail(EPHMC_ERR_CUDA, "stabilised chain: cuSOLVER / cuBLAS handle");
        if (cudaStreamCreateWithFlags(&w->lane[1].st, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&w->ev[0], cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&w->ev[1], cudaEventDisableTiming) != cudaSuccess) {
            cudaGetLastError();
            return fail(EPHMC_ERR_CUDA, "stabilised chain: second stream");
        }
        w->sol = w->lane[0].sol;
        w->blas = w->lane[0].blas;
    }
    if (w->V != V || w->m != m) {
        cudaFree(w->lane_buf);
        cudaFree(w->mats);
        cudaFree(w->vecs);
        cudaFree(w->ivecs);
        w->lane_buf = w->mats = w->vecs = w->ws = nullptr;
        w->info = w->ivecs = nullptr;
        w->V = V;
        w->m = m;
        int l1 = 0, l2 = 0, l3 = 0;
        double *probe = nullptr;
        if (cusolverDnDgeqrf_bufferSize(w->sol, V, V, probe, V, &l1) != CUSOLVER_STATUS_SUCCESS ||
            cusolverDnDorgqr_bufferSize(w->sol, V, V, V, probe, V, probe, &l2) != CUSOLVER_STATUS_SUCCESS ||
            cusolverDnDgetrf_bufferSize(w->sol, V, V, probe, V, &l3) != CUSOLVER_STATUS_SUCCESS)
            return fail(EPHMC_ERR_CUDA, "stabilised chain: workspace query");
        w->lwork = std::max({l1, l2, l3, 1});
        const size_t VV = (size_t)V * V;
        // per lane: workspace, 2 info words (as one double), tau, norms, perm
        const size_t per_lane = (size_t)w->lwork + 1 + 2 * (size_t)V + ((size_t)V + 1) / 2;
        if (cudaMalloc((void **)&w->lane_buf, sizeof(double) * 2 * per_lane) != cudaSuccess ||
            cudaMalloc((void **)&w->mats, sizeof(double) * (6 * (size_t)m + 3) * VV) != cudaSuccess ||
            cudaMalloc((void **)&w->vecs, sizeof(double) * ((2 * (size_t)m + 3) * V + 8)) != cudaSuccess ||
            cudaMalloc((void **)&w->ivecs, sizeof(int) * 2 * (size_t)V) != cudaSuccess) {
            cudaGetLastError();
            w->V = w->m = 0;
            return fail(EPHMC_ERR_NOMEM, "stabilised chain buffers");
        }
        for (int l = 0; l < 2; ++l) {
            double *base = w->lane_buf + (size_t)l * per_lane;
            StabLane &ln = w->lane[l];
            ln.ws = base;
            ln.info = reinterpret_cast<int *>(base + w->lwork);
            ln.tau = base + w->lwork + 1;
            ln.norms = ln.tau + V;
            ln.perm = reinterpret_cast<int *>(ln.norms + V);
        }
        w->ws = w->lane[0].ws;
        w->info = w->lane[0].info;
    }
    w->lane[0].st = st;
    for (StabLane &ln : w->lane)
        if (cusolverDnSetStream(ln.sol, ln.st) != CUSOLVER_STATUS_SUCCESS ||
            cublasSetStream(ln.blas, ln.st) != CUBLAS_STATUS_SUCCESS)
            return fail(EPHMC_ERR_CUDA, "stabilised chain: set stream");
    return EPHMC_OK;
}

// The stabilised chain of one field x (device): segments from b (top down,
// b[0] = Nt > ... > b[m] = 0).  With want_z, Z_k^T of every segment into the
// top-down y starts w.yst(j), j = m-1-k.  log|det M_hat| and its sign into
// the device words w.parts()[0..1].  jobs_dev: 2m free slots of the
// context's job table, uploaded by ctx_upload_jobs.
int stab_chain(ephmc_ctx *c, StabWork **slot, const double *x, const std::vector<int> &b, bool want_z,
               SliceJob *jobs_dev, int slot0) {
    const int V = (int)c->V, m = (int)b.size() - 1;
    int rc;
    if ((rc = stab_ensure(slot, V, m, c->stream))) return rc;
    StabWork &w = **slot;
    const size_t VV = w.VV();
    cudaStream_t st = c->stream;
    auto seg_s = [&](int k) { return b[m - k]; };
    auto seg_e = [&](int k) { return b[m - 1 - k]; };
    // slice jobs: Q side S_k U_k (k = m-1..0), P side S_k^T U'_k (k = 0..m-2)
    std::vector<SliceJob> jobs;
    for (int k = m - 1; k >= 0; --k) {
        SliceJob j{};
        j.src = k == m - 1 ? nullptr : w.U(k);
        j.dst = w.SU(k);
        j.s_first = seg_e(k) - 1;
        j.s_count = seg_e(k) - seg_s(k);
        j.s_dir = -1;
        j.p_begin = 0;
        j.p_end = kPairs;
        j.p_step = 1;
        jobs.push_back(j);
    }
    if (want_z)
        for (int k = 0; k + 1 < m; ++k) {
            SliceJob j{};
            j.src = k == 0 ? nullptr : w.Up(k);
            j.dst = w.W1();
            j.s_first = seg_s(k);
            j.s_count = seg_e(k) - seg_s(k);
            j.s_dir = +1;
            j.p_begin = 1;
            j.p_end = -1;
            j.p_step = -1;
            jobs.push_back(j);
        }
    if ((rc = ctx_upload_jobs(c, jobs.data(), (int)jobs.size(), slot0, st))) return rc;
    auto apply = [&](int ji, cudaStream_t s2) {
        if (slices_strip_supported(c->lat)) return launch_slices_strip<double>(x, c->c, c->lat, jobs_dev + ji, 1, s2);
        return launch_slices<double, double, double>(Axis::Rows, x, c->c, c->lat, jobs_dev + ji, 1, s2);
    };
    StabLane &q = w.lane[0], &pl = w.lane[1];
    const double one = 1.0, zero = 0.0;
    // P side, bottom up, on lane 1 (forked after the job upload): U'_0 = 1,
    // d' = 1, T'^-1 = 1; each step applies S_k^T to U'_k in lane 1's W
    if (want_z) {
        EPHMC_CUDA(cudaEventRecord(w.ev[0], st));
        EPHMC_CUDA(cudaStreamWaitEvent(pl.st, w.ev[0], 0));
        k_eye<<<blocks(VV), 256, 0, pl.st>>>(w.Up(0), V);
        k_eye<<<blocks(VV), 256, 0, pl.st>>>(w.Tpi(0), V);
        k_ones<<<blocks(V), 256, 0, pl.st>>>(w.dp(0), V, nullptr);
        count_launch(3);
        for (int k = 0; k + 1 < m; ++k) {
            if ((rc = apply(m + k, pl.st))) return rc;
            if ((rc = qr_step(w, pl, w.W1(), w.dp(k), w.Tpi(k), w.Up(k + 1), w.dp(k + 1), w.Tpi(k + 1), nullptr)))
                return rc;
        }
        EPHMC_CUDA(cudaEventRecord(w.ev[1], pl.st));
    }
    // Q side, top down, on the context's stream: U_{m-1} = 1, d = 1, T^-1 = 1
    k_eye<<<blocks(VV), 256, 0, st>>>(w.U(m - 1), V);
    k_eye<<<blocks(VV), 256, 0, st>>>(w.Ti(m - 1), V);
    k_ones<<<blocks(V), 256, 0, st>>>(w.d(m - 1), V, q.info);
    count_launch(3);
    for (int k = m - 1; k >= 0; --k) {
        if ((rc = apply(m - 1 - k, st))) return rc;
        if (k >= 1 && (rc = qr_step(w, q, w.SU(k), w.d(k), w.Ti(k), w.U(k - 1), w.d(k - 1), w.Ti(k - 1), q.info)))
            return rc;
    }
    // log det: one more step absorbs S_0, the whole product = U diag(d) T
    // (U in W, T^-1 in yst(m-1), d in its own slot), and 1 + U D T =
    // U N D_b T with N = U^T T^-1 D_b^-1 + D_s, so
    // log|det M| = log|det N| + sum log d_b, sign = sign det(U N T)
    {
        double *Uw = w.W(), *Tw = w.yst(m - 1), *dw = w.dwhole();
        if ((rc = qr_step(w, q, w.SU(0), w.d(0), w.Ti(0), Uw, dw, Tw, q.info, true))) return rc;
        STAB_BLAS(cublasDgemm(q.blas, CUBLAS_OP_T, CUBLAS_OP_N, V, V, V, &one, Uw, V, Tw, V, &zero, w.N(), V));
        k_form_N_whole<<<blocks(VV), 256, 0, st>>>(w.N(), dw, V);
        count_launch(2);
        STAB_SOLVER(cusolverDnDgetrf(q.sol, V, V, w.N(), V, q.ws, w.piv(), q.info));
        k_logdet_parts<<<1, 1024, 0, st>>>(w.N(), w.piv(), dw, q.info, V, w.parts());
        count_launch(1);
    }
    if (!want_z) {
        EPHMC_CUDA(cudaGetLastError());
        return EPHMC_OK;
    }
    EPHMC_CUDA(cudaStreamWaitEvent(st, w.ev[1], 0));  // join the P side
    // Z_0 = U_0 D_s N_0^-1 with N_0 = T_0^-1 D_b^-1 + S_0 U_0 D_s (U', d', T' = 1):
    // y start of the bottom segment
    EPHMC_CUDA(cudaMemcpyAsync(w.N(), w.Ti(0), sizeof(double) * VV, cudaMemcpyDeviceToDevice, st));
    k_form_N<<<blocks(VV), 256, 0, st>>>(w.N(), w.SU(0), w.d(0), w.dp(0), V);
    count_launch(1);
    STAB_SOLVER(cusolverDnDgetrf(q.sol, V, V, w.N(), V, q.ws, w.piv(), q.info));
    k_eye<<<blocks(VV), 256, 0, st>>>(w.W(), V);
    count_launch(1);
    STAB_SOLVER(cusolverDnDgetrs(q.sol, CUBLAS_OP_N, V, V, w.N(), V, w.piv(), w.W(), V, q.info));
    k_scale_rows_small<<<blocks(VV), 256, 0, st>>>(w.W(), w.d(0), V);
    count_launch(2);
    STAB_BLAS(cublasDgemm(q.blas, CUBLAS_OP_T, CUBLAS_OP_T, V, V, V, &one, w.W(), V, w.U(0), V, &zero, w.yst(m - 1),
                          V));
    count_launch(1);
    // Z_k, k = 1..m-1
    for (int k = 1; k < m; ++k) {
        STAB_BLAS(cublasDgemm(q.blas, CUBLAS_OP_T, CUBLAS_OP_N, V, V, V, &one, w.Tpi(k), V, w.Ti(k), V, &zero, w.N(),
                              V));
        STAB_BLAS(cublasDgemm(q.blas, CUBLAS_OP_T, CUBLAS_OP_N, V, V, V, &one, w.Up(k), V, w.SU(k), V, &zero, w.W(),
                              V));
        k_form_N<<<blocks(VV), 256, 0, st>>>(w.N(), w.W(), w.d(k), w.dp(k), V);
        STAB_SOLVER(cusolverDnDgetrf(q.sol, V, V, w.N(), V, q.ws, w.piv(), q.info));
        k_rhs<<<blocks(VV), 256, 0, st>>>(w.Up(k), w.dp(k), V, w.W());
        STAB_SOLVER(cusolverDnDgetrs(q.sol, CUBLAS_OP_N, V, V, w.N(), V, w.piv(), w.W(), V, q.info));
        k_scale_rows_small<<<blocks(VV), 256, 0, st>>>(w.W(), w.d(k), V);
        STAB_BLAS(cublasDgemm(q.blas, CUBLAS_OP_T, CUBLAS_OP_T, V, V, V, &one, w.W(), V, w.U(k), V, &zero,
                              w.yst(m - 1 - k), V));
        count_launch(8);
    }
    EPHMC_CUDA(cudaGetLastError());
    return EPHMC_OK;
}

double *stab_ystart(StabWork *w) { return w ? w->yst(0) : nullptr; }
double *stab_parts(StabWork *w) { return w ? w->parts() : nullptr; }
void *stab_stack(StabWork *w, size_t bytes) {
    if (!w) return nullptr;
    if (w->stack_bytes < bytes) {
        cudaFree(w->stack);
        w->stack = nullptr;
        w->stack_bytes = 0;
        if (cudaMalloc(&w->stack, bytes) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        w->stack_bytes = bytes;
    }
    return w->stack;
}

}  // namespace ephmc
