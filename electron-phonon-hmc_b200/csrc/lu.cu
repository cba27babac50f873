// FP64 LU with partial pivoting, log|det| and inverse of the fermion matrix.
//
// Replaces LAPACKE_dgetrf + LAPACKE_dgetri in logDetM_and_inv_M_hat
// (simulation/organic_dense_matrix.c:580-595).  The matrix is treated
// column-major exactly as LAPACK does: A(r,c) = M[c*V + r], so a column is a
// contiguous row of the reference's array.  Pivoting picks the first row of
// largest magnitude (LAPACK idamax); log|det| = sum log|U_ii| and the sign
// from the diagonal signs and the pivot parity (:582-589).
//
// Right-looking blocked factorisation, panel width nb:
//   k_lu_panel  one 1024-thread CTA factors the nb-column panel held in shared
//               memory (argmax by warp shuffles + one shared-memory round);
//   k_lu_trail  every CTA owns CB trailing columns in shared memory, applies
//               the panel's row interchanges, the unit-lower triangular solve
//               for its U12 block and the rank-nb update of its rows below;
//               left-of-panel columns only take the interchanges.
// Inverse: A^-1 = U^-1 L^-1 P; k_lu_inverse gives each CTA NR columns of the
// identity (permuted by P), solves L then U in 32-row blocks, writes the
// columns of A^-1 (column-major, i.e. rows of the reference's array).
#include "ephmc_internal.cuh"

#include <cmath>
#include <vector>

namespace ephmc {

namespace {

constexpr int kPanelThreads = 1024;

__device__ __forceinline__ void better(double &bv, int &bi, double v, int i) {
    // larger magnitude wins; on a tie the smaller row index (first maximum)
    if (v > bv || (v == bv && i < bi)) { bv = v; bi = i; }
}

__global__ void __launch_bounds__(kPanelThreads) k_lu_panel(double *__restrict__ M, int V, int j0, int nbc,
                                                           int *__restrict__ ipiv, double *__restrict__ diag,
                                                           int *__restrict__ info) {
    extern __shared__ double P[];  // [nbc][H], H = V - j0 rows j0..V-1
    __shared__ double red_v[32];
    __shared__ int red_i[32];
    __shared__ int piv_s;
    const int H = V - j0;
    const int tid = threadIdx.x, T = blockDim.x;
    for (int f = tid; f < nbc * H; f += T) {
        const int cc = f / H, r = f % H;
        P[f] = M[(size_t)(j0 + cc) * V + j0 + r];
    }
    __syncthreads();
    for (int jj = 0; jj < nbc; ++jj) {
        double *col = P + (size_t)jj * H;
        // argmax |col[r]| for r >= jj
        double bv = -1.0;
        int bi = 0x7fffffff;
        for (int r = jj + tid; r < H; r += T) better(bv, bi, fabs(col[r]), r);
        for (int o = 16; o > 0; o >>= 1) {
            const double ov = __shfl_down_sync(0xffffffffu, bv, o);
            const int oi = __shfl_down_sync(0xffffffffu, bi, o);
            better(bv, bi, ov, oi);
        }
        if ((tid & 31) == 0) { red_v[tid >> 5] = bv; red_i[tid >> 5] = bi; }
        __syncthreads();
        if (tid < 32) {
            bv = (tid < (T >> 5)) ? red_v[tid] : -1.0;
            bi = (tid < (T >> 5)) ? red_i[tid] : 0x7fffffff;
            for (int o = 16; o > 0; o >>= 1) {
                const double ov = __shfl_down_sync(0xffffffffu, bv, o);
                const int oi = __shfl_down_sync(0xffffffffu, bi, o);
                better(bv, bi, ov, oi);
            }
            if (tid == 0) {
                int p = bi;
                if (!(bv > 0.0)) {  // exact zero column (or NaN): no interchange, record singularity
                    p = jj;
                    if (*info == 0) *info = j0 + jj + 1;
                }
                piv_s = p;
                ipiv[j0 + jj] = j0 + p;
            }
        }
        __syncthreads();
        const int p = piv_s;
        if (p != jj) {
            for (int cc = tid; cc < nbc; cc += T) {
                double *cl = P + (size_t)cc * H;
                const double a = cl[jj];
                cl[jj] = cl[p];
                cl[p] = a;
            }
        }
        __syncthreads();
        const double d = col[jj];
        if (tid == 0) diag[j0 + jj] = d;
        if (d != 0.0)
            for (int r = jj + 1 + tid; r < H; r += T) col[r] = col[r] / d;
        __syncthreads();
        // rank-1 update of the panel columns right of jj
        const int w = nbc - jj - 1;
        if (w > 0) {
            const int rows = H - jj - 1;
            for (int f = tid; f < w * rows; f += T) {
                const int cc = jj + 1 + f / rows, r = jj + 1 + f % rows;
                double *cl = P + (size_t)cc * H;
                cl[r] = fma(-col[r], cl[jj], cl[r]);
            }
        }
        __syncthreads();
    }
    for (int f = tid; f < nbc * H; f += T) {
        const int cc = f / H, r = f % H;
        M[(size_t)(j0 + cc) * V + j0 + r] = P[f];
    }
}

// Columns left of the panel: row interchanges only (LAPACK applies them to the L part too).
__global__ void k_lu_swap_left(double *__restrict__ M, int V, int j0, int nbc, const int *__restrict__ ipiv) {
    const int cidx = blockIdx.x * blockDim.x + threadIdx.x;
    if (cidx >= j0) return;
    double *colp = M + (size_t)cidx * V;
    for (int jj = 0; jj < nbc; ++jj) {
        const int j = j0 + jj, p = ipiv[j];
        if (p != j) {
            const double a = colp[j];
            colp[j] = colp[p];
            colp[p] = a;
        }
    }
}

// Trailing columns: interchanges, U12 = L11^-1 A12, A22 -= L21 U12.
template <int CB>
__global__ void k_lu_trail(double *__restrict__ M, int V, int j0, int nbc, const int *__restrict__ ipiv) {
    extern __shared__ double C[];  // [CB][H]
    const int H = V - j0;
    const int c0 = j0 + nbc + blockIdx.x * CB;
    const int ncol = min(CB, V - c0);
    const int tid = threadIdx.x, T = blockDim.x;
    for (int f = tid; f < ncol * H; f += T) {
        const int q = f / H, r = f % H;
        C[f] = M[(size_t)(c0 + q) * V + j0 + r];
    }
    __syncthreads();
    if (tid < ncol) {
        double *cl = C + (size_t)tid * H;
        for (int jj = 0; jj < nbc; ++jj) {
            const int p = ipiv[j0 + jj] - j0;
            if (p != jj) {
                const double a = cl[jj];
                cl[jj] = cl[p];
                cl[p] = a;
            }
        }
        // unit lower triangular solve with L11 = A(j0+jj, j0+ii), ii < jj
        for (int jj = 1; jj < nbc; ++jj) {
            double acc = cl[jj];
            for (int ii = 0; ii < jj; ++ii) acc = fma(-M[(size_t)(j0 + ii) * V + j0 + jj], cl[ii], acc);
            cl[jj] = acc;
        }
    }
    __syncthreads();
    // rank-nb update of rows j0+nbc .. V-1
    for (int r = nbc + tid; r < H; r += T) {
        double acc[CB];
#pragma unroll
        for (int q = 0; q < CB; ++q) acc[q] = (q < ncol) ? C[(size_t)q * H + r] : 0.0;
        for (int jj = 0; jj < nbc; ++jj) {
            const double l = M[(size_t)(j0 + jj) * V + j0 + r];
#pragma unroll
            for (int q = 0; q < CB; ++q) acc[q] = fma(-l, C[(size_t)q * H + jj], acc[q]);
        }
#pragma unroll
        for (int q = 0; q < CB; ++q)
            if (q < ncol) C[(size_t)q * H + r] = acc[q];
    }
    __syncthreads();
    for (int f = tid; f < ncol * H; f += T) {
        const int q = f / H, r = f % H;
        M[(size_t)(c0 + q) * V + j0 + r] = C[f];
    }
}

// NR columns of A^-1 per CTA.  b = P e_c, solve L y = b (unit lower), U x = y.
template <int NR>
__global__ void k_lu_inverse(const double *__restrict__ LU, int V, const int *__restrict__ ipiv,
                             double *__restrict__ X) {
    extern __shared__ double b[];  // [V][NR]
    __shared__ double blk[32][33];
    __shared__ int pos_s[NR];
    const int tid = threadIdx.x, T = blockDim.x;
    const int c0 = blockIdx.x * NR;
    const int nr = min(NR, V - c0);
    // where the single 1 of P e_c ends up after the interchanges 0..V-1
    if (tid < nr) {
        int pos = c0 + tid;
        for (int j = 0; j < V; ++j) {
            const int p = ipiv[j];
            if (pos == j) pos = p;
            else if (pos == p) pos = j;
        }
        pos_s[tid] = pos;
    }
    __syncthreads();
    for (int f = tid; f < V * NR; f += T) {
        const int r = f / NR, q = f % NR;
        b[f] = (q < nr && r == pos_s[q]) ? 1.0 : 0.0;
    }
    __syncthreads();
    const int warp = tid >> 5, lane = tid & 31, nwarps = T >> 5;
    // ---- forward: L y = b
    for (int kb = 0; kb < V; kb += 32) {
        const int bs = min(32, V - kb);
        for (int f = tid; f < 32 * 32; f += T) {
            const int rr = f % 32, kk = f / 32;  // L(kb+rr, kb+kk)
            blk[rr][kk] = (rr < bs && kk < bs) ? LU[(size_t)(kb + kk) * V + kb + rr] : 0.0;
        }
        __syncthreads();
        for (int q = warp; q < nr; q += nwarps) {
            double val = (lane < bs) ? b[(size_t)(kb + lane) * NR + q] : 0.0;
            for (int kk = 0; kk < bs; ++kk) {
                const double yk = __shfl_sync(0xffffffffu, val, kk);
                if (lane > kk) val = fma(-blk[lane][kk], yk, val);
            }
            if (lane < bs) b[(size_t)(kb + lane) * NR + q] = val;
        }
        __syncthreads();
        for (int r = kb + bs + tid; r < V; r += T) {
            double acc[NR];
#pragma unroll
            for (int q = 0; q < NR; ++q) acc[q] = b[(size_t)r * NR + q];
            for (int kk = 0; kk < bs; ++kk) {
                const double l = LU[(size_t)(kb + kk) * V + r];
#pragma unroll
                for (int q = 0; q < NR; ++q) acc[q] = fma(-l, b[(size_t)(kb + kk) * NR + q], acc[q]);
            }
#pragma unroll
            for (int q = 0; q < NR; ++q) b[(size_t)r * NR + q] = acc[q];
        }
        __syncthreads();
    }
    // ---- backward: U x = y
    for (int kend = V; kend > 0; kend -= 32) {
        const int kb = max(0, kend - 32), bs = kend - kb;
        for (int f = tid; f < 32 * 32; f += T) {
            const int rr = f % 32, kk = f / 32;  // U(kb+rr, kb+kk)
            blk[rr][kk] = (rr < bs && kk < bs) ? LU[(size_t)(kb + kk) * V + kb + rr] : 0.0;
        }
        __syncthreads();
        for (int q = warp; q < nr; q += nwarps) {
            double val = (lane < bs) ? b[(size_t)(kb + lane) * NR + q] : 0.0;
            for (int kk = bs - 1; kk >= 0; --kk) {
                double xk = 0.0;
                if (lane == kk) val = val / blk[kk][kk];
                xk = __shfl_sync(0xffffffffu, val, kk);
                if (lane < kk) val = fma(-blk[lane][kk], xk, val);
            }
            if (lane < bs) b[(size_t)(kb + lane) * NR + q] = val;
        }
        __syncthreads();
        for (int r = tid; r < kb; r += T) {
            double acc[NR];
#pragma unroll
            for (int q = 0; q < NR; ++q) acc[q] = b[(size_t)r * NR + q];
            for (int kk = 0; kk < bs; ++kk) {
                const double u = LU[(size_t)(kb + kk) * V + r];
#pragma unroll
                for (int q = 0; q < NR; ++q) acc[q] = fma(-u, b[(size_t)(kb + kk) * NR + q], acc[q]);
            }
#pragma unroll
            for (int q = 0; q < NR; ++q) b[(size_t)r * NR + q] = acc[q];
        }
        __syncthreads();
    }
    for (int f = tid; f < nr * V; f += T) {
        const int q = f / V, r = f % V;
        X[(size_t)(c0 + q) * V + r] = b[(size_t)r * NR + q];
    }
}

// log|det| and sign from the diagonal of U and the pivots (parallel sum).
__global__ void k_lu_logdet(const double *__restrict__ diag, const int *__restrict__ ipiv, int V,
                            double *__restrict__ out) {
    __shared__ double s_l[32];
    __shared__ int s_n[32];
    double l = 0.0;
    int neg = 0;
    for (int i = threadIdx.x; i < V; i += blockDim.x) {
        const double d = diag[i];
        l += log(fabs(d));
        if (!(d > 0)) neg ^= 1;
        if (ipiv[i] != i) neg ^= 1;
    }
    for (int o = 16; o > 0; o >>= 1) {
        l += __shfl_down_sync(0xffffffffu, l, o);
        neg ^= __shfl_down_sync(0xffffffffu, neg, o);
    }
    if ((threadIdx.x & 31) == 0) { s_l[threadIdx.x >> 5] = l; s_n[threadIdx.x >> 5] = neg; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        int n = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) { t += s_l[w]; n ^= s_n[w]; }
        out[0] = t;
        out[1] = n ? -1.0 : 1.0;
    }
}

int panel_width(int V) {
    const size_t budget = 200 * 1024 / sizeof(double);
    int nb = 16;
    while (nb > 1 && (size_t)nb * V > budget) nb >>= 1;
    return nb;
}

}  // namespace

int lu_alloc(LUWork &w, int V) {
    w.V = V;
    EPHMC_CUDA(cudaMalloc(&w.ipiv, sizeof(int) * V));
    EPHMC_CUDA(cudaMalloc(&w.diag, sizeof(double) * (V + 2)));
    EPHMC_CUDA(cudaMalloc(&w.info, sizeof(int) * 2));
    EPHMC_CUDA(cudaMalloc(&w.X, sizeof(double) * (size_t)V * V));
    return EPHMC_OK;
}

void lu_free(LUWork &w) {
    if (w.ipiv) cudaFree(w.ipiv);
    if (w.diag) cudaFree(w.diag);
    if (w.info) cudaFree(w.info);
    if (w.X) cudaFree(w.X);
    w = LUWork{};
}

int lu_factor(double *M, LUWork &w, cudaStream_t st) {
    const int V = w.V;
    const int nb = panel_width(V);
    EPHMC_CUDA(cudaMemsetAsync(w.info, 0, sizeof(int) * 2, st));
    const size_t psmem_max = (size_t)nb * V * sizeof(double);
    EPHMC_CUDA(cudaFuncSetAttribute(k_lu_panel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)psmem_max));
    constexpr int CB = 8;
    const size_t tsmem_max = (size_t)CB * V * sizeof(double);
    EPHMC_CUDA(cudaFuncSetAttribute(k_lu_trail<CB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tsmem_max));
    for (int j0 = 0; j0 < V; j0 += nb) {
        const int nbc = std::min(nb, V - j0);
        const int H = V - j0;
        k_lu_panel<<<1, kPanelThreads, (size_t)nbc * H * sizeof(double), st>>>(M, V, j0, nbc, w.ipiv, w.diag, w.info); ephmc::count_launch(1);
        EPHMC_CUDA(cudaGetLastError());
        if (j0 > 0) {
            k_lu_swap_left<<<(j0 + 127) / 128, 128, 0, st>>>(M, V, j0, nbc, w.ipiv); ephmc::count_launch(1);
            EPHMC_CUDA(cudaGetLastError());
        }
        const int ntrail = V - j0 - nbc;
        if (ntrail > 0) {
            k_lu_trail<CB><<<(ntrail + CB - 1) / CB, 256, (size_t)CB * H * sizeof(double), st>>>(M, V, j0, nbc, w.ipiv); ephmc::count_launch(1);
            EPHMC_CUDA(cudaGetLastError());
        }
    }
    return EPHMC_OK;
}

int lu_logdet_inverse(double *M, LUWork &w, double *logdet, int *sign, int *ipiv_host, cudaStream_t st) {
    const int V = w.V;
    int rc = lu_factor(M, w, st);
    if (rc != EPHMC_OK) return rc;
    k_lu_logdet<<<1, 1024, 0, st>>>(w.diag, w.ipiv, V, w.diag + V); ephmc::count_launch(1);
    EPHMC_CUDA(cudaGetLastError());
    int info = 0;
    double ld[2] = {0, 1};
    EPHMC_CUDA(cudaMemcpyAsync(&info, w.info, sizeof(int), cudaMemcpyDeviceToHost, st));
    EPHMC_CUDA(cudaMemcpyAsync(ld, w.diag + V, sizeof(double) * 2, cudaMemcpyDeviceToHost, st));
    if (ipiv_host) EPHMC_CUDA(cudaMemcpyAsync(ipiv_host, w.ipiv, sizeof(int) * V, cudaMemcpyDeviceToHost, st));
    EPHMC_CUDA(cudaStreamSynchronize(st));
    if (ipiv_host)
        for (int i = 0; i < V; ++i) ipiv_host[i] += 1;  // LAPACK 1-based
    if (logdet) *logdet = ld[0];
    if (sign) *sign = ld[1] < 0 ? -1 : 1;
    if (info != 0) return EPHMC_ERR_SINGULAR;
    const size_t need = (size_t)V * V;
    constexpr int NR = 8;
    const size_t ismem = (size_t)V * NR * sizeof(double);
    EPHMC_CUDA(cudaFuncSetAttribute(k_lu_inverse<NR>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ismem));
    k_lu_inverse<NR><<<(V + NR - 1) / NR, 256, ismem, st>>>(M, V, w.ipiv, w.X); ephmc::count_launch(1);
    EPHMC_CUDA(cudaGetLastError());
    EPHMC_CUDA(cudaMemcpyAsync(M, w.X, need * sizeof(double), cudaMemcpyDeviceToDevice, st));
    return EPHMC_OK;
}

}  // namespace ephmc
