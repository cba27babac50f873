// FP64 log|det| and in-place inverse of the fermion matrix by blocked
// Gauss-Jordan elimination with partial pivoting.
//
// Replaces LAPACKE_dgetrf + LAPACKE_dgetri in logDetM_and_inv_M_hat
// (simulation/organic_dense_matrix.c:580-595).  The matrix is seen
// column-major as LAPACK sees it: A(r,c) = M[c*V + r], so column c is the
// contiguous row c of the reference's array.  Pivot rows are chosen among the
// rows not yet used as pivots exactly as dgetrf chooses them (largest
// magnitude, first on ties), so the pivot sequence and U's diagonal are those
// of the LU factorisation: log|det| = sum log|U_ii|, the sign from the
// diagonal signs and the pivot parity (:582-589), pivots reported 1-based.
//
// Per panel of nb columns p (rows P = p, others O):
//   k_gj_panel   one 1024-thread CTA, every thread owns one row of the panel
//                in registers: LU with partial pivoting of rows >= j0 (argmax by
//                __reduce_max_sync on the bit pattern of |a|), then
//                D^-1 = U11^-1 L11^-1 and the new panel columns
//                (rows P: D^-1; rows below: -L21 L11^-1; rows above: -C D^-1);
//   k_gj_update  every CTA owns CB other columns in shared memory: applies the
//                panel's interchanges, sets rows P to D^-1 A(P, col) and
//                updates the other rows A(O, col) -= K A(P, col) with
//                K = A(O, p) D^-1 = -(new panel columns).
// After the last panel the interchanges are undone as column permutations.
// 2V^3 flops in V/nb rank-nb updates over the full matrix (GEMM-shaped, L2
// resident at V = 1024), with no separate triangular-solve phase.
#include "ephmc_internal.cuh"

#include <algorithm>
#include <cmath>

namespace ephmc {

namespace {

constexpr int kPanelThreads = 1024;

// |a| as an ordered 64-bit key (non-negative doubles order like their bits)
__device__ __forceinline__ unsigned long long abs_key(double a) {
    return (unsigned long long)__double_as_longlong(fabs(a));
}

// argmax over the warp of (key, row): larger key wins, smaller row on ties
__device__ __forceinline__ void warp_argmax(unsigned long long &key, int &row) {
    const unsigned hi = (unsigned)(key >> 32), lo = (unsigned)key;
    const unsigned mhi = __reduce_max_sync(0xffffffffu, hi);
    const unsigned mlo = __reduce_max_sync(0xffffffffu, hi == mhi ? lo : 0u);
    const bool win = (hi == mhi) && (lo == mlo);
    const int r = (int)__reduce_min_sync(0xffffffffu, win ? (unsigned)row : 0x7fffffffu);
    key = ((unsigned long long)mhi << 32) | mlo;
    row = r;
}

template <int NB, int RPT>
__global__ void __launch_bounds__(kPanelThreads) k_gj_panel(double *__restrict__ M, int V, int j0, int nbc,
                                                           int *__restrict__ ipiv, double *__restrict__ diag,
                                                           int *__restrict__ info) {
    __shared__ double pivrow[NB], swaprow[NB];
    __shared__ double Lt[NB][NB + 1], Ut[NB][NB + 1], Dinv[NB][NB + 1], Linv[NB][NB + 1];
    __shared__ unsigned long long red_k[32];
    __shared__ int red_r[32];
    __shared__ int piv_s;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    double a[RPT][NB];
#pragma unroll
    for (int i = 0; i < RPT; ++i) {
        const int r = tid + i * kPanelThreads;
#pragma unroll
        for (int c = 0; c < NB; ++c) a[i][c] = (r < V && c < nbc) ? M[(size_t)(j0 + c) * V + r] : 0.0;
    }
#pragma unroll
    for (int jj = 0; jj < NB; ++jj) {
        if (jj < nbc) {
            const int j = j0 + jj;
            unsigned long long bk = 0;
            int br = 0x7fffffff;
#pragma unroll
            for (int i = 0; i < RPT; ++i) {
                const int r = tid + i * kPanelThreads;
                if (r >= j && r < V) {
                    const unsigned long long k = abs_key(a[i][jj]);
                    if (k > bk || (k == bk && r < br)) {
                        bk = k;
                        br = r;
                    }
                }
            }
            warp_argmax(bk, br);
            if (lane == 0) {
                red_k[warp] = bk;
                red_r[warp] = br;
            }
            __syncthreads();
            if (warp == 0) {
                bk = red_k[lane];
                br = red_r[lane];
                warp_argmax(bk, br);
                if (lane == 0) {
                    int p = br;
                    if (bk == 0ull || p >= V) {  // exact zero column: no interchange, singular
                        p = j;
                        if (*info == 0) *info = j + 1;
                    }
                    piv_s = p;
                    ipiv[j] = p;
                }
            }
            __syncthreads();
            const int p = piv_s;
            // rows j and p trade places: owner of p publishes the pivot row, owner of j its own
#pragma unroll
            for (int i = 0; i < RPT; ++i) {
                const int r = tid + i * kPanelThreads;
                if (r == p) {
#pragma unroll
                    for (int c = 0; c < NB; ++c) pivrow[c] = a[i][c];
                }
                if (r == j && p != j) {
#pragma unroll
                    for (int c = 0; c < NB; ++c) swaprow[c] = a[i][c];
                }
            }
            __syncthreads();
            const double d = pivrow[jj];
            if (tid == 0) diag[j] = d;
            const double inv_d = 1.0 / d;
#pragma unroll
            for (int i = 0; i < RPT; ++i) {
                const int r = tid + i * kPanelThreads;
                if (r == j) {
#pragma unroll
                    for (int c = 0; c < NB; ++c) a[i][c] = pivrow[c];
                } else if (r == p) {
#pragma unroll
                    for (int c = 0; c < NB; ++c) a[i][c] = swaprow[c];
                }
                if (r > j && r < V && d != 0.0) {
                    const double l = a[i][jj] * inv_d;
                    a[i][jj] = l;
#pragma unroll
                    for (int c = jj + 1; c < NB; ++c) a[i][c] = fma(-l, pivrow[c], a[i][c]);
                }
            }
        }
    }
    // pivot block rows -> L11 (unit lower) and U11
#pragma unroll
    for (int i = 0; i < RPT; ++i) {
        const int r = tid + i * kPanelThreads;
        if (r >= j0 && r < j0 + nbc) {
            const int rr = r - j0;
#pragma unroll
            for (int c = 0; c < NB; ++c) {
                Lt[rr][c] = (c < rr) ? a[i][c] : (c == rr ? 1.0 : 0.0);
                Ut[rr][c] = (c >= rr) ? a[i][c] : 0.0;
            }
        }
    }
    __syncthreads();
    // Linv = L11^-1 and Uinv (kept in Dinv) column by column, one thread per column
    if (tid < nbc) {
        const int cc = tid;
        for (int rr = 0; rr < nbc; ++rr) {
            double s = (rr == cc) ? 1.0 : 0.0;
            for (int k = cc; k < rr; ++k) s = fma(-Lt[rr][k], Linv[k][cc], s);
            Linv[rr][cc] = (rr < cc) ? 0.0 : s;
        }
        for (int rr = nbc - 1; rr >= 0; --rr) {
            double s = (rr == cc) ? 1.0 : 0.0;
            for (int k = rr + 1; k <= cc; ++k) s = fma(-Ut[rr][k], Dinv[k][cc], s);
            Dinv[rr][cc] = (rr > cc) ? 0.0 : s / Ut[rr][rr];
        }
    }
    __syncthreads();
    // D^-1 = Uinv Linv, written over Ut
    if (tid < nbc * nbc) {
        const int rr = tid / nbc, cc = tid % nbc;
        double s = 0.0;
        for (int k = rr; k < nbc; ++k) s = fma(Dinv[rr][k], Linv[k][cc], s);
        Ut[rr][cc] = s;
    }
    __syncthreads();
    // new panel columns
#pragma unroll
    for (int i = 0; i < RPT; ++i) {
        const int r = tid + i * kPanelThreads;
        if (r >= V) continue;
        const int kind = (r >= j0 && r < j0 + nbc) ? 0 : (r >= j0 + nbc ? 1 : 2);
#pragma unroll
        for (int c = 0; c < NB; ++c) {
            if (c >= nbc) break;
            double s = 0.0;
            if (kind == 0) {  // rows P: D^-1
                s = Ut[r - j0][c];
            } else if (kind == 1) {  // rows below: -L21 L11^-1
#pragma unroll
                for (int k = 0; k < NB; ++k)
                    if (k >= c && k < nbc) s = fma(a[i][k], Linv[k][c], s);
                s = -s;
            } else {  // rows above the panel: -C D^-1
#pragma unroll
                for (int k = 0; k < NB; ++k)
                    if (k < nbc) s = fma(a[i][k], Ut[k][c], s);
                s = -s;
            }
            M[(size_t)(j0 + c) * V + r] = s;
        }
    }
}

// every column outside the panel, CB per CTA (blocks skip the panel)
template <int NB, int CB>
__global__ void k_gj_update(double *__restrict__ M, int V, int j0, int nbc, const int *__restrict__ ipiv) {
    extern __shared__ double C[];  // [CB][V]
    __shared__ double Dn[NB][NB + 1];
    __shared__ double R[NB][CB];
    __shared__ double Cp[NB][CB];
    const int tid = threadIdx.x, T = blockDim.x;
    const int nleft = (j0 + CB - 1) / CB;
    int c0, cend;
    if ((int)blockIdx.x < nleft) {
        c0 = blockIdx.x * CB;
        cend = min(c0 + CB, j0);
    } else {
        c0 = j0 + nbc + ((int)blockIdx.x - nleft) * CB;
        cend = min(c0 + CB, V);
    }
    const int ncol = cend - c0;
    if (ncol <= 0) return;
    __shared__ int pv[NB];
    for (int f = tid; f < ncol * V; f += T) C[f] = M[(size_t)c0 * V + f];
    for (int f = tid; f < nbc * nbc; f += T) {
        const int rr = f % nbc, cc = f / nbc;
        Dn[rr][cc] = M[(size_t)(j0 + cc) * V + j0 + rr];
    }
    if (tid < nbc) pv[tid] = ipiv[j0 + tid];
    __syncthreads();
    if (tid < ncol) {
        double *cl = C + (size_t)tid * V;
        for (int jj = 0; jj < nbc; ++jj) {
            const int j = j0 + jj, p = pv[jj];
            if (p != j) {
                const double t = cl[j];
                cl[j] = cl[p];
                cl[p] = t;
            }
        }
    }
    __syncthreads();
    // pivot rows after the interchanges (A_PO) and R = D^-1 A_PO
    for (int f = tid; f < nbc * ncol; f += T) {
        const int jj = f % nbc, q = f / nbc;
        Cp[jj][q] = C[(size_t)q * V + j0 + jj];
    }
    __syncthreads();
    for (int f = tid; f < nbc * ncol; f += T) {
        const int jj = f % nbc, q = f / nbc;
        double s = 0.0;
        for (int k = 0; k < nbc; ++k) s = fma(Dn[jj][k], Cp[k][q], s);
        R[jj][q] = s;
    }
    __syncthreads();
    // rows P: R; other rows: A - K A_PO with K = -(new panel columns)
    for (int r = tid; r < V; r += T) {
        if (r >= j0 && r < j0 + nbc) {
            for (int q = 0; q < ncol; ++q) C[(size_t)q * V + r] = R[r - j0][q];
        } else {
            double acc[CB];
#pragma unroll
            for (int q = 0; q < CB; ++q) acc[q] = (q < ncol) ? C[(size_t)q * V + r] : 0.0;
            double kr[NB];  // = -K(r, jj): all NB loads issued before the FMAs
#pragma unroll
            for (int jj = 0; jj < NB; ++jj) kr[jj] = (jj < nbc) ? M[(size_t)(j0 + jj) * V + r] : 0.0;
#pragma unroll
            for (int jj = 0; jj < NB; ++jj) {
                if (jj < nbc) {
#pragma unroll
                    for (int q = 0; q < CB; ++q) acc[q] = fma(kr[jj], Cp[jj][q], acc[q]);
                }
            }
#pragma unroll
            for (int q = 0; q < CB; ++q)
                if (q < ncol) C[(size_t)q * V + r] = acc[q];
        }
    }
    __syncthreads();
    for (int f = tid; f < ncol * V; f += T) M[(size_t)c0 * V + f] = C[f];
}

// composed column permutation: applying the interchanges last-first as column
// swaps leaves column c of the result at column src[c] of the elimination output
__global__ void k_compose_perm(const int *__restrict__ ipiv, int V, int *__restrict__ perm) {
    extern __shared__ int src[];  // [V] permutation, then [V] pivots
    int *pv = src + V;
    for (int c = threadIdx.x; c < V; c += blockDim.x) {
        src[c] = c;
        pv[c] = ipiv[c];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = V - 1; k >= 0; --k) {
            const int p = pv[k];
            const int t = src[k];
            src[k] = src[p];
            src[p] = t;
        }
    }
    __syncthreads();
    for (int c = threadIdx.x; c < V; c += blockDim.x) perm[c] = src[c];
}

__global__ void k_gather_rows(const double *__restrict__ A, double *__restrict__ X, int V,
                              const int *__restrict__ perm) {
    const int c = blockIdx.x;
    const int s = perm[c];
    for (int r = threadIdx.x; r < V; r += blockDim.x) X[(size_t)c * V + r] = A[(size_t)s * V + r];
}

// log|det| and sign from U's diagonal and the pivots (parallel sum)
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
    if ((threadIdx.x & 31) == 0) {
        s_l[threadIdx.x >> 5] = l;
        s_n[threadIdx.x >> 5] = neg;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        int n = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
            t += s_l[w];
            n ^= s_n[w];
        }
        out[0] = t;
        out[1] = n ? -1.0 : 1.0;
    }
}

template <int NB, int RPT>
int run_panels(double *M, LUWork &w, cudaStream_t st) {
    const int V = w.V;
    constexpr int CB = 8;
    const size_t usmem = (size_t)CB * V * sizeof(double);
    if (usmem > 200 * 1024) return EPHMC_ERR_UNSUPPORTED;
    EPHMC_CUDA(cudaFuncSetAttribute(k_gj_update<NB, CB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)usmem));
    for (int j0 = 0; j0 < V; j0 += NB) {
        const int nbc = std::min(NB, V - j0);
        k_gj_panel<NB, RPT><<<1, kPanelThreads, 0, st>>>(M, V, j0, nbc, w.ipiv, w.diag, w.info);
        ephmc::count_launch(1);
        EPHMC_CUDA(cudaGetLastError());
        const int nblocks = (j0 + CB - 1) / CB + (V - j0 - nbc + CB - 1) / CB;
        if (nblocks > 0) {
            k_gj_update<NB, CB><<<nblocks, 256, usmem, st>>>(M, V, j0, nbc, w.ipiv);
            ephmc::count_launch(1);
            EPHMC_CUDA(cudaGetLastError());
        }
    }
    return EPHMC_OK;
}

}  // namespace

int lu_alloc(LUWork &w, int V) {
    w.V = V;
    EPHMC_CUDA(cudaMalloc(&w.ipiv, sizeof(int) * 2 * V));  // pivots, then the composed permutation
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

int lu_logdet_inverse(double *M, LUWork &w, double *logdet, int *sign, int *ipiv_host, cudaStream_t st) {
    const int V = w.V;
    EPHMC_CUDA(cudaMemsetAsync(w.info, 0, sizeof(int) * 2, st));
    int rc;
    if (V <= 1024) rc = run_panels<16, 1>(M, w, st);
    else if (V <= 2048) rc = run_panels<8, 2>(M, w, st);
    else if (V <= 4096) rc = run_panels<4, 4>(M, w, st);
    else rc = EPHMC_ERR_UNSUPPORTED;
    if (rc != EPHMC_OK) return rc;
    k_lu_logdet<<<1, 1024, 0, st>>>(w.diag, w.ipiv, V, w.diag + V);
    ephmc::count_launch(1);
    EPHMC_CUDA(cudaGetLastError());
    int *perm = w.ipiv + V;
    k_compose_perm<<<1, 1024, 2 * sizeof(int) * V, st>>>(w.ipiv, V, perm);
    ephmc::count_launch(1);
    k_gather_rows<<<V, 256, 0, st>>>(M, w.X, V, perm);
    ephmc::count_launch(1);
    EPHMC_CUDA(cudaGetLastError());
    EPHMC_CUDA(cudaMemcpyAsync(M, w.X, sizeof(double) * (size_t)V * V, cudaMemcpyDeviceToDevice, st));
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
    return EPHMC_OK;
}

}  // namespace ephmc
