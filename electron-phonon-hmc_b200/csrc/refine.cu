// Reference-algorithm force: refinement of G_t and the link contraction, FP64.
//
// refine_QM1P (simulation/organic_dense_matrix.c:383-442) turns G_t into
//   D = a_lin0 A + a_quad0 (H A + A H) + a_lin1 B + a_quad1 (H B + B H)
// with A = G_t with pair 1 applied to its columns and B = G_t with pair 0
// applied to its rows (two quadratic pairs, pair order {0,1}).  force()
// (simulation/organic_hmc.c:107-126) then reads only the link entries
// D[i][n] + D[n][i].  This kernel evaluates exactly those entries from A and B:
// (H A)[a][b] is the stencil on row a of A at site b, (A H)[a][b] the stencil on
// column b at site a, each summed in the reference's event order, and D is
// accumulated in the reference's order (G = a_lin*loc; G = fma(a_quad, loc+loc2, G)).
// Work is O(V) per slice instead of the reference's four full V x V stencil
// passes, with identical arithmetic for every entry the force uses.
#include "ephmc_internal.cuh"

namespace ephmc {

namespace {

// stencil of row `row` of M evaluated at site `site`: mu M[row][site] + sum_e fac_e M[row][src_e(site)]
__device__ __forceinline__ double stencil_row(const double *__restrict__ M, int V, int row, int site,
                                              const double *__restrict__ fac, const int *__restrict__ ev_src,
                                              const int *__restrict__ ev_fac, double mu) {
    const double *Mr = M + (size_t)row * V;
    double acc = mu * Mr[site];
#pragma unroll
    for (int e = 0; e < 6; ++e) acc = fma(fac[ev_fac[e * V + site]], Mr[ev_src[e * V + site]], acc);
    return acc;
}

// stencil of column `col` of M evaluated at site `site`
__device__ __forceinline__ double stencil_col(const double *__restrict__ M, int V, int col, int site,
                                              const double *__restrict__ fac, const int *__restrict__ ev_src,
                                              const int *__restrict__ ev_fac, double mu) {
    double acc = mu * M[(size_t)site * V + col];
#pragma unroll
    for (int e = 0; e < 6; ++e)
        acc = fma(fac[ev_fac[e * V + site]], M[(size_t)ev_src[e * V + site] * V + col], acc);
    return acc;
}

__device__ __forceinline__ double d_entry(const double *A, const double *B, int V, int a, int b,
                                          const double *fac, const int *ev_src, const int *ev_fac,
                                          const Couplings &c) {
    const double Aab = A[(size_t)a * V + b], Bab = B[(size_t)a * V + b];
    const double A1 = stencil_row(A, V, a, b, fac, ev_src, ev_fac, c.mu);
    const double A2 = stencil_col(A, V, b, a, fac, ev_src, ev_fac, c.mu);
    const double B1 = stencil_row(B, V, a, b, fac, ev_src, ev_fac, c.mu);
    const double B2 = stencil_col(B, V, b, a, fac, ev_src, ev_fac, c.mu);
    double d = c.a_lin[0] * Aab;
    d = fma(c.a_quad[0], A1 + A2, d);
    d = fma(c.a_lin[1], Bab, d);
    d = fma(c.a_quad[1], B1 + B2, d);
    return d;
}

// one CTA per slice of the batch; the slice's hopping table in shared memory
__global__ void k_link_refine(const double *__restrict__ x, Couplings c, const int *__restrict__ ev_src,
                              const int *__restrict__ ev_fac, const int *__restrict__ nbr,
                              const double *__restrict__ Aall, const double *__restrict__ Ball, int V,
                              int t0, unsigned flavors, int schur_clamp, int single_particle,
                              double sp_weight, double *__restrict__ force) {
    extern __shared__ double fac[];
    const int tb = blockIdx.y;
    const int t = t0 + tb;
    const double *xs = x + (size_t)t * 3 * V;
    for (int e = threadIdx.x; e < 3 * V; e += blockDim.x) {
        const int k = e % 3;
        fac[e] = fma(-c.kappa[k], xs[e], c.t[k]);
    }
    __syncthreads();
    const double *A = Aall + (size_t)tb * V * V;
    const double *B = Ball + (size_t)tb * V * V;
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;  // (site, link)
    if (idx >= 3 * V) return;
    const int i = idx / 3, k = idx % 3;
    const int n = nbr[k * V + i];
    double proj = d_entry(A, B, V, i, n, fac, ev_src, ev_fac, c) + d_entry(A, B, V, n, i, fac, ev_src, ev_fac, c);
    if (schur_clamp && fabs(proj) > 2) proj = proj > 0 ? 2 : -2;
    double f = -c.kappa[k] * proj * (double)flavors;
    if (single_particle) f *= sp_weight;
    force[((size_t)t * V + i) * 3 + k] = f;
}

__global__ void k_copy(double *__restrict__ d, const double *__restrict__ s, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) d[i] = s[i];
}

__global__ void k_fill(double *__restrict__ d, double v, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) d[i] = v;
}

__global__ void k_identity(double *__restrict__ M, int V) {
    const size_t n = (size_t)V * V;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        M[i] = (i / V == i % V) ? 1.0 : 0.0;
}

// in-place transpose with 32x32 tiles; blocks above the diagonal swap with their mirror
__global__ void k_transpose(double *M, int V) {
    __shared__ double ta[32][33], tb[32][33];
    const int bi = blockIdx.y, bj = blockIdx.x;
    if (bj < bi) return;
    const int tx = threadIdx.x, ty = threadIdx.y;  // 32 x 8
    for (int yy = ty; yy < 32; yy += 8) {
        const int r = bi * 32 + yy, cidx = bj * 32 + tx;
        if (r < V && cidx < V) ta[yy][tx] = M[(size_t)r * V + cidx];
        const int r2 = bj * 32 + yy, c2 = bi * 32 + tx;
        if (r2 < V && c2 < V) tb[yy][tx] = M[(size_t)r2 * V + c2];
    }
    __syncthreads();
    for (int yy = ty; yy < 32; yy += 8) {
        const int r = bi * 32 + yy, cidx = bj * 32 + tx;
        if (r < V && cidx < V) M[(size_t)r * V + cidx] = tb[tx][yy];
        const int r2 = bj * 32 + yy, c2 = bi * 32 + tx;
        if (r2 < V && c2 < V && bi != bj) M[(size_t)r2 * V + c2] = ta[tx][yy];
    }
}

}  // namespace

int launch_link_refine(const double *x, const Couplings &c, const LatticeDev &lat, const double *A,
                       const double *B, int t0, int nb, unsigned flavors, int schur_clamp,
                       int single_particle, double logdet, double *force, cudaStream_t st) {
    const int V = lat.V;
    const int threads = 128;
    dim3 grid((3 * V + threads - 1) / threads, nb);
    const size_t smem = 3 * (size_t)V * sizeof(double);
    if (smem > 48 * 1024)
        EPHMC_CUDA(cudaFuncSetAttribute(k_link_refine, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_link_refine<<<grid, threads, smem, st>>>(x, c, lat.ev_src, lat.ev_fac, lat.nbr, A, B, V, t0, flavors,
                                               schur_clamp, single_particle, exp(-logdet), force); ephmc::count_launch(1);
    EPHMC_CUDA(cudaGetLastError());
    return EPHMC_OK;
}

int launch_copy(double *dst, const double *src, size_t n, cudaStream_t st) {
    k_copy<<<592, 256, 0, st>>>(dst, src, n); ephmc::count_launch(1);
    EPHMC_CUDA(cudaGetLastError());
    return EPHMC_OK;
}

int launch_fill(double *p, double v, size_t n, cudaStream_t st) {
    k_fill<<<592, 256, 0, st>>>(p, v, n); ephmc::count_launch(1);
    EPHMC_CUDA(cudaGetLastError());
    return EPHMC_OK;
}

int launch_identity(double *M, int V, cudaStream_t st) {
    k_identity<<<592, 256, 0, st>>>(M, V); ephmc::count_launch(1);
    EPHMC_CUDA(cudaGetLastError());
    return EPHMC_OK;
}

int launch_transpose(double *M, int V, cudaStream_t st) {
    dim3 grid((V + 31) / 32, (V + 31) / 32), block(32, 8);
    k_transpose<<<grid, block, 0, st>>>(M, V); ephmc::count_launch(1);
    EPHMC_CUDA(cudaGetLastError());
    return EPHMC_OK;
}

}  // namespace ephmc
