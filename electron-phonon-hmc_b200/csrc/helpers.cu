// Small device kernels behind the drop-in surface: single stencil applications
// (rows or columns, reference summation order), the antisymmetric current
// operator, dense helpers and the phonon-side reductions.
#include "ephmc_internal.cuh"

#include <algorithm>
#include <cstring>

namespace ephmc {

namespace {

// out = (mu + K) in on every row (cols=false) or column (cols=true) of nmat
// V x V matrices; one thread per (vector, site).
__global__ void k_stencil(const double *__restrict__ xs, Couplings c, const int *__restrict__ ev_src,
                          const int *__restrict__ ev_fac, const double *__restrict__ in, double *__restrict__ out,
                          int V, int nvec, int cols, double add_in) {
    const size_t n = (size_t)nvec * V;
    for (size_t f = blockIdx.x * (size_t)blockDim.x + threadIdx.x; f < n; f += (size_t)gridDim.x * blockDim.x) {
        const int vec = (int)(f / V), j = (int)(f % V);
        const size_t base = cols ? (size_t)vec : (size_t)vec * V;
        const size_t stride = cols ? (size_t)V : 1;
        double acc = c.mu * in[base + j * stride];
#pragma unroll
        for (int e = 0; e < 6; ++e) {
            const int fi = ev_fac[e * V + j];
            const int k = fi % 3;
            const double fac = fma(-c.kappa[k], xs[fi], c.t[k]);
            acc = fma(fac, in[base + (size_t)ev_src[e * V + j] * stride], acc);
        }
        out[base + j * stride] = (add_in != 0.0) ? in[base + j * stride] + acc : acc;
    }
}

// w = I_k v: antisymmetric hopping along link k, scatter order of
// apply_current_to_v (simulation/organic_dense_matrix.c:226-249):
// w[i] += fac_i v[n_i]  then  w[n_i] += -fac_i v[i], in increasing i.
__global__ void k_current(const double *__restrict__ xs, Couplings c, const int *__restrict__ nbr,
                          const int *__restrict__ rev_order, const double *__restrict__ v, double *__restrict__ w,
                          int V, int k) {
    // one thread per site j: contributions from (j, here) and (i with n_i = j, there), in (i, type) order
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= V) return;
    const int n = nbr[k * V + j];
    const int i = rev_order[j];  // the site whose k-neighbour is j
    const double fj = fma(-c.kappa[k], xs[3 * j + k], c.t[k]);
    const double fi = fma(-c.kappa[k], xs[3 * i + k], c.t[k]);
    const double here = fj * v[n];
    const double there = -fi * v[i];
    double acc = 0.0;
    if (i < j) {
        acc += there;
        acc += here;
    } else if (i > j) {
        acc += here;
        acc += there;
    } else {  // self-link (L = 1 along k): here then there in the same iteration
        acc += here;
        acc += there;
    }
    w[j] = acc;
}

__global__ void k_combine_refine(double *__restrict__ G, const double *__restrict__ X, const double *__restrict__ X1,
                                 const double *__restrict__ X2, size_t n, double al, double aq, int first) {
    for (size_t f = blockIdx.x * (size_t)blockDim.x + threadIdx.x; f < n; f += (size_t)gridDim.x * blockDim.x) {
        double g = first ? al * X[f] : fma(al, X[f], G[f]);
        g = fma(aq, X1[f] + X2[f], g);
        G[f] = g;
    }
}

// y[i] = sum_k m[i*n+k] x[k] (tr = 0) or y[k] = sum_i m[i*n+k] x[i] (tr = 1)
__global__ void k_matvec(const double *__restrict__ m, const double *__restrict__ x, double *__restrict__ y, int n,
                         int tr) {
    const int o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= n) return;
    double acc = 0.0;
    if (!tr)
        for (int k = 0; k < n; ++k) acc += m[(size_t)o * n + k] * x[k];
    else
        for (int i = 0; i < n; ++i) acc += m[(size_t)i * n + o] * x[i];
    y[o] = acc;
}

// rows i of m2 replaced by m1 * m2[i,:] (mat_mat_mul, simulation/organic_dense_matrix.c:40-45)
__global__ void k_matmat_rows(const double *__restrict__ m1, const double *__restrict__ m2, double *__restrict__ out,
                              int n) {
    const size_t f = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (f >= (size_t)n * n) return;
    const int i = (int)(f / n), o = (int)(f % n);
    double acc = 0.0;
    for (int k = 0; k < n; ++k) acc += m1[(size_t)o * n + k] * m2[(size_t)i * n + k];
    out[f] = acc;
}

__global__ void k_transpose_rect(const double *__restrict__ x, double *__restrict__ y, int n1, int n2) {
    const size_t f = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (f >= (size_t)n1 * n2) return;
    const int i = (int)(f / n1), j = (int)(f % n1);
    y[(size_t)j * n2 + i] = x[f];
}

__global__ void k_trace(const double *__restrict__ m, int n, double *__restrict__ out) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        double tr = 0;
        for (int i = 0; i < n; ++i) tr += m[(size_t)i * (n + 1)];
        out[0] = tr;
    }
}

// p_dot (+)= -omega x + (x_{t+1} - 2 x_t + x_{t-1}) / omega (boson_force, simulation/organic_bosons.c:179-194)
__global__ void k_boson_force(const double *__restrict__ x, double *__restrict__ pd, double omega, int ld, int nt,
                              int overwrite) {
    const size_t n = (size_t)ld * nt;
    for (size_t f = blockIdx.x * (size_t)blockDim.x + threadIdx.x; f < n; f += (size_t)gridDim.x * blockDim.x) {
        const int t = (int)(f / ld), e = (int)(f % ld);
        const double xp = x[(size_t)((t + 1) % nt) * ld + e], xm = x[(size_t)((t + nt - 1) % nt) * ld + e];
        double v = overwrite ? 0.0 : pd[f];
        v -= omega * x[f];
        v += (xp - 2 * x[f] + xm) / omega;
        pd[f] = v;
    }
}

// per-link sum_t (x_t - mean)^2 partials (higher_Matsubaras_norm, simulation/organic_bosons.c:36-53)
__global__ void k_matsubara(const double *__restrict__ x, int ld, int nt, double *__restrict__ part) {
    __shared__ double red[256];
    double acc = 0.0;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < ld; e += gridDim.x * blockDim.x) {
        double m = 0.0;
        for (int t = 0; t < nt; ++t) m += x[(size_t)t * ld + e];
        m /= (double)nt;
        for (int t = 0; t < nt; ++t) {
            const double d = x[(size_t)t * ld + e] - m;
            acc = fma(d, d, acc);
        }
    }
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

// sum and sum of squares partials
__global__ void k_moments(const double *__restrict__ x, size_t n, double *__restrict__ part) {
    __shared__ double s1[256], s2[256];
    double a = 0, b = 0;
    for (size_t f = blockIdx.x * (size_t)blockDim.x + threadIdx.x; f < n; f += (size_t)gridDim.x * blockDim.x) {
        a += x[f];
        b = fma(x[f], x[f], b);
    }
    s1[threadIdx.x] = a;
    s2[threadIdx.x] = b;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) {
            s1[threadIdx.x] += s1[threadIdx.x + o];
            s2[threadIdx.x] += s2[threadIdx.x + o];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        part[2 * blockIdx.x] = s1[0];
        part[2 * blockIdx.x + 1] = s2[0];
    }
}

// greens[tau][a][b] = sum_i x_0[i][a] x_tau[i][b] / ns (phonon_correlator, simulation/organic_dense_matrix.c:526-545)
__global__ void k_phonon_corr(const double *__restrict__ x, int ns, int nt, double *__restrict__ g) {
    const int tau = blockIdx.x;
    const int ab = threadIdx.x;  // 0..8
    if (ab >= 9) return;
    const int a = ab / 3, b = ab % 3;
    double s = 0.0;
    for (int i = 0; i < ns; ++i) s += x[(size_t)i * 3 + a] * x[(size_t)tau * ns * 3 + (size_t)i * 3 + b];
    g[(size_t)tau * 9 + ab] = s / ns;
}

// p_dot[t,i,k] = -kappa_k (D[i][n] + D[n][i]) flavors from one full matrix D for every slice
// (force with CONSTANT_FORCE, simulation/organic_hmc.c:100-127)
__global__ void k_contract_full(const double *__restrict__ D, Couplings c, const int *__restrict__ nbr, int V, int nt,
                                unsigned flavors, int schur, int sp, double spw, double *__restrict__ force) {
    const size_t n = (size_t)nt * V * 3;
    for (size_t f = blockIdx.x * (size_t)blockDim.x + threadIdx.x; f < n; f += (size_t)gridDim.x * blockDim.x) {
        const int k = (int)(f % 3), i = (int)((f / 3) % V);
        const int nb = nbr[k * V + i];
        double proj = D[(size_t)i * V + nb] + D[(size_t)nb * V + i];
        if (schur && fabs(proj) > 2) proj = proj > 0 ? 2 : -2;
        double v = -c.kappa[k] * proj * (double)flavors;
        if (sp) v *= spw;
        force[f] = v;
    }
}

__global__ void k_add_diag(double *__restrict__ M, int V, double v) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < V) M[(size_t)i * (V + 1)] += v;
}

// v = v + fma(a_lin, w, a_quad z), the pair step of apply_2nd_order_mu_K_to_v (:176-178)
__global__ void k_pair_combine(double *__restrict__ v, const double *__restrict__ w, const double *__restrict__ z,
                               double al, double aq, size_t n) {
    for (size_t f = blockIdx.x * (size_t)blockDim.x + threadIdx.x; f < n; f += (size_t)gridDim.x * blockDim.x)
        v[f] = v[f] + fma(al, w[f], aq * z[f]);
}

__global__ void k_axpy(double *__restrict__ y, const double *__restrict__ x, double a, size_t n) {
    for (size_t f = blockIdx.x * (size_t)blockDim.x + threadIdx.x; f < n; f += (size_t)gridDim.x * blockDim.x)
        y[f] = fma(a, x[f], y[f]);
}

}  // namespace

int launch_stencil(const double *xs, const Couplings &c, const LatticeDev &lat, const double *in, double *out,
                   int nvec, bool cols, bool add_in, cudaStream_t st) {
    const size_t n = (size_t)nvec * lat.V;
    const int blocks = (int)std::min<size_t>((n + 255) / 256, 4096);
    k_stencil<<<blocks, 256, 0, st>>>(xs, c, lat.ev_src, lat.ev_fac, in, out, lat.V, nvec, cols ? 1 : 0,
                                      add_in ? 1.0 : 0.0);
    count_launch(1);
    EPHMC_CUDA(cudaGetLastError());
    return EPHMC_OK;
}

int launch_current(const double *xs, const Couplings &c, const LatticeDev &lat, const int *rev_k, const double *v,
                   double *w, int k, cudaStream_t st) {
    k_current<<<(lat.V + 127) / 128, 128, 0, st>>>(xs, c, lat.nbr, rev_k, v, w, lat.V, k);
    count_launch(1);
    EPHMC_CUDA(cudaGetLastError());
    return EPHMC_OK;
}

int launch_combine_refine(double *G, const double *X, const double *X1, const double *X2, size_t n, double al,
                          double aq, bool first, cudaStream_t st) {
    k_combine_refine<<<1184, 256, 0, st>>>(G, X, X1, X2, n, al, aq, first ? 1 : 0);
    count_launch(1);
    EPHMC_CUDA(cudaGetLastError());
    return EPHMC_OK;
}

int launch_matvec(const double *m, const double *x, double *y, int n, bool tr, cudaStream_t st) {
    k_matvec<<<(n + 127) / 128, 128, 0, st>>>(m, x, y, n, tr ? 1 : 0);
    count_launch(1);
    EPHMC_CUDA(cudaGetLastError());
    return EPHMC_OK;
}

int launch_matmat_rows(const double *m1, const double *m2, double *out, int n, cudaStream_t st) {
    const size_t nn = (size_t)n * n;
    k_matmat_rows<<<(unsigned)((nn + 255) / 256), 256, 0, st>>>(m1, m2, out, n);
    count_launch(1);
    EPHMC_CUDA(cudaGetLastError());
    return EPHMC_OK;
}

int launch_transpose_rect(const double *x, double *y, int n1, int n2, cudaStream_t st) {
    const size_t nn = (size_t)n1 * n2;
    k_transpose_rect<<<(unsigned)((nn + 255) / 256), 256, 0, st>>>(x, y, n1, n2);
    count_launch(1);
    EPHMC_CUDA(cudaGetLastError());
    return EPHMC_OK;
}

int launch_trace(const double *m, int n, double *out_dev, cudaStream_t st) {
    k_trace<<<1, 32, 0, st>>>(m, n, out_dev);
    count_launch(1);
    EPHMC_CUDA(cudaGetLastError());
    return EPHMC_OK;
}

int launch_boson_force(const double *x, double *pd, double omega, int ld, int nt, bool overwrite, cudaStream_t st) {
    k_boson_force<<<592, 256, 0, st>>>(x, pd, omega, ld, nt, overwrite ? 1 : 0);
    count_launch(1);
    EPHMC_CUDA(cudaGetLastError());
    return EPHMC_OK;
}

// part needs 2 * 64 doubles; result sums into out[0] (sum), out[1] (sum of squares) on the host
int device_moments(const double *x, size_t n, double *part_dev, double out[2], cudaStream_t st) {
    k_moments<<<64, 256, 0, st>>>(x, n, part_dev);
    count_launch(1);
    EPHMC_CUDA(cudaGetLastError());
    double h[128];
    EPHMC_CUDA(cudaMemcpyAsync(h, part_dev, sizeof(h), cudaMemcpyDeviceToHost, st));
    EPHMC_CUDA(cudaStreamSynchronize(st));
    out[0] = out[1] = 0;
    for (int b = 0; b < 64; ++b) {
        out[0] += h[2 * b];
        out[1] += h[2 * b + 1];
    }
    return EPHMC_OK;
}

int device_matsubara_norm(const double *x, int ld, int nt, double *part_dev, double *out, cudaStream_t st) {
    k_matsubara<<<64, 256, 0, st>>>(x, ld, nt, part_dev);
    count_launch(1);
    EPHMC_CUDA(cudaGetLastError());
    double h[64];
    EPHMC_CUDA(cudaMemcpyAsync(h, part_dev, sizeof(h), cudaMemcpyDeviceToHost, st));
    EPHMC_CUDA(cudaStreamSynchronize(st));
    double s = 0;
    for (int b = 0; b < 64; ++b) s += h[b];
    *out = s;
    return EPHMC_OK;
}

int launch_phonon_corr(const double *x, int ns, int nt, double *g, cudaStream_t st) {
    k_phonon_corr<<<nt, 32, 0, st>>>(x, ns, nt, g);
    count_launch(1);
    EPHMC_CUDA(cudaGetLastError());
    return EPHMC_OK;
}

int launch_contract_full(const double *D, const Couplings &c, const LatticeDev &lat, int nt, unsigned flavors,
                         int schur, int sp, double spw, double *force, cudaStream_t st) {
    k_contract_full<<<592, 256, 0, st>>>(D, c, lat.nbr, lat.V, nt, flavors, schur, sp, spw, force);
    count_launch(1);
    EPHMC_CUDA(cudaGetLastError());
    return EPHMC_OK;
}

int launch_add_diag(double *M, int V, double v, cudaStream_t st) {
    k_add_diag<<<(V + 127) / 128, 128, 0, st>>>(M, V, v);
    count_launch(1);
    EPHMC_CUDA(cudaGetLastError());
    return EPHMC_OK;
}

int launch_pair_combine(double *v, const double *w, const double *z, double al, double aq, size_t n, cudaStream_t st) {
    k_pair_combine<<<(unsigned)std::min<size_t>((n + 255) / 256, 1184), 256, 0, st>>>(v, w, z, al, aq, n);
    count_launch(1);
    EPHMC_CUDA(cudaGetLastError());
    return EPHMC_OK;
}

namespace {
constexpr int kParamBytes = 3968;  // payload of one launch, inside the 4 KB kernel-parameter space
struct ParamChunk {
    unsigned char b[kParamBytes];
};
__global__ void k_write_bytes(unsigned char *__restrict__ dst, ParamChunk c, int n) {
    for (int i = threadIdx.x; i < n; i += blockDim.x) dst[i] = c.b[i];
}
}  // namespace

namespace {
thread_local bool g_uncached = false;
}
void uploads_uncached(bool on) { g_uncached = on; }
bool uploads_are_uncached() { return g_uncached; }

int upload_small(void *dst, const void *src, size_t bytes, cudaStream_t st) {
    const unsigned char *s = static_cast<const unsigned char *>(src);
    unsigned char *d = static_cast<unsigned char *>(dst);
    for (size_t off = 0; off < bytes; off += kParamBytes) {
        const int n = (int)std::min<size_t>(kParamBytes, bytes - off);
        ParamChunk c;
        std::memcpy(c.b, s + off, n);
        k_write_bytes<<<1, 256, 0, st>>>(d + off, c, n);
        count_launch(1);
        EPHMC_CUDA(cudaGetLastError());
    }
    return EPHMC_OK;
}

int launch_axpy(double *y, const double *x, double a, size_t n, cudaStream_t st) {
    k_axpy<<<592, 256, 0, st>>>(y, x, a, n);
    count_launch(1);
    EPHMC_CUDA(cudaGetLastError());
    return EPHMC_OK;
}

}  // namespace ephmc
