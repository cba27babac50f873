// Fourier acceleration of the phonon update, FP64.
//
// The reference transforms 3V real series of length Nt (series e at
// x[t*3V + e]) with FFTW r2c / c2r plans (simulation/organic_hmc.c:317-322),
// acts mode by mode and transforms back:
//   evolve_bosons          (simulation/organic_bosons.c:126-150)
//   sample_fourier_momenta (:76-100), sample_free_bosons (:55-74)
//   energy_fourier_momenta (:102-124)
//   evolve_bosons_approx_step (:152-177), the kinetic step of classical
//   Fourier acceleration
// Here one kernel does transform -> per-mode update -> inverse transform for a
// tile of 32 series held in shared memory, so x and p are read and written
// once (HBM-bound: 2 x 8 x 3V x Nt bytes in, the same out).  The transform is
// a direct real DFT against a shared twiddle table (Nt <= 512), with FFTW's
// unnormalised conventions; the per-mode constants are computed on the host
// with the reference's formulas and passed in.
#include "ephmc_internal.cuh"

#include <map>
#include <mutex>

#include <cmath>
#include <vector>

namespace ephmc {

namespace {

constexpr int kTile = 32;   // series per CTA
constexpr int kRowsY = 8;   // threadIdx.y extent

// forward: X[k] = sum_t a[t] e^{-2 pi i t k / n}, k = 0..n/2
__device__ void dft_fwd(const double *a, double *Xr, double *Xi, int n, const double *cs, const double *sn,
                        int e) {
    const int nc = n / 2 + 1;
    for (int k = threadIdx.y; k < nc; k += kRowsY) {
        double re = 0.0, im = 0.0;
        for (int t = 0; t < n; ++t) {
            const int m = (t * k) % n;
            const double v = a[t * kTile + e];
            re = fma(v, cs[m], re);
            im = fma(-v, sn[m], im);
        }
        Xr[k * kTile + e] = re;
        Xi[k * kTile + e] = im;
    }
}

// inverse (c2r): a[t] = Re X0 + 2 sum_{0<k<n/2} Re(X[k] e^{2 pi i t k/n}) + Re X[n/2] (-1)^t
__device__ void dft_inv(const double *Xr, const double *Xi, double *a, int n, const double *cs, const double *sn,
                        int e) {
    const int nc = n / 2 + 1;
    for (int t = threadIdx.y; t < n; t += kRowsY) {
        double acc = Xr[e];
        for (int k = 1; k < nc; ++k) {
            const int m = (t * k) % n;
            const double term = fma(Xr[k * kTile + e], cs[m], -Xi[k * kTile + e] * sn[m]);
            if (2 * k == n) acc += (t & 1) ? -Xr[k * kTile + e] : Xr[k * kTile + e];
            else acc = fma(2.0, term, acc);
        }
        a[t * kTile + e] = acc;
    }
}

__device__ void load_twiddles(double *cs, double *sn, int n) {
    const int tid = threadIdx.y * kTile + threadIdx.x;
    for (int m = tid; m < n; m += kTile * kRowsY) {
        double s, c;
        sincospi(2.0 * (double)m / (double)n, &s, &c);
        cs[m] = c;
        sn[m] = s;
    }
}

// mode: 0 evolve (x,p), 1 scale p by modes[k] (momentum refresh), 2 scale x by modes[k] (free bosons),
// 3 x <- (x + modes[k] p) c mode by mode, p read only (classical acceleration's kinetic step)
__global__ void k_fa(double *__restrict__ x, double *__restrict__ p, int ld, int n, const double *__restrict__ mc,
                     const double *__restrict__ ms, double c, int mode) {
    extern __shared__ double sm[];
    const int nc = n / 2 + 1;
    double *cs = sm, *sn = cs + n;
    double *ax = sn + n, *ap = ax + (size_t)n * kTile;
    double *xr = ap + (size_t)n * kTile, *xi = xr + (size_t)nc * kTile;
    double *pr = xi + (size_t)nc * kTile, *pi = pr + (size_t)nc * kTile;
    const int e0 = blockIdx.x * kTile;
    const int e = threadIdx.x;
    const bool valid = e0 + e < ld;
    load_twiddles(cs, sn, n);
    for (int t = threadIdx.y; t < n; t += kRowsY) {
        if (mode != 1) ax[t * kTile + e] = valid ? x[(size_t)t * ld + e0 + e] : 0.0;
        if (mode != 2) ap[t * kTile + e] = valid ? p[(size_t)t * ld + e0 + e] : 0.0;
    }
    __syncthreads();
    if (mode != 1) dft_fwd(ax, xr, xi, n, cs, sn, e);
    if (mode != 2) dft_fwd(ap, pr, pi, n, cs, sn, e);
    __syncthreads();
    for (int k = threadIdx.y; k < nc; k += kRowsY) {
        const int o = k * kTile + e;
        if (mode == 0) {
            // x' = c x + (s/f2) p ; p' = c p - (s f2) x   (c, s already divided by n)
            const double s1w = mc[k], sw = ms[k];
            const double x0r = xr[o], x0i = xi[o], p0r = pr[o], p0i = pi[o];
            xr[o] = c * x0r + s1w * p0r;
            xi[o] = c * x0i + s1w * p0i;
            pr[o] = c * p0r - sw * x0r;
            pi[o] = c * p0i - sw * x0i;
        } else if (mode == 1) {
            pr[o] *= mc[k];
            pi[o] *= mc[k];
        } else if (mode == 3) {
            // xc += (h / freq2) pc ; xc *= 1/n   (:170-173)
            xr[o] = fma(mc[k], pr[o], xr[o]) * c;
            xi[o] = fma(mc[k], pi[o], xi[o]) * c;
        } else {
            xr[o] *= mc[k];
            xi[o] *= mc[k];
        }
    }
    __syncthreads();
    if (mode != 1) dft_inv(xr, xi, ax, n, cs, sn, e);
    if (mode != 2 && mode != 3) dft_inv(pr, pi, ap, n, cs, sn, e);
    __syncthreads();
    if (valid) {
        for (int t = threadIdx.y; t < n; t += kRowsY) {
            if (mode != 1) x[(size_t)t * ld + e0 + e] = ax[t * kTile + e];
            if (mode != 2 && mode != 3) p[(size_t)t * ld + e0 + e] = ap[t * kTile + e];
        }
    }
}

// per-CTA partial of sum_k w_k |P_k|^2; w from the host
__global__ void k_fa_energy(const double *__restrict__ p, int ld, int n, const double *__restrict__ wk,
                            double *__restrict__ partial) {
    extern __shared__ double sm[];
    const int nc = n / 2 + 1;
    double *cs = sm, *sn = cs + n, *ap = sn + n;
    double *pr = ap + (size_t)n * kTile, *pi = pr + (size_t)nc * kTile;
    __shared__ double red[kTile * kRowsY];
    const int e0 = blockIdx.x * kTile, e = threadIdx.x;
    const bool valid = e0 + e < ld;
    load_twiddles(cs, sn, n);
    for (int t = threadIdx.y; t < n; t += kRowsY) ap[t * kTile + e] = valid ? p[(size_t)t * ld + e0 + e] : 0.0;
    __syncthreads();
    dft_fwd(ap, pr, pi, n, cs, sn, e);
    __syncthreads();
    double s = 0.0;
    for (int k = threadIdx.y; k < nc; k += kRowsY) {
        const double a = pr[k * kTile + e], b = pi[k * kTile + e];
        s += (a * a + b * b) * wk[k];
    }
    red[threadIdx.y * kTile + e] = s;
    __syncthreads();
    if (threadIdx.y == 0 && e == 0) {
        double t = 0.0;
        for (int i = 0; i < kTile * kRowsY; ++i) t += red[i];
        partial[blockIdx.x] = t;
    }
}

__global__ void k_sum(const double *__restrict__ a, int n, double *__restrict__ out) {
    __shared__ double red[256];
    double s = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) s += a[i];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[0] = red[0];
}

size_t fa_smem(int n, bool two) {
    const int nc = n / 2 + 1;
    return sizeof(double) * (2 * (size_t)n + (two ? 2 : 1) * (size_t)n * kTile + (two ? 4 : 2) * (size_t)nc * kTile);
}

// freq2_k = omega + (2 sin(pi k / Nt))^2 / omega   (simulation/organic_bosons.c:136)
double freq2(double omega, int k, int n) {
    const double matsubara = 3.141592653589793 / n;  // M_PI, simulation/organic_aux.h:7
    return omega + std::pow(2 * std::sin(matsubara * k), 2) / omega;
}

// host mode table -> device scratch (pageable copy: the source is consumed before return)
// what each scratch buffer's table region holds (upload cache, see fa_forget_tables)
std::mutex g_tab_mu;
std::map<const double *, std::vector<double>> g_tab;

int upload_modes(const std::vector<double> &h, double *scratch, cudaStream_t st, double **out) {
    *out = scratch;
    {
        std::lock_guard<std::mutex> l(g_tab_mu);
        auto it = g_tab.find(scratch);
        if (it != g_tab.end() && it->second == h && !uploads_are_uncached()) return EPHMC_OK;
    }
    if (int e = upload_small(scratch, h.data(), sizeof(double) * h.size(), st)) return e;
    std::lock_guard<std::mutex> l(g_tab_mu);
    g_tab[scratch] = h;
    return EPHMC_OK;
}

}  // namespace

void fa_forget_tables(const double *scratch) {
    std::lock_guard<std::mutex> l(g_tab_mu);
    g_tab.erase(scratch);
}

int fa_evolve(double *x, double *p, int ld, int n, double omega, double h, double *scratch, cudaStream_t st) {
    if (n < 1 || n > 512) return EPHMC_ERR_UNSUPPORTED;
    const int nc = n / 2 + 1;
    const double c = std::cos(h) / n, s = std::sin(h) / n;  // :131
    std::vector<double> tab(2 * nc);
    for (int k = 0; k < nc; ++k) {
        const double f2 = freq2(omega, k, n);
        tab[k] = s / f2;       // s1w
        tab[nc + k] = s * f2;  // sw
    }
    double *d = nullptr;
    int rc = upload_modes(tab, scratch, st, &d);
    if (rc) return rc;
    const size_t smem = fa_smem(n, true);
    EPHMC_CUDA(cudaFuncSetAttribute(k_fa, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_fa<<<(ld + kTile - 1) / kTile, dim3(kTile, kRowsY), smem, st>>>(x, p, ld, n, d, d + nc, c, 0); ephmc::count_launch(1);
    EPHMC_CUDA(cudaGetLastError());
    return EPHMC_OK;
}

// x <- x + inverse transform of (h / freq2_k) P_k, normalised by 1/n
// (evolve_bosons_approx_step, simulation/organic_bosons.c:152-177); omega is
// the accelerated frequency sqrt(cfa_mass^2 + omega^2) the caller passes
int fa_approx_step(double *x, const double *p, int ld, int n, double omega, double h, double *scratch,
                   cudaStream_t st) {
    if (n < 1 || n > 512) return EPHMC_ERR_UNSUPPORTED;
    const int nc = n / 2 + 1;
    std::vector<double> tab(nc);
    for (int k = 0; k < nc; ++k) tab[k] = h / freq2(omega, k, n);  // inv_mass (:167)
    double *d = nullptr;
    int rc = upload_modes(tab, scratch, st, &d);
    if (rc) return rc;
    const size_t smem = fa_smem(n, true);
    EPHMC_CUDA(cudaFuncSetAttribute(k_fa, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_fa<<<(ld + kTile - 1) / kTile, dim3(kTile, kRowsY), smem, st>>>(x, const_cast<double *>(p), ld, n, d, d,
                                                                      1.0 / n, 3);
    ephmc::count_launch(1);
    EPHMC_CUDA(cudaGetLastError());
    return EPHMC_OK;
}

// mode 1: momenta, amplitude sqrt(freq2)/n (:88-96); mode 2: free bosons, 1/sqrt(freq2)/n (:62-70)
int fa_scale_modes(double *v, int ld, int n, double omega, int mode, double *scratch, cudaStream_t st) {
    if (n < 1 || n > 512) return EPHMC_ERR_UNSUPPORTED;
    const int nc = n / 2 + 1;
    std::vector<double> tab(nc);
    for (int k = 0; k < nc; ++k) {
        const double fr = std::sqrt(freq2(omega, k, n));
        tab[k] = (mode == 1) ? fr / n : 1. / fr / n;
    }
    double *d = nullptr;
    int rc = upload_modes(tab, scratch, st, &d);
    if (rc) return rc;
    const size_t smem = fa_smem(n, true);
    EPHMC_CUDA(cudaFuncSetAttribute(k_fa, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    if (mode == 1) k_fa<<<(ld + kTile - 1) / kTile, dim3(kTile, kRowsY), smem, st>>>(nullptr, v, ld, n, d, d, 0.0, 1);
    else k_fa<<<(ld + kTile - 1) / kTile, dim3(kTile, kRowsY), smem, st>>>(v, nullptr, ld, n, d, d, 0.0, 2);
    ephmc::count_launch(1);
    EPHMC_CUDA(cudaGetLastError());
    return EPHMC_OK;
}

// sum_k |P_k|^2 * 0.5 / n / freq2_k, doubled for 0 < k < (n+1)/2 (:102-124); result in out_dev[0]
int fa_energy(const double *p, int ld, int n, double omega, double *out_dev, double *scratch, cudaStream_t st) {
    if (n < 1 || n > 512) return EPHMC_ERR_UNSUPPORTED;
    const int nc = n / 2 + 1, center = (n + 1) / 2;
    const int nblk = (ld + kTile - 1) / kTile;
    std::vector<double> tab(nc);  // the per-CTA partials follow at d + nc (written, not accumulated)
    for (int k = 0; k < nc; ++k) {
        double w = .5 / n / freq2(omega, k, n);
        if (k > 0 && k < center) w *= 2;
        tab[k] = w;
    }
    double *d = nullptr;
    int rc = upload_modes(tab, scratch, st, &d);
    if (rc) return rc;
    const int nc2 = n / 2 + 1;
    const size_t smem = sizeof(double) * (2 * (size_t)n + (size_t)n * kTile + 2 * (size_t)nc2 * kTile);
    EPHMC_CUDA(cudaFuncSetAttribute(k_fa_energy, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_fa_energy<<<nblk, dim3(kTile, kRowsY), smem, st>>>(p, ld, n, d, d + nc); ephmc::count_launch(1);
    EPHMC_CUDA(cudaGetLastError());
    k_sum<<<1, 256, 0, st>>>(d + nc, nblk, out_dev); ephmc::count_launch(1);
    EPHMC_CUDA(cudaGetLastError());
    return EPHMC_OK;
}

}  // namespace ephmc

namespace ephmc {
size_t fa_scratch_doubles(int ld, int nt) { return 2 * (size_t)(nt / 2 + 1) + (size_t)(ld + 31) / 32 + 8; }
}  // namespace ephmc
