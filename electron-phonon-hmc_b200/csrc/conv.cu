// Smearing of the static-disorder histograms (optical conductivity) and their
// transform to Euclidean time: the computations of organic_conv
// (simulation/organic_conv.c:9-115), one GPU thread per output entry.
//
//   sigma_w(omega; width)  = pi/2 tanhc(omega/2) h sum_i sigma_i [L(omega - i h) + L(omega + i h)]
//                            L = Lorentzian of half-width `width` (:78-90, :96-111);
//                            width 0: the bin of omega, unsmeared
//   sigma_t(t; width)      = h sum_i sigma_i K(t, i h, width)          (:113-121)
//                            K: the tanh-sinh integral of calc_integral_sigma
//                            (:19-49) / pi, or the Matsubara sum of
//                            matsubara_integral (:51-63) when nt_matsubara > 0
//
// The sums over bins run in the reference's order, one thread per output
// entry; the quadrature terms of sigma_t are computed in parallel first, one
// thread per (t, width, bin).
#include "ephmc_internal.cuh"

#include <cmath>
#include <vector>

namespace ephmc {

namespace {

// the reference's constants (simulation/organic_aux.h:7-10)
constexpr double kPi = 3.141592653589793;
constexpr double kHalfPi = 1.570796326794897;

__device__ double d_tanhc(double x) { return x != 0.0 ? tanh(x) / x : 1.0; }

// sigma_of_w (:9-17)
__device__ double d_sigma_of_w(double w, double t, double omega, double width) {
    const double effW = -(w * width + omega);
    t *= effW;
    return exp(t) / (1 + w * w) * (1 + exp(effW - 2 * t)) / (1 + exp(effW));
}

// calc_integral_sigma (:19-49): tanh-sinh quadrature, step 0.03, at most 200
// nodes, stopped at the first term below DBL_EPSILON of the running sum
__device__ double d_integral_sigma(double t, double omega, double width) {
    if (t > .5) t = 1 - t;
    if (t == 0) return kPi;
    const double h = 0.03;
    double sum = kHalfPi * d_sigma_of_w(0, t, omega, width);
    for (unsigned i = 1; i < 200; i++) {
        const double x = i * h;
        const double sh_x = kHalfPi * sinh(x);
        const double ch_x = kHalfPi * cosh(x);
        const double ch_sh_x = cosh(sh_x);
        const double w = sinh(sh_x);
        const double val = d_sigma_of_w(w, t, omega, width) + d_sigma_of_w(w, t, -omega, width);
        const double term = val * (ch_x * ch_sh_x);
        if (term >= 2.220446049250313e-16 * sum)
            sum += term;
        else
            break;
    }
    return h * sum;
}

// matsubara_integral (:51-63): Re[cos(z (t - 1/2)) / cos(z/2)] + sum over
// fermionic frequencies, z = width + i omega
__device__ double d_matsubara(double t, double omega, double width, unsigned nt) {
    // cos(a + ib) = cos a cosh b - i sin a sinh b
    const double a1 = width * (t - .5), b1 = omega * (t - .5);
    const double nr = cos(a1) * cosh(b1), ni = -sin(a1) * sinh(b1);
    const double a2 = .5 * width, b2 = .5 * omega;
    const double dr = cos(a2) * cosh(b2), di = -sin(a2) * sinh(b2);
    const double den = dr * dr + di * di;
    double sum = (nr * dr + ni * di) / den;
    for (unsigned i = 0; i < nt; i++) {
        const double freq = (2 * i + 1) * kPi;
        // 4 width sin(freq t) / (width^2 + (i freq - omega)^2), real part
        const double dre = width * width + omega * omega - freq * freq, dim = -2 * freq * omega;
        const double num = 4 * width * sin(freq * t);
        sum += num * dre / (dre * dre + dim * dim);
    }
    return sum;
}

// eval_GK_kernel (:65-75)
__device__ double d_gk_kernel(double t, double omega, double width, unsigned nt) {
    if (nt) return d_matsubara(t, omega, width, nt);
    if (width == 0) return d_sigma_of_w(0, t, omega, 1);
    return d_integral_sigma(t, omega, width) / kPi;
}

__device__ double d_lorentz(double x, double width) { return width / (kPi * (width * width + x * x)); }

// out[i][k] = smeared_sigma_w(i h, sigma, widths[k], h, n) (:92-111)
__global__ void k_conv_w(const double *__restrict__ sigma, int n, double h, const double *__restrict__ widths,
                         int ns, double *__restrict__ out) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n * ns) return;
    const int i = e / ns, k = e % ns;
    const double omega = i * h, width = widths[k];
    double r;
    if (width == 0) {
        const unsigned bin = (unsigned)(omega / h + .5);
        const double s = bin < (unsigned)n ? sigma[bin] : 0.0;
        r = bin == 0 ? s : kPi * .5 * d_tanhc(.5 * omega) * s;
    } else {
        double sum = 0;
        for (int b = 0; b < n; b++) {
            const double x0 = b * h;
            sum += sigma[b] * (d_lorentz(omega - x0, width) + d_lorentz(omega + x0, width));
        }
        r = kPi * .5 * d_tanhc(.5 * omega) * h * sum;
    }
    out[e] = r;
}

// terms[(it*ns + k)*n + b] = sigma[b] * eval_GK_kernel(it/nt, b h, widths[k], nt_m)
__global__ void k_conv_t_terms(const double *__restrict__ sigma, int n, double h, const double *__restrict__ widths,
                               int ns, int nt, int nrows, unsigned nt_m, double *__restrict__ terms) {
    const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (size_t)nrows * ns * n) return;
    const int b = (int)(e % n);
    const int k = (int)((e / n) % ns);
    const int it = (int)(e / ((size_t)n * ns));
    const double t = (double)it / nt;
    terms[e] = sigma[b] * d_gk_kernel(t, b * h, widths[k], nt_m);
}

// out[it][k] = h * (sum over b in order of terms)
__global__ void k_conv_t_sum(const double *__restrict__ terms, int n, double h, int nout, double *__restrict__ out) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nout) return;
    const double *p = terms + (size_t)e * n;
    double sum = 0;
    for (int b = 0; b < n; b++) sum += p[b];
    out[e] = h * sum;
}

// device copies of the inputs and the output buffer of one call
struct ConvBufs {
    double *sigma = nullptr, *widths = nullptr, *out = nullptr, *terms = nullptr;
    ~ConvBufs() {
        cudaFree(sigma);
        cudaFree(widths);
        cudaFree(out);
        cudaFree(terms);
    }
};

int conv_upload(ConvBufs &b, const double *sigma, unsigned n, const double *widths, unsigned ns, size_t nout,
                size_t nterms) {
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        set_status(EPHMC_ERR_NO_DEVICE, "no CUDA device");
        return EPHMC_ERR_NO_DEVICE;
    }
    if (cudaMalloc(&b.sigma, sizeof(double) * n) != cudaSuccess ||
        cudaMalloc(&b.widths, sizeof(double) * ns) != cudaSuccess ||
        cudaMalloc(&b.out, sizeof(double) * nout) != cudaSuccess ||
        (nterms && cudaMalloc(&b.terms, sizeof(double) * nterms) != cudaSuccess)) {
        cudaGetLastError();
        set_status(EPHMC_ERR_NOMEM, "conv: device allocation");
        return EPHMC_ERR_NOMEM;
    }
    EPHMC_CUDA(cudaMemcpy(b.sigma, sigma, sizeof(double) * n, cudaMemcpyDefault));
    EPHMC_CUDA(cudaMemcpy(b.widths, widths, sizeof(double) * ns, cudaMemcpyDefault));
    return EPHMC_OK;
}

}  // namespace

}  // namespace ephmc

using namespace ephmc;

extern "C" {

EPHMC_API int ephmc_conv_sigma_w(const double *sigma, unsigned n, double h, const double *widths, unsigned n_smear,
                                 double *out) {
    clear_status();
    if (!sigma || !widths || !out || n == 0 || n_smear == 0 || !(h > 0)) {
        set_status(EPHMC_ERR_ARG, "ephmc_conv_sigma_w arguments");
        return EPHMC_ERR_ARG;
    }
    const size_t nout = (size_t)n * n_smear;
    if (nout > (size_t)INT32_MAX) {
        set_status(EPHMC_ERR_ARG, "ephmc_conv_sigma_w: output too large");
        return EPHMC_ERR_ARG;
    }
    ConvBufs b;
    if (conv_upload(b, sigma, n, widths, n_smear, nout, 0) != EPHMC_OK) return last_status();
    k_conv_w<<<(unsigned)((nout + 255) / 256), 256>>>(b.sigma, (int)n, h, b.widths, (int)n_smear, b.out);
    count_launch(1);
    EPHMC_CUDA(cudaGetLastError());
    EPHMC_CUDA(cudaMemcpy(out, b.out, sizeof(double) * nout, cudaMemcpyDefault));
    return EPHMC_OK;
}

EPHMC_API int ephmc_conv_sigma_t(const double *sigma, unsigned n, double h, const double *widths, unsigned n_smear,
                                 unsigned nt, unsigned nt_matsubara, double *out) {
    clear_status();
    if (!sigma || !widths || !out || n == 0 || n_smear == 0 || nt == 0 || !(h > 0)) {
        set_status(EPHMC_ERR_ARG, "ephmc_conv_sigma_t arguments");
        return EPHMC_ERR_ARG;
    }
    const unsigned nrows = nt / 2 + 1;
    const size_t nout = (size_t)nrows * n_smear, nterms = nout * n;
    if (nterms > ((size_t)1 << 31)) {
        set_status(EPHMC_ERR_ARG, "ephmc_conv_sigma_t: (nt/2+1) * widths * bins too large");
        return EPHMC_ERR_ARG;
    }
    ConvBufs b;
    if (conv_upload(b, sigma, n, widths, n_smear, nout, nterms) != EPHMC_OK) return last_status();
    k_conv_t_terms<<<(unsigned)((nterms + 255) / 256), 256>>>(b.sigma, (int)n, h, b.widths, (int)n_smear, (int)nt,
                                                              (int)nrows, nt_matsubara, b.terms);
    count_launch(1);
    EPHMC_CUDA(cudaGetLastError());
    k_conv_t_sum<<<(unsigned)((nout + 255) / 256), 256>>>(b.terms, (int)n, h, (int)nout, b.out);
    count_launch(1);
    EPHMC_CUDA(cudaGetLastError());
    EPHMC_CUDA(cudaMemcpy(out, b.out, sizeof(double) * nout, cudaMemcpyDefault));
    return EPHMC_OK;
}

}  // extern "C"
