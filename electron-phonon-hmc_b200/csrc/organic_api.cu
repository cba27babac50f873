// Drop-in surface: the reference's function names and prototypes
// (simulation/organic_dense_matrix.h, organic_hmc.h, organic_bosons.h) over the
// library's device contexts.  Declarations: include/ephmc_organic.h.
//
// Contexts are created on first use per (device, lattice, Nt) and kept; the
// couplings and flags of every call are applied before it runs.  Caller
// pointers are used in place when they are device memory and staged through
// the context otherwise, so the reference's own host code runs unchanged.
#include "ephmc_internal.cuh"
#include "../../include/ephmc_organic.h"

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

using namespace ephmc;

// The host program's own MT19937-64 stream, when it links the reference's
// mt19937-64.o / organic_random.o; otherwise the library's copy below.
extern "C" {
void init_genrand64(unsigned long seed) __attribute__((weak));
double genrand64_real2(void) __attribute__((weak));
void random_vector(double *x, unsigned N) __attribute__((weak));
}

struct fftw_plan_s {
    int kind;  // 0 r2c, 1 c2r
    int n, howmany;
    void *in, *out;
};

namespace {

// ---------------------------------------------------------------- RNG
// Published 64-bit Mersenne Twister (Nishimura 2000), the generator of
// simulation/mt19937-64.c, and the Box-Muller pairs of random_vector
// (simulation/organic_random.c:11-22).
struct MT64 {
    static constexpr int N = 312, M = 156;
    uint64_t s[N];
    int pos = N + 1;
    void seed(uint64_t v) {
        s[0] = v;
        for (int i = 1; i < N; ++i) s[i] = 6364136223846793005ULL * (s[i - 1] ^ (s[i - 1] >> 62)) + (uint64_t)i;
        pos = N;
    }
    uint64_t next() {
        if (pos >= N) {
            if (pos == N + 1) seed(5489ULL);
            for (int i = 0; i < N; ++i) {
                const uint64_t y = (s[i] & 0xFFFFFFFF80000000ULL) | (s[(i + 1) % N] & 0x7FFFFFFFULL);
                uint64_t v = s[(i + M) % N] ^ (y >> 1);
                if (y & 1ULL) v ^= 0xB5026F5AA96619E9ULL;
                s[i] = v;
            }
            pos = 0;
        }
        uint64_t z = s[pos++];
        z ^= (z >> 29) & 0x5555555555555555ULL;
        z ^= (z << 17) & 0x71D67FFFEDA60000ULL;
        z ^= (z << 37) & 0xFFF7EEE000000000ULL;
        z ^= z >> 43;
        return z;
    }
    double real2() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
};
MT64 g_mt;
std::mutex g_rng_mu;

void rng_seed(unsigned long long s) {
    if (init_genrand64) init_genrand64((unsigned long)s);
    else {
        std::lock_guard<std::mutex> l(g_rng_mu);
        g_mt.seed(s);
    }
}
double rng_real2() {
    if (genrand64_real2) return genrand64_real2();
    std::lock_guard<std::mutex> l(g_rng_mu);
    return g_mt.real2();
}
void rng_normals(double *x, unsigned n) {
    if (random_vector) {
        random_vector(x, n);
        return;
    }
    for (unsigned k = 0; k < n; k += 2) {
        const double u1 = std::sqrt(-2 * std::log(rng_real2()));
        const double u2 = 6.283185307179586 * rng_real2();  // M_2PI, simulation/organic_aux.h:9
        x[k] = u1 * std::cos(u2);
        x[(k + 1) % n] = u1 * std::sin(u2);
    }
}

// ---------------------------------------------------------------- context registry
std::mutex g_reg_mu;
std::map<std::tuple<int, unsigned, unsigned, uint64_t>, ephmc_ctx *> g_reg;
int g_dropin_mode = EPHMC_FORCE_REFERENCE;

uint64_t hash_nnt(const unsigned *nnt, unsigned ns) {
    uint64_t h = 1469598103934665603ULL;
    for (size_t i = 0; i < 12 * (size_t)ns; ++i) {
        h ^= nnt[i];
        h *= 1099511628211ULL;
    }
    return h;
}

bool devp(const void *p) {
    if (!p) return false;
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

// neighbour table: host copy of a caller's table (host or device)
std::vector<unsigned> host_nnt(const unsigned *nnt, unsigned ns) {
    std::vector<unsigned> h(12 * (size_t)ns);
    if (devp(nnt)) cudaMemcpy(h.data(), nnt, sizeof(unsigned) * h.size(), cudaMemcpyDeviceToHost);
    else std::memcpy(h.data(), nnt, sizeof(unsigned) * h.size());
    return h;
}

ephmc_ctx *get_ctx(const unsigned *nnt, unsigned ns, unsigned nt, const double *t, const double *kappa, double mu,
                   double omega, unsigned flavors, const organic_flags *mode) {
    int dev = 0;
    cudaGetDevice(&dev);
    const std::vector<unsigned> h = host_nnt(nnt, ns);
    const auto key = std::make_tuple(dev, ns, nt, hash_nnt(h.data(), ns));
    double tt[3] = {0, 0, 0}, kk[3] = {0, 0, 0};
    if (t)
        for (int k = 0; k < 3; ++k) tt[k] = t[k];
    if (kappa)
        for (int k = 0; k < 3; ++k) kk[k] = kappa[k];
    ephmc_ctx *c = nullptr;
    {
        std::lock_guard<std::mutex> l(g_reg_mu);
        auto it = g_reg.find(key);
        if (it != g_reg.end()) c = it->second;
    }
    if (!c) {
        if (ephmc_ctx_create_nnt(&c, h.data(), ns, nt, tt, kk, mu, omega, flavors, mode, dev) != EPHMC_OK) {
            std::fprintf(stderr, "ephmc: %s\n", ephmc_last_error_message());
            return nullptr;
        }
        std::lock_guard<std::mutex> l(g_reg_mu);
        g_reg[key] = c;
    }
    ephmc_ctx_set_params(c, tt, kk, mu, omega, flavors);
    ephmc_ctx_set_flags(c, mode);
    return c;
}

// slice-level context (Nt = 1) for functions that see one slice of fields
ephmc_ctx *slice_ctx(const unsigned *nnt, unsigned ns, const double *t, const double *kappa, double mu) {
    return get_ctx(nnt, ns, 1, t, kappa, mu, 0.0, 1, nullptr);
}

// a periodic triangular lattice table for functions that only see ns (the
// neighbour table does not enter them): the L1 = ns, L2 = 1 ring
std::vector<unsigned> &ring_nnt(unsigned ns) {
    static thread_local std::map<unsigned, std::vector<unsigned>> cache;
    auto &v = cache[ns];
    if (v.empty()) {
        v.resize(12 * (size_t)ns);
        triangular_lattice(ns, 1, v.data());
    }
    return v;
}

ephmc_ctx *lu_ctx(unsigned ns) {
    auto &r = ring_nnt(ns);
    const double z[3] = {0, 0, 0};
    return get_ctx(r.data(), ns, 1, z, z, 0.0, 0.0, 1, nullptr);
}

void report(const char *fn) {
    std::fprintf(stderr, "ephmc %s: %s\n", fn, ephmc_last_error_message());
}

// device view of n doubles of a caller pointer; copied back by sync() if host
struct DView {
    double *user = nullptr, *d = nullptr;
    size_t n = 0;
    bool owned = false;
    DView() = default;
    DView(double *u, size_t count) : user(u), n(count) {
        if (!u) return;
        if (devp(u)) {
            d = u;
        } else {
            if (cudaMalloc(&d, sizeof(double) * n) != cudaSuccess) {
                cudaGetLastError();
                d = nullptr;
                return;
            }
            owned = true;
            cudaMemcpy(d, u, sizeof(double) * n, cudaMemcpyHostToDevice);
        }
    }
    DView(const DView &) = delete;
    DView &operator=(const DView &) = delete;
    void back() {
        if (owned && d) cudaMemcpy(user, d, sizeof(double) * n, cudaMemcpyDeviceToHost);
    }
    ~DView() {
        if (owned && d) cudaFree(d);
    }
};

// --------------------------------------------------------------- contractions of the correlator output
// contr_gr_mat / contr_gr_triangle / contract_greens (simulation/organic_lattice.c:62-106)
double contract_greens_h(const double *gr, const double *mat, unsigned nn, unsigned tau) {
    const unsigned n = nn / 2;
    const double *g = gr + (size_t)n * n * tau;
    if (mat) {
        double contr = 0;
        for (unsigned c = 0; c < 2; ++c) {
            double sum = 0;
            for (unsigned a = 0; a < n; ++a) sum += mat[c * n + a] * g[a];
            contr += sum * sum;
        }
        return contr;
    }
    double contr = 0;
    for (unsigned a = 0; a < n; ++a)
        for (unsigned b = 0; b <= a; ++b) contr += g[a * n + b] + g[b * n + a];
    contr *= .5;
    contr -= g[n - 1] + g[(n - 1) * n];
    return contr;
}

}  // namespace

extern "C" {

// ================================================================== RNG / plans / mode
void ephmc_rng_seed(unsigned long long seed) { rng_seed(seed); }
double ephmc_rng_real2(void) { return rng_real2(); }
void ephmc_random_vector(double *x, unsigned n) { rng_normals(x, n); }
void ephmc_set_dropin_force_mode(int m) { g_dropin_mode = m; }

fftw_plan ephmc_fftw_plan_many_dft_r2c(int rank, const int *n, int howmany, double *in, const int *, int, int,
                                       ephmc_dcomplex *out, const int *, int, int, unsigned) {
    if (rank != 1 || !n) return nullptr;
    return new fftw_plan_s{0, n[0], howmany, in, out};
}
fftw_plan ephmc_fftw_plan_many_dft_c2r(int rank, const int *n, int howmany, ephmc_dcomplex *in, const int *, int, int,
                                       double *out, const int *, int, int, unsigned) {
    if (rank != 1 || !n) return nullptr;
    return new fftw_plan_s{1, n[0], howmany, in, out};
}
void ephmc_fftw_destroy_plan(fftw_plan p) { delete p; }

// ================================================================== organic_dense_matrix.h
// mat_mul (simulation/organic_dense_matrix.c:27-32)
void mat_mul(double *m, double *x, double *y, unsigned n) {
    DView M(m, (size_t)n * n), X(x, n), Y(y, n);
    launch_matvec(M.d, X.d, Y.d, (int)n, false, 0);
    cudaDeviceSynchronize();
    Y.back();
}
// mat_mul_tr (:34-38)
void mat_mul_tr(double *m, double *x, double *y, unsigned n) {
    DView M(m, (size_t)n * n), X(x, n), Y(y, n);
    launch_matvec(M.d, X.d, Y.d, (int)n, true, 0);
    cudaDeviceSynchronize();
    Y.back();
}
// mat_mat_mul (:40-45): every row of m2 replaced by m1 * row; y ends holding the last row
void mat_mat_mul(double *m1, double *m2, double *y, unsigned n) {
    DView A(m1, (size_t)n * n), B(m2, (size_t)n * n), Y(y, n);
    double *tmp = nullptr;
    if (cudaMalloc(&tmp, sizeof(double) * (size_t)n * n) != cudaSuccess) return;
    launch_matmat_rows(A.d, B.d, tmp, (int)n, 0);
    cudaMemcpy(B.d, tmp, sizeof(double) * (size_t)n * n, cudaMemcpyDeviceToDevice);
    cudaMemcpy(Y.d, tmp + (size_t)(n - 1) * n, sizeof(double) * n, cudaMemcpyDeviceToDevice);
    cudaFree(tmp);
    B.back();
    Y.back();
}
// construct_id (:47-55)
void construct_id(double *m, unsigned n) {
    DView M(m, (size_t)n * n);
    launch_identity(M.d, (int)n, 0);
    cudaDeviceSynchronize();
    M.back();
}
// transpose (:57-71)
void transpose(double *m, unsigned n) {
    DView M(m, (size_t)n * n);
    launch_transpose(M.d, (int)n, 0);
    cudaDeviceSynchronize();
    M.back();
}
// transpose_rect (:73-85)
void transpose_rect(double *x, double *y, unsigned n1, unsigned n2) {
    DView X(x, (size_t)n1 * n2), Y(y, (size_t)n1 * n2);
    launch_transpose_rect(X.d, Y.d, (int)n1, (int)n2, 0);
    cudaDeviceSynchronize();
    Y.back();
}
// trace (:87-93)
double trace(double *m, unsigned n) {
    DView M(m, (size_t)n * n);
    double *o = nullptr;
    if (cudaMalloc(&o, sizeof(double)) != cudaSuccess) return NAN;
    launch_trace(M.d, (int)n, o, 0);
    double v = 0;
    cudaMemcpy(&v, o, sizeof(double), cudaMemcpyDeviceToHost);
    cudaFree(o);
    return v;
}
// apply_mu_K_to_v (:96-120)
void apply_mu_K_to_v(double *x, double *v, double *w, double *t, double *kappa, double mu, unsigned *nnt, unsigned ns,
                     unsigned) {
    ephmc_ctx *c = slice_ctx(nnt, ns, t, kappa, mu);
    if (!c || ephmc_apply_stencil_rows(c, x, v, w, 1, 0) != EPHMC_OK) report("apply_mu_K_to_v");
}
// apply_mu_K_to_M (:123-131): every row replaced by (mu + K) row; w receives the same rows
void apply_mu_K_to_M(double *x, double *M, double *w, double *t, double *kappa, double mu, unsigned *nnt, unsigned ns,
                     unsigned) {
    ephmc_ctx *c = slice_ctx(nnt, ns, t, kappa, mu);
    if (!c) return report("apply_mu_K_to_M");
    const size_t VV = (size_t)ns * ns;
    DView Md(M, VV);
    if (ephmc_apply_stencil_rows(c, x, Md.d, c->work + 2 * VV, ns, 0) != EPHMC_OK) return report("apply_mu_K_to_M");
    cudaMemcpy(Md.d, c->work + 2 * VV, sizeof(double) * VV, cudaMemcpyDeviceToDevice);
    if (w) {
        if (devp(w)) cudaMemcpy(w, Md.d, sizeof(double) * VV, cudaMemcpyDeviceToDevice);
        else cudaMemcpy(w, Md.d, sizeof(double) * VV, cudaMemcpyDeviceToHost);
    }
    Md.back();
}
// set_taylor_pair_order (:133-159): the order is fixed at library load ({0,1} for two pairs)
void set_taylor_pair_order(void) {}
// apply_K_plus_1_v (:162-166): w = (mu+K) v, v += w
void apply_K_plus_1_v(double *x, double *v, double *w, double *t, double *kappa, double mu, unsigned *nnt, unsigned ns,
                      unsigned nn) {
    apply_mu_K_to_v(x, v, w, t, kappa, mu, nnt, ns, nn);
    DView V(v, ns), W(w, ns);
    launch_axpy(V.d, W.d, 1.0, ns, 0);
    cudaDeviceSynchronize();
    V.back();
}
// apply_2nd_order_mu_K_to_v (:168-183): v += 2 Re(a) Hv + |a|^2 H^2 v; w = Hv, w+ns = H^2 v
void apply_2nd_order_mu_K_to_v(double *x, double *v, double *w, double *t, double *kappa, double mu, unsigned *nnt,
                               unsigned ns, unsigned nn, ephmc_dcomplex a) {
    const double re = __real__ a, im = __imag__ a;
    const double a_lin = 2 * re, a_quad = std::pow(std::hypot(re, im), 2);
    apply_mu_K_to_v(x, v, w, t, kappa, mu, nnt, ns, nn);
    DView V(v, ns), W(w, 2 * (size_t)ns);
    if (im != 0) {
        ephmc_ctx *c = slice_ctx(nnt, ns, t, kappa, mu);
        if (!c) return;
        ephmc_apply_stencil_rows(c, x, W.d, W.d + ns, 1, 0);
        launch_pair_combine(V.d, W.d, W.d + ns, a_lin, a_quad, ns, 0);  // v + fma(a_lin, w, a_quad z)
        cudaDeviceSynchronize();
    } else {
        launch_axpy(V.d, W.d, a_lin, ns, 0);
        cudaDeviceSynchronize();
    }
    V.back();
    W.back();
}
// apply_pair_expansion_mu_K_to_v / apply_exp_mu_K_to_v (:186-207)
void apply_pair_expansion_mu_K_to_v(double *x, double *v, double *w, double *t, double *kappa, double mu, unsigned *nnt,
                                    unsigned ns, unsigned, int revert, int stop) {
    ephmc_ctx *c = slice_ctx(nnt, ns, t, kappa, mu);
    (void)w;
    if (!c || ephmc_apply_exp_rows(c, x, v, 1, revert, stop) != EPHMC_OK) report("apply_pair_expansion_mu_K_to_v");
}
void apply_exp_mu_K_to_v(double *x, double *v, double *w, double *t, double *kappa, double mu, unsigned *nnt,
                         unsigned ns, unsigned nn, int revert, int stop) {
    apply_pair_expansion_mu_K_to_v(x, v, w, t, kappa, mu, nnt, ns, nn, revert, stop);
}
// apply_exp_mu_K_to_M (:209-216)
void apply_exp_mu_K_to_M(double *x, double *M, double *w, double *t, double *kappa, double mu, unsigned *nnt,
                         unsigned ns, unsigned, int revert, int stop) {
    ephmc_ctx *c = slice_ctx(nnt, ns, t, kappa, mu);
    (void)w;
    if (!c || ephmc_apply_exp_rows(c, x, M, ns, revert, stop) != EPHMC_OK) report("apply_exp_mu_K_to_M");
}
// construct_hamilton (:218-224): ham = (mu + K) applied to the identity
void construct_hamilton(double *x, double *ham, double *w, double *t, double *kappa, double mu, unsigned *nnt,
                        unsigned ns, unsigned nn) {
    construct_id(ham, ns);
    apply_mu_K_to_M(x, ham, w, t, kappa, mu, nnt, ns, nn);
}
// apply_current_to_v (:226-249)
void apply_current_to_v(double *x, double *v, double *w, double *t, double *kappa, unsigned *nnt, unsigned ns,
                        unsigned, unsigned k) {
    ephmc_ctx *c = slice_ctx(nnt, ns, t, kappa, 0.0);
    if (!c || ephmc_apply_current(c, x, v, w, k) != EPHMC_OK) report("apply_current_to_v");
}
// construct_M_hat (:251-265)
void construct_M_hat(double *x, double *M_hat, double *w, double *t, double *kappa, double mu, unsigned *nnt,
                     unsigned ns, unsigned, unsigned nt, organic_flags *mode) {
    (void)w;
    ephmc_ctx *c = get_ctx(nnt, ns, nt, t, kappa, mu, 0.0, 1, mode);
    if (!c || ephmc_construct_M_hat(c, x, M_hat) != EPHMC_OK) report("construct_M_hat");
}
// construct_QM1P (:267-309): G at one slice, refined
void construct_QM1P(double *x, double *M_hat, double *QM1P, double *w, double *t, double *kappa, double mu,
                    unsigned *nnt, unsigned ns, unsigned nn, unsigned nt, int time, organic_flags *mode) {
    (void)w;
    (void)nn;
    if (mode && mode->schur_form_inv) {
        // the Schur branch (:270-279): 1 - M_hat^-1, or M_hat itself with SINGLE_PARTICLE
        const size_t VV = (size_t)ns * ns;
        DView G(QM1P, VV), M(M_hat, VV);
        if (!G.d || !M.d) return report("construct_QM1P");
        if (mode->single_particle)
            cudaMemcpy(G.d, M.d, sizeof(double) * VV, cudaMemcpyDeviceToDevice);
        else if (launch_one_minus(G.d, M.d, (int)ns, 0) != EPHMC_OK)
            return report("construct_QM1P");
        cudaDeviceSynchronize();
        G.back();
        return;
    }
    ephmc_ctx *c = get_ctx(nnt, ns, nt, t, kappa, mu, 0.0, 1, mode);
    if (!c) return report("construct_QM1P");
    const size_t VV = (size_t)ns * ns, dim = (size_t)nt * ns * 3;
    DView X(x, dim), G(QM1P, VV);
    if (mode && mode->single_particle) launch_identity(G.d, (int)ns, 0);
    else {
        DView Mi(M_hat, VV);
        cudaMemcpy(G.d, Mi.d, sizeof(double) * VV, cudaMemcpyDeviceToDevice);
    }
    std::vector<SliceJob> jobs;
    const int after = (int)nt - 1 - time;
    SliceJob j{};
    j.src = G.d;
    j.dst = G.d;
    j.s_first = (int)nt - 1;
    j.s_count = after;
    j.s_dir = -1;
    j.p_begin = 0;
    j.p_end = kPairs;
    j.p_step = 1;
    if (after > 0) {
        ctx_upload_jobs(c, &j, 1, 0, 0);
        launch_slices<double, double, double>(Axis::Rows, X.d, c->c, c->lat, c->jobs, 1, 0);
    }
    if (time > 0) {
        j.s_first = 0;
        j.s_count = time;
        j.s_dir = 1;
        ctx_upload_jobs(c, &j, 1, 0, 0);
        launch_slices<double, double, double>(Axis::Cols, X.d, c->c, c->lat, c->jobs, 1, 0);
    }
    cudaDeviceSynchronize();
    if (ephmc_refine_G(c, X.d, G.d, (unsigned)time) != EPHMC_OK) return report("construct_QM1P");
    G.back();
}
// construct_all_QM1P (:311-381)
void construct_all_QM1P(double *x, double *M_hat, double *QM1P, double *w, int *perm, double *t, double *kappa,
                        double mu, unsigned *nnt, unsigned ns, unsigned, unsigned nt, organic_flags *mode) {
    (void)w;
    ephmc_ctx *c = get_ctx(nnt, ns, nt, t, kappa, mu, 0.0, 1, mode);
    std::vector<int> pm(2 * (size_t)nt);
    if (!c || ephmc_all_G(c, x, M_hat, QM1P, pm.data()) != EPHMC_OK) return report("construct_all_QM1P");
    if (perm) {
        if (devp(perm)) cudaMemcpy(perm, pm.data(), sizeof(int) * pm.size(), cudaMemcpyHostToDevice);
        else std::memcpy(perm, pm.data(), sizeof(int) * pm.size());
    }
}
// refine_QM1P (:383-442)
void refine_QM1P(double *x, double *QM1P, double *w, double *t, double *kappa, double mu, unsigned *nnt, unsigned ns,
                 unsigned, int time) {
    (void)w;
    ephmc_ctx *c = slice_ctx(nnt, ns, t, kappa, mu);
    if (!c) return report("refine_QM1P");
    const size_t ld = 3 * (size_t)ns;
    std::vector<double> xs(ld);
    if (devp(x)) cudaMemcpy(xs.data(), x + (size_t)time * ld, sizeof(double) * ld, cudaMemcpyDeviceToHost);
    else std::memcpy(xs.data(), x + (size_t)time * ld, sizeof(double) * ld);
    if (ephmc_refine_G(c, xs.data(), QM1P, 0) != EPHMC_OK) report("refine_QM1P");
}
// refine_QM1P_approx (:444-449)
void refine_QM1P_approx(double *x, double *QM1P, double *w, double *t, double *kappa, double mu, unsigned *nnt,
                        unsigned ns, unsigned nn, int time) {
    apply_mu_K_to_M(x + (size_t)time * ns * nn / 2, QM1P, w, t, kappa, mu, nnt, ns, nn);
}
// phonon_correlator (:526-545)
void phonon_correlator(double *x, unsigned ns, unsigned, unsigned nt, double *greens) {
    DView X(x, (size_t)nt * ns * 3), G(greens, (size_t)nt * 9);
    launch_phonon_corr(X.d, (int)ns, (int)nt, G.d, 0);
    cudaDeviceSynchronize();
    G.back();
}
// logDetM_and_inv_M_hat (:547-607)
double logDetM_and_inv_M_hat(double *M_hat, double *w, int *p, unsigned ns, unsigned flavors, organic_flags *mode) {
    (void)w;
    if (mode && mode->single_particle) return std::log(trace(M_hat, ns));
    ephmc_ctx *c = lu_ctx(ns);
    if (!c) return NAN;
    if (mode && mode->schur_form_inv) {
        // the Schur-form inverse is M_hat^-1 unless the reference's regularisation applies (schur.cu)
        DView Md(M_hat, (size_t)ns * ns);
        if (!Md.d || schur_check(&c->schur, Md.d, (int)ns, c->work, c->stream) != EPHMC_OK) {
            report("logDetM_and_inv_M_hat");
            return NAN;
        }
    }
    double ld = 0;
    int sign = 1;
    std::vector<int> piv(ns);
    const int rc = ephmc_logdet_inverse(c, M_hat, piv.data(), &ld, &sign);
    if (rc != EPHMC_OK && rc != EPHMC_ERR_SINGULAR) report("logDetM_and_inv_M_hat");
    if (p) {
        if (devp(p)) cudaMemcpy(p, piv.data(), sizeof(int) * ns, cudaMemcpyHostToDevice);
        else std::memcpy(p, piv.data(), sizeof(int) * ns);
    }
    if (sign < 0 && (flavors % 2)) {
        std::printf("Negative determinant!\n");
        add_warning(EPHMC_WARN_NEGATIVE_DET);
    }
    return ld;
}

// ================================================================== organic_bosons.h
// hot_start (simulation/organic_bosons.c:16-34)
void hot_start(double *x, double omega, unsigned ns, unsigned nn, unsigned nt) {
    const unsigned ld = ns * nn / 2;
    const double sd = std::sqrt(0.5 / std::tanh(0.5 * nt * omega));
    std::vector<double> h((size_t)ld * nt);
    for (unsigned k = 0; k < ld; k += 2) {
        const double u1 = sd * std::sqrt(-2 * std::log(rng_real2()));
        const double u2 = 6.283185307179586 * rng_real2();
        for (unsigned i = 0; i < nt; ++i) {
            h[k + (size_t)i * ld] = u1 * std::cos(u2);
            h[(k + 1) % ld + (size_t)i * ld] = u1 * std::sin(u2);
        }
    }
    if (devp(x)) cudaMemcpy(x, h.data(), sizeof(double) * h.size(), cudaMemcpyHostToDevice);
    else std::memcpy(x, h.data(), sizeof(double) * h.size());
}
// higher_Matsubaras_norm (:36-53)
double higher_Matsubaras_norm(double *x, unsigned *, unsigned ns, unsigned nn, unsigned nt) {
    DView X(x, (size_t)nt * ns * nn / 2);
    double *part = nullptr;
    if (cudaMalloc(&part, sizeof(double) * 64) != cudaSuccess) return NAN;
    double r = 0;
    device_matsubara_norm(X.d, (int)(ns * nn / 2), (int)nt, part, &r, 0);
    cudaFree(part);
    return r;
}

static ephmc_ctx *fa_ctx(unsigned ns, unsigned nt, double omega) {
    auto &r = ring_nnt(ns);
    const double z[3] = {0, 0, 0};
    return get_ctx(r.data(), ns, nt, z, z, 0.0, omega, 1, nullptr);
}

// sample_free_bosons (:55-74); x is the buffer fft[0] transforms
void sample_free_bosons(double *x, ephmc_dcomplex *, double omega, unsigned ns, unsigned, unsigned nt,
                        const fftw_plan *) {
    const size_t dim = (size_t)nt * ns * 3;
    std::vector<double> h(dim);
    rng_normals(h.data(), (unsigned)dim);
    ephmc_ctx *c = fa_ctx(ns, nt, omega);
    if (!c) return;
    if (devp(x)) cudaMemcpy(x, h.data(), sizeof(double) * dim, cudaMemcpyHostToDevice);
    else std::memcpy(x, h.data(), sizeof(double) * dim);
    if (ephmc_fa_scale_free_bosons(c, x) != EPHMC_OK) report("sample_free_bosons");
}
// sample_fourier_momenta (:76-100)
void sample_fourier_momenta(double *p, ephmc_dcomplex *, double omega, unsigned ns, unsigned, unsigned nt,
                            const fftw_plan *, organic_flags *mode) {
    const size_t dim = (size_t)nt * ns * 3;
    std::vector<double> h(dim);
    rng_normals(h.data(), (unsigned)dim);
    if (devp(p)) cudaMemcpy(p, h.data(), sizeof(double) * dim, cudaMemcpyHostToDevice);
    else std::memcpy(p, h.data(), sizeof(double) * dim);
    if (mode && mode->no_fourier_acc) return;
    ephmc_ctx *c = fa_ctx(ns, nt, omega);
    if (!c) return;
    ephmc_ctx_set_flags(c, mode);
    if (ephmc_fa_scale_momenta(c, p) != EPHMC_OK) report("sample_fourier_momenta");
}
// energy_fourier_momenta (:102-124); p is the buffer fft[1] transforms
double energy_fourier_momenta(ephmc_dcomplex *, double omega, unsigned ns, unsigned, unsigned nt, const fftw_plan *fft) {
    if (!fft || !fft[1]) return NAN;
    ephmc_ctx *c = fa_ctx(ns, nt, omega);
    double e = NAN;
    if (!c) {
        report("energy_fourier_momenta");
        return e;
    }
    // omega is used as given (energy_momenta passes the accelerated one)
    ephmc_flags f = c->flags;
    f.classical_fourier_acc = 0;
    ephmc_ctx_set_flags(c, &f);
    if (ephmc_fa_energy(c, static_cast<double *>(fft[1]->in), &e) != EPHMC_OK) report("energy_fourier_momenta");
    return e;
}
// evolve_bosons (:126-150): x and p are the buffers of plans 0 and 1
void evolve_bosons(ephmc_dcomplex *, double omega, unsigned ns, unsigned, unsigned nt, const fftw_plan *fft, double h) {
    if (!fft || !fft[0] || !fft[1]) return;
    ephmc_ctx *c = fa_ctx(ns, nt, omega);
    if (!c || ephmc_fa_evolve(c, static_cast<double *>(fft[0]->in), static_cast<double *>(fft[1]->in), h) != EPHMC_OK)
        report("evolve_bosons");
}
// evolve_bosons_approx_step (:152-177): x and p are the buffers of plans 0 and 1
void evolve_bosons_approx_step(ephmc_dcomplex *, double omega, unsigned ns, unsigned, unsigned nt,
                               const fftw_plan *fft, double h, organic_flags *mode) {
    if (!fft || !fft[0] || !fft[1]) return;
    ephmc_ctx *c = fa_ctx(ns, nt, omega);
    if (!c) return report("evolve_bosons_approx_step");
    ephmc_ctx_set_flags(c, mode);
    if (ephmc_fa_approx_step(c, static_cast<double *>(fft[0]->in), static_cast<double *>(fft[1]->in), h) != EPHMC_OK)
        report("evolve_bosons_approx_step");
}
// boson_force (:179-194)
void boson_force(double *x, double *p_dot, double omega, unsigned ns, unsigned nn, unsigned nt, int overwrite) {
    const size_t dim = (size_t)nt * ns * nn / 2;
    DView X(x, dim), P(p_dot, dim);
    launch_boson_force(X.d, P.d, omega, (int)(ns * nn / 2), (int)nt, overwrite != 0, 0);
    cudaDeviceSynchronize();
    P.back();
}

// ================================================================== organic_hmc.h (pieces)
// energy_momenta (simulation/organic_hmc.c:56-65)
double energy_momenta(double *p, ephmc_dcomplex *pc, double omega, unsigned ns, unsigned nn, unsigned nt,
                      const fftw_plan *fft, organic_flags *mode) {
    const size_t dim = (size_t)nt * ns * nn / 2;
    if (mode && mode->no_fourier_acc) {
        DView P(p, dim);
        double *part = nullptr;
        if (cudaMalloc(&part, sizeof(double) * 128) != cudaSuccess) return NAN;
        double mom[2];
        device_moments(P.d, dim, part, mom, 0);
        cudaFree(part);
        return .5 * dim * (mom[1] / dim);
    }
    (void)pc;
    (void)fft;
    ephmc_ctx *c = fa_ctx(ns, nt, omega);
    if (!c) return NAN;
    ephmc_ctx_set_flags(c, mode);
    double e = NAN;
    if (ephmc_fa_energy(c, p, &e) != EPHMC_OK) report("energy_momenta");
    return e;
}
// hamilton (:67-84)
double hamilton(double *x, double *, double logDetM, double energyP, double omega, unsigned flavors, unsigned ns,
                unsigned, unsigned nt) {
    auto &r = ring_nnt(ns);
    const double z[3] = {0, 0, 0};
    ephmc_ctx *c = get_ctx(r.data(), ns, nt, z, z, 0.0, omega, flavors, nullptr);
    double H = NAN;
    if (!c || ephmc_hamilton(c, x, logDetM, energyP, &H) != EPHMC_OK) report("hamilton");
    return H;
}
// force (:86-134)
void force(double *x, double *p_dot, double *M_hat, double *QM1P, double *w, int *perm, double *t, double *kappa,
           double mu, double omega, unsigned flavors, unsigned *nnt, unsigned ns, unsigned, unsigned nt, double logDetM,
           organic_flags *mode) {
    (void)QM1P;
    (void)w;
    (void)perm;
    ephmc_ctx *c = get_ctx(nnt, ns, nt, t, kappa, mu, omega, flavors, mode);
    if (!c || ephmc_force(c, x, M_hat, logDetM, p_dot, g_dropin_mode) != EPHMC_OK) report("force");
}
// check_force (:20-54): central differences of -flavors*logdet, step eps^(1/3)
double check_force(double *x, double *p, double *p_dot, double *M_hat, double *w, int *perm, double *t, double *kappa,
                   double mu, double omega, unsigned flavors, unsigned *nnt, unsigned ns, unsigned nn, unsigned nt,
                   organic_flags *mode) {
    (void)p;
    (void)w;
    (void)perm;
    (void)M_hat;
    ephmc_ctx *c = get_ctx(nnt, ns, nt, t, kappa, mu, omega, flavors, mode);
    if (!c) return NAN;
    const size_t dim = (size_t)nt * ns * nn / 2, VV = (size_t)ns * ns;
    const double delta = std::pow(2.220446049250313e-16, 1. / 3);
    std::vector<double> xh(dim), pd(dim);
    if (devp(x)) cudaMemcpy(xh.data(), x, sizeof(double) * dim, cudaMemcpyDeviceToHost);
    else std::memcpy(xh.data(), x, sizeof(double) * dim);
    if (devp(p_dot)) cudaMemcpy(pd.data(), p_dot, sizeof(double) * dim, cudaMemcpyDeviceToHost);
    else std::memcpy(pd.data(), p_dot, sizeof(double) * dim);
    double *Md = c->work;
    double err = 0, nrm = 0;
    for (size_t i = 0; i < dim; ++i) {
        const double keep = xh[i];
        double e[2];
        for (int s = 0; s < 2; ++s) {
            xh[i] = keep + (s == 0 ? delta : -delta);
            ephmc_construct_M_hat(c, xh.data(), Md);
            double ld = 0;
            int sg = 1;
            if (mode && mode->single_particle) {
                double tr = 0;
                launch_trace(Md, (int)ns, c->scratch, c->stream);
                cudaMemcpy(&tr, c->scratch, sizeof(double), cudaMemcpyDeviceToHost);
                ld = std::log(tr);
            } else {
                ephmc_logdet_inverse(c, Md, nullptr, &ld, &sg);
            }
            e[s] = -ld * flavors;
        }
        const double fd = -(e[0] - e[1]) / (2 * delta);
        err += (pd[i] - fd) * (pd[i] - fd);
        nrm += (std::fabs(pd[i]) + std::fabs(fd)) * (std::fabs(pd[i]) + std::fabs(fd));
        xh[i] = keep;
    }
    (void)VV;
    return std::sqrt(err / nrm);
}
// update_x (:136-165)
void update_x(double *x, double *p, double *p_dot, ephmc_dcomplex *xc, double omega, unsigned ns, unsigned nn,
              unsigned nt, const fftw_plan *fft, double h, double half, organic_flags *mode) {
    (void)xc;
    (void)fft;
    const size_t dim = (size_t)nt * ns * nn / 2;
    if (mode && mode->no_fourier_acc) {
        DView X(x, dim), P(p, dim);
        launch_axpy(X.d, P.d, h * std::fabs(half), dim, 0);
        cudaDeviceSynchronize();
        X.back();
        return;
    }
    if (mode && mode->classical_fourier_acc) {
        ephmc_ctx *c = fa_ctx(ns, nt, omega);
        if (!c) return report("update_x");
        ephmc_ctx_set_flags(c, mode);
        DView X(x, dim), P(p, dim), PD(p_dot, dim);
        if (classical_update_x(c, X.d, P.d, PD.d, h, half) != EPHMC_OK) return report("update_x");
        cudaStreamSynchronize(c->stream);
        X.back();
        P.back();
        PD.back();
        return;
    }
    ephmc_ctx *c = fa_ctx(ns, nt, omega);
    if (!c || ephmc_fa_evolve(c, x, p, std::fabs(half) * h) != EPHMC_OK) report("update_x");
}

}  // extern "C"

namespace ephmc {
double dropin_contract_greens(const double *gr, const double *mat, unsigned nn, unsigned tau) {
    return contract_greens_h(gr, mat, nn, tau);
}
double dropin_rng_real2() { return rng_real2(); }
void dropin_rng_normals(double *x, unsigned n) { rng_normals(x, n); }
void dropin_rng_seed(unsigned long long s) { rng_seed(s); }
int dropin_force_mode() { return g_dropin_mode; }
}  // namespace ephmc
