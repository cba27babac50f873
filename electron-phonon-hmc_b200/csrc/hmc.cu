// HMC driver of the drop-in surface: leap_frog, trajectory, run_hmc and the
// correlator, with every field, matrix and work array resident on the GPU;
// the host keeps the MT19937-64 stream, the scalars of the Metropolis step
// and the output files.  Reference: simulation/organic_hmc.c:136-353,
// organic_dense_matrix.c:451-524, organic_aux.c:51-70.
#include "ephmc_internal.cuh"
#include "../../include/ephmc_organic.h"

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <vector>

using namespace ephmc;

namespace {

constexpr unsigned kNumRes = 12;  // NUM_RES, simulation/organic_aux.h:4
constexpr double kPi = 3.141592653589793;

bool devp(const void *p) {
    if (!p) return false;
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

// device view of a caller array (staged when it is host memory)
struct Dev {
    double *user = nullptr, *d = nullptr;
    size_t n = 0;
    bool owned = false;
    Dev(double *u, size_t count, bool copy_in = true) : user(u), n(count) {
        if (!u) return;
        if (devp(u)) {
            d = u;
            return;
        }
        if (cudaMalloc(&d, sizeof(double) * n) != cudaSuccess) {
            cudaGetLastError();
            d = nullptr;
            return;
        }
        owned = true;
        if (copy_in) cudaMemcpy(d, u, sizeof(double) * n, cudaMemcpyHostToDevice);
    }
    Dev(const Dev &) = delete;
    Dev &operator=(const Dev &) = delete;
    void back() {
        if (owned && d) cudaMemcpy(user, d, sizeof(double) * n, cudaMemcpyDeviceToHost);
    }
    ~Dev() {
        if (owned && d) cudaFree(d);
    }
};

ephmc_ctx *ctx_for(unsigned *nnt, unsigned ns, unsigned nt, double *t, double *kappa, double mu, double omega,
                   unsigned flavors, organic_flags *mode) {
    std::vector<unsigned> h(12 * (size_t)ns);
    if (devp(nnt)) cudaMemcpy(h.data(), nnt, sizeof(unsigned) * h.size(), cudaMemcpyDeviceToHost);
    else std::memcpy(h.data(), nnt, sizeof(unsigned) * h.size());
    // one context per call shape; the registry of the drop-in surface keeps it
    static thread_local std::vector<std::pair<std::vector<unsigned>, ephmc_ctx *>> cache;
    for (auto &e : cache)
        if (e.second->nt == nt && e.first == h) {
            ephmc_ctx_set_params(e.second, t, kappa, mu, omega, flavors);
            ephmc_ctx_set_flags(e.second, mode);
            return e.second;
        }
    ephmc_ctx *c = nullptr;
    if (ephmc_ctx_create_nnt(&c, h.data(), ns, nt, t, kappa, mu, omega, flavors, mode, -1) != EPHMC_OK) {
        std::fprintf(stderr, "ephmc: %s\n", ephmc_last_error_message());
        return nullptr;
    }
    cache.emplace_back(h, c);
    return c;
}

double logdet_dev(ephmc_ctx *c, double *M, unsigned ns, unsigned flavors) {
    double ld = 0;
    if (c->flags.single_particle) {
        launch_trace(M, (int)ns, c->scratch, c->stream);
        double tr = 0;
        cudaMemcpy(&tr, c->scratch, sizeof(double), cudaMemcpyDeviceToHost);
        return std::log(tr);
    }
    if (c->flags.schur_form_inv && schur_check(&c->schur, M, (int)ns, c->work, c->stream) != EPHMC_OK) {
        std::fprintf(stderr, "ephmc logDetM_and_inv_M_hat: %s\n", ephmc_last_error_message());
        return NAN;
    }
    int sign = 1;
    ephmc_logdet_inverse(c, M, nullptr, &ld, &sign);
    if (sign < 0 && (flavors % 2)) std::printf("Negative determinant!\n");
    return ld;
}

// the FA momentum refresh: host MT normals -> device, Fourier scaling
void refresh_momenta(ephmc_ctx *c, double *p_dev, size_t dim) {
    std::vector<double> h(dim);
    dropin_rng_normals(h.data(), (unsigned)dim);
    cudaMemcpy(p_dev, h.data(), sizeof(double) * dim, cudaMemcpyHostToDevice);
    if (!c->flags.no_fourier_acc) ephmc_fa_scale_momenta(c, p_dev);
}

double kinetic(ephmc_ctx *c, double *p_dev, size_t dim) {
    if (c->flags.no_fourier_acc) {
        double mom[2];
        device_moments(p_dev, dim, c->cc_part, mom, c->stream);
        return .5 * dim * (mom[1] / dim);
    }
    double e = 0;
    ephmc_fa_energy(c, p_dev, &e);
    return e;
}

void update_x_dev(ephmc_ctx *c, double *x, double *p, double *p_dot, size_t dim, double h, double half) {
    if (c->flags.classical_fourier_acc && !c->flags.no_fourier_acc) {
        if (classical_update_x(c, x, p, p_dot, h, half) != EPHMC_OK)
            std::fprintf(stderr, "ephmc update_x: %s\n", ephmc_last_error_message());
        cudaStreamSynchronize(c->stream);
        return;
    }
    if (c->flags.no_fourier_acc) {
        launch_axpy(x, p, h * std::fabs(half), dim, c->stream);
        cudaStreamSynchronize(c->stream);
    } else {
        ephmc_fa_evolve(c, x, p, std::fabs(half) * h);
    }
}

// update_x (simulation/organic_hmc.c:136-165) issued without a host wait
int update_x_async(ephmc_ctx *c, double *x, double *p, double *p_dot, size_t dim, double h, double half) {
    if (c->flags.classical_fourier_acc && !c->flags.no_fourier_acc) return classical_update_x(c, x, p, p_dot, h, half);
    if (c->flags.no_fourier_acc) return launch_axpy(x, p, h * std::fabs(half), dim, c->stream);
    return fa_evolve(x, p, 3 * (int)c->V, (int)c->nt, c->omega, std::fabs(half) * h, c->scratch, c->stream);
}

bool leapfrog_async_ok(const ephmc_ctx *c) { return !c->flags.single_particle && !c->flags.schur_form_inv; }

// leap_frog (simulation/organic_hmc.c:167-190) on device buffers; M_hat ends
// holding the inverse of the last step
void leap_frog_dev(ephmc_ctx *c, double *x, double *p, double *p_dot, double *M_hat, unsigned steps,
                   double traj_length, int force_mode) {
    const size_t dim = (size_t)c->nt * c->V * 3, VV = (size_t)c->V * c->V;
    if (leapfrog_async_ok(c)) {
        unsigned neg = 0;
        if (ephmc_leapfrog(c, x, p, steps, traj_length, force_mode, &neg) != EPHMC_OK)
            std::fprintf(stderr, "ephmc leap_frog: %s\n", ephmc_last_error_message());
        for (unsigned s = 0; s < neg; ++s) std::printf("Negative determinant!\n");
        cudaMemcpyAsync(p_dot, c->force, sizeof(double) * dim, cudaMemcpyDeviceToDevice, c->stream);
        cudaMemcpyAsync(M_hat, c->M, sizeof(double) * VV, cudaMemcpyDeviceToDevice, c->stream);
        cudaStreamSynchronize(c->stream);
        return;
    }
    const double h = steps ? traj_length / steps : 2 * traj_length;
    double half = .5;
    update_x_dev(c, x, p, p_dot, dim, h, half);
    half = 1;
    for (unsigned s = 1; s <= steps; ++s) {
        double ld = 0;
        if (ephmc_eval(c, x, p_dot, &ld, force_mode) != EPHMC_OK)
            std::fprintf(stderr, "ephmc leap_frog: %s\n", ephmc_last_error_message());
        if (ephmc_last_warnings() & EPHMC_WARN_NEGATIVE_DET) std::printf("Negative determinant!\n");
        cudaMemcpyAsync(M_hat, c->M, sizeof(double) * VV, cudaMemcpyDeviceToDevice, c->stream);
        launch_axpy(p, p_dot, h, dim, c->stream);
        if (s == steps) half = -.5;
        update_x_dev(c, x, p, p_dot, dim, h, half);
    }
    cudaStreamSynchronize(c->stream);
}

// trajectory (simulation/organic_hmc.c:192-294) on the device block of the
// reference's layout x|p|p_dot|x_old|M_hat|M_hat_old|QM1P[nt]|R_0t|w
short trajectory_dev(ephmc_ctx *c, double *xb, double *results, double *greens, int iteration, unsigned meas_freq,
                     double *contr_mat, unsigned steps, double traj_length, double *old, FILE *res_out,
                     FILE *corr_out) {
    const unsigned ns = c->V, nt = c->nt, nn = 6;
    const size_t dim = (size_t)nt * ns * 3, VV = (size_t)ns * ns;
    double *x = xb, *p = x + dim, *p_dot = p + dim, *x_old = p_dot + dim;
    double *M_hat = x_old + dim, *M_old = M_hat + VV, *QM1P = M_old + VV;
    const ephmc_flags &mode = c->flags;
    const int fmode = dropin_force_mode();
    double logDetM = 0, energy = 0, boltzmann = 1;
    short acc = 1;
    if (!mode.zero_filling) {
        const double logDetM_old = old[0];
        cudaMemcpy(x_old, x, sizeof(double) * dim, cudaMemcpyDeviceToDevice);
        cudaMemcpy(M_old, M_hat, sizeof(double) * VV, cudaMemcpyDeviceToDevice);
        refresh_momenta(c, p, dim);
        double energyP = kinetic(c, p, dim);
        double energy_old = 0;
        ephmc_hamilton(c, x, logDetM_old, energyP, &energy_old);
        leap_frog_dev(c, x, p, p_dot, M_hat, steps, traj_length, fmode);
        ephmc_construct_M_hat(c, x, M_hat);
        logDetM = logdet_dev(c, M_hat, ns, c->flavors);
        energyP = kinetic(c, p, dim);
        ephmc_hamilton(c, x, logDetM, energyP, &energy);
        boltzmann = std::exp(energy_old - energy);
        if (!(boltzmann > dropin_rng_real2())) {  // reject (NaN-safe as the reference)
            cudaMemcpy(x, x_old, sizeof(double) * dim, cudaMemcpyDeviceToDevice);
            cudaMemcpy(M_hat, M_old, sizeof(double) * VV, cudaMemcpyDeviceToDevice);
            logDetM = logDetM_old;
            energy = energy_old;
            acc = 0;
        }
        old[0] = logDetM;
    } else {
        std::vector<double> h(dim);
        dropin_rng_normals(h.data(), (unsigned)dim);
        cudaMemcpy(x, h.data(), sizeof(double) * dim, cudaMemcpyHostToDevice);
        ephmc_fa_scale_free_bosons(c, x);
        ephmc_construct_M_hat(c, x, M_hat);
        logDetM = 0;
        ephmc_hamilton(c, x, 0, 0, &energy);
    }
    if (iteration % (int)meas_freq == 0) {
        if (greens) {
            double *gd = nullptr;
            cudaMalloc(&gd, sizeof(double) * nt * 9);
            cc_correlator_dev(c, x, M_hat, QM1P, c->work + (size_t)ns * ns, gd, logDetM);
            cudaMemcpy(greens, gd, sizeof(double) * nt * 9, cudaMemcpyDeviceToHost);
            cudaFree(gd);
            if (corr_out) {  // fprint_corr (simulation/organic_aux.c:51-60)
                for (unsigned i = 0; i < nt; ++i)
                    std::fprintf(corr_out, "%d\t%.15g\n", i,
                                 dropin_contract_greens(greens, contr_mat, nn, i) * (double)(nt * nt));
                std::fflush(corr_out);
            }
        }
        if (results) {
            double mom[2];
            device_moments(x, dim, c->cc_part, mom, c->stream);
            results[0] = mom[0] / dim;        // average(x)
            results[1] = mom[1] / dim - 0.5;  // average_sq(x) - 1/2
            results[2] = energy;
            results[3] = -logDetM;
            device_matsubara_norm(x, 3 * (int)ns, (int)nt, c->cc_part, &results[4], c->stream);
            launch_trace(M_hat, (int)ns, c->scratch, c->stream);
            double tr = 0;
            cudaMemcpy(&tr, c->scratch, sizeof(double), cudaMemcpyDeviceToHost);
            results[5] = (!mode.zero_filling && !mode.single_particle) ? 1 - tr / ns : tr / ns;
            results[6] = acc;
            results[7] = boltzmann;
            // average_links (simulation/organic_aux.c:199-210): sum over slices and sites / ns
            std::vector<double> xh(dim);
            cudaMemcpy(xh.data(), x, sizeof(double) * dim, cudaMemcpyDeviceToHost);
            for (unsigned k = 0; k < 3; ++k) results[8 + k] = 0;
            for (size_t i = 0; i < (size_t)ns * nt; ++i)
                for (unsigned k = 0; k < 3; ++k) results[8 + k] += xh[i * 3 + k];
            for (unsigned k = 0; k < 3; ++k) results[8 + k] /= ns;
            if (greens) results[11] = dropin_contract_greens(greens, contr_mat, nn, nt / 2) * nt * nt / kPi;
            if (res_out) {  // fprint_results (simulation/organic_aux.c:62-70)
                for (unsigned k = 0; k < kNumRes; ++k) std::fprintf(res_out, "%.15g\t", results[k]);
                std::fprintf(res_out, "\n");
                std::fflush(res_out);
            }
        }
    }
    return acc;
}

// ---------------------------------------------------------------- leapfrog pieces
int leapfrog_prepare(ephmc_ctx *c, double *x, double *p, unsigned steps, int force_mode) {
    if (!c || !x || !p) {
        set_status(EPHMC_ERR_ARG, "ephmc_leapfrog arguments");
        return EPHMC_ERR_ARG;
    }
    if (force_mode < EPHMC_FORCE_REFERENCE || force_mode > EPHMC_FORCE_MIXED) {
        set_status(EPHMC_ERR_ARG, "force mode");
        return EPHMC_ERR_ARG;
    }
    if (!leapfrog_async_ok(c)) {
        set_status(EPHMC_ERR_UNSUPPORTED,
                   "ephmc_leapfrog: SINGLE_PARTICLE and SCHUR_FORM_INV forces need each step's log det on the host");
        return EPHMC_ERR_UNSUPPORTED;
    }
    EPHMC_CUDA(cudaSetDevice(c->device));
    if (!devp(x) || !devp(p)) {
        set_status(EPHMC_ERR_ARG, "ephmc_leapfrog: x and p must be device memory");
        return EPHMC_ERR_ARG;
    }
    if (steps > c->md_cap) {
        cudaFree(c->md_log);
        c->md_log = nullptr;
        c->md_cap = 0;
        if (cudaMalloc(&c->md_log, sizeof(double) * 3 * steps) != cudaSuccess) {
            cudaGetLastError();
            set_status(EPHMC_ERR_NOMEM, "ephmc_leapfrog: step log");
            return EPHMC_ERR_NOMEM;
        }
        c->md_cap = steps;
        if (c->lf_graph) {  // the step log moved
            cudaGraphExecDestroy(c->lf_graph);
            c->lf_graph = nullptr;
        }
    }
    return EPHMC_OK;
}

// every operation of the trajectory on stream st (c->stream == st), no host wait
int leapfrog_issue(ephmc_ctx *c, double *x, double *p, unsigned steps, double traj_length, int force_mode,
                   cudaStream_t st) {
    const size_t dim = (size_t)c->nt * c->V * 3;
    const double h = steps ? traj_length / steps : 2 * traj_length;
    int rc = update_x_async(c, x, p, c->force, dim, h, .5);
    for (unsigned s = 1; s <= steps && rc == EPHMC_OK; ++s) {
        if ((rc = eval_async(c, x, force_mode))) break;
        double *lg = c->md_log + 3 * (size_t)(s - 1);
        cudaMemcpyAsync(lg, c->lu.diag + c->V, 2 * sizeof(double), cudaMemcpyDeviceToDevice, st);
        cudaMemcpyAsync(lg + 2, c->lu.info, 2 * sizeof(int), cudaMemcpyDeviceToDevice, st);
        if ((rc = launch_axpy(p, c->force, h, dim, st))) break;
        rc = update_x_async(c, x, p, c->force, dim, h, s == steps ? -.5 : 1.0);
    }
    return rc;
}

// wait for the trajectory on st, then read each step's log det, sign and status
int leapfrog_collect(ephmc_ctx *c, unsigned steps, int rc, cudaStream_t st, unsigned *negative_steps) {
    std::vector<double> lg(3 * (size_t)steps);
    if (steps) cudaMemcpyAsync(lg.data(), c->md_log, sizeof(double) * lg.size(), cudaMemcpyDeviceToHost, st);
    const cudaError_t e = cudaStreamSynchronize(st);
    if (rc != EPHMC_OK) return rc;
    if (e != cudaSuccess) {
        set_status(EPHMC_ERR_CUDA, cudaGetErrorString(e));
        return EPHMC_ERR_CUDA;
    }
    unsigned neg = 0;
    for (unsigned s = 0; s < steps; ++s) {
        int info[2];
        std::memcpy(info, &lg[3 * (size_t)s + 2], sizeof(info));
        if (info[1] != 0) {
            lu_reset_sync(c->lu, st);
            cudaStreamSynchronize(st);
            set_status(EPHMC_ERR_TIMEOUT, "LU: a panel wait of the dataflow kernel ran out; the result is invalid");
            return EPHMC_ERR_TIMEOUT;
        }
        if (info[0] != 0) {
            set_status(EPHMC_ERR_SINGULAR, "zero pivot in an MD step");
            return EPHMC_ERR_SINGULAR;
        }
        if (lg[3 * (size_t)s + 1] < 0 && (c->flavors % 2)) ++neg;
    }
    if (steps) {
        c->last_logdet = lg[3 * (size_t)(steps - 1)];
        c->last_sign = lg[3 * (size_t)(steps - 1) + 1] < 0 ? -1 : 1;
        c->have_inverse = true;
    }
    if (neg) add_warning(EPHMC_WARN_NEGATIVE_DET);
    if (negative_steps) *negative_steps = neg;
    return EPHMC_OK;
}

}  // namespace

extern "C" {

// leap_frog (simulation/organic_hmc.c:167-190) on device x and p with every
// step issued before any host wait: per step sweep 1 + LU + force, p += h F,
// update_x.  The log det, sign and LU status of each step stay on the device
// and are read once at the end.
int ephmc_leapfrog(ephmc_ctx *c, double *x, double *p, unsigned steps, double traj_length, int force_mode,
                   unsigned *negative_steps) {
    clear_status();
    int rc = leapfrog_prepare(c, x, p, steps, force_mode);
    if (rc) return rc;
    rc = leapfrog_issue(c, x, p, steps, traj_length, force_mode, c->stream);
    return leapfrog_collect(c, steps, rc, c->stream, negative_steps);
}

int ephmc_leapfrog_graph(ephmc_ctx *c, double *x, double *p, unsigned steps, double traj_length, int force_mode,
                         unsigned *negative_steps) {
    clear_status();
    int rc = leapfrog_prepare(c, x, p, steps, force_mode);
    if (rc) return rc;
    if (c->stabilize && force_mode != EPHMC_FORCE_REFERENCE && !c->flags.constant_force) {
        set_status(EPHMC_ERR_UNSUPPORTED,
                   "ephmc_leapfrog_graph: the stabilised chain's cuSOLVER factorisations are not captured; use "
                   "ephmc_leapfrog");
        return EPHMC_ERR_UNSUPPORTED;
    }
    if (force_mode == EPHMC_FORCE_REFERENCE || c->flags.constant_force)
        if ((rc = ensure_ref_buffers(c))) return rc;
    if (force_mode == EPHMC_FORCE_MIXED && !c->flags.constant_force)
        if ((rc = ensure_seg_buffers(c))) return rc;
    // the graph runs on the context's private stream, ordered after the work
    // already queued on the caller's stream and before what follows there
    if (!c->batch_stream) {
        if (cudaStreamCreateWithFlags(&c->batch_stream, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&c->batch_ev[0], cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&c->batch_ev[1], cudaEventDisableTiming) != cudaSuccess) {
            cudaGetLastError();
            set_status(EPHMC_ERR_CUDA, "ephmc_leapfrog_graph: stream creation");
            return EPHMC_ERR_CUDA;
        }
    }
    cudaStream_t gs = c->batch_stream, caller = c->stream;
    const LeapfrogKey key{x, p, steps, traj_length, force_mode, c->param_gen};
    if (!c->lf_graph || !(c->lf_key == key)) {
        if (c->lf_graph) cudaGraphExecDestroy(c->lf_graph);
        c->lf_graph = nullptr;
        cudaStream_t keep = c->stream;
        c->stream = gs;
        uploads_uncached(true);  // the graph must carry every table it reads
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamBeginCapture(gs, cudaStreamCaptureModeRelaxed);
        if (e == cudaSuccess) {
            rc = leapfrog_issue(c, x, p, steps, traj_length, force_mode, gs);
            e = cudaStreamEndCapture(gs, &g);
        }
        uploads_uncached(false);
        c->stream = keep;
        if (rc == EPHMC_OK && e == cudaSuccess && g) {
            e = cudaGraphInstantiate(&c->lf_graph, g, 0);
            if (e != cudaSuccess) c->lf_graph = nullptr;
        }
        if (g) cudaGraphDestroy(g);
        if (rc != EPHMC_OK || e != cudaSuccess || !c->lf_graph) {
            cudaGetLastError();
            ctx_forget_uploads(c);
            if (rc == EPHMC_OK) {
                char msg[200];
                std::snprintf(msg, sizeof msg, "ephmc_leapfrog_graph: capture failed (%s)", cudaGetErrorString(e));
                set_status(EPHMC_ERR_CUDA, msg);
                rc = EPHMC_ERR_CUDA;
            }
            return rc;
        }
        c->lf_key = key;
        // the captured uploads rewrote the tables: the host shadows no longer know them
        ctx_forget_uploads(c);
    }
    cudaEventRecord(c->batch_ev[0], caller);
    cudaStreamWaitEvent(gs, c->batch_ev[0], 0);
    if (cudaGraphLaunch(c->lf_graph, gs) != cudaSuccess) {
        cudaGetLastError();
        set_status(EPHMC_ERR_CUDA, "ephmc_leapfrog_graph: graph launch");
        return EPHMC_ERR_CUDA;
    }
    cudaEventRecord(c->batch_ev[1], gs);
    cudaStreamWaitEvent(caller, c->batch_ev[1], 0);
    // the tables the graph left on the device differ from what the shadows hold
    ctx_forget_uploads(c);
    return leapfrog_collect(c, steps, EPHMC_OK, gs, negative_steps);
}

// leap_frog (simulation/organic_hmc.c:167-190)
void leap_frog(double *x, double *p, double *p_dot, ephmc_dcomplex *xc, double *M_hat, double *QM1P, double *w,
               int *perm, double *t, double *kappa, double mu, double omega, unsigned flavors, unsigned *nnt,
               unsigned ns, unsigned, unsigned nt, unsigned steps, double traj_length, const fftw_plan *fft,
               organic_flags *mode) {
    (void)xc;
    (void)QM1P;
    (void)w;
    (void)perm;
    (void)fft;
    ephmc_ctx *c = ctx_for(nnt, ns, nt, t, kappa, mu, omega, flavors, mode);
    if (!c) return;
    const size_t dim = (size_t)nt * ns * 3;
    Dev X(x, dim), P(p, dim), PD(p_dot, dim), M(M_hat, (size_t)ns * ns, false);
    leap_frog_dev(c, X.d, P.d, PD.d, M.d, steps, traj_length, dropin_force_mode());
    X.back();
    P.back();
    PD.back();
    M.back();
}

// trajectory (simulation/organic_hmc.c:192-294): x is the base of the reference's block
// x | p | p_dot | x_old | M_hat | M_hat_old | QM1P[Nt V^2] | R_0t | w[5 V^2].
// A device block is used in place.  For a host block the context keeps a
// device block of that layout between calls, and a call moves only what the
// trajectory reads (x and M_hat, the current field and its inverse) and the
// parts a caller can use afterwards (x, p, p_dot, x_old, M_hat, M_hat_old);
// the rest is work space (QM1P, R_0t, w), about (Nt + 6) V^2 doubles that are
// not copied.
short trajectory(double *x, ephmc_dcomplex *xc, int *perm, double *t, double *kappa, double mu, double omega,
                 unsigned flavors, double *contr_mat, unsigned *nnt, unsigned ns, unsigned, unsigned nt, unsigned steps,
                 double traj_length, double *results, double *greens, int iteration, unsigned meas_freq,
                 const fftw_plan *fft, double *old, FILE *res_out, FILE *corr_out, organic_flags *mode) {
    (void)xc;
    (void)perm;
    (void)fft;
    ephmc_ctx *c = ctx_for(nnt, ns, nt, t, kappa, mu, omega, flavors, mode);
    if (!c) return 0;
    const size_t dim = (size_t)nt * ns * 3, VV = (size_t)ns * ns;
    const size_t total = 4 * dim + (8 + (size_t)nt) * VV;
    if (devp(x))
        return trajectory_dev(c, x, results, greens, iteration, meas_freq, contr_mat, steps, traj_length, old, res_out,
                              corr_out);
    if (c->dropin_block_n < total) {
        cudaFree(c->dropin_block);
        c->dropin_block = nullptr;
        c->dropin_block_n = 0;
        if (cudaMalloc(&c->dropin_block, sizeof(double) * total) != cudaSuccess) {
            cudaGetLastError();
            std::fprintf(stderr, "ephmc trajectory: no device memory for the state block\n");
            return 0;
        }
        c->dropin_block_n = total;
    }
    double *d = c->dropin_block;
    const size_t off_M = 4 * dim;
    cudaMemcpy(d, x, sizeof(double) * dim, cudaMemcpyHostToDevice);                      // x
    cudaMemcpy(d + off_M, x + off_M, sizeof(double) * VV, cudaMemcpyHostToDevice);      // M_hat
    const short acc = trajectory_dev(c, d, results, greens, iteration, meas_freq, contr_mat, steps, traj_length, old,
                                     res_out, corr_out);
    cudaMemcpy(x, d, sizeof(double) * 4 * dim, cudaMemcpyDeviceToHost);                 // x, p, p_dot, x_old
    cudaMemcpy(x + off_M, d + off_M, sizeof(double) * 2 * VV, cudaMemcpyDeviceToHost);  // M_hat, M_hat_old
    return acc;
}

// cc_correlator (simulation/organic_dense_matrix.c:451-524)
void cc_correlator(double *x, double *M_hat, double *R_t0, double *R_0t, double *w, double *t, double *kappa, double mu,
                   unsigned *nnt, unsigned ns, unsigned, unsigned nt, double *greens, double logDetM,
                   organic_flags *mode) {
    (void)w;
    ephmc_ctx *c = ctx_for(nnt, ns, nt, t, kappa, mu, 0.0, 1, mode);
    if (!c) return;
    const size_t dim = (size_t)nt * ns * 3, VV = (size_t)ns * ns;
    Dev X(x, dim), Mi(M_hat, VV), Rt(R_t0, VV * nt, false), G(greens, (size_t)nt * 9, false);
    double *r0t = c->work + VV;  // R_0t on the device, advanced slice by slice
    if (cc_correlator_dev(c, X.d, Mi.d, Rt.d, r0t, G.d, logDetM) != EPHMC_OK) {
        std::fprintf(stderr, "ephmc cc_correlator: %s\n", ephmc_last_error_message());
        return;
    }
    cudaStreamSynchronize(c->stream);
    if (R_0t) {  // the reference leaves R_0t after Nt-1 slices
        if (devp(R_0t))
            cudaMemcpy(R_0t, r0t, sizeof(double) * VV, cudaMemcpyDeviceToDevice);
        else
            cudaMemcpy(R_0t, r0t, sizeof(double) * VV, cudaMemcpyDeviceToHost);
    }
    Rt.back();
    G.back();
}

unsigned ephmc_run_hmc_seeded(unsigned long long seed, double *greens, unsigned l1, unsigned l2, unsigned nt,
                              double *t, double *kappa, double mu, double omega, unsigned flavors, double *contr_mat,
                              unsigned steps, double traj_length, unsigned therm, unsigned meas, unsigned meas_freq,
                              const char *res_name, const char *corr_name, organic_flags *mode) {
    const unsigned ns = l1 * l2, nn = 6;
    std::vector<unsigned> nnt(12 * (size_t)ns);
    triangular_lattice(l1, l2, nnt.data());
    const size_t dim = (size_t)nt * ns * 3, VV = (size_t)ns * ns;
    const unsigned greens_dim = nt * 9;
    double *results = greens + (size_t)greens_dim * meas / meas_freq;
    ephmc_ctx *c = ctx_for(nnt.data(), ns, nt, t, kappa, mu, omega, flavors, mode);
    if (!c) return 0;
    double *xb = nullptr;
    if (cudaMalloc(&xb, sizeof(double) * (4 * dim + (8 + (size_t)nt) * VV)) != cudaSuccess) {
        cudaGetLastError();
        std::fprintf(stderr, "ephmc run_hmc: device allocation failed\n");
        return 0;
    }
    FILE *res_out = res_name ? std::fopen(res_name, "a") : nullptr;
    FILE *corr_out = corr_name ? std::fopen(corr_name, "a") : nullptr;
    dropin_rng_seed(seed);
    // sample_free_bosons (simulation/organic_hmc.c:325)
    {
        std::vector<double> h(dim);
        dropin_rng_normals(h.data(), (unsigned)dim);
        cudaMemcpy(xb, h.data(), sizeof(double) * dim, cudaMemcpyHostToDevice);
        ephmc_fa_scale_free_bosons(c, xb);
    }
    double *M_hat = xb + 4 * dim;
    ephmc_construct_M_hat(c, xb, M_hat);
    double logDetM = 0;
    if (!c->flags.zero_filling) logDetM = logdet_dev(c, M_hat, ns, flavors);
    for (unsigned i = 0; i < therm; ++i)
        trajectory_dev(c, xb, nullptr, nullptr, -1, meas_freq, contr_mat, steps, traj_length, &logDetM, nullptr,
                       nullptr);
    for (unsigned i = 0; i < meas; ++i)
        trajectory_dev(c, xb, results + (size_t)(i / meas_freq) * kNumRes,
                       greens ? greens + (size_t)(i / meas_freq) * greens_dim : nullptr, (int)i, meas_freq, contr_mat,
                       steps, traj_length, &logDetM, res_out, corr_out);
    cudaFree(xb);
    if (res_out) std::fclose(res_out);
    if (corr_out) std::fclose(corr_out);
    (void)nn;
    return meas / meas_freq * (greens_dim + kNumRes);
}

// run_hmc (simulation/organic_hmc.c:296-353), seeded with time(NULL) as the
// reference, or with the value of the environment variable EPHMC_SEED if set.
// EPHMC_FORCE (reference, adjoint or mixed) selects the force algorithm of a
// host program that cannot call ephmc_set_dropin_force_mode itself, such as
// the reference's unchanged organic_main; the default is the reference's.
unsigned run_hmc(double *greens, unsigned l1, unsigned l2, unsigned nt, double *t, double *kappa, double mu,
                 double omega, unsigned flavors, double *contr_mat, unsigned steps, double traj_length, unsigned therm,
                 unsigned meas, unsigned meas_freq, const char *res_name, const char *corr_name, organic_flags *mode) {
    unsigned long long seed = (unsigned long long)std::time(nullptr);
    if (const char *s = std::getenv("EPHMC_SEED")) seed = std::strtoull(s, nullptr, 10);
    if (const char *f = std::getenv("EPHMC_FORCE")) {
        if (!std::strcmp(f, "reference")) ephmc_set_dropin_force_mode(EPHMC_FORCE_REFERENCE);
        else if (!std::strcmp(f, "adjoint")) ephmc_set_dropin_force_mode(EPHMC_FORCE_ADJOINT_FP64);
        else if (!std::strcmp(f, "mixed")) ephmc_set_dropin_force_mode(EPHMC_FORCE_MIXED);
    }
    return ephmc_run_hmc_seeded(seed, greens, l1, l2, nt, t, kappa, mu, omega,
                                flavors, contr_mat, steps, traj_length, therm, meas, meas_freq, res_name, corr_name,
                                mode);
}

}  // extern "C"
