// Native entry points for the phonon side of the step: Fourier-accelerated
// MD update, momentum refresh scaling, kinetic energy, free-boson sampling
// and the action, all on the context's device buffers.
#include "ephmc_internal.cuh"

#include <cmath>

using namespace ephmc;

namespace {

bool dev_ptr(const void *p) {
    if (!p) return false;
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

int fail(int s, const char *m) {
    set_status(s, m);
    return s;
}

// in-place operation on a caller buffer of n doubles through device buffer `dev`
struct Staged {
    double *user;
    double *d;
    bool host;
};

int stage(ephmc_ctx *c, double *user, double *dev, size_t n, Staged &s) {
    s.user = user;
    s.host = !dev_ptr(user);
    s.d = s.host ? dev : user;
    if (s.host) EPHMC_CUDA(cudaMemcpyAsync(dev, user, sizeof(double) * n, cudaMemcpyHostToDevice, c->stream));
    return EPHMC_OK;
}

int unstage(ephmc_ctx *c, const Staged &s, size_t n) {
    if (s.host) EPHMC_CUDA(cudaMemcpyAsync(s.user, s.d, sizeof(double) * n, cudaMemcpyDeviceToHost, c->stream));
    EPHMC_CUDA(cudaStreamSynchronize(c->stream));
    return EPHMC_OK;
}

// partial sums of x^2 and (x_{t+1} - x_t)^2 (periodic in t) per CTA
__global__ void k_action(const double *__restrict__ x, size_t ld, int nt, double *__restrict__ part) {
    __shared__ double s_pot[256], s_kin[256];
    double pot = 0, kin = 0;
    const size_t n = ld * nt;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const size_t t = i / ld, e = i % ld;
        const double a = x[i];
        const double b = x[((t + 1) % nt) * ld + e];
        pot = fma(a, a, pot);
        kin = fma(b - a, b - a, kin);
    }
    s_pot[threadIdx.x] = pot;
    s_kin[threadIdx.x] = kin;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) {
            s_pot[threadIdx.x] += s_pot[threadIdx.x + o];
            s_kin[threadIdx.x] += s_kin[threadIdx.x + o];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        part[2 * blockIdx.x] = s_pot[0];
        part[2 * blockIdx.x + 1] = s_kin[0];
    }
}

__global__ void k_action_final(const double *__restrict__ part, int nblk, double *__restrict__ out) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        double pot = 0, kin = 0;
        for (int b = 0; b < nblk; ++b) {
            pot += part[2 * b];
            kin += part[2 * b + 1];
        }
        out[0] = pot;
        out[1] = kin;
    }
}

}  // namespace

extern "C" {

// evolve_bosons (simulation/organic_bosons.c:126-150): exact harmonic flow for time h
int ephmc_fa_evolve(ephmc_ctx *c, double *x, double *p, double h) {
    if (!c || !x || !p) return fail(EPHMC_ERR_ARG, "ephmc_fa_evolve");
    EPHMC_CUDA(cudaSetDevice(c->device));
    const size_t dim = (size_t)c->nt * c->V * 3;
    Staged sx{}, sp{};
    int rc;
    if ((rc = stage(c, x, c->x, dim, sx))) return rc;
    if ((rc = stage(c, p, c->force, dim, sp))) return rc;
    if ((rc = fa_evolve(sx.d, sp.d, 3 * (int)c->V, (int)c->nt, c->omega, h, c->scratch, c->stream)))
        return fail(rc, "fa_evolve");
    if ((rc = unstage(c, sx, dim))) return rc;
    return unstage(c, sp, dim);
}

// Fourier part of sample_fourier_momenta (simulation/organic_bosons.c:81-99):
// p holds N(0,1) normals on entry, the accelerated momenta on exit
int ephmc_fa_scale_momenta(ephmc_ctx *c, double *p) {
    if (!c || !p) return fail(EPHMC_ERR_ARG, "ephmc_fa_scale_momenta");
    EPHMC_CUDA(cudaSetDevice(c->device));
    const size_t dim = (size_t)c->nt * c->V * 3;
    Staged sp{};
    int rc;
    if ((rc = stage(c, p, c->force, dim, sp))) return rc;
    double om = c->omega;
    if (c->flags.classical_fourier_acc) om = std::sqrt(c->flags.cfa_mass * c->flags.cfa_mass + om * om);
    if ((rc = fa_scale_modes(sp.d, 3 * (int)c->V, (int)c->nt, om, 1, c->scratch, c->stream)))
        return fail(rc, "fa_scale_modes");
    return unstage(c, sp, dim);
}

// Fourier part of sample_free_bosons (simulation/organic_bosons.c:60-73)
int ephmc_fa_scale_free_bosons(ephmc_ctx *c, double *x) {
    if (!c || !x) return fail(EPHMC_ERR_ARG, "ephmc_fa_scale_free_bosons");
    EPHMC_CUDA(cudaSetDevice(c->device));
    const size_t dim = (size_t)c->nt * c->V * 3;
    Staged sx{};
    int rc;
    if ((rc = stage(c, x, c->x, dim, sx))) return rc;
    if ((rc = fa_scale_modes(sx.d, 3 * (int)c->V, (int)c->nt, c->omega, 2, c->scratch, c->stream)))
        return fail(rc, "fa_scale_modes");
    return unstage(c, sx, dim);
}

// energy_fourier_momenta (simulation/organic_bosons.c:102-124)
int ephmc_fa_energy(ephmc_ctx *c, const double *p, double *energy) {
    if (!c || !p || !energy) return fail(EPHMC_ERR_ARG, "ephmc_fa_energy");
    EPHMC_CUDA(cudaSetDevice(c->device));
    const size_t dim = (size_t)c->nt * c->V * 3;
    const double *pd = p;
    if (!dev_ptr(p)) {
        EPHMC_CUDA(cudaMemcpyAsync(c->force, p, sizeof(double) * dim, cudaMemcpyHostToDevice, c->stream));
        pd = c->force;
    }
    double om = c->omega;
    if (c->flags.classical_fourier_acc) om = std::sqrt(c->flags.cfa_mass * c->flags.cfa_mass + om * om);
    double *out = c->scratch + c->scratch_n - 4;
    int rc = fa_energy(pd, 3 * (int)c->V, (int)c->nt, om, out, c->scratch, c->stream);
    if (rc) return fail(rc, "fa_energy");
    EPHMC_CUDA(cudaMemcpyAsync(energy, out, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    EPHMC_CUDA(cudaStreamSynchronize(c->stream));
    return EPHMC_OK;
}

// evolve_bosons_approx_step (simulation/organic_bosons.c:152-177): x moves by
// h times the accelerated velocity, mode by mode, at frequency
// sqrt(cfa_mass^2 + omega^2) when CLASSICAL_FOURIER_ACC is set
int ephmc_fa_approx_step(ephmc_ctx *c, double *x, const double *p, double h) {
    if (!c || !x || !p) return fail(EPHMC_ERR_ARG, "ephmc_fa_approx_step");
    EPHMC_CUDA(cudaSetDevice(c->device));
    const size_t dim = (size_t)c->nt * c->V * 3;
    Staged sx{}, sp{};
    int rc;
    if ((rc = stage(c, x, c->x, dim, sx))) return rc;
    if ((rc = stage(c, const_cast<double *>(p), c->force, dim, sp))) return rc;
    double om = c->omega;
    if (c->flags.classical_fourier_acc) om = std::sqrt(c->flags.cfa_mass * c->flags.cfa_mass + om * om);
    if ((rc = fa_approx_step(sx.d, sp.d, 3 * (int)c->V, (int)c->nt, om, h, c->scratch, c->stream)))
        return fail(rc, "fa_approx_step");
    return unstage(c, sx, dim);
}

// hamilton (simulation/organic_hmc.c:67-84)
int ephmc_hamilton(ephmc_ctx *c, const double *x, double logdet, double energyP, double *H) {
    if (!c || !x || !H) return fail(EPHMC_ERR_ARG, "ephmc_hamilton");
    EPHMC_CUDA(cudaSetDevice(c->device));
    const size_t ld = (size_t)c->V * 3, dim = ld * c->nt;
    const double *xd = x;
    if (!dev_ptr(x)) {
        EPHMC_CUDA(cudaMemcpyAsync(c->x, x, sizeof(double) * dim, cudaMemcpyHostToDevice, c->stream));
        xd = c->x;
    }
    const int nblk = 64;
    double *part = c->scratch + (c->scratch_n - 8 - ephmc::kActionScratch);  // 2*nblk + 2 doubles
    k_action<<<nblk, 256, 0, c->stream>>>(xd, ld, (int)c->nt, part); ephmc::count_launch(1);
    k_action_final<<<1, 32, 0, c->stream>>>(part, nblk, part + 2 * nblk); ephmc::count_launch(1);
    EPHMC_CUDA(cudaGetLastError());
    double pk[2];
    EPHMC_CUDA(cudaMemcpyAsync(pk, part + 2 * nblk, sizeof(pk), cudaMemcpyDeviceToHost, c->stream));
    EPHMC_CUDA(cudaStreamSynchronize(c->stream));
    *H = -logdet * c->flavors + energyP + (pk[1] / c->omega + pk[0] * c->omega) / 2;
    return EPHMC_OK;
}

}  // extern "C"

namespace ephmc {

// update_x with CLASSICAL_FOURIER_ACC (simulation/organic_hmc.c:142-163): the
// leapfrog step h is split into cfa_steps sub-steps of the harmonic boson
// force (plain omega) and the accelerated kinetic step (accelerated omega);
// half = 0.5 is the first half step, -0.5 the last, 1 a full step.  x, p,
// p_dot: device buffers of the context's shape, on the context's stream.
int classical_update_x(ephmc_ctx *c, double *x, double *p, double *p_dot, double h, double half) {
    const int ld = 3 * (int)c->V, nt = (int)c->nt;
    const size_t dim = (size_t)nt * ld;
    const unsigned steps = c->flags.cfa_steps ? c->flags.cfa_steps : 1;
    double om = c->omega;
    const double om_acc = std::sqrt(c->flags.cfa_mass * c->flags.cfa_mass + om * om);
    h /= steps;
    int rc;
    auto kick = [&](double w) -> int {  // p += w * (boson force at x)
        int r = launch_boson_force(x, p_dot, om, ld, nt, true, c->stream);
        return r ? r : launch_axpy(p, p_dot, w, dim, c->stream);
    };
    auto drift = [&](double w) { return fa_approx_step(x, p, ld, nt, om_acc, w, c->scratch, c->stream); };
    if (half != .5) {
        if ((rc = kick(.5 * h))) return rc;
        for (unsigned k = 0; k < steps / 2; ++k) {
            if ((rc = drift(h))) return rc;
            if ((rc = kick(h))) return rc;
        }
        if ((rc = drift(.5 * h))) return rc;
    }
    if (half != -.5) {
        if ((rc = drift(.5 * h))) return rc;
        for (unsigned k = 0; k < steps / 2; ++k) {
            if ((rc = kick(h))) return rc;
            if ((rc = drift(h))) return rc;
        }
        if ((rc = kick(.5 * h))) return rc;
    }
    return EPHMC_OK;
}

}  // namespace ephmc
