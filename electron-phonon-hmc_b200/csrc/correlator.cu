// Current-current correlator (measurement), FP64.
//
// cc_correlator (simulation/organic_dense_matrix.c:451-524):
//   R_t0[tau] = B_tau ... B_{Nt-1} M^-1   (rows propagated, one chain)
//   R_0t(tau) = B_{tau-1} ... B_0 M^-T     (rows propagated, one chain)
//   g_ab(tau) = sum_{i,j} chi_ia(0) chi_jb(tau) [ R_t0[j][i] R_0t[jb][ia] + R_t0[jb][ia] R_0t[j][i]
//                                            - R_t0[jb][i] R_0t[j][ia] - R_t0[j][ia] R_0t[jb][i] ]
//   greens[tau][a][b] = g / ns   (single particle: g e^{-logdet})
// R_t0 is one launch of the slice kernel that keeps every state (the caller's
// Nt V^2 buffer, as the reference's R_t0); R_0t is a single V x V matrix that
// advances one slice after each tau's contraction, as in the reference, so
// no second Nt V^2 stack is held.  Each tau's Wick contraction is one launch
// over j with the 9 (a,b) sums reduced per block.
#include "ephmc_internal.cuh"

namespace ephmc {

namespace {

__global__ void k_cc_contract(const double *__restrict__ x, Couplings c, const int *__restrict__ nbr,
                              const double *__restrict__ Rt0, const double *__restrict__ R0t, int V, int tau,
                              double *__restrict__ part) {
    const int j = blockIdx.x;
    const size_t VV = (size_t)V * V;
    const double *A = Rt0 + (size_t)tau * VV;  // R_t0 at tau
    const double *B = R0t;                     // R_0t at tau
    const double *x0 = x, *xt = x + (size_t)tau * 3 * V;
    double acc[9];
#pragma unroll
    for (int ab = 0; ab < 9; ++ab) acc[ab] = 0.0;
    int jb[3];
    double chj[3];
#pragma unroll
    for (int b = 0; b < 3; ++b) {
        jb[b] = nbr[b * V + j];
        chj[b] = fma(-c.kappa[b], xt[3 * j + b], c.t[b]);
    }
    for (int i = threadIdx.x; i < V; i += blockDim.x) {
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const int ia = nbr[a * V + i];
            const double chi = fma(-c.kappa[a], x0[3 * i + a], c.t[a]);
#pragma unroll
            for (int b = 0; b < 3; ++b) {
                const int jj = jb[b];
                double corr = A[(size_t)j * V + i] * B[(size_t)jj * V + ia];
                corr += A[(size_t)jj * V + ia] * B[(size_t)j * V + i];
                corr -= A[(size_t)jj * V + i] * B[(size_t)j * V + ia];
                corr -= A[(size_t)j * V + ia] * B[(size_t)jj * V + i];
                acc[a * 3 + b] += chi * chj[b] * corr;
            }
        }
    }
    __shared__ double red[9][256];
#pragma unroll
    for (int ab = 0; ab < 9; ++ab) red[ab][threadIdx.x] = acc[ab];
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o)
#pragma unroll
            for (int ab = 0; ab < 9; ++ab) red[ab][threadIdx.x] += red[ab][threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x < 9) part[((size_t)tau * V + j) * 9 + threadIdx.x] = red[threadIdx.x][0];
}

__global__ void k_cc_final(const double *__restrict__ part, int V, int nt, double scale, double *__restrict__ greens) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nt * 9) return;
    const int tau = f / 9, ab = f % 9;
    double g = 0.0;
    for (int j = 0; j < V; ++j) g += part[((size_t)tau * V + j) * 9 + ab];
    greens[f] = g * scale;
}

}  // namespace

int cc_correlator_dev(ephmc_ctx *c, const double *x, const double *Minv, double *R_t0, double *R_0t, double *greens,
                      double logdet) {
    const int V = (int)c->V, nt = (int)c->nt;
    const size_t VV = (size_t)V * V;
    cudaStream_t st = c->stream;
    const bool plain = !(c->flags.zero_filling || c->flags.single_particle);
    double *start_t0 = c->work, *start_0t = R_0t;  // R_0t: one matrix, advanced slice by slice
    int rc;
    if (plain) {
        if ((rc = launch_copy(start_t0, Minv, VV, st))) return rc;
        if ((rc = launch_copy(start_0t, Minv, VV, st))) return rc;
        if ((rc = launch_transpose(start_0t, V, st))) return rc;  // only the transposed R_0t is used
    } else {
        if ((rc = launch_identity(start_t0, V, st))) return rc;
        if ((rc = launch_identity(start_0t, V, st))) return rc;
    }
    // R_t0 chain: slices Nt-1 .. 0 applied to rows, state after slice tau kept at R_t0[tau]
    SliceJob j1{};
    j1.src = start_t0;
    j1.dst = R_t0;
    j1.stack = R_t0;
    j1.stack_off = 0;
    j1.s_first = nt - 1;
    j1.s_count = nt;
    j1.s_dir = -1;
    j1.p_begin = 0;
    j1.p_end = kPairs;
    j1.p_step = 1;
    // R_0t: slice tau applied to the rows in place after tau's contraction
    std::vector<SliceJob> jobs{j1};
    for (int tau = 0; tau + 1 < nt; ++tau) {
        SliceJob j2 = j1;
        j2.src = R_0t;
        j2.dst = R_0t;
        j2.stack = nullptr;
        j2.s_first = tau;
        j2.s_count = 1;
        j2.s_dir = 1;
        jobs.push_back(j2);
    }
    if ((rc = ctx_upload_jobs(c, jobs.data(), (int)jobs.size(), 0, st))) return rc;
    if ((rc = launch_slices<double, double, double>(Axis::Rows, x, c->c, c->lat, c->jobs, 1, st))) return rc;
    double *part = c->cc_part;  // nt * V * 9 doubles
    for (int tau = 0; tau < nt; ++tau) {
        k_cc_contract<<<V, 256, 0, st>>>(x, c->c, c->lat.nbr, R_t0, R_0t, V, tau, part);
        count_launch(1);
        EPHMC_CUDA(cudaGetLastError());
        if (tau + 1 < nt &&
            (rc = launch_slices<double, double, double>(Axis::Rows, x, c->c, c->lat, c->jobs + 1 + tau, 1, st)))
            return rc;
    }
    const double scale = c->flags.single_particle ? std::exp(-logdet) : 1.0 / V;
    k_cc_final<<<(nt * 9 + 127) / 128, 128, 0, st>>>(part, V, nt, scale, greens);
    count_launch(1);
    EPHMC_CUDA(cudaGetLastError());
    return EPHMC_OK;
}

}  // namespace ephmc
