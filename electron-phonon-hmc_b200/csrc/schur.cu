// SCHUR_FORM_INV (simulation/organic_dense_matrix.c:556-603, organic_hmc.c:116,
// construct_QM1P :270-279).
//
// The reference writes M_hat - 1 = Z T Z^T (real Schur form, dgees), and then
// zeroes every entry of T below eps = max Re(ev) * DBL_EPSILON / 1e-3. It does
// this only when min Re(ev) < -1 or eps > 1. It factors T + 1 and returns
// M_hat^-1 = Z (T + 1)^-1 Z^T.  When the regularisation does not trigger,
// Z (T + 1)^-1 Z^T is M_hat^-1 and det(T + 1) = det M_hat (Z is orthogonal),
// so the inverse and log det are those of the LU of M_hat itself.  Here the
// eigenvalues of M_hat - 1 (cuSOLVER Xgeev, values only) decide the
// condition; when it triggers, the zeroed entries depend on the Schur basis
// the solver picks and there is no GPU real Schur decomposition to pick one:
// that case returns EPHMC_ERR_UNSUPPORTED with the eigenvalue bounds.
// The force clamp |G_ij + G_ji| <= 2 of organic_hmc.c:116 applies in every
// force algorithm (k_schur_clamp for the adjoint paths, which never form G).
#include "ephmc_internal.cuh"

#include <cusolverDn.h>

#include <cfloat>
#include <cstdio>
#include <vector>

namespace ephmc {

namespace {

__global__ void k_add_diag(double *A, int V, double a) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < V) A[(size_t)i * V + i] += a;
}

// G = 1 - M (construct_QM1P's Schur branch, :272-274)
__global__ void k_one_minus(double *G, const double *M, int V) {
    const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (size_t)V * V) return;
    const size_t i = e / V, j = e % V;
    G[e] = -M[e] + (i == j ? 1.0 : 0.0);
}

// p = -kappa_k * proj * f  ->  proj = -p / (kappa_k f), clamped to [-2, 2]
__global__ void k_schur_clamp(double *force, size_t n, double k0, double k1, double k2, double f) {
    const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    const int k = (int)(e % 3);
    const double kap = k == 0 ? k0 : (k == 1 ? k1 : k2);
    if (kap == 0.0 || f == 0.0) return;
    const double proj = -force[e] / (kap * f);
    if (fabs(proj) > 2) force[e] = -kap * (proj > 0 ? 2.0 : -2.0) * f;
}

}  // namespace

struct SchurSolver {
    int V = 0;
    cusolverDnHandle_t h = nullptr;
    cusolverDnParams_t p = nullptr;
    void *dwork = nullptr;
    size_t dbytes = 0;
    std::vector<char> hwork;
    double *W = nullptr;  // V complex eigenvalues
    int *info = nullptr;
};

void schur_free(SchurSolver *s) {
    if (!s) return;
    if (s->p) cusolverDnDestroyParams(s->p);
    if (s->h) cusolverDnDestroy(s->h);
    cudaFree(s->dwork);
    cudaFree(s->W);
    cudaFree(s->info);
    cudaGetLastError();
    delete s;
}

namespace {

int schur_init(SchurSolver *s, double *A, int V) {
    if (cusolverDnCreate(&s->h) != CUSOLVER_STATUS_SUCCESS) {
        s->h = nullptr;
        set_status(EPHMC_ERR_CUDA, "SCHUR_FORM_INV: cusolverDnCreate");
        return EPHMC_ERR_CUDA;
    }
    if (cusolverDnCreateParams(&s->p) != CUSOLVER_STATUS_SUCCESS) {
        s->p = nullptr;
        set_status(EPHMC_ERR_CUDA, "SCHUR_FORM_INV: cusolverDnCreateParams");
        return EPHMC_ERR_CUDA;
    }
    if (cudaMalloc(&s->W, sizeof(double) * 2 * V) != cudaSuccess || cudaMalloc(&s->info, sizeof(int)) != cudaSuccess) {
        cudaGetLastError();
        set_status(EPHMC_ERR_NOMEM, "SCHUR_FORM_INV: device allocation");
        return EPHMC_ERR_NOMEM;
    }
    size_t hbytes = 0;
    if (cusolverDnXgeev_bufferSize(s->h, s->p, CUSOLVER_EIG_MODE_NOVECTOR, CUSOLVER_EIG_MODE_NOVECTOR, V, CUDA_R_64F,
                                   A, V, CUDA_C_64F, s->W, CUDA_R_64F, nullptr, 1, CUDA_R_64F, nullptr, 1, CUDA_R_64F,
                                   &s->dbytes, &hbytes) != CUSOLVER_STATUS_SUCCESS) {
        set_status(EPHMC_ERR_CUDA, "SCHUR_FORM_INV: cusolverDnXgeev_bufferSize");
        return EPHMC_ERR_CUDA;
    }
    if (cudaMalloc(&s->dwork, std::max<size_t>(s->dbytes, 16)) != cudaSuccess) {
        cudaGetLastError();
        set_status(EPHMC_ERR_NOMEM, "SCHUR_FORM_INV: device allocation of the eigenvalue workspace");
        return EPHMC_ERR_NOMEM;
    }
    s->hwork.resize(std::max<size_t>(hbytes, 16));
    s->V = V;
    return EPHMC_OK;
}

}  // namespace

// The regularisation condition of logDetM_and_inv_M_hat's Schur branch
// (:556-575) for the device matrix M (V x V, any layout: eigenvalues of M
// and M^T agree); scratch: V*V doubles of device memory.
int schur_check(SchurSolver **slot, const double *M, int V, double *scratch, cudaStream_t st) {
    if (!*slot || (*slot)->V != V) {
        schur_free(*slot);
        *slot = new SchurSolver();
        const int rc = schur_init(*slot, scratch, V);
        if (rc != EPHMC_OK) {
            schur_free(*slot);
            *slot = nullptr;
            return rc;
        }
    }
    SchurSolver *s = *slot;
    EPHMC_CUDA(cudaMemcpyAsync(scratch, M, sizeof(double) * V * V, cudaMemcpyDeviceToDevice, st));
    k_add_diag<<<(V + 255) / 256, 256, 0, st>>>(scratch, V, -1.0);
    count_launch(1);
    EPHMC_CUDA(cudaGetLastError());
    if (cusolverDnSetStream(s->h, st) != CUSOLVER_STATUS_SUCCESS ||
        cusolverDnXgeev(s->h, s->p, CUSOLVER_EIG_MODE_NOVECTOR, CUSOLVER_EIG_MODE_NOVECTOR, V, CUDA_R_64F, scratch, V,
                        CUDA_C_64F, s->W, CUDA_R_64F, nullptr, 1, CUDA_R_64F, nullptr, 1, CUDA_R_64F, s->dwork,
                        s->dbytes, s->hwork.data(), s->hwork.size(), s->info) != CUSOLVER_STATUS_SUCCESS) {
        set_status(EPHMC_ERR_CUDA, "SCHUR_FORM_INV: cusolverDnXgeev");
        return EPHMC_ERR_CUDA;
    }
    std::vector<double> w(2 * (size_t)V);
    int info = 0;
    EPHMC_CUDA(cudaMemcpyAsync(w.data(), s->W, sizeof(double) * 2 * V, cudaMemcpyDeviceToHost, st));
    EPHMC_CUDA(cudaMemcpyAsync(&info, s->info, sizeof(int), cudaMemcpyDeviceToHost, st));
    EPHMC_CUDA(cudaStreamSynchronize(st));
    if (info != 0) {
        set_status(EPHMC_ERR_CUDA, "SCHUR_FORM_INV: the eigenvalue iteration did not converge");
        return EPHMC_ERR_CUDA;
    }
    double min_ev = w[0], max_ev = w[0];
    for (int i = 1; i < V; i++) {
        if (w[2 * i] < min_ev) min_ev = w[2 * i];
        if (w[2 * i] > max_ev) max_ev = w[2 * i];
    }
    const double eps = max_ev * DBL_EPSILON / 1e-3;
    if (min_ev < -1 || eps > 1) {
        char msg[256];
        std::snprintf(msg, sizeof msg,
                      "SCHUR_FORM_INV: the reference's regularisation of the Schur factor applies (min Re ev of "
                      "M_hat - 1 = %.6g, max = %.6g); it depends on the Schur basis and is not implemented",
                      min_ev, max_ev);
        set_status(EPHMC_ERR_UNSUPPORTED, msg);
        return EPHMC_ERR_UNSUPPORTED;
    }
    return EPHMC_OK;
}

int launch_one_minus(double *G, const double *M, int V, cudaStream_t st) {
    const size_t n = (size_t)V * V;
    k_one_minus<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(G, M, V);
    count_launch(1);
    EPHMC_CUDA(cudaGetLastError());
    return EPHMC_OK;
}

int launch_schur_clamp(double *force, size_t n, const double kappa[3], double f, cudaStream_t st) {
    k_schur_clamp<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(force, n, kappa[0], kappa[1], kappa[2], f);
    count_launch(1);
    EPHMC_CUDA(cudaGetLastError());
    return EPHMC_OK;
}

}  // namespace ephmc
