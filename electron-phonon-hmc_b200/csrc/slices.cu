// Slice propagators B_t = f_1(H_t) f_0(H_t) applied to the vectors of V x V
// matrices, FP64, in the summation order of the reference.
//
// Reference: apply_mu_K_to_v / apply_2nd_order_mu_K_to_v / apply_exp_mu_K_to_M
// (simulation/organic_dense_matrix.c:96-120, 168-216).  The reference applies
// the stencil to each contiguous length-V row of a matrix; "Rows" does that,
// "Cols" does the same to each column, which is what the reference obtains by
// transpose -> apply to rows -> transpose (construct_all_QM1P :349-360,
// refine_QM1P :410-424), without the two transposes.
//
// Layout in HBM: matrices are V*V doubles, row-major, rows contiguous.
// One CTA keeps R vectors (8V bytes each) plus their stencil image w and the
// slice's hopping table in shared memory and applies the whole slice sequence
// of its job before writing back, so HBM sees one read and one write per job
// regardless of the number of slices (the unfused bound would be 16 V^2 bytes
// per slice).  The sum for w[j] = mu v[j] + sum_e fac_e v[src_e] is taken in
// the reference's scatter order via the per-site event table, with fma as gcc
// contracts the reference source (fac = t - kappa x fused, w += fac v fused,
// v + fma(a_lin, w, a_quad z) for a pair), so results are bit-identical.
#include "ephmc_internal.cuh"

namespace ephmc {

namespace {

template <typename T> __device__ __forceinline__ T ld_as(const void *p, size_t i);
template <> __device__ __forceinline__ double ld_as<double>(const void *p, size_t i) {
    return static_cast<const double *>(p)[i];
}

template <typename T> __device__ __forceinline__ void st_as(void *p, size_t i, double v);
template <> __device__ __forceinline__ void st_as<double>(void *p, size_t i, double v) {
    static_cast<double *>(p)[i] = v;
}
template <> __device__ __forceinline__ void st_as<float>(void *p, size_t i, double v) {
    static_cast<float *>(p)[i] = static_cast<float>(v);
}

// S sites per thread (site j = threadIdx.x + s*blockDim.x), R vectors per CTA.
// WIDE: one CTA of at most 320 threads per SM, so that the S = 8 sites' hopping
// tables stay in registers (168 instead of 64; with 64 they spill 880 bytes):
// M_hat at 48x48, Nt = 128 takes 25.6 ms instead of 39.1.
template <typename StackT, bool COLS, int S, bool WIDE>
__global__ void __launch_bounds__(WIDE ? 320 : 512, WIDE ? 1 : 2) k_slices(const double *__restrict__ x, Couplings c,
                         const int *__restrict__ ev_src, const int *__restrict__ ev_fac,
                         const SliceJob *__restrict__ jobs, int V, int R) {
    extern __shared__ double smem[];
    double *v = smem;               // [R][V]
    double *w = v + (size_t)R * V;  // [R][V]
    double *fac = w + (size_t)R * V;  // [3V]

    const SliceJob job = jobs[blockIdx.y];
    const int T = blockDim.x, tid = threadIdx.x;
    const int vec0 = blockIdx.x * R;
    const int nvec = min(R, V - vec0);
    if (nvec <= 0) return;
    const size_t VV = (size_t)V * V;

    int src[S][6];
#pragma unroll
    for (int s = 0; s < S; ++s) {
        const int j = tid + s * T;
#pragma unroll
        for (int e = 0; e < 6; ++e) src[s][e] = (j < V) ? ev_src[e * V + j] : 0;
    }

    // ---- load the vectors
    if (job.src == nullptr) {
        for (int f = tid; f < R * V; f += T) {
            const int r = f / V, j = f % V;
            v[f] = (r < nvec && j == vec0 + r) ? 1.0 : 0.0;
        }
    } else if (!COLS) {
        for (int f = tid; f < nvec * V; f += T) v[f] = ld_as<double>(job.src, (size_t)vec0 * V + f);
    } else {
        for (int f = tid; f < nvec * V; f += T) {
            const int r = f % nvec, j = f / nvec;
            v[r * V + j] = ld_as<double>(job.src, (size_t)j * V + vec0 + r);
        }
    }

    for (int it = 0; it < job.s_count; ++it) {
        const int sl = job.s_first + it * job.s_dir;
        __syncthreads();
        const double *xs = x + (size_t)sl * 3 * V;
        for (int e = tid; e < 3 * V; e += T) {
            const int k = e % 3;
            fac[e] = fma(-c.kappa[k], xs[e], c.t[k]);
        }
        __syncthreads();
        double f[S][6];
#pragma unroll
        for (int s = 0; s < S; ++s) {
            const int j = tid + s * T;
#pragma unroll
            for (int e = 0; e < 6; ++e) f[s][e] = (j < V) ? fac[ev_fac[e * V + j]] : 0.0;
        }
        for (int p = job.p_begin; p != job.p_end; p += job.p_step) {
            const double al = c.a_lin[p], aq = c.a_quad[p];
            const bool cplx = c.cplx[p] != 0;
            // w = (mu + K) v
            for (int r = 0; r < nvec; ++r) {
                const double *vr = v + (size_t)r * V;
                double *wr = w + (size_t)r * V;
#pragma unroll
                for (int s = 0; s < S; ++s) {
                    const int j = tid + s * T;
                    if (j < V) {
                        double acc = c.mu * vr[j];
#pragma unroll
                        for (int e = 0; e < 6; ++e) acc = fma(f[s][e], vr[src[s][e]], acc);
                        wr[j] = acc;
                    }
                }
            }
            __syncthreads();
            // z = (mu + K) w at the own site; v += a_lin w + a_quad z
            for (int r = 0; r < nvec; ++r) {
                double *vr = v + (size_t)r * V;
                const double *wr = w + (size_t)r * V;
#pragma unroll
                for (int s = 0; s < S; ++s) {
                    const int j = tid + s * T;
                    if (j < V) {
                        if (cplx) {
                            double acc = c.mu * wr[j];
#pragma unroll
                            for (int e = 0; e < 6; ++e) acc = fma(f[s][e], wr[src[s][e]], acc);
                            vr[j] = vr[j] + fma(al, wr[j], aq * acc);
                        } else {
                            vr[j] = fma(al, wr[j], vr[j]);
                        }
                    }
                }
            }
            __syncthreads();
        }
        if (job.stack != nullptr && (it + 1 < job.s_count || job.dst == nullptr)) {
            StackT *dst = static_cast<StackT *>(job.stack) + (size_t)(sl + job.stack_off) * VV;
            if (!COLS) {
                for (int f = tid; f < nvec * V; f += T) st_as<StackT>(dst, (size_t)vec0 * V + f, v[f]);
            } else {
                for (int f = tid; f < nvec * V; f += T) {
                    const int r = f % nvec, j = f / nvec;
                    st_as<StackT>(dst, (size_t)j * V + vec0 + r, v[r * V + j]);
                }
            }
        }
    }
    __syncthreads();
    if (job.dst == nullptr) return;
    if (job.add_identity) {
        for (int r = tid; r < nvec; r += T) v[(size_t)r * V + vec0 + r] += 1.0;
        __syncthreads();
    }
    if (!COLS) {
        for (int f = tid; f < nvec * V; f += T) st_as<double>(job.dst, (size_t)vec0 * V + f, v[f]);
    } else {
        for (int f = tid; f < nvec * V; f += T) {
            const int r = f % nvec, j = f / nvec;
            st_as<double>(job.dst, (size_t)j * V + vec0 + r, v[r * V + j]);
        }
    }
}

struct Shape {
    int S, T, R;
    size_t smem;
};

size_t shape_smem(int V, int R) { return ((size_t)2 * R * V + 3 * (size_t)V) * sizeof(double); }

Shape pick_shape(const LatticeDev &lat) {
    const int V = lat.V;
    Shape sh{};
    const int opts[5] = {1, 2, 4, 8, 16};
    sh.S = 16;
    for (int o : opts) {
        if ((V + o - 1) / o <= 512) { sh.S = o; break; }
    }
    const int per = (V + sh.S - 1) / sh.S;
    sh.T = ((per + 31) / 32) * 32;
    // vectors per CTA: as many as fit in ~100 KB beside the hopping table
    const size_t budget = 100 * 1024;
    int R = (int)((budget / sizeof(double) - 3 * (size_t)V) / (2 * (size_t)V));
    if (R < 1) R = 1;
    if (R > 8) R = 8;
    sh.R = R;
    // a tuned shape (ephmc_ctx_autotune) replaces the rule when it is valid
    const int tS = lat.tune_slices_S, tR = lat.tune_slices_R;
    if ((tS == 1 || tS == 2 || tS == 4 || tS == 8 || tS == 16) && (V + tS - 1) / tS <= 512) {
        sh.S = tS;
        sh.T = (((V + tS - 1) / tS + 31) / 32) * 32;
    }
    if (tR >= 1 && shape_smem(V, tR) <= 227 * 1024) sh.R = tR;
    sh.smem = shape_smem(V, sh.R);
    return sh;
}

template <typename StackT, bool COLS>
int launch_axis(const double *x, const Couplings &c, const LatticeDev &lat, const SliceJob *jobs,
                int njobs, cudaStream_t st) {
    const int V = lat.V;
    Shape sh = pick_shape(lat);
    if (sh.smem > 227 * 1024) {
        set_status(EPHMC_ERR_UNSUPPORTED, "slice propagation: a vector and its stencil image exceed shared memory");
        return EPHMC_ERR_UNSUPPORTED;
    }
    dim3 grid((V + sh.R - 1) / sh.R, njobs);
    void (*kern)(const double *, Couplings, const int *, const int *, const SliceJob *, int, int) = nullptr;
    switch (sh.S) {
        case 1: kern = k_slices<StackT, COLS, 1, false>; break;
        case 2: kern = k_slices<StackT, COLS, 2, false>; break;
        case 4: kern = k_slices<StackT, COLS, 4, false>; break;
        case 8: kern = sh.T <= 320 ? k_slices<StackT, COLS, 8, true> : k_slices<StackT, COLS, 8, false>; break;
        default: kern = k_slices<StackT, COLS, 16, false>; break;
    }
    EPHMC_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh.smem));
    kern<<<grid, sh.T, sh.smem, st>>>(x, c, lat.ev_src, lat.ev_fac, jobs, V, sh.R); ephmc::count_launch(1);
    EPHMC_CUDA(cudaGetLastError());
    return EPHMC_OK;
}

}  // namespace

template <typename Real, typename Store, typename StackT>
int launch_slices(Axis axis, const double *x, const Couplings &c, const LatticeDev &lat,
                  const SliceJob *jobs_dev, int njobs, cudaStream_t st) {
    static_assert(sizeof(Real) == 8 && sizeof(Store) == 8, "FP64 slice kernels");
    if (njobs <= 0) return EPHMC_OK;
    if (axis == Axis::Rows) return launch_axis<StackT, false>(x, c, lat, jobs_dev, njobs, st);
    return launch_axis<StackT, true>(x, c, lat, jobs_dev, njobs, st);
}

template int launch_slices<double, double, double>(Axis, const double *, const Couplings &,
                                                   const LatticeDev &, const SliceJob *, int,
                                                   cudaStream_t);
template int launch_slices<double, double, float>(Axis, const double *, const Couplings &,
                                                  const LatticeDev &, const SliceJob *, int,
                                                  cudaStream_t);

}  // namespace ephmc
