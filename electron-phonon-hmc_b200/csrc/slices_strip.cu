// Slice propagation (sweep 1: M_hat and the q stack) for lattices with
// L1 = 32, with the lattice held in registers.
//
// Same products as k_slices (slices.cu) -- B_t = pair 1 (pair 0) applied to
// the rows of the identity, slice Nt-1 first, the state after each slice
// spilled to the stack -- summed in a different order, so M_hat agrees with
// the reference to rounding rather than bitwise.  Used by the adjoint and
// mixed force paths; the reference path keeps k_slices.
//
// Layout: warp w of the CTA owns rows b = H w .. H w + H-1 of the lattice,
// lane a the column a, for each of the CTA's R vectors; a thread keeps its H
// sites of every vector in registers.  A stencil reads the row neighbours
// (a +- 1) by warp shuffles; the rows above and below inside the strip are
// the thread's own registers, and the two rows just outside the strip come
// from the neighbouring warps through shared memory (one barrier per stencil
// for all R vectors).  Shared-memory traffic per site and stencil drops from
// eight operand loads/stores to the strip ends' share.
#include "ephmc_internal.cuh"

#include <algorithm>

namespace ephmc {

namespace {

constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ double shfl_from(double v, int src) { return __shfl_sync(kFull, v, src); }

// coefficients of the six hopping terms at one site (see stencil())
struct Hop {
    double f0, f1, f2, f0l, f1d, f2dr;
};

// (H v)(a, b) = mu v + f0 v(a+1,b) + f0(a-1,b) v(a-1,b) + f1 v(a,b+1)
//             + f1(a,b-1) v(a,b-1) + f2 v(a-1,b+1) + f2(a+1,b-1) v(a+1,b-1)
__device__ __forceinline__ double stencil(const Hop &h, double mu, double v, double l, double r, double up,
                                          double down, double upleft, double downright) {
    const double s1 = fma(h.f0, r, mu * v);
    const double s2 = fma(h.f1, up, h.f0l * l);
    const double s3 = fma(h.f2, upleft, h.f1d * down);
    return (s1 + s2) + fma(h.f2dr, downright, s3);
}

template <typename T> __device__ __forceinline__ void st_val(T *p, double v);
template <> __device__ __forceinline__ void st_val<double>(double *p, double v) { *p = v; }
template <> __device__ __forceinline__ void st_val<float>(float *p, double v) { *p = (float)v; }

// w[r][h] = (mu + K) v[r][h] for the thread's H sites of R vectors; edge
// exchange through shared memory (edge[2][R][nw][32]: bottom and top rows)
template <int R, int H>
__device__ __forceinline__ void apply_H(const double (&v)[R][H], double (&w)[R][H], const Hop (&hp)[H],
                                        double mu, double *edge, int nw, int warp, int lane) {
    const int below = (warp + nw - 1) % nw, above = (warp + 1) % nw;
    double *bot = edge, *top = edge + (size_t)R * nw * 32;
#pragma unroll
    for (int r = 0; r < R; ++r) {
        bot[(r * nw + warp) * 32 + lane] = v[r][0];
        top[(r * nw + warp) * 32 + lane] = v[r][H - 1];
    }
    __syncthreads();
    const int lm = (lane + 31) & 31, lp = (lane + 1) & 31;
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const double dn = top[(r * nw + below) * 32 + lane];  // row H w - 1
        const double upx = bot[(r * nw + above) * 32 + lane]; // row H w + H
        double L[H], Rt[H];
#pragma unroll
        for (int h = 0; h < H; ++h) {
            L[h] = shfl_from(v[r][h], lm);
            Rt[h] = shfl_from(v[r][h], lp);
        }
        const double dnR = shfl_from(dn, lp);   // (a+1, row below the strip)
        const double upL = shfl_from(upx, lm);  // (a-1, row above the strip)
#pragma unroll
        for (int h = 0; h < H; ++h) {
            const double up = (h + 1 < H) ? v[r][h + 1] : upx;
            const double down = (h > 0) ? v[r][h - 1] : dn;
            const double ul = (h + 1 < H) ? L[h + 1] : upL;
            const double dr = (h > 0) ? Rt[h - 1] : dnR;
            w[r][h] = stencil(hp[h], mu, v[r][h], L[h], Rt[h], up, down, ul, dr);
        }
    }
    __syncthreads();  // the edge buffer is reused by the next stencil
}

template <typename StackT, int R, int H>
__global__ void __launch_bounds__(256) k_slices_strip(const double *__restrict__ x, Couplings cp,
                                                      const SliceJob *__restrict__ jobs, int L2) {
    extern __shared__ double edge[];  // [2][R][nw][32]
    const SliceJob job = jobs[blockIdx.y];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (int)(blockDim.x >> 5);
    const int V = 32 * L2;
    const size_t VV = (size_t)V * V;
    const int vec0 = blockIdx.x * R;
    const int b0 = H * warp;
    const double mu = cp.mu;

    double v[R][H], w[R][H];
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int c = vec0 + r;
#pragma unroll
        for (int h = 0; h < H; ++h) {
            const int i = (b0 + h) * 32 + lane;
            if (job.src == nullptr) v[r][h] = (c < V && i == c) ? 1.0 : 0.0;
            else v[r][h] = (c < V) ? static_cast<const double *>(job.src)[(size_t)c * V + i] : 0.0;
        }
    }
    const int lm = (lane + 31) & 31, lp = (lane + 1) & 31;
    for (int it = 0; it < job.s_count; ++it) {
        const int sl = job.s_first + it * job.s_dir;
        const double *xs = x + (size_t)sl * 3 * V;
        // hopping coefficients of the thread's sites (row below the strip for f1d, f2dr)
        Hop hp[H];
        {
            const int bd = (b0 + L2 - 1) % L2;
            double f1_prev = fma(-cp.kappa[1], xs[3 * (bd * 32 + lane) + 1], cp.t[1]);
            double f2_prev = fma(-cp.kappa[2], xs[3 * (bd * 32 + lane) + 2], cp.t[2]);
#pragma unroll
            for (int h = 0; h < H; ++h) {
                const int i = (b0 + h) * 32 + lane;
                hp[h].f0 = fma(-cp.kappa[0], xs[3 * i + 0], cp.t[0]);
                hp[h].f1 = fma(-cp.kappa[1], xs[3 * i + 1], cp.t[1]);
                hp[h].f2 = fma(-cp.kappa[2], xs[3 * i + 2], cp.t[2]);
                hp[h].f0l = shfl_from(hp[h].f0, lm);
                hp[h].f1d = f1_prev;
                hp[h].f2dr = shfl_from(f2_prev, lp);
                f1_prev = hp[h].f1;
                f2_prev = hp[h].f2;
            }
        }
        for (int p = job.p_begin; p != job.p_end; p += job.p_step) {
            // p is 0 or 1; selecting avoids indexing the parameter struct at run time
            const double al = p ? cp.a_lin[1] : cp.a_lin[0], aq = p ? cp.a_quad[1] : cp.a_quad[0];
            apply_H<R, H>(v, w, hp, mu, edge, nw, warp, lane);
            if (p ? cp.cplx[1] : cp.cplx[0]) {
                double z[R][H];
                apply_H<R, H>(w, z, hp, mu, edge, nw, warp, lane);
#pragma unroll
                for (int r = 0; r < R; ++r)
#pragma unroll
                    for (int h = 0; h < H; ++h) v[r][h] = v[r][h] + fma(al, w[r][h], aq * z[r][h]);
            } else {
#pragma unroll
                for (int r = 0; r < R; ++r)
#pragma unroll
                    for (int h = 0; h < H; ++h) v[r][h] = fma(al, w[r][h], v[r][h]);
            }
        }
        if (job.stack != nullptr && (it + 1 < job.s_count || job.dst == nullptr)) {
            StackT *dst = static_cast<StackT *>(job.stack) + (size_t)(sl + job.stack_off) * VV;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const int c = vec0 + r;
                if (c < V)
#pragma unroll
                    for (int h = 0; h < H; ++h) st_val<StackT>(dst + (size_t)c * V + (b0 + h) * 32 + lane, v[r][h]);
            }
        }
    }
    double *dst = static_cast<double *>(job.dst);
    if (dst == nullptr) return;
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int c = vec0 + r;
        if (c >= V) continue;
#pragma unroll
        for (int h = 0; h < H; ++h) {
            const int i = (b0 + h) * 32 + lane;
            dst[(size_t)c * V + i] = v[r][h] + ((job.add_identity && i == c) ? 1.0 : 0.0);
        }
    }
}

template <typename StackT, int R, int H>
int launch_strip(const double *x, const Couplings &c, const LatticeDev &lat, const SliceJob *jobs, int njobs,
                 cudaStream_t st) {
    const int V = lat.V, L2 = lat.l2, nw = L2 / H;
    const size_t smem = sizeof(double) * 2 * R * (size_t)nw * 32;
    dim3 grid((V + R - 1) / R, njobs);
    k_slices_strip<StackT, R, H><<<grid, 32 * nw, smem, st>>>(x, c, jobs, L2);
    ephmc::count_launch(1);
    EPHMC_CUDA(cudaGetLastError());
    return EPHMC_OK;
}

}  // namespace

bool slices_strip32_supported(const LatticeDev &lat) {
    return lat.l1 == 32 && lat.l2 >= 4 && lat.l2 % 4 == 0 && lat.l2 / 4 <= 8;
}

bool slices_strip_supported(const LatticeDev &lat) { return slices_strip32_supported(lat) || slices_tile_supported(lat); }

template <typename StackT>
int launch_slices_strip(const double *x, const Couplings &c, const LatticeDev &lat, const SliceJob *jobs_dev,
                        int njobs, cudaStream_t st) {
    if (!slices_strip32_supported(lat)) return launch_slices_tile<StackT>(x, c, lat, jobs_dev, njobs, st);
    if (njobs <= 0) return EPHMC_OK;
    return launch_strip<StackT, 2, 4>(x, c, lat, jobs_dev, njobs, st);
}

template int launch_slices_strip<float>(const double *, const Couplings &, const LatticeDev &, const SliceJob *, int,
                                        cudaStream_t);
template int launch_slices_strip<double>(const double *, const Couplings &, const LatticeDev &, const SliceJob *,
                                         int, cudaStream_t);

}  // namespace ephmc

// ---------------------------------------------------------------- FP32 variant
// The stacks of the segmented mixed force start from the identity at each
// segment's top and run at most one segment (<= 16 slices by default), so they
// are propagated in FP32: the two vectors of a CTA are the halves of float2
// pairs and every stencil is one packed FP32 instruction (fma/mul/add
// .rn.f32x2) for both.  Same layout as the FP64 kernel above.
namespace ephmc {

namespace {

using P2 = float2;
__device__ __forceinline__ P2 p2fma(P2 a, P2 b, P2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ P2 p2mul(P2 a, P2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ P2 p2add(P2 a, P2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ P2 p2dup(float c) { return make_float2(c, c); }
__device__ __forceinline__ P2 p2shfl(P2 v, int src) {
    return make_float2(__shfl_sync(0xffffffffu, v.x, src), __shfl_sync(0xffffffffu, v.y, src));
}

struct HopF {
    P2 f0, f1, f2, f0l, f1d, f2dr;
};

__device__ __forceinline__ P2 stencil_f(const HopF &h, P2 mu, P2 v, P2 l, P2 r, P2 up, P2 down, P2 upleft,
                                        P2 downright) {
    const P2 s1 = p2fma(h.f0, r, p2mul(mu, v));
    const P2 s2 = p2fma(h.f1, up, p2mul(h.f0l, l));
    const P2 s3 = p2fma(h.f2, upleft, p2mul(h.f1d, down));
    return p2add(p2add(s1, s2), p2fma(h.f2dr, downright, s3));
}

__device__ __forceinline__ void group_bar(int g, int nthreads) {
    asm volatile("bar.sync %0, %1;" ::"r"(1 + g), "r"(nthreads) : "memory");
}

// w = (mu + K) v for the thread's H sites of both vectors; edge rows through
// shared memory (edge[2][nw][32] pairs of the thread's group), one group
// barrier before and one after
template <int H>
__device__ __forceinline__ void apply_H_f(const P2 (&v)[H], P2 (&w)[H], const HopF (&hp)[H], P2 mu, P2 *edge, int nw,
                                          int warp, int lane, int g) {
    const int below = (warp + nw - 1) % nw, above = (warp + 1) % nw;
    P2 *bot = edge, *top = edge + (size_t)nw * 32;
    bot[warp * 32 + lane] = v[0];
    top[warp * 32 + lane] = v[H - 1];
    group_bar(g, 32 * nw);
    const int lm = (lane + 31) & 31, lp = (lane + 1) & 31;
    const P2 dn = top[below * 32 + lane];
    const P2 upx = bot[above * 32 + lane];
    P2 L[H], Rt[H];
#pragma unroll
    for (int h = 0; h < H; ++h) {
        L[h] = p2shfl(v[h], lm);
        Rt[h] = p2shfl(v[h], lp);
    }
    const P2 dnR = p2shfl(dn, lp), upL = p2shfl(upx, lm);
#pragma unroll
    for (int h = 0; h < H; ++h) {
        const P2 up = (h + 1 < H) ? v[h + 1] : upx;
        const P2 down = (h > 0) ? v[h - 1] : dn;
        const P2 ul = (h + 1 < H) ? L[h + 1] : upL;
        const P2 dr = (h > 0) ? Rt[h - 1] : dnR;
        w[h] = stencil_f(hp[h], mu, v[h], L[h], Rt[h], up, down, ul, dr);
    }
    group_bar(g, 32 * nw);
}

// jobs with an identity start and no destination (every state, the last
// included, goes to the FP32 stack).  A CTA has G independent groups of
// nw = L2/H warps (named barriers per group); work item = (job, vector pair),
// taken grid-stride by the groups, so that a grid of one CTA per SM can run
// beside the LU on the SMs the LU leaves idle.
template <int H, int G>
__global__ void __launch_bounds__(512, 1) k_slices_strip_f32(const double *__restrict__ x, Couplings cp,
                                                             const SliceJob *__restrict__ jobs, int njobs, int L2) {
    extern __shared__ P2 edge_f[];  // [G][2][nw][32]
    const int lane = threadIdx.x & 31, nw = L2 / H;
    const int g = (int)(threadIdx.x >> 5) / nw, warp = (int)(threadIdx.x >> 5) - g * nw;
    P2 *edge_g = edge_f + (size_t)g * 2 * nw * 32;
    const int V = 32 * L2;
    const size_t VV = (size_t)V * V;
    const int b0 = H * warp;
    const P2 mu = p2dup((float)cp.mu);
    const int pairs = V / 2;  // V = 32 L2 is even: both vectors of a pair live
    for (int item = blockIdx.x * G + g; item < njobs * pairs; item += gridDim.x * G) {
    const SliceJob job = jobs[item / pairs];
    const int c0 = (item % pairs) * 2, c1 = c0 + 1;
    P2 v[H], w[H];
#pragma unroll
    for (int h = 0; h < H; ++h) {
        const int i = (b0 + h) * 32 + lane;
        v[h] = make_float2(i == c0 ? 1.f : 0.f, i == c1 ? 1.f : 0.f);
    }
    const int lm = (lane + 31) & 31, lp = (lane + 1) & 31;
    for (int it = 0; it < job.s_count; ++it) {
        const int sl = job.s_first + it * job.s_dir;
        const double *xs = x + (size_t)sl * 3 * V;
        HopF hp[H];
        {
            const int bd = (b0 + L2 - 1) % L2;
            float f1p = (float)fma(-cp.kappa[1], xs[3 * (bd * 32 + lane) + 1], cp.t[1]);
            float f2p = (float)fma(-cp.kappa[2], xs[3 * (bd * 32 + lane) + 2], cp.t[2]);
#pragma unroll
            for (int h = 0; h < H; ++h) {
                const int i = (b0 + h) * 32 + lane;
                const float f0 = (float)fma(-cp.kappa[0], xs[3 * i + 0], cp.t[0]);
                const float f1 = (float)fma(-cp.kappa[1], xs[3 * i + 1], cp.t[1]);
                const float f2 = (float)fma(-cp.kappa[2], xs[3 * i + 2], cp.t[2]);
                hp[h].f0 = p2dup(f0);
                hp[h].f1 = p2dup(f1);
                hp[h].f2 = p2dup(f2);
                hp[h].f0l = p2dup(__shfl_sync(0xffffffffu, f0, lm));
                hp[h].f1d = p2dup(f1p);
                hp[h].f2dr = p2dup(__shfl_sync(0xffffffffu, f2p, lp));
                f1p = f1;
                f2p = f2;
            }
        }
        for (int p = job.p_begin; p != job.p_end; p += job.p_step) {
            const P2 al = p2dup((float)(p ? cp.a_lin[1] : cp.a_lin[0]));
            const P2 aq = p2dup((float)(p ? cp.a_quad[1] : cp.a_quad[0]));
            apply_H_f<H>(v, w, hp, mu, edge_g, nw, warp, lane, g);
            if (p ? cp.cplx[1] : cp.cplx[0]) {
                P2 z[H];
                apply_H_f<H>(w, z, hp, mu, edge_g, nw, warp, lane, g);
#pragma unroll
                for (int h = 0; h < H; ++h) v[h] = p2add(v[h], p2fma(al, w[h], p2mul(aq, z[h])));
            } else {
#pragma unroll
                for (int h = 0; h < H; ++h) v[h] = p2fma(al, w[h], v[h]);
            }
        }
        float *dst = static_cast<float *>(job.stack) + (size_t)(sl + job.stack_off) * VV;
#pragma unroll
        for (int h = 0; h < H; ++h) {
            const int i = (b0 + h) * 32 + lane;
            dst[(size_t)c0 * V + i] = v[h].x;
            dst[(size_t)c1 * V + i] = v[h].y;
        }
    }
    }
}

}  // namespace

int launch_slices_strip_identity_f32(const double *x, const Couplings &c, const LatticeDev &lat,
                                     const SliceJob *jobs_dev, int njobs, cudaStream_t st, int max_ctas) {
    if (!slices_strip32_supported(lat)) return EPHMC_ERR_UNSUPPORTED;
    if (njobs <= 0) return EPHMC_OK;
    constexpr int H = 4, G = 2;
    const int V = lat.V, L2 = lat.l2, nw = L2 / H;
    if (G * nw * 32 > 512) return EPHMC_ERR_UNSUPPORTED;
    const size_t smem = sizeof(P2) * G * 2 * (size_t)nw * 32;
    const int items = njobs * (V / 2);
    const int need = (items + G - 1) / G;
    const int grid = max_ctas > 0 ? std::min(need, max_ctas) : need;
    k_slices_strip_f32<H, G><<<grid, G * 32 * nw, smem, st>>>(x, c, jobs_dev, njobs, L2);
    count_launch(1);
    EPHMC_CUDA(cudaGetLastError());
    return EPHMC_OK;
}

}  // namespace ephmc
