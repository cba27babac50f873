// Slice propagation (sweep 1, the y chain and FP32-stored stacks) for lattices
// with L1 != 32, with the lattice held in registers.
//
// The same products as k_slices (slices.cu) and k_slices_strip
// (slices_strip.cu) -- B_t = pair 1 (pair 0) applied to the rows of the job's
// start matrix, slice s_first first, states spilled to the stack -- summed in
// the order of k_slices_strip, so results agree with the reference's
// (simulation/organic_dense_matrix.c:168-216, construct_M_hat :251-265) to
// rounding rather than bit for bit.
//
// Layout: a lattice row of L1 sites is held by NCL = L1 / W lanes of a group
// of LPR lanes (NCL <= LPR; lanes past NCL idle), W consecutive columns per
// lane; a warp holds G = 32 / LPR groups, and group g of warp w owns the strip
// s = G w + g of H rows.  A thread keeps its H x W sites of each of the CTA's R
// vectors in registers.  A stencil takes the column neighbours inside the
// thread's W columns from its registers and across lanes by warp shuffles
// (two per row instead of two per site), the rows inside the strip from its
// registers, and the two rows just outside the strip from the neighbouring
// strips through shared memory (one barrier per stencil for all R vectors).
#include "ephmc_internal.cuh"

#include <algorithm>

namespace ephmc {

namespace {

constexpr unsigned kFull = 0xffffffffu;

template <typename Real> struct HopT {
    Real f0, f1, f2, f0l, f1d, f2dr;
};

// (H v)(a, b) = mu v + f0 v(a+1,b) + f0(a-1,b) v(a-1,b) + f1 v(a,b+1)
//             + f1(a,b-1) v(a,b-1) + f2 v(a-1,b+1) + f2(a+1,b-1) v(a+1,b-1),
// in the summation order of the L1 = 32 strip kernel
template <typename Real>
__device__ __forceinline__ Real stencil_t(const HopT<Real> &h, Real mu, Real v, Real l, Real r, Real up, Real down,
                                          Real upleft, Real downright) {
    const Real s1 = fma(h.f0, r, mu * v);
    const Real s2 = fma(h.f1, up, h.f0l * l);
    const Real s3 = fma(h.f2, upleft, h.f1d * down);
    return (s1 + s2) + fma(h.f2dr, downright, s3);
}

template <typename T, typename Real> __device__ __forceinline__ void st_t(T *p, Real v) { *p = (T)v; }

// The hopping field of one slice (3V doubles) into shared memory by
// asynchronous copies spread over the CTA: 16 bytes per copy when x and the
// slice size allow it, else 8.  The caller commits the group and waits for it
// with cp.async.wait_group (a hardware wait; no copy is left in flight at exit).
__device__ __forceinline__ void stage_field(double *dst, const double *src, int n3, bool vec16) {
    if (vec16) {
        for (int e = 2 * (int)threadIdx.x; e < n3; e += 2 * (int)blockDim.x)
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((unsigned)__cvta_generic_to_shared(dst + e)),
                         "l"(src + e)
                         : "memory");
    } else {
        for (int e = (int)threadIdx.x; e < n3; e += (int)blockDim.x)
            asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"((unsigned)__cvta_generic_to_shared(dst + e)),
                         "l"(src + e)
                         : "memory");
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
}

// Thread geometry of the tile layout
struct Tile {
    int L1, L2, NS;  // lattice extents, strips
    int s, a0, b0;   // this thread's strip, first column, first row
    int lm, lp;      // lanes holding the columns left of a0 and right of a0 + W - 1
    bool act;        // the lane holds sites
};

template <int W, int LPR, int H>
__device__ __forceinline__ Tile tile_of(int L1, int L2) {
    constexpr int G = 32 / LPR;
    Tile t;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int g = lane / LPR, cl = lane % LPR, ncl = L1 / W;
    t.L1 = L1;
    t.L2 = L2;
    t.NS = L2 / H;
    t.s = warp * G + g;
    t.act = cl < ncl;
    t.a0 = t.act ? cl * W : 0;  // idle lanes mirror column 0 (read only, never stored)
    t.b0 = t.s * H;
    t.lm = g * LPR + (t.act ? (cl == 0 ? ncl - 1 : cl - 1) : 0);
    t.lp = g * LPR + (t.act ? (cl + 1 == ncl ? 0 : cl + 1) : 0);
    return t;
}

// w = (mu + K) v for the thread's H x W sites of R vectors; the strips' bottom
// and top rows through shared memory (edge[2][R][NS][L1])
template <typename Real, int R, int H, int W>
__device__ __forceinline__ void apply_H_tile(const Real (&v)[R][H][W], Real (&w)[R][H][W],
                                             const HopT<Real> (&hp)[H][W], Real mu, Real *edge, const Tile &t) {
    Real *bot = edge, *top = edge + (size_t)R * t.NS * t.L1;
    if (t.act) {
#pragma unroll
        for (int r = 0; r < R; ++r)
#pragma unroll
            for (int c = 0; c < W; ++c) {
                bot[((size_t)r * t.NS + t.s) * t.L1 + t.a0 + c] = v[r][0][c];
                top[((size_t)r * t.NS + t.s) * t.L1 + t.a0 + c] = v[r][H - 1][c];
            }
    }
    __syncthreads();
    const int sb = t.s == 0 ? t.NS - 1 : t.s - 1, sa = t.s + 1 == t.NS ? 0 : t.s + 1;
#pragma unroll
    for (int r = 0; r < R; ++r) {
        Real dn[W], upx[W];
#pragma unroll
        for (int c = 0; c < W; ++c) {
            dn[c] = top[((size_t)r * t.NS + sb) * t.L1 + t.a0 + c];   // row b0 - 1
            upx[c] = bot[((size_t)r * t.NS + sa) * t.L1 + t.a0 + c];  // row b0 + H
        }
        Real Lh[H], Rh[H];  // (a0 - 1, b0 + h), (a0 + W, b0 + h)
#pragma unroll
        for (int h = 0; h < H; ++h) {
            Lh[h] = __shfl_sync(kFull, v[r][h][W - 1], t.lm);
            Rh[h] = __shfl_sync(kFull, v[r][h][0], t.lp);
        }
        const Real upL = __shfl_sync(kFull, upx[W - 1], t.lm);  // (a0 - 1, b0 + H)
        const Real dnR = __shfl_sync(kFull, dn[0], t.lp);       // (a0 + W, b0 - 1)
#pragma unroll
        for (int h = 0; h < H; ++h)
#pragma unroll
            for (int c = 0; c < W; ++c) {
                const Real l = c > 0 ? v[r][h][c - 1] : Lh[h];
                const Real rt = c + 1 < W ? v[r][h][c + 1] : Rh[h];
                const Real up = h + 1 < H ? v[r][h + 1][c] : upx[c];
                const Real down = h > 0 ? v[r][h - 1][c] : dn[c];
                const Real ul = h + 1 < H ? (c > 0 ? v[r][h + 1][c - 1] : Lh[h + 1]) : (c > 0 ? upx[c - 1] : upL);
                const Real dr = h > 0 ? (c + 1 < W ? v[r][h - 1][c + 1] : Rh[h - 1]) : (c + 1 < W ? dn[c + 1] : dnR);
                w[r][h][c] = stencil_t<Real>(hp[h][c], mu, v[r][h][c], l, rt, up, down, ul, dr);
            }
    }
    __syncthreads();  // the edge buffer is reused by the next stencil
}

// byte offset of the staged hopping fields after the edge rows
__host__ __device__ constexpr size_t tile_field_offset(size_t edge_bytes) { return (edge_bytes + 15) / 16 * 16; }

// Real: the arithmetic (double; float for stacks that start from the
// identity and only feed the mixed force, as in the L1 = 32 FP32 kernel)
template <typename Real, typename StackT, int R, int H, int W, int LPR, int MAXT>
__global__ void __launch_bounds__(MAXT) k_slices_tile(const double *__restrict__ x, Couplings cp,
                                                      const SliceJob *__restrict__ jobs, int L1, int L2) {
    extern __shared__ __align__(16) unsigned char smem_t[];
    Real *edge_t = reinterpret_cast<Real *>(smem_t);  // [2][R][NS][L1]
    const SliceJob job = jobs[blockIdx.y];
    const Tile t = tile_of<W, LPR, H>(L1, L2);
    const int V = L1 * L2;
    // the slices' hopping fields, [2][3V] doubles after the edge rows (16-byte
    // aligned): slice it + 1 is copied while slice it is computed
    const int n3 = 3 * V;
    double *xbuf = reinterpret_cast<double *>(smem_t + tile_field_offset(sizeof(Real) * 2 * R * (size_t)t.NS * L1));
    const bool vec16 = (reinterpret_cast<uintptr_t>(x) & 15) == 0 && (n3 & 1) == 0;
    const size_t VV = (size_t)V * V;
    const int vec0 = blockIdx.x * R;
    const Real mu = (Real)cp.mu;

    Real v[R][H][W], w[R][H][W];
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int c = vec0 + r;
#pragma unroll
        for (int h = 0; h < H; ++h)
#pragma unroll
            for (int k = 0; k < W; ++k) {
                const int i = (t.b0 + h) * L1 + t.a0 + k;
                if (job.src == nullptr) v[r][h][k] = (t.act && c < V && i == c) ? Real(1) : Real(0);
                else v[r][h][k] = (t.act && c < V) ? (Real) static_cast<const double *>(job.src)[(size_t)c * V + i] : Real(0);
            }
    }
    const int bd = t.b0 == 0 ? L2 - 1 : t.b0 - 1;  // the row below the strip
    if (job.s_count > 0) stage_field(xbuf, x + (size_t)job.s_first * n3, n3, vec16);
    for (int it = 0; it < job.s_count; ++it) {
        const int sl = job.s_first + it * job.s_dir;
        asm volatile("cp.async.wait_group 0;" ::: "memory");  // this thread's copies of slice it
        __syncthreads();  // everyone's, and every thread is past slice it - 1 (its buffer is free)
        if (it + 1 < job.s_count)
            stage_field(xbuf + (size_t)((it + 1) & 1) * n3, x + (size_t)(sl + job.s_dir) * n3, n3, vec16);
        const double *xs = xbuf + (size_t)(it & 1) * n3;
        // hopping coefficients of the thread's sites (its own links), and of
        // the neighbours they take from (left: link 0, below: link 1, below
        // right: link 2) from its registers, the neighbouring lanes, or, for
        // the strip's bottom row, the row below
        HopT<Real> hp[H][W];
#pragma unroll
        for (int h = 0; h < H; ++h)
#pragma unroll
            for (int k = 0; k < W; ++k) {
                const double *xi = xs + 3 * ((t.b0 + h) * L1 + t.a0 + k);
                hp[h][k].f0 = (Real)fma(-cp.kappa[0], xi[0], cp.t[0]);
                hp[h][k].f1 = (Real)fma(-cp.kappa[1], xi[1], cp.t[1]);
                hp[h][k].f2 = (Real)fma(-cp.kappa[2], xi[2], cp.t[2]);
            }
#pragma unroll
        for (int h = 0; h < H; ++h) {
            const Real f0w = __shfl_sync(kFull, hp[h][W - 1].f0, t.lm);  // (a0 - 1, b)
#pragma unroll
            for (int k = 0; k < W; ++k) hp[h][k].f0l = k > 0 ? hp[h][k - 1].f0 : f0w;
        }
#pragma unroll
        for (int h = H - 1; h > 0; --h) {
            const Real f2e = __shfl_sync(kFull, hp[h - 1][0].f2, t.lp);  // (a0 + W, b - 1)
#pragma unroll
            for (int k = 0; k < W; ++k) {
                hp[h][k].f1d = hp[h - 1][k].f1;
                hp[h][k].f2dr = k + 1 < W ? hp[h - 1][k + 1].f2 : f2e;
            }
        }
#pragma unroll
        for (int k = 0; k < W; ++k) {
            const int a = t.a0 + k, ar = a + 1 == L1 ? 0 : a + 1;
            hp[0][k].f1d = (Real)fma(-cp.kappa[1], xs[3 * (bd * L1 + a) + 1], cp.t[1]);
            hp[0][k].f2dr = (Real)fma(-cp.kappa[2], xs[3 * (bd * L1 + ar) + 2], cp.t[2]);
        }
        for (int p = job.p_begin; p != job.p_end; p += job.p_step) {
            // p is 0 or 1; selecting avoids indexing the parameter struct at run time
            const Real al = (Real)(p ? cp.a_lin[1] : cp.a_lin[0]), aq = (Real)(p ? cp.a_quad[1] : cp.a_quad[0]);
            apply_H_tile<Real, R, H, W>(v, w, hp, mu, edge_t, t);
            if (p ? cp.cplx[1] : cp.cplx[0]) {
                Real z[R][H][W];
                apply_H_tile<Real, R, H, W>(w, z, hp, mu, edge_t, t);
#pragma unroll
                for (int r = 0; r < R; ++r)
#pragma unroll
                    for (int h = 0; h < H; ++h)
#pragma unroll
                        for (int k = 0; k < W; ++k) v[r][h][k] = v[r][h][k] + fma(al, w[r][h][k], aq * z[r][h][k]);
            } else {
#pragma unroll
                for (int r = 0; r < R; ++r)
#pragma unroll
                    for (int h = 0; h < H; ++h)
#pragma unroll
                        for (int k = 0; k < W; ++k) v[r][h][k] = fma(al, w[r][h][k], v[r][h][k]);
            }
        }
        if (job.stack != nullptr && (it + 1 < job.s_count || job.dst == nullptr) && t.act) {
            StackT *dst = static_cast<StackT *>(job.stack) + (size_t)(sl + job.stack_off) * VV;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const int c = vec0 + r;
                if (c < V)
#pragma unroll
                    for (int h = 0; h < H; ++h)
#pragma unroll
                        for (int k = 0; k < W; ++k)
                            st_t<StackT>(dst + (size_t)c * V + (t.b0 + h) * L1 + t.a0 + k, v[r][h][k]);
            }
        }
    }
    double *dst = static_cast<double *>(job.dst);
    if (dst == nullptr || !t.act) return;
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int c = vec0 + r;
        if (c >= V) continue;
#pragma unroll
        for (int h = 0; h < H; ++h)
#pragma unroll
            for (int k = 0; k < W; ++k) {
                const int i = (t.b0 + h) * L1 + t.a0 + k;
                dst[(size_t)c * V + i] = (double)v[r][h][k] + ((job.add_identity && i == c) ? 1.0 : 0.0);
            }
    }
}

// Tile shapes by L1: W columns per lane, LPR lanes per row group, H rows per
// strip, R vectors per CTA.  Threads per CTA: 32 L2 / (H G).
struct TileShape {
    int W, LPR, H, R, maxT;
};

bool tile_shape(int L1, int L2, TileShape &s) {
    switch (L1) {
    case 48: s = {3, 16, 2, 1, 384}; break;
    case 24: s = {3, 8, 1, 2, 256}; break;
    case 16: s = {1, 16, 2, 2, 256}; break;
    case 12: s = {1, 16, 2, 2, 256}; break;  // 12 of 16 lanes per row
    case 8: s = {1, 8, 2, 4, 256}; break;
    default: return false;
    }
    const int G = 32 / s.LPR;
    if (L2 < 2 || L2 % s.H != 0 || (L2 / s.H) % G != 0) return false;
    const int threads = 32 * (L2 / s.H) / G;
    const size_t smem = sizeof(double) * 2 * s.R * (size_t)(L2 / s.H) * L1;
    return threads >= 32 && threads <= s.maxT && smem <= 48 * 1024;
}

template <typename Real, typename StackT, int R, int H, int W, int LPR, int MAXT>
int launch_tile(const double *x, const Couplings &c, const LatticeDev &lat, const SliceJob *jobs, int njobs,
                cudaStream_t st) {
    constexpr int G = 32 / LPR;
    const int V = lat.V, L1 = lat.l1, L2 = lat.l2, NS = L2 / H;
    const int threads = 32 * NS / G;
    if (threads > MAXT) return EPHMC_ERR_UNSUPPORTED;
    const size_t edge = sizeof(Real) * 2 * R * (size_t)NS * L1;
    if (edge > 48 * 1024) return EPHMC_ERR_UNSUPPORTED;
    const size_t smem = tile_field_offset(edge) + 2 * 3 * sizeof(double) * (size_t)V;  // + two slices' fields
    if (smem > 227 * 1024) return EPHMC_ERR_UNSUPPORTED;
    auto kern = k_slices_tile<Real, StackT, R, H, W, LPR, MAXT>;
    EPHMC_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    dim3 grid((V + R - 1) / R, njobs);
    kern<<<grid, threads, smem, st>>>(x, c, jobs, L1, L2);
    ephmc::count_launch(1);
    EPHMC_CUDA(cudaGetLastError());
    return EPHMC_OK;
}

}  // namespace

bool slices_tile_supported(const LatticeDev &lat) {
    TileShape s;
    return tile_shape(lat.l1, lat.l2, s);
}

template <typename StackT>
int launch_slices_tile(const double *x, const Couplings &c, const LatticeDev &lat, const SliceJob *jobs_dev,
                       int njobs, cudaStream_t st) {
    TileShape s;
    if (!tile_shape(lat.l1, lat.l2, s)) return EPHMC_ERR_UNSUPPORTED;
    if (njobs <= 0) return EPHMC_OK;
    switch (lat.l1) {
    case 48: return launch_tile<double, StackT, 1, 2, 3, 16, 384>(x, c, lat, jobs_dev, njobs, st);
    case 24: return launch_tile<double, StackT, 2, 1, 3, 8, 256>(x, c, lat, jobs_dev, njobs, st);
    case 16:
    case 12: return launch_tile<double, StackT, 2, 2, 1, 16, 256>(x, c, lat, jobs_dev, njobs, st);
    case 8: return launch_tile<double, StackT, 4, 2, 1, 8, 256>(x, c, lat, jobs_dev, njobs, st);
    default: return EPHMC_ERR_UNSUPPORTED;
    }
}

// Stacks from the identity in FP32 arithmetic (twice the vectors per CTA)
int launch_slices_tile_identity_f32(const double *x, const Couplings &c, const LatticeDev &lat,
                                    const SliceJob *jobs_dev, int njobs, cudaStream_t st) {
    TileShape s;
    if (!tile_shape(lat.l1, lat.l2, s)) return EPHMC_ERR_UNSUPPORTED;
    if (njobs <= 0) return EPHMC_OK;
    switch (lat.l1) {
    case 48: return launch_tile<float, float, 2, 2, 3, 16, 384>(x, c, lat, jobs_dev, njobs, st);
    case 24: return launch_tile<float, float, 4, 1, 3, 8, 256>(x, c, lat, jobs_dev, njobs, st);
    case 16:
    case 12: return launch_tile<float, float, 4, 2, 1, 16, 256>(x, c, lat, jobs_dev, njobs, st);
    case 8: return launch_tile<float, float, 8, 2, 1, 8, 256>(x, c, lat, jobs_dev, njobs, st);
    default: return EPHMC_ERR_UNSUPPORTED;
    }
}

template int launch_slices_tile<float>(const double *, const Couplings &, const LatticeDev &, const SliceJob *, int,
                                       cudaStream_t);
template int launch_slices_tile<double>(const double *, const Couplings &, const LatticeDev &, const SliceJob *, int,
                                        cudaStream_t);

}  // namespace ephmc
