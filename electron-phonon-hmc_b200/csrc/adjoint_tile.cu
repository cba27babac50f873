// Adjoint sweep 2 in FP32 for lattices with L1 = 8, 12, 16, 24, with the
// lattice held in registers (the register-tile layout of slices_tile.cu).
//
// Same quantities and formulas as k_adjoint_strip (adjoint_strip.cu) -- the
// force of simulation/organic_hmc.c:86-134 through the adjoint of the slice
// chain, levels A-D per slice and the link contraction of refine_QM1P
// (simulation/organic_dense_matrix.c:383-442) -- on the tile layout: NCL =
// L1 / W lanes of a group of LPR lanes hold a lattice row, W consecutive
// columns per lane; a warp holds 32 / LPR groups, each a strip of H rows.  A
// CTA has KG independent vector groups (named barriers per group); a group
// carries two vectors, the halves of packed FP32 pairs, through the slices
// of its segment.  Column neighbours come from
// the thread's registers or, at the block's edges, by warp shuffles (two per
// row); the rows just outside a strip from shared memory.  In the link
// contraction a thread forms, for each of its sites, the right link, the up
// link and the up-left link of its right neighbour (a+1, b), whose up-left
// site (a, b+1) is the thread's own up neighbour; link sums meet in a
// shared-memory accumulator and go to the FP64 force with one atomic per
// (site, link) and slice.
#include "ephmc_internal.cuh"

namespace ephmc {

namespace {

constexpr unsigned kFullA = 0xffffffffu;
constexpr int kSlotsT = 9;  // edge rows exchanged at the widest level

// packed FP32 pairs (the kernel's vector type is a template parameter; the
// shapes in use all carry two vectors per group)
template <typename VT> struct VOps;
template <> struct VOps<float2> {
    static constexpr int kVec = 2;
    static __device__ __forceinline__ float2 fma_(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
    static __device__ __forceinline__ float2 mul(float2 a, float2 b) { return __fmul2_rn(a, b); }
    static __device__ __forceinline__ float2 add(float2 a, float2 b) { return __fadd2_rn(a, b); }
    static __device__ __forceinline__ float2 dup(float c) { return make_float2(c, c); }
    static __device__ __forceinline__ float2 shfl(float2 v, int src) {
        return make_float2(__shfl_sync(kFullA, v.x, src), __shfl_sync(kFullA, v.y, src));
    }
    static __device__ __forceinline__ float sum(float2 v) { return v.x + v.y; }
    static __device__ __forceinline__ float2 make(float a, float b) { return make_float2(a, b); }
    static __device__ __forceinline__ float lo(float2 v) { return v.x; }
    static __device__ __forceinline__ float hi(float2 v) { return v.y; }
};

// FP32 hopping coefficients of one site
struct HopS {
    float f0, f1, f2, f0l, f1d, f2dr;
};

template <typename VT>
__device__ __forceinline__ VT stencil_v(const HopS &h, VT mu, VT v, VT l, VT r, VT up, VT down, VT upleft,
                                        VT downright) {
    using O = VOps<VT>;
    const VT s1 = O::fma_(O::dup(h.f0), r, O::mul(mu, v));
    const VT s2 = O::fma_(O::dup(h.f1), up, O::mul(O::dup(h.f0l), l));
    const VT s3 = O::fma_(O::dup(h.f2), upleft, O::mul(O::dup(h.f1d), down));
    return O::add(O::add(s1, s2), O::fma_(O::dup(h.f2dr), downright, s3));
}

__device__ __forceinline__ void vgroup_sync(int g, int nthreads) {
    asm volatile("bar.sync %0, %1;" ::"r"(1 + g), "r"(nthreads) : "memory");
}

// Geometry of a thread in its vector group
struct TileA {
    int L1, L2, NS;
    int s, a0, b0, lm, lp;
    bool act;
};

// Edge rows of one group and buffer: [kSlotsT][NS][L1]
template <typename VT> struct EdgesT {
    VT *base;
    int NS, L1;
    __device__ VT *row(int slot, int strip) const { return base + ((size_t)slot * NS + strip) * L1; }
};

// out = H in for the thread's H x W sites; the rows outside the strip from the
// edge slots slot_bot (bottom rows) and slot_top (top rows) of buffer E
template <typename VT, int H, int W>
__device__ __forceinline__ void stencil_tile(const VT (&in)[H][W], VT (&out)[H][W], const HopS (&hp)[H][W], VT mu,
                                             const EdgesT<VT> &E, int slot_bot, int slot_top, const TileA &t) {
    using O = VOps<VT>;
    const int sb = t.s == 0 ? t.NS - 1 : t.s - 1, sa = t.s + 1 == t.NS ? 0 : t.s + 1;
    VT dn[W], upx[W];
#pragma unroll
    for (int c = 0; c < W; ++c) {
        dn[c] = E.row(slot_top, sb)[t.a0 + c];
        upx[c] = E.row(slot_bot, sa)[t.a0 + c];
    }
    VT Lh[H], Rh[H];
#pragma unroll
    for (int h = 0; h < H; ++h) {
        Lh[h] = O::shfl(in[h][W - 1], t.lm);
        Rh[h] = O::shfl(in[h][0], t.lp);
    }
    const VT upL = O::shfl(upx[W - 1], t.lm), dnR = O::shfl(dn[0], t.lp);
#pragma unroll
    for (int h = 0; h < H; ++h)
#pragma unroll
        for (int c = 0; c < W; ++c) {
            const VT l = c > 0 ? in[h][c - 1] : Lh[h];
            const VT rt = c + 1 < W ? in[h][c + 1] : Rh[h];
            const VT up = h + 1 < H ? in[h + 1][c] : upx[c];
            const VT down = h > 0 ? in[h - 1][c] : dn[c];
            const VT ul = h + 1 < H ? (c > 0 ? in[h + 1][c - 1] : Lh[h + 1]) : (c > 0 ? upx[c - 1] : upL);
            const VT dr = h > 0 ? (c + 1 < W ? in[h - 1][c + 1] : Rh[h - 1]) : (c + 1 < W ? dn[c + 1] : dnR);
            out[h][c] = stencil_v<VT>(hp[h][c], mu, in[h][c], l, rt, up, down, ul, dr);
        }
}

template <typename VT, int H, int W>
__device__ __forceinline__ void put_rows(const EdgesT<VT> &E, int slot_bot, int slot_top, const VT (&v)[H][W],
                                         const TileA &t) {
    if (!t.act) return;
#pragma unroll
    for (int c = 0; c < W; ++c) {
        E.row(slot_bot, t.s)[t.a0 + c] = v[0][c];
        E.row(slot_top, t.s)[t.a0 + c] = v[H - 1][c];
    }
}

// the quantities of one site entering the link contraction, with
// L1 = a0 q + b0 Hq and L3 = a1 f0q + b1 H f0q formed once per site
template <typename VT> struct SiteT {
    VT q, L1, f0q, L3, y, hy, f1y, hf1y;
};

template <typename VT> __device__ __forceinline__ SiteT<VT> shfl_site_t(const SiteT<VT> &s, int src) {
    using O = VOps<VT>;
    return SiteT<VT>{O::shfl(s.q, src),  O::shfl(s.L1, src), O::shfl(s.f0q, src), O::shfl(s.L3, src),
                     O::shfl(s.y, src),  O::shfl(s.hy, src), O::shfl(s.f1y, src), O::shfl(s.hf1y, src)};
}

// link (i, n) entry of D + D^T:
//   d = L1_i f1y_n + L1_n f1y_i + b0 (q_i Hf1y_n + q_n Hf1y_i)
//     + L3_i y_n + L3_n y_i + b1 (f0q_i Hy_n + f0q_n Hy_i)
template <typename VT>
__device__ __forceinline__ VT link_term_t(const SiteT<VT> &i, const SiteT<VT> &n, VT aq0, VT aq1) {
    using O = VOps<VT>;
    const VT d1 = O::fma_(i.L1, n.f1y, O::mul(n.L1, i.f1y));
    const VT e1 = O::fma_(aq0, O::fma_(i.q, n.hf1y, O::mul(n.q, i.hf1y)), d1);
    const VT d3 = O::fma_(i.L3, n.y, O::mul(n.L3, i.y));
    const VT e3 = O::fma_(aq1, O::fma_(i.f0q, n.hy, O::mul(n.f0q, i.hy)), d3);
    return O::add(e1, e3);
}

__device__ __forceinline__ double pick3t(const double (&a)[3], int k) { return k == 0 ? a[0] : k == 1 ? a[1] : a[2]; }

// MODE 0: all slices from M^-1; 1: one segment of a checkpointed sweep
// (AdjointRange t0, t1, q_top, y_in, y_out); 2: the segment grid
// (AdjointRange seg_*), one segment per blockIdx.y
template <typename VT, int W, int LPR, int H, int KG, int MAXT, int MODE>
__global__ void __launch_bounds__(MAXT, 1) k_adjoint_tile(const double *__restrict__ x, Couplings cp,
                                                         const float *__restrict__ qstack,
                                                         const double *__restrict__ Minv, int L1, int L2, int nt,
                                                         double pref, double *__restrict__ force,
                                                         AdjointRange rg_in) {
    using O = VOps<VT>;
    constexpr int Gl = 32 / LPR, NV = VOps<VT>::kVec;
    AdjointRange rg = rg_in;
    if (MODE == 0) rg = AdjointRange{0, nt, nullptr, nullptr, nullptr, true};
    extern __shared__ __align__(16) float sm_t[];
    const int V = L1 * L2, NS = L2 / H, NWg = NS / Gl;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int g = warp / NWg, wl = warp - g * NWg;
    TileA t;
    {
        const int gl = lane / LPR, cl = lane % LPR, ncl = L1 / W;
        t.L1 = L1;
        t.L2 = L2;
        t.NS = NS;
        t.s = wl * Gl + gl;
        t.act = cl < ncl;
        t.a0 = t.act ? cl * W : 0;
        t.b0 = t.s * H;
        t.lm = gl * LPR + (t.act ? (cl == 0 ? ncl - 1 : cl - 1) : 0);
        t.lp = gl * LPR + (t.act ? (cl + 1 == ncl ? 0 : cl + 1) : 0);
    }
    float *acc = sm_t;  // [2][V][3] link sums, by slice parity
    VT *edges = reinterpret_cast<VT *>(sm_t + 6 * V);
    const size_t ebuf = (size_t)kSlotsT * NS * L1;
    EdgesT<VT> eb[2];
#pragma unroll
    for (int k = 0; k < 2; ++k) eb[k] = EdgesT<VT>{edges + (2 * g + k) * ebuf, NS, L1};
    const VT mu = O::dup((float)cp.mu);
    const VT al0 = O::dup((float)cp.a_lin[0]), aq0 = O::dup((float)cp.a_quad[0]);
    const VT al1 = O::dup((float)cp.a_lin[1]), aq1 = O::dup((float)cp.a_quad[1]);
    const size_t VV = (size_t)V * V;
    const int cv0 = (blockIdx.x * KG + g) * NV;
    const int cv1 = NV == 2 ? cv0 + 1 : cv0;
    const bool live = cv0 < V;  // (NV = 2: V is even, both vectors are live together)
    int q_id_slice = nt - 1;
    if (MODE == 2) {
        const int j = rg.seg_j0 + (int)blockIdx.y;
        rg.t1 = nt - j * rg.seg_C;
        rg.t0 = max(0, rg.t1 - rg.seg_C);
        q_id_slice = rg.t1 - 1;
        qstack += rg.seg_regions ? (size_t)j * rg.seg_C * VV : 0;
        rg.y_start += rg.seg_regions ? (size_t)j * VV : 0;
        rg.q_top = nullptr;
        rg.y_out = nullptr;
    }
    const int c0v = live ? cv0 : 0, c1v = live ? cv1 : 0;  // idle groups read vector 0, store nothing

    const float *y_in = static_cast<const float *>(rg.y_in);
    VT y[H][W];
#pragma unroll
    for (int h = 0; h < H; ++h)
#pragma unroll
        for (int k = 0; k < W; ++k) {
            const int i = (t.b0 + h) * L1 + t.a0 + k;
            if (MODE == 2)
                y[h][k] = O::make((float)rg.y_start[(size_t)c0v * V + i], (float)rg.y_start[(size_t)c1v * V + i]);
            else
                y[h][k] = y_in ? O::make(y_in[(size_t)c0v * V + i], y_in[(size_t)c1v * V + i])
                               : O::make((float)Minv[(size_t)i * V + c0v], (float)Minv[(size_t)i * V + c1v]);
        }
    for (int e = threadIdx.x; e < 6 * V; e += blockDim.x) acc[e] = 0.f;
    __syncthreads();
    const int nthr = 32 * NWg;
    const int bd = t.b0 == 0 ? L2 - 1 : t.b0 - 1;

    for (int ts = rg.t0; ts < rg.t1; ++ts) {
        float *acc_t = acc + (ts & 1) * 3 * V;
        const double *xs = x + (size_t)ts * 3 * V;
        // own links from x; the neighbours' from registers, the neighbouring
        // lanes, or (the strip's bottom row) the row below
        HopS hp[H][W];
#pragma unroll
        for (int h = 0; h < H; ++h)
#pragma unroll
            for (int k = 0; k < W; ++k) {
                const double *xi = xs + 3 * ((t.b0 + h) * L1 + t.a0 + k);
                hp[h][k].f0 = (float)fma(-cp.kappa[0], __ldg(xi + 0), cp.t[0]);
                hp[h][k].f1 = (float)fma(-cp.kappa[1], __ldg(xi + 1), cp.t[1]);
                hp[h][k].f2 = (float)fma(-cp.kappa[2], __ldg(xi + 2), cp.t[2]);
            }
#pragma unroll
        for (int h = 0; h < H; ++h) {
            const float f0w = __shfl_sync(kFullA, hp[h][W - 1].f0, t.lm);
#pragma unroll
            for (int k = 0; k < W; ++k) hp[h][k].f0l = k > 0 ? hp[h][k - 1].f0 : f0w;
        }
#pragma unroll
        for (int h = H - 1; h > 0; --h) {
            const float f2e = __shfl_sync(kFullA, hp[h - 1][0].f2, t.lp);
#pragma unroll
            for (int k = 0; k < W; ++k) {
                hp[h][k].f1d = hp[h - 1][k].f1;
                hp[h][k].f2dr = k + 1 < W ? hp[h - 1][k + 1].f2 : f2e;
            }
        }
#pragma unroll
        for (int k = 0; k < W; ++k) {
            const int a = t.a0 + k, ar = a + 1 == L1 ? 0 : a + 1;
            hp[0][k].f1d = (float)fma(-cp.kappa[1], __ldg(xs + 3 * (bd * L1 + a) + 1), cp.t[1]);
            hp[0][k].f2dr = (float)fma(-cp.kappa[2], __ldg(xs + 3 * (bd * L1 + ar) + 2), cp.t[2]);
        }
        // q(t): the stack entry t - t0, the segment's FP64 checkpoint (its last
        // slice, checkpointed evaluation), or e_c (slice nt-1; the top slice of
        // a segment of the grid)
        VT q[H][W];
        {
            const bool top = rg.q_top != nullptr && ts == rg.t1 - 1;
            const float *qs = qstack + (size_t)(ts - rg.t0) * VV;
#pragma unroll
            for (int h = 0; h < H; ++h)
#pragma unroll
                for (int k = 0; k < W; ++k) {
                    const int i = (t.b0 + h) * L1 + t.a0 + k;
                    q[h][k] = (ts == q_id_slice) ? O::make(i == cv0 ? 1.f : 0.f, i == cv1 ? 1.f : 0.f)
                              : top ? O::make((float)rg.q_top[(size_t)c0v * V + i], (float)rg.q_top[(size_t)c1v * V + i])
                                    : O::make(__ldg(qs + (size_t)c0v * V + i), __ldg(qs + (size_t)c1v * V + i));
                }
        }
        VT hq[H][W], hy[H][W], f0q[H][W], f1y[H][W], hf0q[H][W], hf1y[H][W];
        // level A: hq = H q, hy = H y
        put_rows<VT, H, W>(eb[0], 0, 1, q, t);
        put_rows<VT, H, W>(eb[0], 2, 3, y, t);
        vgroup_sync(g, nthr);
        stencil_tile<VT, H, W>(q, hq, hp, mu, eb[0], 0, 1, t);
        stencil_tile<VT, H, W>(y, hy, hp, mu, eb[0], 2, 3, t);
        // level B: f0q = q + a0 hq + b0 H hq, f1y = y + a1 hy + b1 H hy
        put_rows<VT, H, W>(eb[1], 0, 1, hq, t);
        put_rows<VT, H, W>(eb[1], 2, 3, hy, t);
        vgroup_sync(g, nthr);
        {
            VT z[H][W];
            stencil_tile<VT, H, W>(hq, z, hp, mu, eb[1], 0, 1, t);
#pragma unroll
            for (int h = 0; h < H; ++h)
#pragma unroll
                for (int k = 0; k < W; ++k) f0q[h][k] = O::add(q[h][k], O::fma_(al0, hq[h][k], O::mul(aq0, z[h][k])));
            stencil_tile<VT, H, W>(hy, z, hp, mu, eb[1], 2, 3, t);
#pragma unroll
            for (int h = 0; h < H; ++h)
#pragma unroll
                for (int k = 0; k < W; ++k) f1y[h][k] = O::add(y[h][k], O::fma_(al1, hy[h][k], O::mul(aq1, z[h][k])));
        }
        // level C: hf0q = H f0q, hf1y = H f1y
        put_rows<VT, H, W>(eb[0], 0, 1, f0q, t);
        put_rows<VT, H, W>(eb[0], 2, 3, f1y, t);
        vgroup_sync(g, nthr);
        stencil_tile<VT, H, W>(f0q, hf0q, hp, mu, eb[0], 0, 1, t);
        stencil_tile<VT, H, W>(f1y, hf1y, hp, mu, eb[0], 2, 3, t);
        // level D: the link contraction, then the next y; edges: hf1y
        // bottom/top rows and the bottom rows of seven link quantities (with
        // hf1y's bottom row, the up neighbours of the strip's top row)
        {
            const EdgesT<VT> &E = eb[1];
            put_rows<VT, H, W>(E, 0, 1, hf1y, t);
            if (t.act) {
#pragma unroll
                for (int k = 0; k < W; ++k) {
                    E.row(2, t.s)[t.a0 + k] = q[0][k];
                    E.row(3, t.s)[t.a0 + k] = O::fma_(al0, q[0][k], O::mul(aq0, hq[0][k]));
                    E.row(4, t.s)[t.a0 + k] = f0q[0][k];
                    E.row(5, t.s)[t.a0 + k] = O::fma_(al1, f0q[0][k], O::mul(aq1, hf0q[0][k]));
                    E.row(6, t.s)[t.a0 + k] = y[0][k];
                    E.row(7, t.s)[t.a0 + k] = hy[0][k];
                    E.row(8, t.s)[t.a0 + k] = f1y[0][k];
                }
            }
            vgroup_sync(g, nthr);
            const int sa = t.s + 1 == NS ? 0 : t.s + 1;
#pragma unroll
            for (int h = 0; h < H; ++h) {
                const int b = t.b0 + h;
                SiteT<VT> sr[W];
#pragma unroll
                for (int k = 0; k < W; ++k)
                    sr[k] = SiteT<VT>{q[h][k], O::fma_(al0, q[h][k], O::mul(aq0, hq[h][k])), f0q[h][k],
                                      O::fma_(al1, f0q[h][k], O::mul(aq1, hf0q[h][k])), y[h][k], hy[h][k],
                                      f1y[h][k], hf1y[h][k]};
                const SiteT<VT> rn = shfl_site_t<VT>(sr[0], t.lp);  // (a0 + W, b)
#pragma unroll
                for (int k = 0; k < W; ++k) {
                    const int a = t.a0 + k, ar = a + 1 == L1 ? 0 : a + 1;
                    SiteT<VT> up;
                    if (h + 1 < H) {
                        const int hu = h + 1 < H ? h + 1 : h;
                        up = SiteT<VT>{q[hu][k], O::fma_(al0, q[hu][k], O::mul(aq0, hq[hu][k])), f0q[hu][k],
                                       O::fma_(al1, f0q[hu][k], O::mul(aq1, hf0q[hu][k])), y[hu][k], hy[hu][k],
                                       f1y[hu][k], hf1y[hu][k]};
                    } else {
                        up = SiteT<VT>{E.row(2, sa)[a], E.row(3, sa)[a], E.row(4, sa)[a], E.row(5, sa)[a],
                                       E.row(6, sa)[a], E.row(7, sa)[a], E.row(8, sa)[a], E.row(0, sa)[a]};
                    }
                    const SiteT<VT> &right = k + 1 < W ? sr[k + 1 < W ? k + 1 : k] : rn;
                    const VT lr = link_term_t<VT>(sr[k], right, aq0, aq1);  // site (a, b), link 0
                    const VT lu = link_term_t<VT>(sr[k], up, aq0, aq1);     // site (a, b), link 1
                    const VT lul = link_term_t<VT>(right, up, aq0, aq1);    // site (a+1, b), link 2
                    if (t.act && live) {
                        atomicAdd(acc_t + 3 * (b * L1 + a) + 0, O::sum(lr));
                        atomicAdd(acc_t + 3 * (b * L1 + a) + 1, O::sum(lu));
                        atomicAdd(acc_t + 3 * (b * L1 + ar) + 2, O::sum(lul));
                    }
                }
            }
            VT z[H][W];
            stencil_tile<VT, H, W>(hf1y, z, hp, mu, E, 0, 1, t);
#pragma unroll
            for (int h = 0; h < H; ++h)
#pragma unroll
                for (int k = 0; k < W; ++k) y[h][k] = O::add(f1y[h][k], O::fma_(al0, hf1y[h][k], O::mul(aq0, z[h][k])));
        }
        // every group's sums of slice t are in acc_t: add them to the force and
        // clear the buffer, which slice t+2 reuses (after the next barrier)
        __syncthreads();
        for (int e = threadIdx.x; e < 3 * V; e += blockDim.x) {
            atomicAdd(force + (size_t)ts * 3 * V + e, -pick3t(cp.kappa, e % 3) * pref * (double)acc_t[e]);
            acc_t[e] = 0.f;
        }
    }
    if (MODE != 2 && rg.y_out != nullptr && t.act && live) {
        float *y_out = static_cast<float *>(rg.y_out);
#pragma unroll
        for (int h = 0; h < H; ++h)
#pragma unroll
            for (int k = 0; k < W; ++k) {
                const int i = (t.b0 + h) * L1 + t.a0 + k;
                y_out[(size_t)cv0 * V + i] = O::lo(y[h][k]);
                if (NV == 2) y_out[(size_t)cv1 * V + i] = O::hi(y[h][k]);
            }
    }
}

struct AdjShape {
    int W, LPR, H, KG, maxT;
};

bool adj_tile_shape(int L1, int L2, AdjShape &s) {
    // (not L1 = 48: one vector per CTA at 384 threads and 221 KB of shared
    // memory left one vector in flight per SM, and the shared-memory kernel
    // k_adjoint was faster there: 22 against 34 ms per 48x48, Nt = 128 force)
    switch (L1) {
    case 24: s = {3, 8, 1, 2, 384}; break;
    case 16: s = {1, 16, 2, 2, 256}; break;
    case 12: s = {1, 16, 2, 2, 256}; break;
    case 8: s = {1, 8, 2, 2, 256}; break;
    default: return false;
    }
    const int Gl = 32 / s.LPR;
    if (L2 < 2 || L2 % s.H != 0 || (L2 / s.H) % Gl != 0) return false;
    const int threads = s.KG * 32 * (L2 / s.H) / Gl;
    const size_t vt = sizeof(float2);
    const size_t smem = sizeof(float) * 6 * (size_t)L1 * L2 + vt * 2 * s.KG * (size_t)kSlotsT * (L2 / s.H) * L1;
    return threads >= 32 && threads <= s.maxT && smem <= 227 * 1024;
}

template <typename VT, int W, int LPR, int H, int KG, int MAXT>
int launch_adj_tile(const double *x, const Couplings &c, const LatticeDev &lat, const float *qstack,
                    const double *Minv, int nt, double pref, double *force, cudaStream_t st, const AdjointRange &rg,
                    bool range, int seg_count) {
    constexpr int Gl = 32 / LPR, NV = VOps<VT>::kVec;
    const int V = lat.V, L1 = lat.l1, L2 = lat.l2, NS = L2 / H;
    const int threads = KG * 32 * (NS / Gl);
    if (threads > MAXT) return EPHMC_ERR_UNSUPPORTED;
    const size_t smem = sizeof(float) * 6 * (size_t)V + sizeof(VT) * 2 * KG * (size_t)kSlotsT * NS * L1;
    if (smem > 227 * 1024) return EPHMC_ERR_UNSUPPORTED;
    const int per_cta = KG * NV;
    const dim3 grid((V + per_cta - 1) / per_cta, rg.seg_C > 0 ? (unsigned)seg_count : 1u);
    void (*kern)(const double *, Couplings, const float *, const double *, int, int, int, double, double *,
                 AdjointRange) = rg.seg_C > 0 ? k_adjoint_tile<VT, W, LPR, H, KG, MAXT, 2>
                                 : range      ? k_adjoint_tile<VT, W, LPR, H, KG, MAXT, 1>
                                              : k_adjoint_tile<VT, W, LPR, H, KG, MAXT, 0>;
    EPHMC_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    kern<<<grid, threads, smem, st>>>(x, c, qstack, Minv, L1, L2, nt, pref, force, rg);
    ephmc::count_launch(1);
    EPHMC_CUDA(cudaGetLastError());
    return EPHMC_OK;
}

}  // namespace

bool adjoint_tile_supported(const LatticeDev &lat) {
    AdjShape s;
    return adj_tile_shape(lat.l1, lat.l2, s);
}

int launch_adjoint_tile(const double *x, const Couplings &c, const LatticeDev &lat, const float *qstack,
                        const double *Minv, int nt, unsigned flavors, int single_particle, double logdet,
                        double *force, cudaStream_t st, const AdjointRange *range, int seg_count) {
    if (!adjoint_tile_supported(lat)) return EPHMC_ERR_UNSUPPORTED;
    double pref = (double)flavors;
    if (single_particle) pref *= exp(-logdet);
    AdjointRange rg{0, nt, nullptr, nullptr, nullptr, true};
    if (range) rg = *range;
    if (rg.zero_force) EPHMC_CUDA(cudaMemsetAsync(force, 0, sizeof(double) * (size_t)nt * lat.V * 3, st));
    const bool r = range != nullptr;
    switch (lat.l1) {
    case 24: return launch_adj_tile<float2, 3, 8, 1, 2, 384>(x, c, lat, qstack, Minv, nt, pref, force, st, rg, r, seg_count);
    case 16:
    case 12: return launch_adj_tile<float2, 1, 16, 2, 2, 256>(x, c, lat, qstack, Minv, nt, pref, force, st, rg, r, seg_count);
    case 8: return launch_adj_tile<float2, 1, 8, 2, 2, 256>(x, c, lat, qstack, Minv, nt, pref, force, st, rg, r, seg_count);
    default: return EPHMC_ERR_UNSUPPORTED;
    }
}

}  // namespace ephmc
