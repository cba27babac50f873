// Adjoint sweep 2 in FP32 for lattices with L1 = 32, with the lattice held
// in registers (the layout of slices_strip.cu).
//
// Same quantities as k_adjoint (adjoint.cu) -- the force of
// simulation/organic_hmc.c:86-134 through the adjoint of the slice chain --
// with the same formulas, summed in a different order.
//
// A CTA has G = 2 independent groups of nw = L2/4 warps; each group carries
// two vectors through all slices, held as the two halves of float2 pairs so
// that every stencil, combination and link product is one packed FP32
// instruction (fma/mul/add .rn.f32x2) for both vectors.  Warp w of a group
// owns rows 4w .. 4w+3, lane a the column a; a thread keeps its 4 sites of
// the pair in registers.  Per slice and group:
//   level A  hq = H q, hy = H y
//   level B  f0q = q + a0 hq + b0 H hq,  f1y = y + a1 hy + b1 H hy
//   level C  hf0q = H f0q, hf1y = H f1y
//   level D  y <- f1y + a0 hf1y + b0 H hf1y, and the link contraction
// Row neighbours (a +- 1) come from warp shuffles; the rows just outside a
// warp's strip from the neighbouring warps through shared memory, one named
// barrier per level for the group (edge buffers alternate between levels, so
// one barrier suffices).  In the link contraction a thread fetches the eight
// quantities of its right neighbour (a+1) once and forms both the right link
// of its own site and the up-left link of that neighbour, whose up-left site
// (a, b+1) is the thread's own.  Link sums of the CTA's 4 vectors meet in a
// shared-memory accumulator; after one barrier per slice the CTA adds them to
// the FP64 force with one atomic per (site, link).
#include "ephmc_internal.cuh"

namespace ephmc {

namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kR = 2;         // vectors per group: the .x and .y halves of every pair
constexpr int kH = 4;         // rows per warp
constexpr int kG = 2;         // groups per CTA
constexpr int kSlots = 9;     // edge rows exchanged at the widest level

using P = float2;

__device__ __forceinline__ P pfma(P a, P b, P c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ P pmul(P a, P b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ P padd(P a, P b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ P pdup(float c) { return make_float2(c, c); }
__device__ __forceinline__ P pshfl(P v, int src) {
    return make_float2(__shfl_sync(kFull, v.x, src), __shfl_sync(kFull, v.y, src));
}

// hopping coefficients of one site, the same value in both halves
struct HopP {
    P f0, f1, f2, f0l, f1d, f2dr;
};

// (H v)(a, b) = mu v + f0 v(a+1,b) + f0(a-1,b) v(a-1,b) + f1 v(a,b+1)
//             + f1(a,b-1) v(a,b-1) + f2 v(a-1,b+1) + f2(a+1,b-1) v(a+1,b-1)
__device__ __forceinline__ P stencil(const HopP &h, P mu, P v, P l, P r, P up, P down, P upleft, P downright) {
    const P s1 = pfma(h.f0, r, pmul(mu, v));
    const P s2 = pfma(h.f1, up, pmul(h.f0l, l));
    const P s3 = pfma(h.f2, upleft, pmul(h.f1d, down));
    return padd(padd(s1, s2), pfma(h.f2dr, downright, s3));
}

__device__ __forceinline__ void group_sync(int g, int nthreads) {
    asm volatile("bar.sync %0, %1;" ::"r"(1 + g), "r"(nthreads) : "memory");
}

// edge buffer of a group: [kSlots][nw][32] pairs
struct Edges {
    P *base;
    int nw, wg, lane;
    __device__ P *at(int slot, int warp) const { return base + (slot * nw + warp) * 32 + lane; }
    __device__ void put(int slot, P v) const { *at(slot, wg) = v; }
    __device__ P below(int slot) const { return *at(slot, (wg + nw - 1) % nw); }
    __device__ P above(int slot) const { return *at(slot, (wg + 1) % nw); }
};

// out = H in for the thread's rows, given the edge rows dn (row below the
// strip) and up (row above)
__device__ __forceinline__ void stencil_rows(const P (&in)[kH], P (&out)[kH], const HopP (&hp)[kH], P mu, P dn,
                                             P upx, int lm, int lp) {
    P L[kH], Rt[kH];
#pragma unroll
    for (int h = 0; h < kH; ++h) {
        L[h] = pshfl(in[h], lm);
        Rt[h] = pshfl(in[h], lp);
    }
    const P dnR = pshfl(dn, lp), upL = pshfl(upx, lm);
#pragma unroll
    for (int h = 0; h < kH; ++h) {
        const P up = (h + 1 < kH) ? in[h + 1] : upx;
        const P down = (h > 0) ? in[h - 1] : dn;
        const P ul = (h + 1 < kH) ? L[h + 1] : upL;
        const P dr = (h > 0) ? Rt[h - 1] : dnR;
        out[h] = stencil(hp[h], mu, in[h], L[h], Rt[h], up, down, ul, dr);
    }
}

// the quantities of one site entering the link contraction, with
// L1 = a0 q + b0 Hq and L3 = a1 f0q + b1 H f0q formed once per site
struct Site {
    P q, L1, f0q, L3, y, hy, f1y, hf1y;
};

__device__ __forceinline__ Site shfl_site(const Site &s, int src) {
    return Site{pshfl(s.q, src),  pshfl(s.L1, src), pshfl(s.f0q, src), pshfl(s.L3, src),
                pshfl(s.y, src),  pshfl(s.hy, src), pshfl(s.f1y, src), pshfl(s.hf1y, src)};
}

// link (i, n) entry of D + D^T:
//   d = L1_i f1y_n + L1_n f1y_i + b0 (q_i Hf1y_n + q_n Hf1y_i)
//     + L3_i y_n + L3_n y_i + b1 (f0q_i Hy_n + f0q_n Hy_i)
__device__ __forceinline__ P link_term(const Site &i, const Site &n, P aq0, P aq1) {
    const P d1 = pfma(i.L1, n.f1y, pmul(n.L1, i.f1y));
    const P e1 = pfma(aq0, pfma(i.q, n.hf1y, pmul(n.q, i.hf1y)), d1);
    const P d3 = pfma(i.L3, n.y, pmul(n.L3, i.y));
    const P e3 = pfma(aq1, pfma(i.f0q, n.hy, pmul(n.f0q, i.hy)), d3);
    return padd(e1, e3);
}

__device__ __forceinline__ double pick3(const double (&a)[3], int k) { return k == 0 ? a[0] : k == 1 ? a[1] : a[2]; }

// MODE 0: all slices from M^-1 (the range fields are not read); 1: one
// segment of a checkpointed sweep (AdjointRange t0, t1, q_top, y_in, y_out);
// 2: the segment grid (AdjointRange seg_*), one segment per blockIdx.y
template <int MODE>
__global__ void __launch_bounds__(512, 1) k_adjoint_strip(const double *__restrict__ x, Couplings cp,
                                                          const float *__restrict__ qstack,
                                                          const double *__restrict__ Minv, int L2, int nt,
                                                          double pref, double *__restrict__ force,
                                                          AdjointRange rg_in) {
    AdjointRange rg = rg_in;
    if (MODE == 0) rg = AdjointRange{0, nt, nullptr, nullptr, nullptr, true};
    extern __shared__ float sm[];
    const int V = 32 * L2, nw = L2 / kH;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int g = warp / nw, wg = warp - g * nw;
    const int b0 = kH * wg;
    const int lm = (lane + 31) & 31, lp = (lane + 1) & 31;
    const size_t edge_pairs = (size_t)kSlots * nw * 32;
    float *acc = sm;  // [2][V][3] link sums, by slice parity
    P *edges = reinterpret_cast<P *>(sm + 6 * V);
    Edges eb[2];
#pragma unroll
    for (int k = 0; k < 2; ++k) eb[k] = Edges{edges + (2 * g + k) * edge_pairs, nw, wg, lane};
    const P mu = pdup((float)cp.mu);
    const P al0 = pdup((float)cp.a_lin[0]), aq0 = pdup((float)cp.a_quad[0]);
    const P al1 = pdup((float)cp.a_lin[1]), aq1 = pdup((float)cp.a_quad[1]);
    const size_t VV = (size_t)V * V;
    // V = 32 L2 is a multiple of the 4 vectors of a CTA: every vector is live
    const int cv0 = (blockIdx.x * kG + g) * kR, cv1 = cv0 + 1;
    // the segment of the grid (MODE 2): slices [t0, t1), identity q at t1 - 1
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

    // y(t0): rows cv0, cv1 of M^-1 (columns of the inverse's array), the rows
    // a previous segment left in rg.y_in, or the segment's FP64 start rows
    const float *y_in = static_cast<const float *>(rg.y_in);
    P y[kH];
#pragma unroll
    for (int h = 0; h < kH; ++h) {
        const int i = (b0 + h) * 32 + lane;
        if (MODE == 2)
            y[h] = make_float2((float)rg.y_start[(size_t)cv0 * V + i], (float)rg.y_start[(size_t)cv1 * V + i]);
        else
            y[h] = y_in ? make_float2(y_in[(size_t)cv0 * V + i], y_in[(size_t)cv1 * V + i])
                        : make_float2((float)Minv[(size_t)i * V + cv0], (float)Minv[(size_t)i * V + cv1]);
    }
    for (int e = threadIdx.x; e < 6 * V; e += blockDim.x) acc[e] = 0.f;
    __syncthreads();

    for (int t = rg.t0; t < rg.t1; ++t) {
        float *acc_t = acc + (t & 1) * 3 * V;
        const double *xs = x + (size_t)t * 3 * V;
        // FP32 hopping coefficients of the thread's sites
        HopP hp[kH];
        {
            const int bd = (b0 + L2 - 1) % L2;
            float f1p = (float)fma(-cp.kappa[1], xs[3 * (bd * 32 + lane) + 1], cp.t[1]);
            float f2p = (float)fma(-cp.kappa[2], xs[3 * (bd * 32 + lane) + 2], cp.t[2]);
#pragma unroll
            for (int h = 0; h < kH; ++h) {
                const int i = (b0 + h) * 32 + lane;
                const float f0 = (float)fma(-cp.kappa[0], xs[3 * i + 0], cp.t[0]);
                const float f1 = (float)fma(-cp.kappa[1], xs[3 * i + 1], cp.t[1]);
                const float f2 = (float)fma(-cp.kappa[2], xs[3 * i + 2], cp.t[2]);
                hp[h].f0 = pdup(f0);
                hp[h].f1 = pdup(f1);
                hp[h].f2 = pdup(f2);
                hp[h].f0l = pdup(__shfl_sync(kFull, f0, lm));
                hp[h].f1d = pdup(f1p);
                hp[h].f2dr = pdup(__shfl_sync(kFull, f2p, lp));
                f1p = f1;
                f2p = f2;
            }
        }
        // q(t): the stack entry t - t0, the segment's FP64 checkpoint (its last
        // slice, checkpointed evaluation), or e_c (slice nt-1; the top slice of
        // a segment of the grid)
        P q[kH];
        {
            const bool top = rg.q_top != nullptr && t == rg.t1 - 1;
            const float *qs = qstack + (size_t)(t - rg.t0) * VV;
#pragma unroll
            for (int h = 0; h < kH; ++h) {
                const int i = (b0 + h) * 32 + lane;
                q[h] = (t == q_id_slice) ? make_float2(i == cv0 ? 1.f : 0.f, i == cv1 ? 1.f : 0.f)
                       : top ? make_float2((float)rg.q_top[(size_t)cv0 * V + i], (float)rg.q_top[(size_t)cv1 * V + i])
                             : make_float2(__ldg(qs + (size_t)cv0 * V + i), __ldg(qs + (size_t)cv1 * V + i));
            }
        }
        P hq[kH], hy[kH], f0q[kH], f1y[kH], hf0q[kH], hf1y[kH];
        // level A: hq = H q, hy = H y
        {
            const Edges &E = eb[0];
            E.put(0, q[0]);
            E.put(1, q[kH - 1]);
            E.put(2, y[0]);
            E.put(3, y[kH - 1]);
            group_sync(g, 32 * nw);
            stencil_rows(q, hq, hp, mu, E.below(1), E.above(0), lm, lp);
            stencil_rows(y, hy, hp, mu, E.below(3), E.above(2), lm, lp);
        }
        // level B: f0q, f1y
        {
            const Edges &E = eb[1];
            E.put(0, hq[0]);
            E.put(1, hq[kH - 1]);
            E.put(2, hy[0]);
            E.put(3, hy[kH - 1]);
            group_sync(g, 32 * nw);
            P z[kH];
            stencil_rows(hq, z, hp, mu, E.below(1), E.above(0), lm, lp);
#pragma unroll
            for (int h = 0; h < kH; ++h) f0q[h] = padd(q[h], pfma(al0, hq[h], pmul(aq0, z[h])));
            stencil_rows(hy, z, hp, mu, E.below(3), E.above(2), lm, lp);
#pragma unroll
            for (int h = 0; h < kH; ++h) f1y[h] = padd(y[h], pfma(al1, hy[h], pmul(aq1, z[h])));
        }
        // level C: hf0q = H f0q, hf1y = H f1y
        {
            const Edges &E = eb[0];
            E.put(0, f0q[0]);
            E.put(1, f0q[kH - 1]);
            E.put(2, f1y[0]);
            E.put(3, f1y[kH - 1]);
            group_sync(g, 32 * nw);
            stencil_rows(f0q, hf0q, hp, mu, E.below(1), E.above(0), lm, lp);
            stencil_rows(f1y, hf1y, hp, mu, E.below(3), E.above(2), lm, lp);
        }
        // level D: next y, then the link contraction; edges: hf1y top/bottom
        // and the bottom rows of the eight link quantities (the up
        // neighbours of the strip's top row)
        {
            const Edges &E = eb[1];
            Site s[kH + 1];
#pragma unroll
            for (int h = 0; h < kH; ++h)
                s[h] = Site{q[h], pfma(al0, q[h], pmul(aq0, hq[h])), f0q[h], pfma(al1, f0q[h], pmul(aq1, hf0q[h])),
                            y[h], hy[h],                              f1y[h], hf1y[h]};
            E.put(0, hf1y[0]);
            E.put(1, hf1y[kH - 1]);
            E.put(2, s[0].q);
            E.put(3, s[0].L1);
            E.put(4, s[0].f0q);
            E.put(5, s[0].L3);
            E.put(6, s[0].y);
            E.put(7, s[0].hy);
            E.put(8, s[0].f1y);
            group_sync(g, 32 * nw);
            s[kH] = Site{E.above(2), E.above(3), E.above(4), E.above(5),
                         E.above(6), E.above(7), E.above(8), E.above(0)};
#pragma unroll
            for (int h = 0; h < kH; ++h) {
                const int i = (b0 + h) * 32 + lane;
                const Site r = shfl_site(s[h], lp);
                const P right = link_term(s[h], r, aq0, aq1);        // site (a, b), link 0
                const P up = link_term(s[h], s[h + 1], aq0, aq1);    // site (a, b), link 1
                const P upleft = link_term(r, s[h + 1], aq0, aq1);   // site (a+1, b), link 2
                atomicAdd(acc_t + 3 * i + 0, right.x + right.y);
                atomicAdd(acc_t + 3 * i + 1, up.x + up.y);
                atomicAdd(acc_t + 3 * ((b0 + h) * 32 + lp) + 2, upleft.x + upleft.y);
            }
            {
                P z[kH];
                stencil_rows(hf1y, z, hp, mu, E.below(1), E.above(0), lm, lp);
#pragma unroll
                for (int h = 0; h < kH; ++h) y[h] = padd(f1y[h], pfma(al0, hf1y[h], pmul(aq0, z[h])));
            }
        }
        // every group's sums of slice t are in acc_t: add them to the force and
        // clear the buffer, which slice t+2 reuses (after the next barrier)
        __syncthreads();
        for (int e = threadIdx.x; e < 3 * V; e += blockDim.x) {
            atomicAdd(force + (size_t)t * 3 * V + e, -pick3(cp.kappa, e % 3) * pref * (double)acc_t[e]);
            acc_t[e] = 0.f;
        }
    }
    if (MODE != 2 && rg.y_out != nullptr) {
        float *y_out = static_cast<float *>(rg.y_out);
#pragma unroll
        for (int h = 0; h < kH; ++h) {
            const int i = (b0 + h) * 32 + lane;
            y_out[(size_t)cv0 * V + i] = y[h].x;
            y_out[(size_t)cv1 * V + i] = y[h].y;
        }
    }
}

}  // namespace

bool adjoint_strip32_supported(const LatticeDev &lat) {
    return lat.l1 == 32 && lat.l2 >= kH && lat.l2 % kH == 0 && kG * (lat.l2 / kH) * 32 <= 512;
}

bool adjoint_strip_supported(const LatticeDev &lat) {
    return adjoint_strip32_supported(lat) || adjoint_tile_supported(lat);
}

int launch_adjoint_strip(const double *x, const Couplings &c, const LatticeDev &lat, const float *qstack,
                         const double *Minv, int nt, unsigned flavors, int single_particle, double logdet,
                         double *force, cudaStream_t st, const AdjointRange *range, int seg_count) {
    if (!adjoint_strip32_supported(lat))
        return launch_adjoint_tile(x, c, lat, qstack, Minv, nt, flavors, single_particle, logdet, force, st, range,
                                   seg_count);
    const int V = lat.V, L2 = lat.l2, nw = L2 / kH;
    const size_t smem = sizeof(float) * (6 * (size_t)V + 2 * (size_t)kG * kSlots * kR * nw * 32);
    if (smem > 227 * 1024) return EPHMC_ERR_UNSUPPORTED;
    double pref = (double)flavors;
    if (single_particle) pref *= exp(-logdet);
    AdjointRange rg{0, nt, nullptr, nullptr, nullptr, true};
    if (range) rg = *range;
    if (rg.zero_force) EPHMC_CUDA(cudaMemsetAsync(force, 0, sizeof(double) * (size_t)nt * V * 3, st));
    const int per_cta = kG * kR;
    const dim3 grid((V + per_cta - 1) / per_cta, rg.seg_C > 0 ? (unsigned)seg_count : 1u);
    void (*kern)(const double *, Couplings, const float *, const double *, int, int, double, double *,
                 AdjointRange) = rg.seg_C > 0 ? k_adjoint_strip<2> : range ? k_adjoint_strip<1> : k_adjoint_strip<0>;
    EPHMC_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    kern<<<grid, kG * nw * 32, smem, st>>>(x, c, qstack, Minv, L2, nt, pref, force, rg);
    ephmc::count_launch(1);
    EPHMC_CUDA(cudaGetLastError());
    return EPHMC_OK;
}

}  // namespace ephmc
