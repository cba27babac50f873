// Adjoint sweep 2 in FP32 for lattices with L1 = 32, with the lattice held
// in registers (the layout of slices_strip.cu).
//
// Same quantities as k_adjoint (adjoint.cu) -- the force of
// simulation/organic_hmc.c:86-134 through the adjoint of the slice chain --
// with the same formulas, summed in a different order.
//
// A CTA has G = 2 independent groups of nw = L2/4 warps; each group carries
// R = 2 vectors through all slices.  Warp w of a group owns rows 4w .. 4w+3,
// lane a the column a; a thread keeps its 4 sites of its group's vectors in
// registers.  Per slice and group:
//   level A  hq = H q, hy = H y
//   level B  f0q = q + a0 hq + b0 H hq,  f1y = y + a1 hy + b1 H hy
//   level C  hf0q = H f0q, hf1y = H f1y
//   level D  y <- f1y + a0 hf1y + b0 H hf1y, and the link contraction
// Row neighbours (a +- 1) come from warp shuffles; the rows just outside a
// warp's strip from the neighbouring warps through shared memory, one named
// barrier per level for the group (edge buffers alternate between levels, so
// one barrier suffices).  Link sums of the CTA's 4 vectors meet in a
// shared-memory accumulator; after one barrier per slice the CTA adds them to
// the FP64 force with one atomic per (site, link).
#include "ephmc_internal.cuh"

namespace ephmc {

namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kR = 2;         // vectors per group
constexpr int kH = 4;         // rows per warp
constexpr int kG = 2;         // groups per CTA
constexpr int kSlots = 9;     // edge rows exchanged at the widest level

struct HopF {
    float f0, f1, f2, f0l, f1d, f2dr;
};

__device__ __forceinline__ float shfl_from(float v, int src) { return __shfl_sync(kFull, v, src); }

// (H v)(a, b) = mu v + f0 v(a+1,b) + f0(a-1,b) v(a-1,b) + f1 v(a,b+1)
//             + f1(a,b-1) v(a,b-1) + f2 v(a-1,b+1) + f2(a+1,b-1) v(a+1,b-1)
__device__ __forceinline__ float stencil(const HopF &h, float mu, float v, float l, float r, float up, float down,
                                         float upleft, float downright) {
    const float s1 = fmaf(h.f0, r, mu * v);
    const float s2 = fmaf(h.f1, up, h.f0l * l);
    const float s3 = fmaf(h.f2, upleft, h.f1d * down);
    return (s1 + s2) + fmaf(h.f2dr, downright, s3);
}

__device__ __forceinline__ void group_sync(int g, int nthreads) {
    asm volatile("bar.sync %0, %1;" ::"r"(1 + g), "r"(nthreads) : "memory");
}

// edge buffer of a group: [kSlots][kR][nw][32] floats
struct Edges {
    float *base;
    int nw, wg, lane;
    __device__ float *at(int slot, int r, int warp) const { return base + ((slot * kR + r) * nw + warp) * 32 + lane; }
    __device__ void put(int slot, int r, float v) const { *at(slot, r, wg) = v; }
    __device__ float below(int slot, int r) const { return *at(slot, r, (wg + nw - 1) % nw); }
    __device__ float above(int slot, int r) const { return *at(slot, r, (wg + 1) % nw); }
};

// out = H in for the thread's rows, given the edge rows dn (row below the
// strip) and up (row above)
__device__ __forceinline__ void stencil_rows(const float (&in)[kH], float (&out)[kH], const HopF (&hp)[kH], float mu,
                                             float dn, float upx, int lm, int lp) {
    float L[kH], Rt[kH];
#pragma unroll
    for (int h = 0; h < kH; ++h) {
        L[h] = shfl_from(in[h], lm);
        Rt[h] = shfl_from(in[h], lp);
    }
    const float dnR = shfl_from(dn, lp), upL = shfl_from(upx, lm);
#pragma unroll
    for (int h = 0; h < kH; ++h) {
        const float up = (h + 1 < kH) ? in[h + 1] : upx;
        const float down = (h > 0) ? in[h - 1] : dn;
        const float ul = (h + 1 < kH) ? L[h + 1] : upL;
        const float dr = (h > 0) ? Rt[h - 1] : dnR;
        out[h] = stencil(hp[h], mu, in[h], L[h], Rt[h], up, down, ul, dr);
    }
}

struct Site8 {
    float q, hq, f0q, hf0q, y, hy, f1y, hf1y;
};

// link (i, n) entry of D + D^T for one vector:
//   L1 = a0 q + b0 Hq,  L3 = a1 f0q + b1 H f0q,
//   d = L1_i f1y_n + L1_n f1y_i + b0 (q_i Hf1y_n + q_n Hf1y_i)
//     + L3_i y_n + L3_n y_i + b1 (f0q_i Hy_n + f0q_n Hy_i)
__device__ __forceinline__ float link_term(const Site8 &i, const Site8 &n, float al0, float aq0, float al1,
                                           float aq1) {
    const float L1i = fmaf(al0, i.q, aq0 * i.hq), L3i = fmaf(al1, i.f0q, aq1 * i.hf0q);
    const float L1n = fmaf(al0, n.q, aq0 * n.hq), L3n = fmaf(al1, n.f0q, aq1 * n.hf0q);
    const float d1 = fmaf(L1i, n.f1y, L1n * i.f1y);
    const float d2 = aq0 * fmaf(i.q, n.hf1y, n.q * i.hf1y);
    const float d3 = fmaf(L3i, n.y, L3n * i.y);
    const float d4 = aq1 * fmaf(i.f0q, n.hy, n.f0q * i.hy);
    return (d1 + d2) + (d3 + d4);
}

__device__ __forceinline__ double pick3(const double (&a)[3], int k) { return k == 0 ? a[0] : k == 1 ? a[1] : a[2]; }

// SEG: a segment of a checkpointed sweep (AdjointRange); without it the
// kernel walks all slices from M^-1 and the range fields are not read
template <bool SEG>
__global__ void __launch_bounds__(512, 1) k_adjoint_strip(const double *__restrict__ x, Couplings cp,
                                                          const float *__restrict__ qstack,
                                                          const double *__restrict__ Minv, int L2, int nt,
                                                          double pref, double *__restrict__ force,
                                                          AdjointRange rg_in) {
    AdjointRange rg = rg_in;
    if (!SEG) rg = AdjointRange{0, nt, nullptr, nullptr, nullptr, true};
    extern __shared__ float sm[];
    const int V = 32 * L2, nw = L2 / kH;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int g = warp / nw, wg = warp - g * nw;
    const int b0 = kH * wg;
    const int lm = (lane + 31) & 31, lp = (lane + 1) & 31;
    const size_t edge_floats = (size_t)kSlots * kR * nw * 32;
    float *acc = sm;  // [2][V][3] link sums, by slice parity
    Edges eb[2];
#pragma unroll
    for (int k = 0; k < 2; ++k) eb[k] = Edges{sm + 6 * V + (2 * g + k) * edge_floats, nw, wg, lane};
    const float mu = (float)cp.mu;
    const float al0 = (float)cp.a_lin[0], aq0 = (float)cp.a_quad[0];
    const float al1 = (float)cp.a_lin[1], aq1 = (float)cp.a_quad[1];
    const size_t VV = (size_t)V * V;
    int cvec[kR];
    bool live[kR];
#pragma unroll
    for (int r = 0; r < kR; ++r) {
        cvec[r] = (blockIdx.x * kG + g) * kR + r;
        live[r] = cvec[r] < V;
    }

    // y(t0): row c of M^-1 (column c of the inverse's array), or the rows a
    // previous segment left in rg.y_in
    const float *y_in = static_cast<const float *>(rg.y_in);
    float y[kR][kH];
#pragma unroll
    for (int r = 0; r < kR; ++r)
#pragma unroll
        for (int h = 0; h < kH; ++h) {
            const int i = (b0 + h) * 32 + lane;
            y[r][h] = !live[r] ? 0.f
                      : y_in  ? y_in[(size_t)cvec[r] * V + i]
                              : (float)Minv[(size_t)i * V + cvec[r]];
        }
    for (int e = threadIdx.x; e < 6 * V; e += blockDim.x) acc[e] = 0.f;
    __syncthreads();

    for (int t = rg.t0; t < rg.t1; ++t) {
        float *acc_t = acc + (t & 1) * 3 * V;
        const double *xs = x + (size_t)t * 3 * V;
        // FP32 hopping coefficients of the thread's sites
        HopF hp[kH];
        {
            const int bd = (b0 + L2 - 1) % L2;
            float f1p = (float)fma(-cp.kappa[1], xs[3 * (bd * 32 + lane) + 1], cp.t[1]);
            float f2p = (float)fma(-cp.kappa[2], xs[3 * (bd * 32 + lane) + 2], cp.t[2]);
#pragma unroll
            for (int h = 0; h < kH; ++h) {
                const int i = (b0 + h) * 32 + lane;
                hp[h].f0 = (float)fma(-cp.kappa[0], xs[3 * i + 0], cp.t[0]);
                hp[h].f1 = (float)fma(-cp.kappa[1], xs[3 * i + 1], cp.t[1]);
                hp[h].f2 = (float)fma(-cp.kappa[2], xs[3 * i + 2], cp.t[2]);
                hp[h].f0l = shfl_from(hp[h].f0, lm);
                hp[h].f1d = f1p;
                hp[h].f2dr = shfl_from(f2p, lp);
                f1p = hp[h].f1;
                f2p = hp[h].f2;
            }
        }
        // q(t): the stack entry t - t0, the segment's FP64 checkpoint (its last
        // slice, checkpointed evaluation), or e_c (slice nt-1)
        float q[kR][kH];
        const bool top = rg.q_top != nullptr && t == rg.t1 - 1;
#pragma unroll
        for (int r = 0; r < kR; ++r) {
            const float *qs = qstack + (size_t)(t - rg.t0) * VV + (size_t)cvec[r] * V;
            const double *qt = top ? rg.q_top + (size_t)cvec[r] * V : nullptr;
#pragma unroll
            for (int h = 0; h < kH; ++h) {
                const int i = (b0 + h) * 32 + lane;
                q[r][h] = !live[r]        ? 0.f
                          : (t == nt - 1) ? (i == cvec[r] ? 1.f : 0.f)
                          : top           ? (float)qt[i]
                                          : __ldg(qs + i);
            }
        }
        float hq[kR][kH], hy[kR][kH], f0q[kR][kH], f1y[kR][kH], hf0q[kR][kH], hf1y[kR][kH];
        // level A: hq = H q, hy = H y
        {
            const Edges &E = eb[0];
#pragma unroll
            for (int r = 0; r < kR; ++r) {
                E.put(0, r, q[r][0]);
                E.put(1, r, q[r][kH - 1]);
                E.put(2, r, y[r][0]);
                E.put(3, r, y[r][kH - 1]);
            }
            group_sync(g, 32 * nw);
#pragma unroll
            for (int r = 0; r < kR; ++r) {
                stencil_rows(q[r], hq[r], hp, mu, E.below(1, r), E.above(0, r), lm, lp);
                stencil_rows(y[r], hy[r], hp, mu, E.below(3, r), E.above(2, r), lm, lp);
            }
        }
        // level B: f0q, f1y
        {
            const Edges &E = eb[1];
#pragma unroll
            for (int r = 0; r < kR; ++r) {
                E.put(0, r, hq[r][0]);
                E.put(1, r, hq[r][kH - 1]);
                E.put(2, r, hy[r][0]);
                E.put(3, r, hy[r][kH - 1]);
            }
            group_sync(g, 32 * nw);
#pragma unroll
            for (int r = 0; r < kR; ++r) {
                float z[kH];
                stencil_rows(hq[r], z, hp, mu, E.below(1, r), E.above(0, r), lm, lp);
#pragma unroll
                for (int h = 0; h < kH; ++h) f0q[r][h] = q[r][h] + fmaf(al0, hq[r][h], aq0 * z[h]);
                stencil_rows(hy[r], z, hp, mu, E.below(3, r), E.above(2, r), lm, lp);
#pragma unroll
                for (int h = 0; h < kH; ++h) f1y[r][h] = y[r][h] + fmaf(al1, hy[r][h], aq1 * z[h]);
            }
        }
        // level C: hf0q = H f0q, hf1y = H f1y
        {
            const Edges &E = eb[0];
#pragma unroll
            for (int r = 0; r < kR; ++r) {
                E.put(0, r, f0q[r][0]);
                E.put(1, r, f0q[r][kH - 1]);
                E.put(2, r, f1y[r][0]);
                E.put(3, r, f1y[r][kH - 1]);
            }
            group_sync(g, 32 * nw);
#pragma unroll
            for (int r = 0; r < kR; ++r) {
                stencil_rows(f0q[r], hf0q[r], hp, mu, E.below(1, r), E.above(0, r), lm, lp);
                stencil_rows(f1y[r], hf1y[r], hp, mu, E.below(3, r), E.above(2, r), lm, lp);
            }
        }
        // level D: next y and the link contraction; edges: hf1y top/bottom and
        // the bottom rows of the other seven vectors (the up neighbours of the
        // strip's top row)
        {
            const Edges &E = eb[1];
#pragma unroll
            for (int r = 0; r < kR; ++r) {
                E.put(0, r, hf1y[r][0]);
                E.put(1, r, hf1y[r][kH - 1]);
                E.put(2, r, q[r][0]);
                E.put(3, r, hq[r][0]);
                E.put(4, r, f0q[r][0]);
                E.put(5, r, hf0q[r][0]);
                E.put(6, r, y[r][0]);
                E.put(7, r, hy[r][0]);
                E.put(8, r, f1y[r][0]);
            }
            group_sync(g, 32 * nw);
            float dsum[kH][3];
#pragma unroll
            for (int h = 0; h < kH; ++h) dsum[h][0] = dsum[h][1] = dsum[h][2] = 0.f;
#pragma unroll
            for (int r = 0; r < kR; ++r) {
                // the eight vectors at the thread's rows and at the row above the strip
                Site8 s[kH + 1];
#pragma unroll
                for (int h = 0; h < kH; ++h)
                    s[h] = Site8{q[r][h], hq[r][h], f0q[r][h], hf0q[r][h], y[r][h], hy[r][h], f1y[r][h], hf1y[r][h]};
                s[kH] = Site8{E.above(2, r), E.above(3, r), E.above(4, r), E.above(5, r),
                              E.above(6, r), E.above(7, r), E.above(8, r), E.above(0, r)};
#pragma unroll
                for (int h = 0; h < kH; ++h) {
                    const Site8 &si = s[h], &su = s[h + 1];
                    const Site8 right{shfl_from(si.q, lp), shfl_from(si.hq, lp), shfl_from(si.f0q, lp),
                                      shfl_from(si.hf0q, lp), shfl_from(si.y, lp), shfl_from(si.hy, lp),
                                      shfl_from(si.f1y, lp), shfl_from(si.hf1y, lp)};
                    const Site8 upleft{shfl_from(su.q, lm), shfl_from(su.hq, lm), shfl_from(su.f0q, lm),
                                       shfl_from(su.hf0q, lm), shfl_from(su.y, lm), shfl_from(su.hy, lm),
                                       shfl_from(su.f1y, lm), shfl_from(su.hf1y, lm)};
                    if (live[r]) {
                        dsum[h][0] += link_term(si, right, al0, aq0, al1, aq1);
                        dsum[h][1] += link_term(si, su, al0, aq0, al1, aq1);
                        dsum[h][2] += link_term(si, upleft, al0, aq0, al1, aq1);
                    }
                }
                float z[kH];
                stencil_rows(hf1y[r], z, hp, mu, E.below(1, r), E.above(0, r), lm, lp);
#pragma unroll
                for (int h = 0; h < kH; ++h) y[r][h] = f1y[r][h] + fmaf(al0, hf1y[r][h], aq0 * z[h]);
            }
#pragma unroll
            for (int h = 0; h < kH; ++h) {
                const int i = (b0 + h) * 32 + lane;
#pragma unroll
                for (int k = 0; k < 3; ++k) atomicAdd(acc_t + 3 * i + k, dsum[h][k]);
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
    if (rg.y_out != nullptr) {
        float *y_out = static_cast<float *>(rg.y_out);
#pragma unroll
        for (int r = 0; r < kR; ++r)
            if (live[r])
#pragma unroll
                for (int h = 0; h < kH; ++h) y_out[(size_t)cvec[r] * V + (b0 + h) * 32 + lane] = y[r][h];
    }
}

}  // namespace

bool adjoint_strip_supported(const LatticeDev &lat) {
    return lat.l1 == 32 && lat.l2 >= kH && lat.l2 % kH == 0 && kG * (lat.l2 / kH) * 32 <= 512;
}

int launch_adjoint_strip(const double *x, const Couplings &c, const LatticeDev &lat, const float *qstack,
                         const double *Minv, int nt, unsigned flavors, int single_particle, double logdet,
                         double *force, cudaStream_t st, const AdjointRange *range) {
    if (!adjoint_strip_supported(lat)) return EPHMC_ERR_UNSUPPORTED;
    const int V = lat.V, L2 = lat.l2, nw = L2 / kH;
    const size_t smem = sizeof(float) * (6 * (size_t)V + 2 * (size_t)kG * kSlots * kR * nw * 32);
    if (smem > 227 * 1024) return EPHMC_ERR_UNSUPPORTED;
    double pref = (double)flavors;
    if (single_particle) pref *= exp(-logdet);
    AdjointRange rg{0, nt, nullptr, nullptr, nullptr, true};
    if (range) rg = *range;
    if (rg.zero_force) EPHMC_CUDA(cudaMemsetAsync(force, 0, sizeof(double) * (size_t)nt * V * 3, st));
    const int per_cta = kG * kR;
    if (range) {
        EPHMC_CUDA(cudaFuncSetAttribute(k_adjoint_strip<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        k_adjoint_strip<true><<<(V + per_cta - 1) / per_cta, kG * nw * 32, smem, st>>>(x, c, qstack, Minv, L2, nt,
                                                                                     pref, force, rg);
    } else {
        EPHMC_CUDA(cudaFuncSetAttribute(k_adjoint_strip<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        k_adjoint_strip<false><<<(V + per_cta - 1) / per_cta, kG * nw * 32, smem, st>>>(x, c, qstack, Minv, L2, nt,
                                                                                      pref, force, rg);
    }
    ephmc::count_launch(1);
    EPHMC_CUDA(cudaGetLastError());
    return EPHMC_OK;
}

}  // namespace ephmc
