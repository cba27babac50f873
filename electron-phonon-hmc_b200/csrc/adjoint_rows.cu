// Adjoint sweep 2 in FP32 for lattices with L1 = 32: one warp per vector, the
// lattice row (a = 0..31) across the lanes, rows b = 0..L2-1 streamed through
// a register pipeline.
//
// Same quantities as k_adjoint (adjoint.cu), i.e. the force of
// simulation/organic_hmc.c:86-134 through the adjoint of the slice chain, with
// the vectors of one slice computed in a different order:
//   level 0  q(b), y(b)                         (stack / carried y, row b = tau)
//   level 1  hq = H q, hy = H y                 (row tau-1)
//   level 2  f0q = q + a0 hq + b0 H hq,  f1y = y + a1 hy + b1 H hy   (tau-2)
//   level 3  hf0q = H f0q, hf1y = H f1y         (tau-3)
//   level 4  yn = f1y + a0 hf1y + b0 H hf1y and the link contraction (tau-4)
// A stencil at row b needs the row below, the row itself and the row above of
// its input; the row above was produced earlier in the same step and the two
// others in the previous two steps, so each level lags the one before by one
// row and keeps its last five rows in a register ring.  Neighbours along the
// row (a +- 1, periodic because L1 = 32 = warp size) come from warp shuffles,
// done once per row and array; the vertical and diagonal neighbours are ring
// entries.  The rows wrap around (periodic L2): the sweep of a slice runs
// steps tau = -4 .. L2+3, and only levels whose inputs are complete commit
// results (rows 0..L2-1 of level 4 at tau = 4 .. L2+3).
//
// The FP32 hopping tables of all slices are built first (k_hop_table); a warp
// reads its row of them, and of the stack, five steps ahead of use.  Per
// slice the link sums of the CTA's W vectors (W warps) meet in a
// shared-memory accumulator, and after one barrier the CTA adds them to the
// FP64 force with one atomic per (site, link).
#include "ephmc_internal.cuh"

#include <algorithm>

namespace ephmc {

namespace {

constexpr int kDepth = 5;  // ring depth = pipeline lag + 1
constexpr unsigned kFull = 0xffffffffu;

// a value with its left (a-1) and right (a+1) neighbours along the row
struct V3 {
    float v, l, r;
};

__device__ __forceinline__ V3 with_neighbours(float v) {
    const int lane = threadIdx.x & 31;
    V3 o;
    o.v = v;
    o.l = __shfl_sync(kFull, v, (lane + 31) & 31);
    o.r = __shfl_sync(kFull, v, (lane + 1) & 31);
    return o;
}

// hopping coefficients seen from site (a, b): own links 0, 1, 2, link 0 of the
// left site, link 1 of the site below, link 2 of the site below-right
struct Cf {
    float f0, f1, f2, f0l, f1d, f2dr;
};

// (H v)(a, b) = mu v + f0 v(a+1,b) + f0(a-1,b) v(a-1,b) + f1 v(a,b+1)
//             + f1(a,b-1) v(a,b-1) + f2 v(a-1,b+1) + f2(a+1,b-1) v(a+1,b-1),
// summed as a shallow tree (the mixed path's FP32 sweep has no reference order)
__device__ __forceinline__ float stencil(const Cf &c, float mu, const V3 &mid, const V3 &up, const V3 &down) {
    const float s1 = fmaf(c.f0, mid.r, mu * mid.v);
    const float s2 = fmaf(c.f1, up.v, c.f0l * mid.l);
    const float s3 = fmaf(c.f2, up.l, c.f1d * down.v);
    return (s1 + s2) + fmaf(c.f2dr, down.r, s3);
}

// row rho (any rho >= -L2) folded into 0..L2-1
__device__ __forceinline__ int wrap_row(int rho, int L2) {
    while (rho < 0) rho += L2;
    while (rho >= L2) rho -= L2;
    return rho;
}

// q of virtual row rho: the stack entry, or e_c when qs is null
__device__ __forceinline__ float load_q(const float *qs, int c, int rho, int L2, int lane) {
    const int i = wrap_row(rho, L2) * 32 + lane;
    return qs ? __ldg(qs + i) : (i == c ? 1.f : 0.f);
}

struct F3 {
    float f0, f1, f2;
};
__device__ __forceinline__ F3 load_hop(const float *tab, int V, int rho, int L2, int lane) {
    const int i = wrap_row(rho, L2) * 32 + lane;
    return F3{__ldg(tab + i), __ldg(tab + V + i), __ldg(tab + 2 * V + i)};
}

// a[k] for a runtime k in 0..2 without indexing the parameter array (which
// would copy the kernel's parameter struct to local memory)
__device__ __forceinline__ double pick3(const double (&a)[3], int k) { return k == 0 ? a[0] : k == 1 ? a[1] : a[2]; }

// FP32 hopping tables of all slices: tab[t][k][i] = t_k - kappa_k x[t][i][k]
__global__ void k_hop_table(const double *__restrict__ x, Couplings cp, int V, int nt, float *__restrict__ tab) {
    const size_t n = (size_t)nt * 3 * V;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
        const size_t t = e / (3 * (size_t)V);
        const int r = (int)(e - t * 3 * V), k = r / V, i = r - k * V;
        tab[e] = (float)fma(-pick3(cp.kappa, k), x[(t * V + i) * 3 + k], pick3(cp.t, k));
    }
}

// the eight vectors of the contraction at one site
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

__global__ void __launch_bounds__(256, 1) k_adjoint_rows(const float *__restrict__ hop, Couplings cp,
                                                         const float *__restrict__ qstack,
                                                         const double *__restrict__ Minv, int L2, int nt,
                                                         double pref, double *__restrict__ force) {
    extern __shared__ float sm[];
    const int V = 32 * L2;
    const int W = (int)(blockDim.x >> 5);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    float *acc = sm;                            // [2][V][3] link sums of the CTA's vectors, by slice parity
    float *ybuf = sm + 6 * V + 2 * V * warp;    // [2][V] this warp's y, current and next
    const int c = blockIdx.x * W + warp;        // this warp's vector
    const bool live = c < V;
    const float mu = (float)cp.mu;
    const float al0 = (float)cp.a_lin[0], aq0 = (float)cp.a_quad[0];
    const float al1 = (float)cp.a_lin[1], aq1 = (float)cp.a_quad[1];
    const size_t VV = (size_t)V * V;

    // y(0): row c of M^-1 (column c of the inverse's array)
    if (live)
        for (int b = 0; b < L2; ++b) ybuf[b * 32 + lane] = (float)Minv[(size_t)(b * 32 + lane) * V + c];
    for (int e = threadIdx.x; e < 6 * V; e += blockDim.x) acc[e] = 0.f;
    __syncthreads();

    for (int t = 0; t < nt; ++t) {
        float *acc_t = acc + (t & 1) * 3 * V;
        if (live) {
            const float *yc = ybuf + (t & 1) * V;
            float *yn_out = ybuf + ((t & 1) ^ 1) * V;
            const float *tab = hop + (size_t)t * 3 * V;
            // q(nt-1) = e_c (qs null); the stack holds slices 0..nt-2
            const float *qs = (t == nt - 1) ? nullptr : qstack + (size_t)t * VV + (size_t)c * V;
            // the first steps read ring slots no row has reached yet; their
            // results are never committed, but the slots start defined
            V3 q[kDepth], y[kDepth], hq[kDepth], hy[kDepth], f0q[kDepth], f1y[kDepth], hf0q[kDepth], hf1y[kDepth];
            Cf cf[kDepth];
            // q and the own hoppings of row rho are loaded five steps before use
            float qpre[kDepth];
            F3 hpre[kDepth];
#pragma unroll
            for (int s = 0; s < kDepth; ++s) {
                q[s] = y[s] = hq[s] = hy[s] = f0q[s] = f1y[s] = hf0q[s] = hf1y[s] = V3{0.f, 0.f, 0.f};
                cf[s] = Cf{0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
                qpre[s] = load_q(qs, c, -4 + s, L2, lane);
                hpre[s] = load_hop(tab, V, -4 + s, L2, lane);
            }
            // steps tau = -4, -3, ...; every ring keeps row rho in slot (rho + 4) % 5,
            // so at step tau = base + u rows tau, tau-1, ..., tau-4 sit in s0..s4
            for (int base = -4; base < L2 + 4; base += kDepth) {
#pragma unroll
                for (int u = 0; u < kDepth; ++u) {
                    const int tau = base + u;
                    const int s0 = u, s1 = (u + 4) % kDepth, s2 = (u + 3) % kDepth, s3 = (u + 2) % kDepth,
                              s4 = (u + 1) % kDepth;
                    // coefficients and level 0 (q, y) of row tau
                    {
                        Cf &n = cf[s0];
                        n.f0 = hpre[s0].f0;
                        n.f1 = hpre[s0].f1;
                        n.f2 = hpre[s0].f2;
                        n.f0l = __shfl_sync(kFull, n.f0, (lane + 31) & 31);
                        n.f1d = cf[s1].f1;
                        n.f2dr = __shfl_sync(kFull, cf[s1].f2, (lane + 1) & 31);
                        q[s0] = with_neighbours(qpre[s0]);
                        y[s0] = with_neighbours(yc[wrap_row(tau, L2) * 32 + lane]);
                        qpre[s0] = load_q(qs, c, tau + kDepth, L2, lane);
                        hpre[s0] = load_hop(tab, V, tau + kDepth, L2, lane);
                    }
                    // level 1: row tau-1 (rows below / at / above: slots s2 / s1 / s0)
                    hq[s1] = with_neighbours(stencil(cf[s1], mu, q[s1], q[s0], q[s2]));
                    hy[s1] = with_neighbours(stencil(cf[s1], mu, y[s1], y[s0], y[s2]));
                    // level 2: row tau-2
                    {
                        const float zq = stencil(cf[s2], mu, hq[s2], hq[s1], hq[s3]);
                        const float zy = stencil(cf[s2], mu, hy[s2], hy[s1], hy[s3]);
                        f0q[s2] = with_neighbours(q[s2].v + fmaf(al0, hq[s2].v, aq0 * zq));
                        f1y[s2] = with_neighbours(y[s2].v + fmaf(al1, hy[s2].v, aq1 * zy));
                    }
                    // level 3: row tau-3
                    hf0q[s3] = with_neighbours(stencil(cf[s3], mu, f0q[s3], f0q[s2], f0q[s4]));
                    hf1y[s3] = with_neighbours(stencil(cf[s3], mu, f1y[s3], f1y[s2], f1y[s4]));
                    // level 4: row tau-4, committed for tau = 4 .. L2+3
                    if (tau >= 4 && tau < L2 + 4) {
                        const int i = (tau - 4) * 32 + lane;
                        // the row below (tau-5) is in s0 until level 3 reaches row tau
                        const float z = stencil(cf[s4], mu, hf1y[s4], hf1y[s3], hf1y[s0]);
                        yn_out[i] = f1y[s4].v + fmaf(al0, hf1y[s4].v, aq0 * z);
                        // link contraction at (a, b): neighbours right (a+1,b), up (a,b+1), up-left (a-1,b+1);
                        // row b+1 of a level is one step younger than row b
                        const Site8 si{q[s4].v, hq[s4].v, f0q[s4].v, hf0q[s4].v,
                                       y[s4].v, hy[s4].v, f1y[s4].v, hf1y[s4].v};
                        const Site8 right{q[s4].r, hq[s4].r, f0q[s4].r, hf0q[s4].r,
                                          y[s4].r, hy[s4].r, f1y[s4].r, hf1y[s4].r};
                        const Site8 up{q[s3].v, hq[s3].v, f0q[s3].v, hf0q[s3].v,
                                       y[s3].v, hy[s3].v, f1y[s3].v, hf1y[s3].v};
                        const Site8 upleft{q[s3].l, hq[s3].l, f0q[s3].l, hf0q[s3].l,
                                           y[s3].l, hy[s3].l, f1y[s3].l, hf1y[s3].l};
                        atomicAdd(acc_t + 3 * i + 0, link_term(si, right, al0, aq0, al1, aq1));
                        atomicAdd(acc_t + 3 * i + 1, link_term(si, up, al0, aq0, al1, aq1));
                        atomicAdd(acc_t + 3 * i + 2, link_term(si, upleft, al0, aq0, al1, aq1));
                    }
                }
            }
        }
        // every warp's sums of slice t are in acc_t: add them to the force and
        // clear the buffer, which slice t+2 reuses (after the next barrier)
        __syncthreads();
        for (int e = threadIdx.x; e < 3 * V; e += blockDim.x) {
            atomicAdd(force + (size_t)t * 3 * V + e, -pick3(cp.kappa, e % 3) * pref * (double)acc_t[e]);
            acc_t[e] = 0.f;
        }
    }
}

}  // namespace

bool adjoint_rows_supported(const LatticeDev &lat) { return lat.l1 == 32 && lat.l2 >= 2 && lat.l2 <= 64; }

size_t adjoint_rows_scratch_floats(int V, int nt) { return (size_t)nt * 3 * V; }

int launch_adjoint_rows(const double *x, const Couplings &c, const LatticeDev &lat, const float *qstack,
                        const double *Minv, int nt, unsigned flavors, int single_particle, double logdet,
                        double *force, float *scratch, cudaStream_t st) {
    if (!adjoint_rows_supported(lat) || !scratch) return EPHMC_ERR_UNSUPPORTED;
    const int V = lat.V, L2 = lat.l2;
    int dev = 0, sms = 0;
    EPHMC_CUDA(cudaGetDevice(&dev));
    EPHMC_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    // vectors (warps) per CTA: spread the V vectors over all SMs, at most 8
    int W = (V + sms - 1) / sms;
    if (W < 1) W = 1;
    if (W > 8) W = 8;
    const size_t smem = sizeof(float) * (6 * (size_t)V + 2 * (size_t)V * W);
    if (smem > 227 * 1024) return EPHMC_ERR_UNSUPPORTED;
    double pref = (double)flavors;
    if (single_particle) pref *= exp(-logdet);
    EPHMC_CUDA(cudaMemsetAsync(force, 0, sizeof(double) * (size_t)nt * V * 3, st));
    const size_t n = (size_t)nt * 3 * V;
    k_hop_table<<<(unsigned)std::min<size_t>((n + 255) / 256, 4 * (size_t)sms), 256, 0, st>>>(x, c, V, nt, scratch);
    ephmc::count_launch(1);
    EPHMC_CUDA(cudaFuncSetAttribute(k_adjoint_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_adjoint_rows<<<(V + W - 1) / W, 32 * W, smem, st>>>(scratch, c, qstack, Minv, L2, nt, pref, force);
    ephmc::count_launch(1);
    EPHMC_CUDA(cudaGetLastError());
    return EPHMC_OK;
}

}  // namespace ephmc
