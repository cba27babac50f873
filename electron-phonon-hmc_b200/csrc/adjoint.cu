// Adjoint (reverse-mode) fermion force, sweep 2.
//
// Same quantity as force() + construct_all_QM1P + refine_QM1P
// (simulation/organic_hmc.c:86-134, organic_dense_matrix.c:311-442), by a
// different association of the same products.  With
//   q_c(t) = Q_t e_c,  Q_t = B_{t+1}...B_{Nt-1}          (sweep 1, stored)
//   y_c(t) = P_t^T M^-T e_c,  P_t = B_0...B_{t-1},  y_c(t+1) = B_t y_c(t)
// the reference's G_t = Q_t M^-1 P_t is sum_c q_c(t) y_c(t)^T, and its refined
// matrix for B_t = f_1 f_0 is
//   D_t = sum_c (a0 q + b0 Hq)(f1 y)^T + b0 q (H f1 y)^T
//             + (a1 f0q + b1 H f0q) y^T + b1 (f0 q)(H y)^T,
// whose link entries D[i][n] + D[n][i] give p_dot[t,i,k] = -kappa_k flavors (...).
// Every vector needed (Hq, f0q, H f0q, Hy, f1y, H f1y) is a by-product of
// propagating q or y through one slice, so a slice costs 7 stencils and an
// O(V) link contraction per vector instead of the reference's
// (3 + log2 Nt) slice propagations of full matrices.
//
// One CTA owns R vectors c and walks t = 0..Nt-1, keeping all nine working
// vectors in shared memory; partial link sums of its R vectors are added to
// the force with one FP64 atomic per (t, site, link).
#include <algorithm>

#include "ephmc_internal.cuh"

namespace ephmc {

namespace {

template <typename Real>
__device__ __forceinline__ Real stencil_at(const Real *__restrict__ v, int j, const int (&src)[6],
                                           const Real (&f)[6], Real mu) {
    Real acc = mu * v[j];
#pragma unroll
    for (int e = 0; e < 6; ++e) acc = fma(f[e], v[src[e]], acc);
    return acc;
}

// MODE 0: all slices from M^-1 (the range fields are not read); 1: one
// segment of a checkpointed sweep (AdjointRange t0, t1, q_top, y_in, y_out);
// 2: the segment grid (AdjointRange seg_*), one segment per blockIdx.y
// WIDE: one CTA per SM of at most 320 threads for S = 8, so that eight
// sites keep their tables in 168 registers instead of spilling (the FP32
// force at 48x48, Nt = 128: 27.2 ms instead of 39.5), or of at most 640
// threads for S = 4: the FP32 sweep's four sites fit in 96 registers, and
// at 48x48 18 warps per SM instead of 9 hide more of the stencils' latency
// (force phase 38.5 -> 33.9 ms)
template <typename Real, typename QT, int S, int MODE, bool WIDE, bool PACK>
__global__ void __launch_bounds__(WIDE ? (S == 4 ? 640 : 320) : 512, 1) k_adjoint(const double *__restrict__ x, Couplings c, const int *__restrict__ ev_src,
                          const int *__restrict__ ev_fac, const int *__restrict__ nbr,
                          const QT *__restrict__ qstack, const double *__restrict__ Minv, int V, int nt,
                          int R, double pref_scale, double *__restrict__ force, AdjointRange rg_in) {
    AdjointRange rg = rg_in;
    if (MODE == 0) rg = AdjointRange{0, nt, nullptr, nullptr, nullptr, true};
    const float *__restrict__ lat_coef = rg_in.coef;  // packed sweep: [nt][6][V]
    // the segment of the grid (MODE 2): slices [t0, t1), identity q at t1 - 1
    int q_id_slice = nt - 1;
    if (MODE == 2) {
        const int j = rg.seg_j0 + (int)blockIdx.y;
        rg.t1 = nt - j * rg.seg_C;
        rg.t0 = max(0, rg.t1 - rg.seg_C);
        q_id_slice = rg.t1 - 1;
        qstack += rg.seg_regions ? (size_t)j * rg.seg_C * V * V : 0;
        rg.y_start += rg.seg_regions ? (size_t)j * V * V : 0;
        rg.q_top = nullptr;
        rg.y_out = nullptr;
        rg.y_in = nullptr;
    }
    extern __shared__ unsigned char smem_raw[];
    Real *base = reinterpret_cast<Real *>(smem_raw);
    const size_t RV = (size_t)R * V;
    Real *q = base, *hq = q + RV, *f0q = hq + RV, *hf0q = f0q + RV;
    Real *y = hf0q + RV, *hy = y + RV, *f1y = hy + RV, *hf1y = f1y + RV, *yn = hf1y + RV;
    Real *fac = yn + RV;  // [3V]

    const int T = blockDim.x, tid = threadIdx.x;
    const int c0 = blockIdx.x * R;
    const int nvec = min(R, V - c0);
    const size_t VV = (size_t)V * V;
    const Real mu = (Real)c.mu;
    const Real al0 = (Real)c.a_lin[0], aq0 = (Real)c.a_quad[0];
    const Real al1 = (Real)c.a_lin[1], aq1 = (Real)c.a_quad[1];

    // A site's three forward neighbours are, on most lattices, consecutive in
    // its event list (its own links sort as one block between the incoming
    // ones): nbr[k][j] = src[p + k] with p in 0..3.  PACK (the FP32 sweep on
    // a lattice where this holds for every site, LatticeDev::nb_in_events)
    // keeps two bits per site in pos instead of three registers per site (at
    // 48x48 it then spills nothing); the FP64 sweep, which spills more that
    // way, and the lattices where a self-link breaks the block keep nb.  On
    // lattices small enough for one site to appear twice, any p whose three
    // entries match gives the same neighbours.
    constexpr bool kPack = PACK;
    int src[S][6], nb[kPack ? 1 : S][3];
    unsigned pos = 0;
#pragma unroll
    for (int s = 0; s < S; ++s) {
        const int j = tid + s * T;
#pragma unroll
        for (int e = 0; e < 6; ++e) src[s][e] = (j < V) ? ev_src[e * V + j] : 0;
        const int n0 = (j < V) ? nbr[j] : 0, n1 = (j < V) ? nbr[V + j] : 0, n2 = (j < V) ? nbr[2 * V + j] : 0;
        if (kPack) {
            unsigned p = 3;
#pragma unroll
            for (int q = 2; q >= 0; --q)
                if (src[s][q] == n0 && src[s][q + 1] == n1 && src[s][q + 2] == n2) p = (unsigned)q;
            pos |= p << (2 * s);
        } else {
            nb[kPack ? 0 : s][0] = n0;
            nb[kPack ? 0 : s][1] = n1;
            nb[kPack ? 0 : s][2] = n2;
        }
    }

    // y(t0): row c of M^-1 (math) = column c of the inverse's array, the rows
    // a previous segment left in rg.y_in, or the segment's FP64 start rows
    if (MODE == 2) {
        const double *yi = rg.y_start + (size_t)c0 * V;
        for (int f = tid; f < nvec * V; f += T) y[f] = (Real)yi[f];
    } else if (rg.y_in != nullptr) {
        const Real *yi = static_cast<const Real *>(rg.y_in) + (size_t)c0 * V;
        for (int f = tid; f < nvec * V; f += T) y[f] = yi[f];
    } else {
        for (int f = tid; f < nvec * V; f += T) {
            const int r = f % nvec, j = f / nvec;
            y[(size_t)r * V + j] = (Real)Minv[(size_t)j * V + c0 + r];
        }
    }

    // The packed sweep does not use fac: with R <= 3 it holds the next slice's
    // q rows, copied from the stack (cp.async) while the slice is computed.
    Real *qn = fac;
    const bool qpre = kPack && R <= 3;
    const bool q16 = (reinterpret_cast<uintptr_t>(qstack) & 15) == 0 && (V & 3) == 0;
    auto prefetch_q = [&](int s, Real *dst) {
        if (s == q_id_slice || (rg.q_top != nullptr && s == rg.t1 - 1)) return;  // e_c or the checkpoint
        const QT *qs = qstack + (size_t)(s - rg.t0) * VV + (size_t)c0 * V;
        const int n = nvec * V;
        if (q16) {
            for (int f = 4 * tid; f < n; f += 4 * T)
                asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(
                                 (unsigned)__cvta_generic_to_shared(dst + f)),
                             "l"(qs + f)
                             : "memory");
        } else {
            for (int f = tid; f < n; f += T)
                asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"((unsigned)__cvta_generic_to_shared(dst + f)),
                             "l"(qs + f)
                             : "memory");
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
    };
    if (qpre && rg.t0 < rg.t1) prefetch_q(rg.t0, q);

    for (int t = rg.t0; t < rg.t1; ++t) {
        if (qpre) asm volatile("cp.async.wait_group 0;" ::: "memory");  // this thread's copies of q(t)
        __syncthreads();  // everyone's; every thread is past slice t - 1 (qn is free)
        if (qpre && t + 1 < rg.t1) prefetch_q(t + 1, qn);
        // the sites' stencil coefficients: the packed sweep loads them from the
        // slice's coefficient table (coalesced, before the barrier below); the
        // others form the slice's link coefficients in fac and gather them
        // through ev_fac after it
        Real fl[S][6];
        if (kPack) {
            const float *cf = lat_coef + (size_t)t * 6 * V;
#pragma unroll
            for (int s = 0; s < S; ++s) {
                const int j = tid + s * T;
#pragma unroll
                for (int e = 0; e < 6; ++e) fl[s][e] = (j < V) ? (Real)__ldg(cf + (size_t)e * V + j) : (Real)0;
            }
        } else {
            const double *xs = x + (size_t)t * 3 * V;
            for (int e = tid; e < 3 * V; e += T) {
                const int k = e % 3;
                fac[e] = (Real)fma(-c.kappa[k], xs[e], c.t[k]);
            }
        }
        if (t == q_id_slice) {
            for (int f = tid; f < nvec * V; f += T) {
                const int r = f / V, j = f % V;
                q[f] = (j == c0 + r) ? (Real)1 : (Real)0;
            }
        } else if (rg.q_top != nullptr && t == rg.t1 - 1) {
            // the segment's last q is its checkpoint, kept in FP64
            const double *qs = rg.q_top + (size_t)c0 * V;
            for (int f = tid; f < nvec * V; f += T) q[f] = (Real)(QT)qs[f];
        } else if (!qpre) {
            const QT *qs = qstack + (size_t)(t - rg.t0) * VV + (size_t)c0 * V;
            for (int f = tid; f < nvec * V; f += T) q[f] = (Real)qs[f];
        }
        __syncthreads();
        if (!kPack) {
#pragma unroll
            for (int s = 0; s < S; ++s) {
                const int j = tid + s * T;
#pragma unroll
                for (int e = 0; e < 6; ++e) fl[s][e] = (j < V) ? fac[ev_fac[e * V + j]] : (Real)0;
            }
        }
        // A: hq = H q, hy = H y
        for (int r = 0; r < nvec; ++r) {
#pragma unroll
            for (int s = 0; s < S; ++s) {
                const int j = tid + s * T;
                if (j < V) {
                    hq[r * V + j] = stencil_at(q + r * V, j, src[s], fl[s], mu);
                    hy[r * V + j] = stencil_at(y + r * V, j, src[s], fl[s], mu);
                }
            }
        }
        __syncthreads();
        // B: f0q = q + a0 hq + b0 H hq ; f1y = y + a1 hy + b1 H hy
        for (int r = 0; r < nvec; ++r) {
#pragma unroll
            for (int s = 0; s < S; ++s) {
                const int j = tid + s * T;
                if (j < V) {
                    const Real zq = stencil_at(hq + r * V, j, src[s], fl[s], mu);
                    f0q[r * V + j] = q[r * V + j] + fma(al0, hq[r * V + j], aq0 * zq);
                    const Real zy = stencil_at(hy + r * V, j, src[s], fl[s], mu);
                    f1y[r * V + j] = y[r * V + j] + fma(al1, hy[r * V + j], aq1 * zy);
                }
            }
        }
        __syncthreads();
        // C: hf0q = H f0q, hf1y = H f1y
        for (int r = 0; r < nvec; ++r) {
#pragma unroll
            for (int s = 0; s < S; ++s) {
                const int j = tid + s * T;
                if (j < V) {
                    hf0q[r * V + j] = stencil_at(f0q + r * V, j, src[s], fl[s], mu);
                    hf1y[r * V + j] = stencil_at(f1y + r * V, j, src[s], fl[s], mu);
                }
            }
        }
        __syncthreads();
        // D: yn = f0 f1 y ; contraction of the link entries
        Real acc[S][3];
#pragma unroll
        for (int s = 0; s < S; ++s)
#pragma unroll
            for (int k = 0; k < 3; ++k) acc[s][k] = (Real)0;
        for (int r = 0; r < nvec; ++r) {
            const Real *Q = q + r * V, *HQ = hq + r * V, *F0Q = f0q + r * V, *HF0Q = hf0q + r * V;
            const Real *Y = y + r * V, *HY = hy + r * V, *F1Y = f1y + r * V, *HF1Y = hf1y + r * V;
#pragma unroll
            for (int s = 0; s < S; ++s) {
                const int i = tid + s * T;
                if (i < V) {
                    const Real z = stencil_at(HF1Y, i, src[s], fl[s], mu);
                    yn[r * V + i] = F1Y[i] + fma(al0, HF1Y[i], aq0 * z);
                    const Real L1i = fma(al0, Q[i], aq0 * HQ[i]);
                    const Real L3i = fma(al1, F0Q[i], aq1 * HF0Q[i]);
#pragma unroll
                    for (int k = 0; k < 3; ++k) {
                        const unsigned p = (pos >> (2 * s)) & 3u;
                        const int n = !kPack  ? nb[kPack ? 0 : s][k]
                                      : p == 0 ? src[s][k]
                                      : p == 1 ? src[s][k + 1]
                                      : p == 2 ? src[s][k + 2]
                                               : src[s][k + 3];
                        const Real L1n = fma(al0, Q[n], aq0 * HQ[n]);
                        const Real L3n = fma(al1, F0Q[n], aq1 * HF0Q[n]);
                        Real d = L1i * F1Y[n];
                        d = fma(L1n, F1Y[i], d);
                        d = fma(aq0, fma(Q[i], HF1Y[n], Q[n] * HF1Y[i]), d);
                        d = fma(L3i, Y[n], d);
                        d = fma(L3n, Y[i], d);
                        d = fma(aq1, fma(F0Q[i], HY[n], F0Q[n] * HY[i]), d);
                        acc[s][k] += d;
                    }
                }
            }
        }
#pragma unroll
        for (int s = 0; s < S; ++s) {
            const int i = tid + s * T;
            if (i < V) {
#pragma unroll
                for (int k = 0; k < 3; ++k)
                    atomicAdd(force + ((size_t)t * V + i) * 3 + k, -c.kappa[k] * pref_scale * (double)acc[s][k]);
            }
        }
        __syncthreads();
        Real *tmp = y;
        y = yn;
        yn = tmp;
        if (qpre) {
            tmp = q;
            q = qn;
            qn = tmp;
        }
    }
    if (MODE != 2 && rg.y_out != nullptr) {
        Real *yo = static_cast<Real *>(rg.y_out) + (size_t)c0 * V;
        for (int f = tid; f < nvec * V; f += T) yo[f] = y[f];
    }
}

// The packed sweep's coefficient table for slices [t0, t1): coef[t][e][j] =
// (float)(t_k - kappa_k x[t][f]), f = ev_fac[e][j], k = f % 3 -- the value the
// unpacked sweep forms in fac[f] and gathers through ev_fac, bit for bit.
__global__ void __launch_bounds__(256) k_adjoint_coef(const double *__restrict__ x, Couplings c,
                                                      const int *__restrict__ ev_fac, int V, int t0, int t1,
                                                      float *__restrict__ coef) {
    const size_t n6 = 6 * (size_t)V, total = (size_t)(t1 - t0) * n6;
    for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < total;
         idx += (size_t)gridDim.x * blockDim.x) {
        const int t = t0 + (int)(idx / n6);
        const int r = (int)(idx % n6);  // e V + j
        const int f = ev_fac[r], k = f % 3;
        const double kap = k == 0 ? c.kappa[0] : k == 1 ? c.kappa[1] : c.kappa[2];
        const double tk = k == 0 ? c.t[0] : k == 1 ? c.t[1] : c.t[2];
        coef[(size_t)t * n6 + r] = (float)fma(-kap, x[(size_t)t * 3 * V + f], tk);
    }
}

template <typename Real, typename QT>
using AdjointKernel = void (*)(const double *, Couplings, const int *, const int *, const int *, const QT *,
                               const double *, int, int, int, double, double *, AdjointRange);

// the instance of a mode; packed neighbours only in the FP32 sweep, and no
// unpacked instance at 640 threads
template <typename Real, typename QT, int S, bool WIDE = false>
AdjointKernel<Real, QT> pick_adjoint(int mode, bool packed) {
    if constexpr (sizeof(Real) == 4) {
        if (packed)
            return mode == 2   ? k_adjoint<Real, QT, S, 2, WIDE, true>
                   : mode == 1 ? k_adjoint<Real, QT, S, 1, WIDE, true>
                               : k_adjoint<Real, QT, S, 0, WIDE, true>;
    }
    if constexpr (WIDE && S == 4)
        return pick_adjoint<Real, QT, S, false>(mode, false);
    else
        return mode == 2   ? k_adjoint<Real, QT, S, 2, WIDE, false>
               : mode == 1 ? k_adjoint<Real, QT, S, 1, WIDE, false>
                           : k_adjoint<Real, QT, S, 0, WIDE, false>;
}

}  // namespace

template <typename Real, typename QT>
int launch_adjoint_sweep(const double *x, const Couplings &c, const LatticeDev &lat, const QT *qstack,
                         const double *Minv, int nt, unsigned flavors, int single_particle, double logdet,
                         double *force, cudaStream_t st, const AdjointRange *range, int seg_count) {
    const int V = lat.V;
    const bool packed = sizeof(Real) == 4 && lat.nb_in_events && lat.coef != nullptr && lat.coef_nt >= nt;
    int S = 16;
    // the fewest sites per thread within the thread limit: 512, or 640 for
    // the packed FP32 sweep at four sites (the FP64 one spills there)
    for (int o : {1, 2, 4, 8, 16})
        if ((V + o - 1) / o <= adjoint_max_threads(o, packed)) { S = o; break; }
    int T = (((V + S - 1) / S) + 31) / 32 * 32;
    const size_t per_vec = 9 * (size_t)V * sizeof(Real);
    const size_t fac_b = 3 * (size_t)V * sizeof(Real);
    const size_t budget = 227 * 1024;  // the sm_100 per-block opt-in maximum
    int R = (int)((budget - fac_b) / per_vec);
    if (R < 1 || fac_b + per_vec > budget) {
        set_status(EPHMC_ERR_UNSUPPORTED, sizeof(Real) == 8
                                              ? "adjoint sweep: nine FP64 vectors of V sites exceed shared memory "
                                                "(V > 2421); use the mixed or the reference force"
                                              : "adjoint sweep: nine FP32 vectors of V sites exceed shared memory");
        return EPHMC_ERR_UNSUPPORTED;
    }
    if (R > 4) R = 4;
    // a tuned shape (ephmc_ctx_autotune) replaces the rule when it is valid
    {
        const int tS = lat.tune_adj_S, tR = lat.tune_adj_R;
        if ((tS == 1 || tS == 2 || tS == 4 || tS == 8 || tS == 16) &&
            (V + tS - 1) / tS <= adjoint_max_threads(tS, packed)) {
            S = tS;
            T = (((V + S - 1) / S) + 31) / 32 * 32;
        }
        if (tR >= 1 && tR <= 4 && fac_b + per_vec * tR <= budget) R = tR;
    }
    const size_t smem = per_vec * R + fac_b;
    double pref = (double)flavors;
    if (single_particle) pref *= exp(-logdet);
    AdjointRange rg{0, nt, nullptr, nullptr, nullptr, true};
    if (range) rg = *range;
    if (rg.zero_force) EPHMC_CUDA(cudaMemsetAsync(force, 0, sizeof(double) * (size_t)nt * V * 3, st));
    const int mode = rg.seg_C > 0 ? 2 : range != nullptr ? 1 : 0;
    AdjointKernel<Real, QT> kern = nullptr;
    switch (S) {
        case 1: kern = pick_adjoint<Real, QT, 1>(mode, packed); break;
        case 2: kern = pick_adjoint<Real, QT, 2>(mode, packed); break;
        case 4:
            kern = T > 512 ? pick_adjoint<Real, QT, 4, true>(mode, packed) : pick_adjoint<Real, QT, 4>(mode, packed);
            break;
        case 8:
            kern = T <= 320 ? pick_adjoint<Real, QT, 8, true>(mode, packed) : pick_adjoint<Real, QT, 8>(mode, packed);
            break;
        default: kern = pick_adjoint<Real, QT, 16>(mode, packed); break;
    }
    EPHMC_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const dim3 grid((V + R - 1) / R, mode == 2 ? (unsigned)seg_count : 1u);
    if (packed) {  // the coefficient table of the slices this launch covers
        int ta = 0, tb = nt;
        if (mode == 1) {
            ta = rg.t0;
            tb = rg.t1;
        } else if (mode == 2) {
            tb = nt - rg.seg_j0 * rg.seg_C;
            ta = nt - (rg.seg_j0 + seg_count) * rg.seg_C > 0 ? nt - (rg.seg_j0 + seg_count) * rg.seg_C : 0;
        }
        if (tb > ta) {
            const size_t total = (size_t)(tb - ta) * 6 * V;
            const unsigned blocks = (unsigned)std::min<size_t>((total + 255) / 256, 148 * 16);
            k_adjoint_coef<<<blocks, 256, 0, st>>>(x, c, lat.ev_fac, V, ta, tb, lat.coef);
            ephmc::count_launch(1);
            EPHMC_CUDA(cudaGetLastError());
        }
        rg.coef = lat.coef;
    }
    kern<<<grid, T, smem, st>>>(x, c, lat.ev_src, lat.ev_fac, lat.nbr, qstack, Minv, V, nt, R, pref, force, rg);
    ephmc::count_launch(1);
    EPHMC_CUDA(cudaGetLastError());
    return EPHMC_OK;
}

template int launch_adjoint_sweep<double, double>(const double *, const Couplings &, const LatticeDev &,
                                                  const double *, const double *, int, unsigned, int, double,
                                                  double *, cudaStream_t, const AdjointRange *, int);
template int launch_adjoint_sweep<float, float>(const double *, const Couplings &, const LatticeDev &,
                                                const float *, const double *, int, unsigned, int, double,
                                                double *, cudaStream_t, const AdjointRange *, int);

}  // namespace ephmc
