// FP64 log|det| and in-place inverse of the fermion matrix by blocked
// Gauss-Jordan elimination with partial pivoting.
//
// Replaces LAPACKE_dgetrf + LAPACKE_dgetri in logDetM_and_inv_M_hat
// (simulation/organic_dense_matrix.c:580-595).  The matrix is seen
// column-major as LAPACK sees it: A(r,c) = M[c*V + r], so column c is the
// contiguous row c of the reference's array.  Pivot rows are chosen among the
// rows not yet used as pivots exactly as dgetrf chooses them (largest
// magnitude, first on ties), so the pivot sequence and U's diagonal are those
// of the LU factorisation: log|det| = sum log|U_ii|, the sign from the
// diagonal signs and the pivot parity (:582-589), pivots reported 1-based.
//
// Per panel of nb columns p (rows P = pivot rows, O = all others):
//   k_gj_panel   one CTA; every thread owns RPT rows of the panel in
//                registers (all V rows).  Each pivot step is a full
//                Gauss-Jordan sweep restricted to the panel columns, with one
//                barrier: every warp publishes its best candidate row (key and
//                values) in a double-buffered table, every warp reduces the
//                table itself, and rows are never moved (pivoted rows are only
//                marked; the LAPACK interchange sequence is rebuilt at the
//                end).  After nb sweeps the panel columns hold exactly the
//                block sweep: rows P = D^-1, rows O = -A(O,p) D^-1, written at
//                each row's logical position.
//   k_gj_update  every CTA owns CB other columns and a copy of the panel in
//                shared memory: applies the panel's interchanges, sets rows P
//                to D^-1 A(P, col) and updates the other rows
//                A(O, col) += (new panel columns) A(P, col).
// After the last panel the interchanges are undone as column permutations.
// 2V^3 flops in V/nb rank-nb updates over the full matrix, L2 resident at
// V = 1024, with no separate triangular-solve phase.
#include "ephmc_internal.cuh"

#include <atomic>

#include <algorithm>
#include <cmath>

namespace ephmc {

namespace {

// |a| as an ordered 64-bit key (non-negative doubles order like their bits)
__device__ __forceinline__ unsigned long long abs_key(double a) {
    return (unsigned long long)__double_as_longlong(fabs(a));
}

// argmax over the warp of (key, row): larger key wins, smaller row on ties;
// returns the lowest lane holding the winner
__device__ __forceinline__ int warp_argmax(unsigned long long &key, int &row) {
    const unsigned hi = (unsigned)(key >> 32), lo = (unsigned)key;
    const unsigned mhi = __reduce_max_sync(0xffffffffu, hi);
    const unsigned mlo = __reduce_max_sync(0xffffffffu, hi == mhi ? lo : 0u);
    const bool win = (hi == mhi) && (lo == mlo);
    const int r = (int)__reduce_min_sync(0xffffffffu, win ? (unsigned)row : 0x7fffffffu);
    const int lane = (int)__reduce_min_sync(0xffffffffu, (win && row == r) ? (threadIdx.x & 31) : 32u);
    key = ((unsigned long long)mhi << 32) | mlo;
    row = r;
    return lane;
}

template <int NB, int RPT, int T>
__global__ void __launch_bounds__(T, 1) k_gj_panel(double *__restrict__ M, int V, int j0, int nbc,
                                                  int *__restrict__ ipiv, double *__restrict__ diag,
                                                  int *__restrict__ info) {
    constexpr int NW = T / 32;
    __shared__ unsigned long long ck[2][NW];
    __shared__ int cr[2][NW];
    __shared__ double crow[2][NW][NB];
    __shared__ int chosen[NB];
    extern __shared__ int perm_s[];  // pos[V] | where[V]
    int *pos = perm_s, *where = perm_s + V;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    double a[RPT][NB];
    bool active[RPT];
#pragma unroll
    for (int i = 0; i < RPT; ++i) {
        const int r = tid + i * T;
        active[i] = (r >= j0 && r < V);
#pragma unroll
        for (int c = 0; c < NB; ++c) a[i][c] = (r < V && c < nbc) ? M[(size_t)(j0 + c) * V + r] : 0.0;
    }
    for (int r = tid; r < V; r += T) {
        pos[r] = r;
        where[r] = r;
    }
#pragma unroll
    for (int jj = 0; jj < NB; ++jj) {
        if (jj < nbc) {
            const int buf = jj & 1;
            unsigned long long bk = 0;
            int br = 0x7fffffff;
#pragma unroll
            for (int i = 0; i < RPT; ++i) {
                const int r = tid + i * T;
                if (active[i]) {
                    const unsigned long long k = abs_key(a[i][jj]);
                    if (k > bk || (k == bk && r < br)) {
                        bk = k;
                        br = r;
                    }
                }
            }
            warp_argmax(bk, br);
#pragma unroll
            for (int i = 0; i < RPT; ++i) {
                if (tid + i * T == br) {
#pragma unroll
                    for (int c = 0; c < NB; ++c) crow[buf][warp][c] = a[i][c];
                }
            }
            if (lane == 0) {
                ck[buf][warp] = bk;
                cr[buf][warp] = br;
            }
            __syncthreads();
            unsigned long long k = (lane < NW) ? ck[buf][lane] : 0ull;
            int p = (lane < NW) ? cr[buf][lane] : 0x7fffffff;
            const int w = warp_argmax(k, p);
            const bool singular = (k == 0ull || p >= V);
            const double *pr = crow[buf][w];
            const double d = pr[jj];
            const double inv_d = singular ? 0.0 : 1.0 / d;
            if (tid == 0) {
                chosen[jj] = singular ? -1 : p;
                diag[j0 + jj] = singular ? 0.0 : d;
                if (singular && *info == 0) *info = j0 + jj + 1;
            }
            // Gauss-Jordan sweep on the panel columns: pivot row scaled by 1/d,
            // every other row r: a_r -= a_r[jj] * (scaled pivot row), a_r[jj] = -a_r[jj] / d
#pragma unroll
            for (int i = 0; i < RPT; ++i) {
                const int r = tid + i * T;
                if (r >= V || singular) continue;
                if (r == p) {
#pragma unroll
                    for (int c = 0; c < NB; ++c) a[i][c] = (c == jj) ? inv_d : pr[c] * inv_d;
                    active[i] = false;
                } else {
                    const double f = a[i][jj];
#pragma unroll
                    for (int c = 0; c < NB; ++c)
                        if (c != jj) a[i][c] = fma(-f, pr[c] * inv_d, a[i][c]);
                    a[i][jj] = -f * inv_d;
                }
            }
        }
    }
    __syncthreads();
    // LAPACK interchange sequence: at step j the row at logical position j
    // trades places with the chosen row
    if (tid == 0) {
        for (int jj = 0; jj < nbc; ++jj) {
            const int j = j0 + jj;
            int pp = chosen[jj];
            if (pp < 0) pp = pos[j];  // zero column: no interchange
            const int q = where[pp];
            ipiv[j] = q;
            const int rj = pos[j];
            pos[q] = rj;
            where[rj] = q;
            pos[j] = pp;
            where[pp] = j;
        }
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < RPT; ++i) {
        const int r = tid + i * T;
        if (r >= V) continue;
        const int row = (r < j0) ? r : where[r];
#pragma unroll
        for (int c = 0; c < NB; ++c)
            if (c < nbc) M[(size_t)(j0 + c) * V + row] = a[i][c];
    }
}

// every column outside the panel, CB per CTA (blocks skip the panel); the new
// panel columns are staged in shared memory next to the CTA's own columns
template <int NB, int CB>
__global__ void __launch_bounds__(256) k_gj_update(double *__restrict__ M, int V, int j0, int nbc,
                                                   const int *__restrict__ ipiv) {
    extern __shared__ double sm[];
    double *C = sm;                  // [CB][V]
    double *Pn = sm + (size_t)CB * V;  // [NB][V] new panel columns
    __shared__ double R[NB][CB];
    __shared__ double Cp[NB][CB];
    __shared__ int pv[NB];
    const int tid = threadIdx.x, T = blockDim.x;
    const int nleft = (j0 + CB - 1) / CB;
    int c0, cend;
    if ((int)blockIdx.x < nleft) {
        c0 = blockIdx.x * CB;
        cend = min(c0 + CB, j0);
    } else {
        c0 = j0 + nbc + ((int)blockIdx.x - nleft) * CB;
        cend = min(c0 + CB, V);
    }
    const int ncol = cend - c0;
    if (ncol <= 0) return;
    for (int f = tid; f < ncol * V; f += T) C[f] = M[(size_t)c0 * V + f];
    for (int f = tid; f < nbc * V; f += T) Pn[f] = M[(size_t)j0 * V + f];
    if (tid < nbc) pv[tid] = ipiv[j0 + tid];
    __syncthreads();
    if (tid < ncol) {
        double *cl = C + (size_t)tid * V;
        for (int jj = 0; jj < nbc; ++jj) {
            const int j = j0 + jj, p = pv[jj];
            if (p != j) {
                const double t = cl[j];
                cl[j] = cl[p];
                cl[p] = t;
            }
        }
    }
    __syncthreads();
    // pivot rows after the interchanges (A_PO) and R = D^-1 A_PO (D^-1 = rows P of the new panel)
    for (int f = tid; f < nbc * ncol; f += T) {
        const int jj = f % nbc, q = f / nbc;
        Cp[jj][q] = C[(size_t)q * V + j0 + jj];
    }
    __syncthreads();
    for (int f = tid; f < nbc * ncol; f += T) {
        const int jj = f % nbc, q = f / nbc;
        double s = 0.0;
        for (int k = 0; k < nbc; ++k) s = fma(Pn[(size_t)k * V + j0 + jj], Cp[k][q], s);
        R[jj][q] = s;
    }
    __syncthreads();
    // rows P: R; other rows: A + (new panel) A_PO.  A_PO is read from shared
    // memory in the loop (volatile), not hoisted into NB x CB registers.
    volatile double(*Cpv)[CB] = Cp;
    for (int r = tid; r < V; r += T) {
        if (r >= j0 && r < j0 + nbc) {
            for (int q = 0; q < ncol; ++q) C[(size_t)q * V + r] = R[r - j0][q];
            continue;
        }
        double acc[CB];
#pragma unroll
        for (int q = 0; q < CB; ++q) acc[q] = (q < ncol) ? C[(size_t)q * V + r] : 0.0;
#pragma unroll
        for (int jj = 0; jj < NB; ++jj) {
            if (jj < nbc) {
                const double kr = Pn[(size_t)jj * V + r];
#pragma unroll
                for (int q = 0; q < CB; ++q) acc[q] = fma(kr, Cpv[jj][q], acc[q]);
            }
        }
#pragma unroll
        for (int q = 0; q < CB; ++q)
            if (q < ncol) C[(size_t)q * V + r] = acc[q];
    }
    __syncthreads();
    for (int f = tid; f < ncol * V; f += T) M[(size_t)c0 * V + f] = C[f];
}

// ---------------------------------------------------------------- dataflow kernel
// One cooperative launch for the whole factorisation and inverse (V <= 1024).
// CTA b owns columns [8b, 8b+8) of A for the entire run, one row per thread,
// in registers.  Panels are processed in order; panel k is CTA k's own block:
//   * CTA k, once its block has received panels 0..k-1, runs the 8 pivot
//     steps on it (Gauss-Jordan sweep restricted to the block) and publishes
//     the swept block, the pivots and U's diagonal, then a ready flag;
//   * every other CTA waits for that flag and applies the block update to its
//     own columns: with K = published block and A_P = its rows at the 8 pivot
//     positions, rows P become K_P A_P and all other rows r add K_r A_P.
// Rows never move.  Each thread tracks the logical position (LAPACK's row
// order after interchanges) of its row by replaying the interchanges, which
// also gives the dgetrf tie-break (first logical row among equal magnitudes)
// and the final placement: the inverse is X(lpos(r), P_j) = Y(r, j), with P_j
// the physical pivot row of step j and Y the array after the last panel.
// The ready flags (sync[1..nblk]) carry a per-call epoch, one more than the
// call counter sync[0] that every CTA reads at its start and the last panel's
// owner advances at its end, so they are never reset and a captured launch
// can be replayed.  The counter sits at word 0 for every V, so calls of
// different sizes on one workspace keep counting up and no flag a smaller
// call left behind matches a later epoch.  Waits are bounded (kLuWaitNs): on
// expiry the CTA sets info[1] and leaves.
constexpr unsigned long long kLuWaitNs = 2000000000ull;
constexpr unsigned kLuWaitPolls = 1u << 26;

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned *p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_u32(unsigned *p, unsigned v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// true once *f == epoch; false when the wait runs out (time or poll count).
// sleep_ns > 0 spaces the polls of waiters that are not on the critical path.
__device__ bool wait_ready(const unsigned *f, unsigned epoch, unsigned sleep_ns) {
    if (ld_acquire_u32(f) == epoch) return true;
    const unsigned long long t0 = global_ns();
    for (unsigned n = 0; n < kLuWaitPolls; ++n) {
        if (sleep_ns) __nanosleep(sleep_ns);
        if (ld_acquire_u32(f) == epoch) return true;
        if (global_ns() - t0 > kLuWaitNs) break;
    }
    return false;
}

// argmax of (key, lp) over the 32 lanes: larger key, then smaller logical
// position.  Returns true in the one lane holding the winner (logical
// positions are distinct); when no lane has a candidate (lp == INT_MAX
// everywhere) lane 0 is the winner.
__device__ __forceinline__ bool warp_argmax_lpos(unsigned long long &key, int &lp) {
    const unsigned hi = (unsigned)(key >> 32), lo = (unsigned)key;
    const unsigned mhi = __reduce_max_sync(0xffffffffu, hi);
    const unsigned mlo = __reduce_max_sync(0xffffffffu, hi == mhi ? lo : 0u);
    const bool win = (hi == mhi) && (lo == mlo);
    const int ml = (int)__reduce_min_sync(0xffffffffu, win ? (unsigned)lp : 0x7fffffffu);
    const bool me = win && lp == ml && (ml != 0x7fffffff || (threadIdx.x & 31) == 0);
    key = ((unsigned long long)mhi << 32) | mlo;
    lp = ml;
    return me;
}

// Same result as warp_argmax_lpos, with a shortcut for the usual case of a
// unique largest high word (sign, exponent and 20 mantissa bits of |value|):
// then that lane wins without comparing low words or positions.  Unlike
// warp_argmax_lpos it leaves key and lp as they were in every lane.
__device__ __forceinline__ bool warp_argmax_fast(unsigned long long &key, int &lp) {
    const unsigned hi = (unsigned)(key >> 32);
    const unsigned mhi = __reduce_max_sync(0xffffffffu, hi);
    const unsigned tied = __ballot_sync(0xffffffffu, hi == mhi);
    if (mhi != 0u && __popc(tied) == 1) return hi == mhi;
    unsigned long long k2 = key;
    int l2 = lp;
    return warp_argmax_lpos(k2, l2);
}

// 1/d by Newton-Raphson iteration for the reciprocal, x <- x + x (1 - d x)
// (the error e = 1 - d x squares at each step; the iteration as written for a
// fused multiply-add in P. Markstein, IA-64 and Elementary Functions, 2000,
// ch. 8), two steps from the hardware approximation of PTX rcp.approx.ftz.f64.
// The approximation flushes subnormal arguments and results to zero, so for
// |d| outside [2^-1021, 2^1021] (subnormal pivots, pivots whose reciprocal is
// subnormal, zero, inf, NaN) the quotient 1.0 / d is taken instead.
__device__ __forceinline__ double recip_nr(double d) {
    const double a = fabs(d);
    if (!(a >= 0x1p-1021 && a <= 0x1p1021)) return 1.0 / d;
    double x;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(x) : "d"(d));
    double e = fma(-d, x, 1.0);
    x = fma(x, e, x);
    e = fma(-d, x, 1.0);
    return fma(x, e, x);
}

template <int NB>
__device__ __forceinline__ void rotate_left(double (&a)[NB]) {
    const double t = a[0];
#pragma unroll
    for (int q = 0; q + 1 < NB; ++q) a[q] = a[q + 1];
    a[NB - 1] = t;
}

// RPT rows per thread (rows tid, tid + T, ...), T = blockDim.x <= MAXT.
template <int NB, int RPT, int MAXT>
__global__ void __launch_bounds__(MAXT, 1) k_gj_dataflow(double *__restrict__ M, int V,
                                                        double *__restrict__ panels, int *__restrict__ ipiv,
                                                        double *__restrict__ diag, int *__restrict__ info,
                                                        unsigned *__restrict__ sync, int withhold) {
    constexpr int MW = MAXT / 32;
    // per warp candidate of a pivot step: |value| key, logical position,
    // physical row, value, and the row already divided by its pivot entry
    __shared__ unsigned long long ck[2][MW];
    __shared__ int cl[2][MW], cphys[2][MW];
    __shared__ double cval[2][MW];
    __shared__ __align__(16) double crow[2][MW][NB];
    __shared__ __align__(16) double Cp[2][NB][NB];
    __shared__ int s_ip[2][NB];
    __shared__ int own_p[NB];
    __shared__ int s_abort;
    __shared__ unsigned s_epoch;
    __shared__ double s_l[MW];
    __shared__ int s_n[MW];

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, T = (int)blockDim.x, NW = T >> 5;
    const int b = blockIdx.x, nblk = gridDim.x;
    const int c0 = b * NB, ncol = min(NB, V - c0);
    unsigned *ready = sync + 1;
    int row[RPT], lpos[RPT];
    double a[RPT][NB];
#pragma unroll
    for (int i = 0; i < RPT; ++i) {
        row[i] = tid + i * T;
        lpos[i] = row[i];
#pragma unroll
        for (int q = 0; q < NB; ++q) a[i][q] = (row[i] < V && q < ncol) ? M[(size_t)(c0 + q) * V + row[i]] : 0.0;
    }
    if (tid == 0) {
        s_abort = 0;
        const unsigned e = __ldcg(sync) + 1u;
        s_epoch = e ? e : 1u;
    }
    __syncthreads();
    const unsigned epoch = s_epoch;

    for (int k = 0; k < nblk; ++k) {
        const int j0 = k * NB, nbc = min(NB, V - j0);
        if (k == b) {
            // the block is rotated one column left after every step, so the
            // pivot column is always a[.][0]; NB rotations in all restore it
            for (int jj = 0; jj < nbc; ++jj) {
                const int j = j0 + jj, buf = jj & 1;
                unsigned long long key = 0ull;
                int lp = 0x7fffffff, bi = 0;
#pragma unroll
                for (int i = 0; i < RPT; ++i) {
                    if (row[i] < V && lpos[i] >= j) {
                        const unsigned long long ki = (unsigned long long)__double_as_longlong(fabs(a[i][0]));
                        if (ki > key || (ki == key && lpos[i] < lp)) {
                            key = ki;
                            lp = lpos[i];
                            bi = i;
                        }
                    }
                }
                if (warp_argmax_fast(key, lp)) {
                    double v[NB];
#pragma unroll
                    for (int q = 0; q < NB; ++q) v[q] = a[0][q];
#pragma unroll
                    for (int i = 1; i < RPT; ++i)
                        if (bi == i) {
#pragma unroll
                            for (int q = 0; q < NB; ++q) v[q] = a[i][q];
                        }
                    const double inv = (key == 0ull) ? 0.0 : recip_nr(v[0]);
                    ck[buf][warp] = key;
                    cl[buf][warp] = lp;
                    cphys[buf][warp] = row[bi];
                    cval[buf][warp] = v[0];
                    crow[buf][warp][0] = inv;
#pragma unroll
                    for (int q = 1; q < NB; ++q) crow[buf][warp][q] = v[q] * inv;
                }
                __syncthreads();
                unsigned long long kb = (lane < NW) ? ck[buf][lane] : 0ull;
                int lb = (lane < NW) ? cl[buf][lane] : 0x7fffffff;
                const bool wme = warp_argmax_fast(kb, lb) && lane < NW;
                const int w = __ffs(__ballot_sync(0xffffffffu, wme)) - 1;
                const int p = cphys[buf][w];
                lb = cl[buf][w];
                double prs[NB];
#pragma unroll
                for (int q = 0; q < NB; q += 2) {
                    const double2 t2 = *reinterpret_cast<const double2 *>(&crow[buf][w][q]);
                    prs[q] = t2.x;
                    prs[q + 1] = t2.y;
                }
                if (tid == 0) {
                    const bool singular = (ck[buf][w] == 0ull);
                    ipiv[j] = lb;
                    diag[j] = singular ? 0.0 : cval[buf][w];
                    own_p[jj] = p;
                    if (singular) atomicCAS(info, 0, j + 1);
                }
#pragma unroll
                for (int i = 0; i < RPT; ++i) {
                    if (row[i] == p) {
#pragma unroll
                        for (int q = 0; q < NB; ++q) a[i][q] = prs[q];
                    } else {
                        const double f = a[i][0];
                        a[i][0] = -f * prs[0];
#pragma unroll
                        for (int q = 1; q < NB; ++q) a[i][q] = fma(-f, prs[q], a[i][q]);
                    }
                    if (lpos[i] == j) lpos[i] = lb;
                    else if (lpos[i] == lb) lpos[i] = j;
                    rotate_left(a[i]);
                }
            }
            for (int e = nbc; e < NB; ++e) {
#pragma unroll
                for (int i = 0; i < RPT; ++i) rotate_left(a[i]);
            }
#pragma unroll
            for (int i = 0; i < RPT; ++i)
#pragma unroll
                for (int q = 0; q < NB; ++q)
                    if (row[i] < V && q < nbc) panels[(size_t)(j0 + q) * V + row[i]] = a[i][q];
            __syncthreads();
            // (withhold: test hook, the flag of that one panel is never set)
            if (tid == 0 && k != withhold) st_release_u32(ready + k, epoch);
        } else {
            const int buf = k & 1;
            // one warp waits and fetches the panel's pivots; the next owner
            // polls without pause, the others space their polls
            if (warp == 0) {
                int ok = 1;
                if (lane == 0) ok = wait_ready(ready + k, epoch, b == k + 1 ? 0u : 256u);
                ok = __shfl_sync(0xffffffffu, ok, 0);
                __syncwarp();
                if (ok) {
                    if (lane < nbc) s_ip[buf][lane] = __ldcg(ipiv + j0 + lane);
                } else if (lane == 0) {
                    s_abort = 1;
                    atomicExch(info + 1, 1);
                }
            }
            __syncthreads();
            if (s_abort) return;
            double kv[RPT][NB];
#pragma unroll
            for (int i = 0; i < RPT; ++i)
#pragma unroll
                for (int m = 0; m < NB; ++m)
                    kv[i][m] = (row[i] < V && m < nbc) ? __ldcg(panels + (size_t)(j0 + m) * V + row[i]) : 0.0;
            bool is_p[RPT];
#pragma unroll
            for (int i = 0; i < RPT; ++i) {
#pragma unroll
                for (int m = 0; m < NB; ++m) {
                    if (m < nbc) {
                        const int j = j0 + m, ip = s_ip[buf][m];
                        if (lpos[i] == j) lpos[i] = ip;
                        else if (lpos[i] == ip) lpos[i] = j;
                    }
                }
                is_p[i] = row[i] < V && lpos[i] >= j0 && lpos[i] < j0 + nbc;
                if (is_p[i]) {
#pragma unroll
                    for (int q = 0; q < NB; ++q) Cp[buf][lpos[i] - j0][q] = a[i][q];
                }
            }
            __syncthreads();
#pragma unroll
            for (int q = 0; q < NB; ++q) {
                double cp[NB];
#pragma unroll
                for (int m = 0; m < NB; ++m) cp[m] = (m < nbc) ? Cp[buf][m][q] : 0.0;
#pragma unroll
                for (int i = 0; i < RPT; ++i) {
                    double s = 0.0;
#pragma unroll
                    for (int m = 0; m < NB; ++m) s = fma(kv[i][m], cp[m], s);
                    a[i][q] = is_p[i] ? s : a[i][q] + s;
                }
            }
        }
    }
    __syncthreads();
    // every panel has been seen: place the inverse, X(lpos, P_j) = Y(r, j)
#pragma unroll
    for (int i = 0; i < RPT; ++i)
#pragma unroll
        for (int q = 0; q < NB; ++q)
            if (row[i] < V && q < ncol) M[(size_t)own_p[q] * V + lpos[i]] = a[i][q];
    // the last panel's owner has acquired every flag: log|det| and sign
    if (b == nblk - 1) {
        double l = 0.0;
        int neg = 0;
        for (int i = tid; i < V; i += T) {
            const double d = __ldcg(diag + i);
            l += log(fabs(d));
            if (!(d > 0)) neg ^= 1;
            if (__ldcg(ipiv + i) != i) neg ^= 1;
        }
        for (int o = 16; o > 0; o >>= 1) {
            l += __shfl_down_sync(0xffffffffu, l, o);
            neg ^= __shfl_down_sync(0xffffffffu, neg, o);
        }
        if (lane == 0) {
            s_l[warp] = l;
            s_n[warp] = neg;
        }
        __syncthreads();
        if (tid == 0) {
            double t = 0.0;
            int n = 0;
            for (int i = 0; i < NW; ++i) {
                t += s_l[i];
                n ^= s_n[i];
            }
            diag[V] = t;
            diag[V + 1] = n ? -1.0 : 1.0;
            sync[0] = epoch;
        }
    }
}

// ---------------------------------------------------------------- two panels per CTA
// The dataflow kernel for 1024 < V <= 2304, where one 8-column panel per CTA
// would need more CTAs (V / 8 > 128) than the SMs hold at one per SM: CTA b
// owns panel b in registers (5 rows per thread, 512 threads) and panel
// b + nCTA in shared memory (8 x 2560 doubles, 160 KB), nCTA = ceil(P / 2)
// for P = V / 8 panels.  The protocol is that of k_gj_dataflow: panels are
// taken in order, the owner runs the 8 pivot steps on its block and
// publishes the swept block, the pivots and U's diagonal with a ready flag
// (per-call epoch, bounded waits), every other CTA applies the block update
// A(O, c) += K(O, :) A(P, c), A(P, c) = K(P, :) A(P, c) to both of its panels.
// The shared-memory panel's pivot steps index its columns directly instead of
// rotating registers.  The update accumulates into the columns (pivot rows
// first set to zero) two multipliers at a time.
constexpr int kLu2Threads = 512, kLu2Rpt = 5;
constexpr int kLu2MaxV = 2304;                   // 2 * 8 panel columns per SM on 144 SMs
constexpr int kLu2Rows = kLu2Threads * kLu2Rpt;  // 2560 rows held (the last ones padding)

__global__ void __launch_bounds__(kLu2Threads, 1) k_gj_dataflow2(double *__restrict__ M, int V,
                                                                double *__restrict__ panels, int *__restrict__ ipiv,
                                                                double *__restrict__ diag, int *__restrict__ info,
                                                                unsigned *__restrict__ sync, int withhold) {
    constexpr int NB = kLuPanel, RPT = kLu2Rpt, MW = kLu2Threads / 32, LD = kLu2Rows;
    __shared__ unsigned long long ck[2][MW];
    __shared__ int cl[2][MW], cphys[2][MW];
    __shared__ double cval[2][MW];
    __shared__ __align__(16) double crow[2][MW][NB];
    __shared__ __align__(16) double CpA[2][NB][NB], CpB[2][NB][NB];  // [buf][q][m]: pivot row m, column q
    __shared__ int s_ip[2][NB];
    __shared__ int own_pA[NB], own_pB[NB];
    __shared__ int s_abort;
    __shared__ unsigned s_epoch;
    __shared__ double s_l[MW];
    __shared__ int s_n[MW];
    extern __shared__ __align__(16) double sB[];  // [NB][LD]: the second panel

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, T = (int)blockDim.x, NW = T >> 5;
    const int b = blockIdx.x, ncta = gridDim.x;
    const int P = (V + NB - 1) / NB;
    const int pA = b, pB = b + ncta;  // pB < P: the CTA has a second panel
    const bool hasB = pB < P;
    const int cA = pA * NB, ncolA = min(NB, V - cA), cB = pB * NB, ncolB = hasB ? min(NB, V - cB) : 0;
    const int last_owner = P - 1 - ncta;  // the owner of panel P - 1 (as its second panel)
    unsigned *ready = sync + 1;
    int row[RPT], lpos[RPT];
    double a[RPT][NB];
#pragma unroll
    for (int i = 0; i < RPT; ++i) {
        row[i] = tid + i * T;
        lpos[i] = row[i];
#pragma unroll
        for (int q = 0; q < NB; ++q) {
            a[i][q] = (row[i] < V && q < ncolA) ? M[(size_t)(cA + q) * V + row[i]] : 0.0;
            sB[q * LD + row[i]] = (row[i] < V && q < ncolB) ? M[(size_t)(cB + q) * V + row[i]] : 0.0;
        }
    }
    if (tid == 0) {
        s_abort = 0;
        const unsigned e = __ldcg(sync) + 1u;
        s_epoch = e ? e : 1u;
    }
    __syncthreads();
    const unsigned epoch = s_epoch;

    // the register panel and the shared-memory panel exchange places
    auto swap_panels = [&]() {
#pragma unroll
        for (int i = 0; i < RPT; ++i)
#pragma unroll
            for (int q = 0; q < NB; ++q) {
                const double t = sB[q * LD + row[i]];
                sB[q * LD + row[i]] = a[i][q];
                a[i][q] = t;
            }
    };

    // Panel k's block update (its swept block K published at columns j0.. of
    // panels) applied to this CTA's register panel (doA) and shared-memory
    // panel (doB); the rows' logical positions already follow panel k.  Row
    // by row: the row's K entries are read once and serve both panels; rows
    // P start from zero (A(P, c) = K(P, :) A(P, c)), the others from their
    // value (A(O, c) += K(O, :) A(P, c)).
    auto apply_panel = [&](int k, int j0, int nbc, bool doA, bool doB) {
        const int buf = k & 1;
        bool is_p[RPT];
#pragma unroll
        for (int i = 0; i < RPT; ++i) {
            is_p[i] = row[i] < V && lpos[i] >= j0 && lpos[i] < j0 + nbc;
            if (is_p[i]) {
                const int m = lpos[i] - j0;
#pragma unroll
                for (int q = 0; q < NB; ++q) {
                    if (doA) CpA[buf][q][m] = a[i][q];
                    if (doB) CpB[buf][q][m] = sB[q * LD + row[i]];
                }
            }
        }
        // a short last panel: the missing pivot rows are zero
        for (int e = tid; nbc < NB && e < NB * NB; e += T)
            if (e % NB >= nbc) {
                CpA[buf][e / NB][e % NB] = 0.0;
                CpB[buf][e / NB][e % NB] = 0.0;
            }
        __syncthreads();
#pragma unroll
        for (int i = 0; i < RPT; ++i) {
            if (row[i] >= V) continue;
            double kr[NB];
#pragma unroll
            for (int m = 0; m < NB; ++m) kr[m] = m < nbc ? __ldcg(panels + (size_t)(j0 + m) * V + row[i]) : 0.0;
            if (doA) {
#pragma unroll
                for (int q = 0; q < NB; ++q) {
                    double acc = is_p[i] ? 0.0 : a[i][q];
#pragma unroll
                    for (int m = 0; m < NB; m += 2) {
                        const double2 cp = *reinterpret_cast<const double2 *>(&CpA[buf][q][m]);
                        acc = fma(kr[m + 1], cp.y, fma(kr[m], cp.x, acc));
                    }
                    a[i][q] = acc;
                }
            }
            if (doB) {
                double *col = sB + row[i];
#pragma unroll
                for (int q = 0; q < NB; ++q) {
                    double acc = is_p[i] ? 0.0 : col[q * LD];
#pragma unroll
                    for (int m = 0; m < NB; m += 2) {
                        const double2 cp = *reinterpret_cast<const double2 *>(&CpB[buf][q][m]);
                        acc = fma(kr[m + 1], cp.y, fma(kr[m], cp.x, acc));
                    }
                    col[q * LD] = acc;
                }
            }
        }
    };

    for (int k = 0; k < P; ++k) {
        const int j0 = k * NB, nbc = min(NB, V - j0);
        if (k == pA || k == pB) {
            // the panel to factor in registers: the second panel trades places
            // with the first for its 8 steps (each thread its own rows)
            const bool second = (k == pB);
            if (second) swap_panels();
            int *own_p = second ? own_pB : own_pA;
            // rotated one column left after every step
            for (int jj = 0; jj < nbc; ++jj) {
                const int j = j0 + jj, buf = jj & 1;
                unsigned long long key = 0ull;
                int lp = 0x7fffffff, bi = 0;
#pragma unroll
                for (int i = 0; i < RPT; ++i) {
                    if (row[i] < V && lpos[i] >= j) {
                        const unsigned long long ki = (unsigned long long)__double_as_longlong(fabs(a[i][0]));
                        if (ki > key || (ki == key && lpos[i] < lp)) {
                            key = ki;
                            lp = lpos[i];
                            bi = i;
                        }
                    }
                }
                if (warp_argmax_fast(key, lp)) {
                    double d = a[0][0];
#pragma unroll
                    for (int i = 1; i < RPT; ++i)
                        if (bi == i) d = a[i][0];
                    const double inv = (key == 0ull) ? 0.0 : recip_nr(d);
                    ck[buf][warp] = key;
                    cl[buf][warp] = lp;
                    cphys[buf][warp] = tid + bi * T;
                    cval[buf][warp] = d;
                    crow[buf][warp][0] = inv;
#pragma unroll
                    for (int i = 0; i < RPT; ++i)
                        if (bi == i) {
#pragma unroll
                            for (int q = 1; q < NB; ++q) crow[buf][warp][q] = a[i][q] * inv;
                        }
                }
                __syncthreads();
                unsigned long long kb = (lane < NW) ? ck[buf][lane] : 0ull;
                int lb = (lane < NW) ? cl[buf][lane] : 0x7fffffff;
                const bool wme = warp_argmax_fast(kb, lb) && lane < NW;
                const int w = __ffs(__ballot_sync(0xffffffffu, wme)) - 1;
                const int p = cphys[buf][w];
                lb = cl[buf][w];
                double prs[NB];
#pragma unroll
                for (int q = 0; q < NB; q += 2) {
                    const double2 t2 = *reinterpret_cast<const double2 *>(&crow[buf][w][q]);
                    prs[q] = t2.x;
                    prs[q + 1] = t2.y;
                }
                if (tid == 0) {
                    const bool singular = (ck[buf][w] == 0ull);
                    ipiv[j] = lb;
                    diag[j] = singular ? 0.0 : cval[buf][w];
                    own_p[jj] = p;
                    if (singular) atomicCAS(info, 0, j + 1);
                }
#pragma unroll
                for (int i = 0; i < RPT; ++i) {
                    if (row[i] == p) {
#pragma unroll
                        for (int q = 0; q < NB; ++q) a[i][q] = prs[q];
                    } else {
                        const double f = a[i][0];
                        a[i][0] = -f * prs[0];
#pragma unroll
                        for (int q = 1; q < NB; ++q) a[i][q] = fma(-f, prs[q], a[i][q]);
                    }
                    if (lpos[i] == j) lpos[i] = lb;
                    else if (lpos[i] == lb) lpos[i] = j;
                    rotate_left(a[i]);
                }
            }
            for (int e = nbc; e < NB; ++e) {
#pragma unroll
                for (int i = 0; i < RPT; ++i) rotate_left(a[i]);
            }
#pragma unroll
            for (int i = 0; i < RPT; ++i)
#pragma unroll
                for (int q = 0; q < NB; ++q)
                    if (row[i] < V && q < nbc) panels[(size_t)(j0 + q) * V + row[i]] = a[i][q];
            __syncthreads();
            if (tid == 0 && k != withhold) st_release_u32(ready + k, epoch);
            // the panel in shared memory takes this panel's update like every
            // other CTA's; then the panels return to their places
            if (hasB) apply_panel(k, j0, nbc, false, true);
            if (second) swap_panels();
        } else {
            const int buf = k & 1;
            if (warp == 0) {
                int ok = 1;
                if (lane == 0) ok = wait_ready(ready + k, epoch, (k + 1 == pA || k + 1 == pB) ? 0u : 256u);
                ok = __shfl_sync(0xffffffffu, ok, 0);
                __syncwarp();
                if (ok) {
                    if (lane < nbc) s_ip[buf][lane] = __ldcg(ipiv + j0 + lane);
                } else if (lane == 0) {
                    s_abort = 1;
                    atomicExch(info + 1, 1);
                }
            }
            __syncthreads();
            if (s_abort) return;
#pragma unroll
            for (int i = 0; i < RPT; ++i)
#pragma unroll
                for (int m = 0; m < NB; ++m) {
                    if (m < nbc) {
                        const int j = j0 + m, ip = s_ip[buf][m];
                        if (lpos[i] == j) lpos[i] = ip;
                        else if (lpos[i] == ip) lpos[i] = j;
                    }
                }
            apply_panel(k, j0, nbc, true, hasB);
        }
    }
    __syncthreads();
    // every panel has been seen: place the inverse, X(lpos, P_j) = Y(r, j)
#pragma unroll
    for (int i = 0; i < RPT; ++i)
#pragma unroll
        for (int q = 0; q < NB; ++q)
            if (row[i] < V) {
                if (q < ncolA) M[(size_t)own_pA[q] * V + lpos[i]] = a[i][q];
                if (q < ncolB) M[(size_t)own_pB[q] * V + lpos[i]] = sB[q * LD + row[i]];
            }
    // the last panel's owner has acquired every flag: log|det| and sign
    if (b == last_owner) {
        double l = 0.0;
        int neg = 0;
        for (int i = tid; i < V; i += T) {
            const double d = __ldcg(diag + i);
            l += log(fabs(d));
            if (!(d > 0)) neg ^= 1;
            if (__ldcg(ipiv + i) != i) neg ^= 1;
        }
        for (int o = 16; o > 0; o >>= 1) {
            l += __shfl_down_sync(0xffffffffu, l, o);
            neg ^= __shfl_down_sync(0xffffffffu, neg, o);
        }
        if (lane == 0) {
            s_l[warp] = l;
            s_n[warp] = neg;
        }
        __syncthreads();
        if (tid == 0) {
            double t = 0.0;
            int n = 0;
            for (int i = 0; i < NW; ++i) {
                t += s_l[i];
                n ^= s_n[i];
            }
            diag[V] = t;
            diag[V + 1] = n ? -1.0 : 1.0;
            sync[0] = epoch;
        }
    }
}

// composed column permutation: applying the interchanges last-first as column
// swaps leaves column c of the result at column src[c] of the elimination output
__global__ void k_compose_perm(const int *__restrict__ ipiv, int V, int *__restrict__ perm) {
    extern __shared__ int src[];  // [V] permutation, then [V] pivots
    int *pv = src + V;
    for (int c = threadIdx.x; c < V; c += blockDim.x) {
        src[c] = c;
        pv[c] = ipiv[c];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = V - 1; k >= 0; --k) {
            const int p = pv[k];
            const int t = src[k];
            src[k] = src[p];
            src[p] = t;
        }
    }
    __syncthreads();
    for (int c = threadIdx.x; c < V; c += blockDim.x) perm[c] = src[c];
}

__global__ void k_gather_rows(const double *__restrict__ A, double *__restrict__ X, int V,
                              const int *__restrict__ perm) {
    const int c = blockIdx.x;
    const int s = perm[c];
    for (int r = threadIdx.x; r < V; r += blockDim.x) X[(size_t)c * V + r] = A[(size_t)s * V + r];
}

// log|det| and sign from U's diagonal and the pivots (parallel sum)
__global__ void k_lu_logdet(const double *__restrict__ diag, const int *__restrict__ ipiv, int V,
                            double *__restrict__ out) {
    __shared__ double s_l[32];
    __shared__ int s_n[32];
    double l = 0.0;
    int neg = 0;
    for (int i = threadIdx.x; i < V; i += blockDim.x) {
        const double d = diag[i];
        l += log(fabs(d));
        if (!(d > 0)) neg ^= 1;
        if (ipiv[i] != i) neg ^= 1;
    }
    for (int o = 16; o > 0; o >>= 1) {
        l += __shfl_down_sync(0xffffffffu, l, o);
        neg ^= __shfl_down_sync(0xffffffffu, neg, o);
    }
    if ((threadIdx.x & 31) == 0) {
        s_l[threadIdx.x >> 5] = l;
        s_n[threadIdx.x >> 5] = neg;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        int n = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
            t += s_l[w];
            n ^= s_n[w];
        }
        out[0] = t;
        out[1] = n ? -1.0 : 1.0;
    }
}

template <int NB, int RPT, int T, int CB>
int run_panels(double *M, LUWork &w, cudaStream_t st) {
    const int V = w.V;
    const size_t usmem = (size_t)(CB + NB) * V * sizeof(double);
    const size_t psmem = 2 * (size_t)V * sizeof(int);
    if (usmem > 210 * 1024 || psmem > 64 * 1024 || V > RPT * T) return EPHMC_ERR_UNSUPPORTED;
    EPHMC_CUDA(cudaFuncSetAttribute(k_gj_update<NB, CB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)usmem));
    EPHMC_CUDA(cudaFuncSetAttribute(k_gj_panel<NB, RPT, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)psmem));
    for (int j0 = 0; j0 < V; j0 += NB) {
        const int nbc = std::min(NB, V - j0);
        k_gj_panel<NB, RPT, T><<<1, T, psmem, st>>>(M, V, j0, nbc, w.ipiv, w.diag, w.info);
        ephmc::count_launch(1);
        EPHMC_CUDA(cudaGetLastError());
        const int nblocks = (j0 + CB - 1) / CB + (V - j0 - nbc + CB - 1) / CB;
        if (nblocks > 0) {
            k_gj_update<NB, CB><<<nblocks, 256, usmem, st>>>(M, V, j0, nbc, w.ipiv);
            ephmc::count_launch(1);
            EPHMC_CUDA(cudaGetLastError());
        }
    }
    return EPHMC_OK;
}

// ephmc_test_lu_withhold_next: the panel whose ready flag the next dataflow
// launch does not set (-1: none)
std::atomic<int> g_lu_withhold{-1};

template <int RPT, int MAXT>
int launch_dataflow(double *M, LUWork &w, int nblk, int T, int sms, cudaStream_t st) {
    int per_sm = 0;
    EPHMC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_gj_dataflow<kLuPanel, RPT, MAXT>, T, 0));
    if ((long)per_sm * sms < nblk) return EPHMC_ERR_UNSUPPORTED;
    const int V = w.V;
    double *panels = w.X;
    int withhold = g_lu_withhold.exchange(-1);  // one call only
    void *args[] = {&M, (void *)&V, &panels, &w.ipiv, &w.diag, &w.info, &w.sync, &withhold};
    EPHMC_CUDA(cudaLaunchCooperativeKernel((const void *)k_gj_dataflow<kLuPanel, RPT, MAXT>, dim3(nblk), dim3(T), args,
                                           0, st));
    ephmc::count_launch(1);
    return EPHMC_OK;
}

// CTA sizes of the dataflow kernel for a given number of rows per thread:
// 256 threads at most, or 512 with 2 rows per thread.  At V = 1024, 512
// threads of 2 rows (128 registers each) take 1.31 ms against 1.45 for 256
// threads of 4 rows: each pivot step's row scan and rank-1 update are half as
// long per thread, with twice the warps to hide them; 1024 threads of one row
// (64 registers) take 1.82 ms.
inline int lu_max_threads(int rpt) { return rpt == 2 ? 512 : 256; }

}  // namespace

bool lu_shape_ok(int V, int rpt) {
    return (rpt == 1 || rpt == 2 || rpt == 4) && (V + rpt - 1) / rpt <= lu_max_threads(rpt);
}

namespace {

// Two panels per CTA (1024 < V <= 2304): all ceil(P/2) CTAs resident at once,
// each with the second panel's 160 KB of shared memory.
int run_dataflow2(double *M, LUWork &w, cudaStream_t st) {
    const int V = w.V;
    if (V <= 1024 || V > kLu2MaxV || w.sync == nullptr || w.sync_words < lu_sync_words(V))
        return EPHMC_ERR_UNSUPPORTED;
    const int P = (V + kLuPanel - 1) / kLuPanel, ncta = (P + 1) / 2;
    int dev = 0, sms = 0, coop = 0;
    EPHMC_CUDA(cudaGetDevice(&dev));
    EPHMC_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    EPHMC_CUDA(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
    if (!coop) return EPHMC_ERR_UNSUPPORTED;
    const size_t smem = sizeof(double) * kLuPanel * (size_t)kLu2Rows;
    EPHMC_CUDA(cudaFuncSetAttribute(k_gj_dataflow2, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    EPHMC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_gj_dataflow2, kLu2Threads, smem));
    if ((long)per_sm * sms < ncta) return EPHMC_ERR_UNSUPPORTED;
    double *panels = w.X;
    int withhold = g_lu_withhold.exchange(-1);  // one call only
    void *args[] = {&M, (void *)&V, &panels, &w.ipiv, &w.diag, &w.info, &w.sync, &withhold};
    EPHMC_CUDA(cudaLaunchCooperativeKernel((const void *)k_gj_dataflow2, dim3(ncta), dim3(kLu2Threads), args, smem,
                                           st));
    ephmc::count_launch(1);
    return EPHMC_OK;
}

// The dataflow kernel needs all ceil(V/8) CTAs resident at once; returns
// EPHMC_ERR_UNSUPPORTED (nothing launched) when they are not; above V = 1024
// the two-panel kernel.
int run_dataflow(double *M, LUWork &w, cudaStream_t st) {
    const int V = w.V;
    if (V > 1024) return run_dataflow2(M, w, st);
    if (w.sync == nullptr || w.sync_words < lu_sync_words(V)) return EPHMC_ERR_UNSUPPORTED;
    const int nblk = (V + kLuPanel - 1) / kLuPanel;
    int dev = 0, sms = 0, coop = 0;
    EPHMC_CUDA(cudaGetDevice(&dev));
    EPHMC_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    EPHMC_CUDA(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
    if (!coop) return EPHMC_ERR_UNSUPPORTED;
    // rows per thread; a tuned choice (ephmc_ctx_autotune) replaces the rule
    // when its CTA size is one of the kernel's
    int rpt = V <= 256 ? 1 : 2;
    if (lu_shape_ok(V, w.tune_rpt)) rpt = w.tune_rpt;
    const int T = ((V + rpt - 1) / rpt + 31) / 32 * 32;
    if (rpt == 1) return launch_dataflow<1, 256>(M, w, nblk, T, sms, st);
    if (rpt == 2) return T > 256 ? launch_dataflow<2, 512>(M, w, nblk, T, sms, st)
                                 : launch_dataflow<2, 256>(M, w, nblk, T, sms, st);
    return launch_dataflow<4, 256>(M, w, nblk, T, sms, st);
}

}  // namespace

int lu_alloc(LUWork &w, int V) {
    w.V = V;
    EPHMC_CUDA(cudaMalloc(&w.ipiv, sizeof(int) * 2 * V));  // pivots, then the composed permutation
    EPHMC_CUDA(cudaMalloc(&w.diag, sizeof(double) * (V + 2)));
    EPHMC_CUDA(cudaMalloc(&w.info, sizeof(int) * 2));
    EPHMC_CUDA(cudaMalloc(&w.X, sizeof(double) * (size_t)V * V));
    w.sync_words = lu_sync_words(V);
    EPHMC_CUDA(cudaMalloc(&w.sync, sizeof(unsigned) * w.sync_words));
    EPHMC_CUDA(cudaMemset(w.sync, 0, sizeof(unsigned) * w.sync_words));
    return EPHMC_OK;
}

void lu_reset_sync(LUWork &w, cudaStream_t st) {
    if (w.sync && w.sync_words) cudaMemsetAsync(w.sync, 0, sizeof(unsigned) * w.sync_words, st);
}

void lu_free(LUWork &w) {
    if (w.ipiv) cudaFree(w.ipiv);
    if (w.diag) cudaFree(w.diag);
    if (w.info) cudaFree(w.info);
    if (w.X) cudaFree(w.X);
    if (w.sync) cudaFree(w.sync);
    w = LUWork{};
}

// Everything up to the inverse in place, asynchronous on st: pivots (0-based,
// LAPACK order) in w.ipiv, U's diagonal in w.diag, log|det| and sign in
// w.diag[V], w.diag[V+1], first zero pivot (1-based) in w.info[0].
int lu_logdet_inverse_async(double *M, LUWork &w, cudaStream_t st) {
    const int V = w.V;
    EPHMC_CUDA(cudaMemsetAsync(w.info, 0, sizeof(int) * 2, st));
    int rc = run_dataflow(M, w, st);
    if (rc == EPHMC_OK) return EPHMC_OK;
    if (rc != EPHMC_ERR_UNSUPPORTED) return rc;
    if (V <= 1024) rc = run_panels<16, 4, 256, 7>(M, w, st);
    else if (V <= 2048) rc = run_panels<8, 4, 512, 4>(M, w, st);
    else if (V <= 4096) rc = run_panels<4, 4, 1024, 2>(M, w, st);
    else rc = EPHMC_ERR_UNSUPPORTED;
    if (rc != EPHMC_OK) return rc;
    k_lu_logdet<<<1, 1024, 0, st>>>(w.diag, w.ipiv, V, w.diag + V);
    ephmc::count_launch(1);
    EPHMC_CUDA(cudaGetLastError());
    int *perm = w.ipiv + V;
    k_compose_perm<<<1, 1024, 2 * sizeof(int) * V, st>>>(w.ipiv, V, perm);
    ephmc::count_launch(1);
    k_gather_rows<<<V, 256, 0, st>>>(M, w.X, V, perm);
    ephmc::count_launch(1);
    EPHMC_CUDA(cudaGetLastError());
    EPHMC_CUDA(cudaMemcpyAsync(M, w.X, sizeof(double) * (size_t)V * V, cudaMemcpyDeviceToDevice, st));
    return EPHMC_OK;
}

int lu_logdet_inverse(double *M, LUWork &w, double *logdet, int *sign, int *ipiv_host, cudaStream_t st) {
    const int V = w.V;
    int rc = lu_logdet_inverse_async(M, w, st);
    if (rc != EPHMC_OK) return rc;
    int info[2] = {0, 0};
    double ld[2] = {0, 1};
    EPHMC_CUDA(cudaMemcpyAsync(info, w.info, sizeof(int) * 2, cudaMemcpyDeviceToHost, st));
    EPHMC_CUDA(cudaMemcpyAsync(ld, w.diag + V, sizeof(double) * 2, cudaMemcpyDeviceToHost, st));
    if (ipiv_host) EPHMC_CUDA(cudaMemcpyAsync(ipiv_host, w.ipiv, sizeof(int) * V, cudaMemcpyDeviceToHost, st));
    EPHMC_CUDA(cudaStreamSynchronize(st));
    if (ipiv_host)
        for (int i = 0; i < V; ++i) ipiv_host[i] += 1;  // LAPACK 1-based
    if (logdet) *logdet = ld[0];
    if (sign) *sign = ld[1] < 0 ? -1 : 1;
    if (info[1] != 0) {
        // flags of the abandoned call could match the next call's epoch
        lu_reset_sync(w, st);
        cudaStreamSynchronize(st);
        set_status(EPHMC_ERR_TIMEOUT, "LU: a panel wait of the dataflow kernel ran out; the result is invalid");
        return EPHMC_ERR_TIMEOUT;
    }
    if (info[0] != 0) return EPHMC_ERR_SINGULAR;
    return EPHMC_OK;
}

}  // namespace ephmc

extern "C" EPHMC_API void ephmc_test_lu_withhold_next(int panel) { ephmc::g_lu_withhold.store(panel); }
