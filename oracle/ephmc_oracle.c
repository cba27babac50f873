/*
 * CPU restatement of the electron-phonon HMC hot path -- TEST ORACLE ONLY.
 *
 * Written for this project from the algorithm of the reference
 * (j-ostmeyer/electron-phonon-hmc, the C files under simulation/).  Every function cites the
 * reference lines it restates.  Nothing here is shipped: only tests/, the smoke
 * check and bench.py's CPU baseline load liboracle.so, as the checker.
 *
 * Pinning: tests compare this restatement against the reference's own C
 * sources compiled unmodified into oracle/_ref/libephref.so (oracle/Makefile).
 * Deliberate differences from the reference:
 *   - LU / inverse are an unblocked partial-pivoting LU and the classic
 *     inverse-of-U-then-solve-with-L inverse, instead of LAPACKE dgetrf/dgetri;
 *     results agree to the reference's own thread-to-thread reproducibility.
 *   - the real DFT for Fourier acceleration is an O(Nt^2) transform with
 *     FFTW's conventions (FFTW3 is not installed).
 */
#include <complex.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "ephmc_oracle.h"

#define OR_TWO_PI 6.283185307179586 /* value of M_2PI, simulation/organic_aux.h:9 */
#define OR_PI 3.141592653589793     /* value of M_PI, simulation/organic_aux.h:7 */
#define OR_NPAIRS 2

/* Taylor-4 factorised into two quadratic pairs, c_p (simulation/taylor-coeff_pairs.h:35-42
   under -DTAYLOR_ORDER_4, the build's choice at simulation/Makefile:14). */
static const double or_coeff_re[OR_NPAIRS] = {1.8294933739891903, 0.1705066260108097};
static const double or_coeff_im[OR_NPAIRS] = {0.9404019519941707, 1.5785318126884535};

/* Pair order for two pairs: set_taylor_pair_order (simulation/organic_dense_matrix.c:133-159)
   with NUM_TAYLOR_PAIRS = 2 yields the identity order {0, 1}. */
static const unsigned or_pair_order[OR_NPAIRS] = {0, 1};

/* ------------------------------------------------------------ MT19937-64 */
/* Published 64-bit Mersenne Twister (Nishimura 2000); the reference uses the
   authors' C code at simulation/mt19937-64.c:73-79 (seeding) and :108-162
   (generation, genrand64_real2 on [0,1)). */
#define MT_N 312
#define MT_M 156
static uint64_t mt_state[MT_N];
static int mt_pos = MT_N + 1;

void or_mt_seed(unsigned long long seed) {
    mt_state[0] = (uint64_t)seed;
    for (int i = 1; i < MT_N; i++) {
        const uint64_t prev = mt_state[i - 1];
        mt_state[i] = 6364136223846793005ULL * (prev ^ (prev >> 62)) + (uint64_t)i;
    }
    mt_pos = MT_N;
}

static uint64_t mt_next(void) {
    if (mt_pos >= MT_N) {
        if (mt_pos == MT_N + 1) or_mt_seed(5489ULL);
        const uint64_t upper = 0xFFFFFFFF80000000ULL, lower = 0x7FFFFFFFULL;
        for (int i = 0; i < MT_N; i++) {
            const uint64_t y = (mt_state[i] & upper) | (mt_state[(i + 1) % MT_N] & lower);
            uint64_t v = mt_state[(i + MT_M) % MT_N] ^ (y >> 1);
            if (y & 1ULL) v ^= 0xB5026F5AA96619E9ULL;
            mt_state[i] = v;
        }
        mt_pos = 0;
    }
    uint64_t z = mt_state[mt_pos++];
    z ^= (z >> 29) & 0x5555555555555555ULL;
    z ^= (z << 17) & 0x71D67FFFEDA60000ULL;
    z ^= (z << 37) & 0xFFF7EEE000000000ULL;
    z ^= z >> 43;
    return z;
}

double or_mt_real2(void) { return (double)(mt_next() >> 11) * (1.0 / 9007199254740992.0); }

/* Box-Muller pairs, cos into even slots, sin into the next (wrapping for odd n):
   random_vector, simulation/organic_random.c:11-22. */
void or_normals(double *x, unsigned n) {
    for (unsigned k = 0; k < n; k += 2) {
        const double r = sqrt(-2 * log(or_mt_real2()));
        const double phi = OR_TWO_PI * or_mt_real2();
        x[k] = r * cos(phi);
        x[(k + 1) % n] = r * sin(phi);
    }
}

/* ------------------------------------------------------------ lattice & parameters */
/* Periodic L1 x L2 triangular lattice, construct_triangular
   (simulation/organic_lattice.c:10-46).  Entries 6i+0..5 are the neighbour
   sites right, left, top-right, bottom-left, top-left, bottom-right; entries
   6(V+i)+0..5 the matching link indices. */
void or_lattice(unsigned l1, unsigned l2, unsigned *nnt) {
    const unsigned V = l1 * l2;
    for (unsigned i = 0; i < V; i++) {
        const unsigned c1 = i % l1, c2 = i / l1;
        const unsigned row = c2 * l1;
        const unsigned up = ((c2 + 1) % l2) * l1, down = ((c2 + l2 - 1) % l2) * l1;
        const unsigned r1 = (c1 + 1) % l1, lf1 = (c1 + l1 - 1) % l1;
        unsigned *s = nnt + 6 * i;
        s[0] = row + r1;       /* right */
        s[1] = row + lf1;      /* left */
        s[2] = up + c1;        /* top right */
        s[3] = down + c1;      /* bottom left */
        s[4] = up + lf1;       /* top left */
        s[5] = down + r1;      /* bottom right */
        unsigned *l = nnt + 6 * (V + i);
        l[0] = 3 * i;
        l[1] = 3 * s[1];
        l[2] = 3 * i + 1;
        l[3] = 3 * s[3] + 1;
        l[4] = 3 * i + 2;
        l[5] = 3 * s[5] + 2;
    }
}

/* Unit conversion of organic_main (simulation/organic_main.c:99-116, with
   ROOM_TEMPERATURE 0.025 at :8). */
void or_convert_params(double beta, unsigned nt, const double *J, const double *lam,
                       double mu0, double omega0, int static_disorder,
                       double *t, double *kappa, double *mu, double *omega) {
    const double x_avg = static_disorder ? 1 : sqrt(.5 / tanh(.5 * omega0 / 0.025));
    double b = static_disorder ? -beta : beta / nt;
    double m = mu0 * b;
    *omega = omega0 * b;
    for (int k = 0; k < 3; k++) {
        t[k] = J[k] * b;
        kappa[k] = lam[k] * t[k] / x_avg;
        m -= 2 * fabs(t[k]);
    }
    *mu = m;
}

/* a = c_p / (2P): linear coefficient 2 Re a and quadratic |a|^2
   (simulation/organic_dense_matrix.c:169,189,192). */
void or_pair_coeffs(double *a_lin, double *a_quad, int *is_complex) {
    for (int p = 0; p < OR_NPAIRS; p++) {
        const unsigned pos = or_pair_order[p];
        const double re = .5 * or_coeff_re[pos] / OR_NPAIRS;
        const double im = .5 * or_coeff_im[pos] / OR_NPAIRS;
        const double mag = hypot(re, im);
        a_lin[p] = 2 * re;
        a_quad[p] = mag * mag;
        is_complex[p] = im != 0;
    }
}

or_model *or_model_new(unsigned l1, unsigned l2, unsigned nt, const double *t,
                       const double *kappa, double mu, double omega,
                       unsigned flavors, const int *flags) {
    or_model *m = calloc(1, sizeof(*m));
    m->l1 = l1; m->l2 = l2; m->ns = l1 * l2; m->nt = nt; m->flavors = flavors;
    for (int k = 0; k < 3; k++) { m->t[k] = t[k]; m->kappa[k] = kappa[k]; }
    m->mu = mu; m->omega = omega;
    if (flags) for (int k = 0; k < 7; k++) m->flags[k] = flags[k];
    m->nnt = malloc(sizeof(unsigned) * 12 * m->ns);
    or_lattice(l1, l2, m->nnt);
    return m;
}

void or_model_free(or_model *m) {
    if (!m) return;
    free(m->nnt);
    free(m);
}

/* ------------------------------------------------------------ stencil */
/* w = (mu + K_t(x)) v in scatter form over the three forward links of every
   site: apply_mu_K_to_v (simulation/organic_dense_matrix.c:96-120). */
void or_apply_mu_K_v(const or_model *m, const double *xs, const double *v, double *w) {
    const unsigned V = m->ns;
    for (unsigned i = 0; i < V; i++) w[i] = m->mu * v[i];
    for (unsigned i = 0; i < V; i++) {
        for (unsigned k = 0; k < 3; k++) {
            const unsigned j = m->nnt[6 * i + 2 * k];
            const double hop = m->t[k] - m->kappa[k] * xs[3 * i + k];
            const double to_i = hop * v[j];
            const double to_j = hop * v[i];
            w[i] += to_i;
            w[j] += to_j;
        }
    }
}

/* v <- v + a_lin H v + a_quad H^2 v (apply_2nd_order_mu_K_to_v, :168-183) */
static void or_apply_pair_v(const or_model *m, const double *xs, double *v, double *scratch,
                            double a_lin, double a_quad, int cplx) {
    const unsigned V = m->ns;
    double *hv = scratch, *hhv = scratch + V;
    or_apply_mu_K_v(m, xs, v, hv);
    if (cplx) {
        or_apply_mu_K_v(m, xs, hv, hhv);
        for (unsigned i = 0; i < V; i++) v[i] += a_lin * hv[i] + a_quad * hhv[i];
    } else {
        for (unsigned i = 0; i < V; i++) v[i] += a_lin * hv[i];
    }
}

/* Pair product in taylor_pair_order: forward pairs [0, stop) or, with revert,
   pairs (stop, P-1] from the last down (apply_pair_expansion_mu_K_to_v, :186-194). */
static void or_apply_exp_v(const or_model *m, const double *xs, double *v, double *scratch,
                           int revert, int stop) {
    double al[OR_NPAIRS], aq[OR_NPAIRS];
    int cx[OR_NPAIRS];
    or_pair_coeffs(al, aq, cx);
    if (revert) {
        for (int p = OR_NPAIRS - 1; p > stop; p--) or_apply_pair_v(m, xs, v, scratch, al[p], aq[p], cx[p]);
    } else {
        for (int p = 0; p < stop; p++) or_apply_pair_v(m, xs, v, scratch, al[p], aq[p], cx[p]);
    }
}

/* Every row of M (apply_exp_mu_K_to_M, :209-216). */
void or_apply_exp_M(const or_model *m, const double *xs, double *M, int revert, int stop) {
    const unsigned V = m->ns;
#pragma omp parallel
    {
        double *scratch = malloc(sizeof(double) * 2 * V);
#pragma omp for
        for (unsigned r = 0; r < V; r++) or_apply_exp_v(m, xs, M + (size_t)r * V, scratch, revert, stop);
        free(scratch);
    }
}

/* Every row of M replaced by (mu + K) row (apply_mu_K_to_M, :123-131). */
static void or_apply_mu_K_M(const or_model *m, const double *xs, double *M) {
    const unsigned V = m->ns;
#pragma omp parallel
    {
        double *w = malloc(sizeof(double) * V);
#pragma omp for
        for (unsigned r = 0; r < V; r++) {
            or_apply_mu_K_v(m, xs, M + (size_t)r * V, w);
            memcpy(M + (size_t)r * V, w, sizeof(double) * V);
        }
        free(w);
    }
}

static void or_transpose(double *M, unsigned n) {
#pragma omp parallel for
    for (unsigned i = 0; i < n; i++)
        for (unsigned j = i + 1; j < n; j++) {
            const double a = M[(size_t)i * n + j];
            M[(size_t)i * n + j] = M[(size_t)j * n + i];
            M[(size_t)j * n + i] = a;
        }
}

static void or_identity(double *M, unsigned n) {
    memset(M, 0, sizeof(double) * (size_t)n * n);
    for (unsigned i = 0; i < n; i++) M[(size_t)i * (n + 1)] = 1;
}

/* M_hat = 1 + B_0 ... B_{Nt-1}: identity rows propagated by slices Nt-1 .. 0,
   then +1 on the diagonal unless ZERO_FILLING / SINGLE_PARTICLE
   (construct_M_hat, simulation/organic_dense_matrix.c:251-265). */
void or_construct_M_hat(const or_model *m, const double *x, double *M) {
    const unsigned V = m->ns;
    or_identity(M, V);
    for (int tau = (int)m->nt - 1; tau >= 0; tau--)
        or_apply_exp_M(m, x + (size_t)tau * V * 3, M, 0, OR_NPAIRS);
    if (!m->flags[1] && !m->flags[3])
        for (unsigned i = 0; i < V; i++) M[(size_t)i * (V + 1)] += 1;
}

/* ------------------------------------------------------------ LU */
/* log|det| and in-place inverse of the column-major matrix A(r,c) = M[c*n+r]
   (logDetM_and_inv_M_hat, simulation/organic_dense_matrix.c:580-595: dgetrf,
   sign from diagonal signs and pivots, dgetri).  Partial pivoting picks the
   first row of largest magnitude, as LAPACK's idamax. */
double or_logdet_inverse(double *M, unsigned n, int *sign_out) {
#define A_(r, c) M[(size_t)(c) * n + (r)]
    int *piv = malloc(sizeof(int) * n);
    double logdet = 0;
    int sign = 1;
    for (unsigned j = 0; j < n; j++) {
        unsigned p = j;
        double best = fabs(A_(j, j));
        for (unsigned r = j + 1; r < n; r++)
            if (fabs(A_(r, j)) > best) { best = fabs(A_(r, j)); p = r; }
        piv[j] = (int)p;
        if (p != j) {
            for (unsigned c = 0; c < n; c++) {
                const double a = A_(j, c);
                A_(j, c) = A_(p, c);
                A_(p, c) = a;
            }
        }
        const double d = A_(j, j);
        if (d != 0)
            for (unsigned r = j + 1; r < n; r++) A_(r, j) /= d;
#pragma omp parallel for if (n - j > 128)
        for (unsigned c = j + 1; c < n; c++) {
            const double f = A_(j, c);
            if (f != 0)
                for (unsigned r = j + 1; r < n; r++) A_(r, c) -= A_(r, j) * f;
        }
    }
    for (unsigned i = 0; i < n; i++) {
        const double d = A_(i, i);
        logdet += log(fabs(d));
        if (d <= 0) sign = -sign;
        if (piv[i] != (int)i) sign = -sign;
    }
    if (sign_out) *sign_out = sign;

    /* inverse of U in place (upper triangle) */
    for (unsigned j = 0; j < n; j++) {
        A_(j, j) = 1 / A_(j, j);
        const double s = -A_(j, j);
        /* column j above the diagonal: inv(U[0:j,0:j]) * U[0:j,j] * s */
        for (unsigned r = 0; r < j; r++) {
            double acc = 0;
            for (unsigned k = r; k < j; k++) acc += A_(r, k) * A_(k, j);
            A_(r, j) = acc;
        }
        for (unsigned r = 0; r < j; r++) A_(r, j) *= s;
    }
    /* solve X * L = inv(U) column by column from the right */
    double *lcol = malloc(sizeof(double) * n);
    for (int j = (int)n - 1; j >= 0; j--) {
        for (unsigned r = (unsigned)j + 1; r < n; r++) {
            lcol[r] = A_(r, j);
            A_(r, j) = 0;
        }
#pragma omp parallel for if (n > 256)
        for (unsigned r = 0; r < n; r++) {
            double acc = A_(r, j);
            for (unsigned k = (unsigned)j + 1; k < n; k++) acc -= A_(r, k) * lcol[k];
            A_(r, j) = acc;
        }
    }
    /* undo the row interchanges as column interchanges, last first */
    for (int j = (int)n - 2; j >= 0; j--) {
        const unsigned p = (unsigned)piv[j];
        if (p != (unsigned)j)
            for (unsigned r = 0; r < n; r++) {
                const double a = A_(r, j);
                A_(r, j) = A_(r, p);
                A_(r, p) = a;
            }
    }
    free(lcol);
    free(piv);
    return logdet;
#undef A_
}

/* ------------------------------------------------------------ force (reference algorithm) */
static unsigned or_ceil_half(unsigned n) { return n / 2 + n % 2; }         /* simulation/organic_aux.c:11-13 */
static unsigned or_ceil_log2(unsigned n) {                                  /* simulation/organic_aux.c:15-19 */
    unsigned l = 0;
    while (n > 1) { n = or_ceil_half(n); l++; }
    return l;
}

/* G_t = Q_t M^-1 P_t for every t by log-depth sharing: each pass halves the
   outstanding slice count; a matrix that still lacks slices spawns a copy
   `chunk` slots later which takes `chunk` slices from the P side while the
   original takes `chunk` slices from the Q side
   (construct_all_QM1P, simulation/organic_dense_matrix.c:311-381). */
void or_all_G(const or_model *m, const double *x, const double *M_inv, double *G) {
    const unsigned V = m->ns, nt = m->nt;
    const size_t md = (size_t)V * V;
    const size_t ld = (size_t)V * 3;
    unsigned *from_q = calloc(nt, sizeof(unsigned)); /* slices taken on the Q side */
    unsigned *from_p = calloc(nt, sizeof(unsigned)); /* slices taken on the P side */
    if (!m->flags[3]) memcpy(G, M_inv, sizeof(double) * md);
    else or_identity(G, V);

    unsigned left = nt - 1;
    const unsigned passes = or_ceil_log2(nt);
    for (unsigned r = 0; r < passes; r++) {
        const unsigned chunk = or_ceil_half(left);
        for (int i = (int)nt - 1; i >= 0; i--) {
            if (!(i == 0 || from_q[i] || from_p[i])) continue;
            const unsigned j = (unsigned)i + chunk;
            if (j < nt && from_q[j] == 0 && from_p[j] == 0) {
                double *Gj = G + j * md;
                memcpy(Gj, G + (size_t)i * md, sizeof(double) * md);
                from_q[j] = from_q[i];
                from_p[j] = from_p[i];
                or_transpose(Gj, V);
                for (unsigned tau = from_p[j]; tau < from_p[j] + chunk; tau++)
                    or_apply_exp_M(m, x + tau * ld, Gj, 0, OR_NPAIRS);
                or_transpose(Gj, V);
                from_p[j] += chunk;
            }
            for (int tau = (int)nt - 1 - (int)from_q[i]; tau > (int)nt - 1 - (int)from_q[i] - (int)chunk; tau--)
                or_apply_exp_M(m, x + (size_t)tau * ld, G + (size_t)i * md, 0, OR_NPAIRS);
            from_q[i] += chunk;
        }
        left -= chunk;
    }
    free(from_q);
    free(from_p);
}

/* G_t -> sum_p [ a_lin X_p + a_quad (H X_p + X_p H) ], X_p = F_<p G F_>p, the
   exact derivative of the factorised polynomial (refine_QM1P,
   simulation/organic_dense_matrix.c:383-442).  F_<p are the pairs before p
   applied to rows, F_>p the pairs after p applied to columns. */
void or_refine(const or_model *m, const double *x, double *G, unsigned t) {
    const unsigned V = m->ns;
    const size_t md = (size_t)V * V;
    const double *xs = x + (size_t)t * V * 3;
    double al[OR_NPAIRS], aq[OR_NPAIRS];
    int cx[OR_NPAIRS];
    or_pair_coeffs(al, aq, cx);
    double *orig = malloc(sizeof(double) * md);
    double *loc = malloc(sizeof(double) * md);
    double *loc2 = malloc(sizeof(double) * md);
    memcpy(orig, G, sizeof(double) * md);
    memset(G, 0, sizeof(double) * md);
    for (int p = 0; p < OR_NPAIRS; p++) {
        memcpy(loc, orig, sizeof(double) * md);
        or_apply_exp_M(m, xs, loc, 0, p);
        or_transpose(loc, V);
        or_apply_exp_M(m, xs, loc, 1, p);
        if (cx[p]) {
            memcpy(loc2, loc, sizeof(double) * md);
            or_apply_mu_K_M(m, xs, loc2);
            or_transpose(loc2, V);
        }
        or_transpose(loc, V);
        for (size_t e = 0; e < md; e++) G[e] += al[p] * loc[e];
        if (cx[p]) {
            or_apply_mu_K_M(m, xs, loc);
            for (size_t e = 0; e < md; e++) G[e] += aq[p] * (loc[e] + loc2[e]);
        }
    }
    free(orig);
    free(loc);
    free(loc2);
}

/* p_dot[t,i,k] = -kappa_k (G[i][n] + G[n][i]) flavors with n the k-th forward
   neighbour; the Schur clamp and single-particle weight as in force
   (simulation/organic_hmc.c:107-126). */
void or_contract(const or_model *m, const double *Gt, unsigned t, double logdet, double *p_dot) {
    const unsigned V = m->ns;
    for (unsigned i = 0; i < V; i++) {
        for (unsigned k = 0; k < 3; k++) {
            const unsigned n = m->nnt[6 * i + 2 * k];
            double proj = Gt[(size_t)i * V + n] + Gt[(size_t)n * V + i];
            if (m->flags[0] && fabs(proj) > 2) proj = proj > 0 ? 2 : -2;
            double f = -m->kappa[k] * proj * m->flavors;
            if (m->flags[3]) f *= exp(-logdet);
            p_dot[((size_t)t * V + i) * 3 + k] = f;
        }
    }
}

/* construct_M_hat + logDetM_and_inv_M_hat + force, the body of leap_frog
   (simulation/organic_hmc.c:177-180); flags other than none are not restated. */
double or_eval_reference(const or_model *m, const double *x, double *p_dot, double *M_inv_out, int *sign_out) {
    const unsigned V = m->ns, nt = m->nt;
    const size_t md = (size_t)V * V;
    double *M = malloc(sizeof(double) * md);
    double *G = malloc(sizeof(double) * md * nt);
    or_construct_M_hat(m, x, M);
    const double logdet = or_logdet_inverse(M, V, sign_out);
    if (M_inv_out) memcpy(M_inv_out, M, sizeof(double) * md);
    or_all_G(m, x, M, G);
    for (unsigned t = 0; t < nt; t++) {
        or_refine(m, x, G + t * md, t);
        or_contract(m, G + t * md, t, logdet, p_dot);
    }
    free(M);
    free(G);
    return logdet;
}

/* ------------------------------------------------------------ adjoint (same math, O(Nt)) */
/* Same quantities as or_eval_reference by reverse-mode accumulation instead of
   explicit G_t matrices.  With q_c(t) = Q_t e_c (Q_t = B_{t+1}..B_{Nt-1}) and
   y_c(t) = P_t^T M^-T e_c (P_t = B_0..B_{t-1}):  G_t = sum_c q_c y_c^T, and
   with B = f_1 f_0 the refined matrix is
     D = sum_c (a0 q + b0 Hq)(f1 y)^T + b0 q (H f1 y)^T
             + (a1 f0q + b1 H f0q) y^T + b1 (f0 q)(H y)^T,
   whose link entries give the force exactly as or_contract.  Rows of the
   working matrices are the vectors q_c, y_c (index c).  Used by the tests to
   pin the GPU adjoint and, with single != 0, to model its float rounding. */
static void round_float(double *a, size_t n) {
    for (size_t i = 0; i < n; i++) a[i] = (double)(float)a[i];
}

static void or_apply_pair_M(const or_model *m, const double *xs, double *M, double *H1, double *H2, int p) {
    /* M <- f_p M (rows); H1 <- H M_in, H2 <- H (H M_in) on the same rows */
    const unsigned V = m->ns;
    double al[OR_NPAIRS], aq[OR_NPAIRS];
    int cx[OR_NPAIRS];
    or_pair_coeffs(al, aq, cx);
#pragma omp parallel for
    for (unsigned r = 0; r < V; r++) {
        double *v = M + (size_t)r * V, *h1 = H1 + (size_t)r * V, *h2 = H2 + (size_t)r * V;
        or_apply_mu_K_v(m, xs, v, h1);
        or_apply_mu_K_v(m, xs, h1, h2);
        for (unsigned i = 0; i < V; i++) v[i] += al[p] * h1[i] + aq[p] * h2[i];
    }
}

static void or_apply_H_M(const or_model *m, const double *xs, const double *M, double *out) {
    const unsigned V = m->ns;
#pragma omp parallel for
    for (unsigned r = 0; r < V; r++) or_apply_mu_K_v(m, xs, M + (size_t)r * V, out + (size_t)r * V);
}

double or_eval_adjoint(const or_model *m, const double *x, double *p_dot, int single) {
    const unsigned V = m->ns, nt = m->nt;
    const size_t md = (size_t)V * V, ld = (size_t)V * 3;
    double al[OR_NPAIRS], aq[OR_NPAIRS];
    int cx[OR_NPAIRS];
    or_pair_coeffs(al, aq, cx);
    double *qs = malloc(sizeof(double) * md * nt); /* q(t) rows, t = 0..nt-1 */
    double *M = malloc(sizeof(double) * md);
    double *h1 = malloc(sizeof(double) * md), *h2 = malloc(sizeof(double) * md);
    /* sweep 1: q(nt-1) = I, q(t-1) = f1 f0 q(t); q(-1) rows are M_hat - 1 */
    or_identity(M, V);
    for (int tau = (int)nt - 1; tau >= 0; tau--) {
        memcpy(qs + (size_t)tau * md, M, sizeof(double) * md);
        or_apply_pair_M(m, x + tau * ld, M, h1, h2, 0);
        or_apply_pair_M(m, x + tau * ld, M, h1, h2, 1);
    }
    if (!m->flags[1] && !m->flags[3])
        for (unsigned i = 0; i < V; i++) M[(size_t)i * (V + 1)] += 1;
    int sign;
    const double logdet = or_logdet_inverse(M, V, &sign);
    /* y(0) rows = rows of M^-1 (math) = columns of the inverse's memory */
    double *y = malloc(sizeof(double) * md), *yn = malloc(sizeof(double) * md);
    for (unsigned r = 0; r < V; r++)
        for (unsigned c = 0; c < V; c++) y[(size_t)r * V + c] = M[(size_t)c * V + r];
    if (single) { round_float(qs, md * nt); round_float(y, md); }
    double *f0q = malloc(sizeof(double) * md), *hq = malloc(sizeof(double) * md);
    double *hf0q = malloc(sizeof(double) * md), *hy = malloc(sizeof(double) * md);
    double *f1y = malloc(sizeof(double) * md), *hf1y = malloc(sizeof(double) * md);
    for (unsigned t = 0; t < nt; t++) {
        const double *xs = x + t * ld;
        const double *q = qs + (size_t)t * md;
        memcpy(f0q, q, sizeof(double) * md);
        or_apply_pair_M(m, xs, f0q, hq, h2, 0);   /* hq = H q, f0q = f0 q */
        or_apply_H_M(m, xs, f0q, hf0q);            /* H f0 q */
        memcpy(f1y, y, sizeof(double) * md);
        or_apply_pair_M(m, xs, f1y, hy, h2, 1);   /* hy = H y, f1y = f1 y */
        memcpy(yn, f1y, sizeof(double) * md);
        or_apply_pair_M(m, xs, yn, hf1y, h2, 0);  /* hf1y = H f1 y, yn = f0 f1 y */
        if (single) {
            round_float(f0q, md); round_float(hq, md); round_float(hf0q, md);
            round_float(hy, md); round_float(f1y, md); round_float(hf1y, md); round_float(yn, md);
        }
#pragma omp parallel for
        for (unsigned i = 0; i < V; i++) {
            for (unsigned k = 0; k < 3; k++) {
                const unsigned n = m->nnt[6 * i + 2 * k];
                double d = 0;
                for (unsigned c = 0; c < V; c++) {
                    const size_t o = (size_t)c * V;
                    for (int sw = 0; sw < 2; sw++) {
                        const unsigned a = sw ? n : i, b = sw ? i : n;
                        d += (al[0] * q[o + a] + aq[0] * hq[o + a]) * f1y[o + b]
                           + aq[0] * q[o + a] * hf1y[o + b]
                           + (al[1] * f0q[o + a] + aq[1] * hf0q[o + a]) * y[o + b]
                           + aq[1] * f0q[o + a] * hy[o + b];
                    }
                }
                double f = -m->kappa[k] * d * m->flavors;
                if (m->flags[3]) f *= exp(-logdet);
                p_dot[((size_t)t * V + i) * 3 + k] = f;
            }
        }
        double *sw = y; y = yn; yn = sw;
    }
    free(f0q); free(hq); free(hf0q); free(hy); free(f1y); free(hf1y);
    free(y); free(yn); free(qs); free(M); free(h1); free(h2);
    return logdet;
}

/* ------------------------------------------------------------ action */
/* -flavors logdet + E_p + (sum (x_{t+1}-x_t)^2 / omega + omega sum x^2) / 2,
   periodic in t (hamilton, simulation/organic_hmc.c:67-84). */
double or_hamilton(const double *x, double logdet, double energyP, double omega,
                   unsigned flavors, unsigned ns, unsigned nt) {
    const size_t ld = (size_t)ns * 3;
    double pot = 0, kin = 0;
    for (unsigned t = 0; t < nt; t++) {
        const double *a = x + t * ld, *b = x + ((t + 1) % nt) * ld;
        for (size_t e = 0; e < ld; e++) {
            pot += a[e] * a[e];
            const double d = b[e] - a[e];
            kin += d * d;
        }
    }
    return -logdet * flavors + energyP + (kin / omega + pot * omega) / 2;
}

/* Central finite differences of -flavors*logdet with step eps^(1/3), relative
   error sqrt(sum (F - F_fd)^2 / sum (|F| + |F_fd|)^2)
   (check_force, simulation/organic_hmc.c:20-54). */
double or_check_force(const or_model *m, const double *x_in, const double *p_dot) {
    const unsigned V = m->ns, nt = m->nt;
    const size_t dim = (size_t)nt * V * 3, md = (size_t)V * V;
    const double delta = pow(2.220446049250313e-16, 1. / 3);
    double *x = malloc(sizeof(double) * dim);
    double *M = malloc(sizeof(double) * md);
    memcpy(x, x_in, sizeof(double) * dim);
    double err = 0, nrm = 0;
    for (size_t i = 0; i < dim; i++) {
        const double keep = x[i];
        x[i] = keep + delta;
        or_construct_M_hat(m, x, M);
        const double ep = -or_logdet_inverse(M, V, NULL) * m->flavors;
        x[i] = keep - delta;
        or_construct_M_hat(m, x, M);
        const double em = -or_logdet_inverse(M, V, NULL) * m->flavors;
        const double f = -(ep - em) / (2 * delta);
        err += (p_dot[i] - f) * (p_dot[i] - f);
        nrm += (fabs(p_dot[i]) + fabs(f)) * (fabs(p_dot[i]) + fabs(f));
        x[i] = keep;
    }
    free(x);
    free(M);
    return sqrt(err / nrm);
}

/* ------------------------------------------------------------ Fourier acceleration */
/* Unnormalised real DFT along t of ld interleaved series x[t*ld + e]:
   Xc[(k*ld + e)*2 + {0,1}] = sum_t x[t*ld+e] exp(-2 pi i t k / nt), k <= nt/2
   (the r2c plans of simulation/organic_hmc.c:319-320). */
void or_rdft_forward(const double *x, double *Xc, unsigned ld, unsigned nt) {
    const unsigned nc = nt / 2 + 1;
    for (unsigned k = 0; k < nc; k++) {
        for (unsigned e = 0; e < ld; e++) {
            long double re = 0, im = 0;
            for (unsigned t = 0; t < nt; t++) {
                const long double ang = OR_TWO_PI * (long double)((unsigned long)t * k % nt) / nt;
                re += x[(size_t)t * ld + e] * cosl(ang);
                im -= x[(size_t)t * ld + e] * sinl(ang);
            }
            Xc[((size_t)k * ld + e) * 2] = (double)re;
            Xc[((size_t)k * ld + e) * 2 + 1] = (double)im;
        }
    }
}

/* Inverse (c2r) with Hermitian completion, unnormalised (plans :321-322). */
void or_rdft_inverse(const double *Xc, double *x, unsigned ld, unsigned nt) {
    const unsigned nc = nt / 2 + 1;
    for (unsigned t = 0; t < nt; t++) {
        for (unsigned e = 0; e < ld; e++) {
            long double acc = Xc[e * 2];
            for (unsigned k = 1; k < nc; k++) {
                const long double ang = OR_TWO_PI * (long double)((unsigned long)t * k % nt) / nt;
                const double re = Xc[((size_t)k * ld + e) * 2], im = Xc[((size_t)k * ld + e) * 2 + 1];
                if (2 * k == nt) acc += re * cosl(ang);
                else acc += 2 * (re * cosl(ang) - im * sinl(ang));
            }
            x[(size_t)t * ld + e] = (double)acc;
        }
    }
}

static double or_freq2(double omega, unsigned k, unsigned nt) {
    const double s = 2 * sin(OR_PI / nt * k);
    return omega + s * s / omega;
}

/* Exact harmonic flow for time h per Matsubara mode
   (evolve_bosons, simulation/organic_bosons.c:126-150). */
void or_evolve_bosons(double *x, double *p, double omega, unsigned ns, unsigned nt, double h) {
    const unsigned ld = ns * 3, nc = nt / 2 + 1;
    double *xc = malloc(sizeof(double) * 2 * ld * nc), *pc = malloc(sizeof(double) * 2 * ld * nc);
    or_rdft_forward(x, xc, ld, nt);
    or_rdft_forward(p, pc, ld, nt);
    const double c = cos(h) / nt, s = sin(h) / nt;
    for (unsigned k = 0; k < nc; k++) {
        const double f2 = or_freq2(omega, k, nt);
        const double sw = s * f2, s1w = s / f2;
        for (unsigned e = 0; e < 2 * ld; e++) {
            const size_t o = (size_t)k * 2 * ld + e;
            const double x0 = xc[o], p0 = pc[o];
            xc[o] = c * x0 + s1w * p0;
            pc[o] = c * p0 - sw * x0;
        }
    }
    or_rdft_inverse(xc, x, ld, nt);
    or_rdft_inverse(pc, p, ld, nt);
    free(xc);
    free(pc);
}

/* p ~ N(0,1), scaled per mode by sqrt(freq2)/Nt in Fourier space
   (sample_fourier_momenta, simulation/organic_bosons.c:76-100). */
void or_sample_fourier_momenta(double *p, double omega, unsigned ns, unsigned nt) {
    const unsigned ld = ns * 3, nc = nt / 2 + 1;
    or_normals(p, ld * nt);
    double *pc = malloc(sizeof(double) * 2 * ld * nc);
    or_rdft_forward(p, pc, ld, nt);
    for (unsigned k = 0; k < nc; k++) {
        const double a = sqrt(or_freq2(omega, k, nt)) / nt;
        for (unsigned e = 0; e < 2 * ld; e++) pc[(size_t)k * 2 * ld + e] *= a;
    }
    or_rdft_inverse(pc, p, ld, nt);
    free(pc);
}

/* sum_k |p_k|^2 / (2 Nt freq2_k), interior modes counted twice
   (energy_fourier_momenta, simulation/organic_bosons.c:102-124). */
double or_energy_fourier_momenta(const double *p, double omega, unsigned ns, unsigned nt) {
    const unsigned ld = ns * 3, nc = nt / 2 + 1, center = (nt + 1) / 2;
    double *pc = malloc(sizeof(double) * 2 * ld * nc);
    or_rdft_forward(p, pc, ld, nt);
    double en = 0;
    for (unsigned k = 0; k < nc; k++) {
        double w = .5 / nt / or_freq2(omega, k, nt);
        if (k > 0 && k < center) w *= 2;
        for (unsigned e = 0; e < ld; e++) {
            const double re = pc[((size_t)k * ld + e) * 2], im = pc[((size_t)k * ld + e) * 2 + 1];
            en += (re * re + im * im) * w;
        }
    }
    free(pc);
    return en;
}

/* x from the free-phonon distribution: normals scaled by 1/(sqrt(freq2) Nt)
   per mode (sample_free_bosons, simulation/organic_bosons.c:55-74). */
void or_sample_free_bosons(double *x, double omega, unsigned ns, unsigned nt) {
    const unsigned ld = ns * 3, nc = nt / 2 + 1;
    or_normals(x, ld * nt);
    double *xc = malloc(sizeof(double) * 2 * ld * nc);
    or_rdft_forward(x, xc, ld, nt);
    for (unsigned k = 0; k < nc; k++) {
        const double a = 1. / sqrt(or_freq2(omega, k, nt)) / nt;
        for (unsigned e = 0; e < 2 * ld; e++) xc[(size_t)k * 2 * ld + e] *= a;
    }
    or_rdft_inverse(xc, x, ld, nt);
    free(xc);
}

/* sum over links of sum_t (x_t - mean_t x)^2 (higher_Matsubaras_norm,
   simulation/organic_bosons.c:36-53). */
double or_higher_matsubaras_norm(const double *x, unsigned ns, unsigned nt) {
    const size_t ld = (size_t)ns * 3;
    double acc = 0;
    for (size_t e = 0; e < ld; e++) {
        double mean = 0;
        for (unsigned t = 0; t < nt; t++) mean += x[t * ld + e];
        mean /= (double)nt;
        for (unsigned t = 0; t < nt; t++) {
            const double d = x[t * ld + e] - mean;
            acc += d * d;
        }
    }
    return acc;
}
