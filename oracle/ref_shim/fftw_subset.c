/*
 * Minimal real DFT implementing the FFTW3 calls the reference makes, for the
 * test oracle only (oracle/_ref).  FFTW3 is not installed in this image.
 *
 * Conventions (FFTW3 manual, "What FFTW Really Computes"):
 *   r2c:  Y[k] = sum_{j<n} X[j] exp(-2 pi i j k / n),  k = 0..n/2
 *   c2r:  X[j] = sum_{k<n} Y[k] exp(+2 pi i j k / n),  with Y[n-k] = conj Y[k]
 *         (imaginary parts of Y[0] and, for even n, Y[n/2] are ignored)
 * Both unnormalised; "many" layout: element j of transform b sits at
 * in[b*idist + j*istride].  Plans bind their buffers at creation, exactly as
 * the reference relies on (simulation/organic_hmc.c:319-322).
 *
 * Twiddles are computed from (j*k mod n) so their error does not grow with j*k.
 * Long double accumulation keeps the O(n^2) sums at double accuracy.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "fftw3.h"

struct fftw_plan_s {
    int kind; /* 0 = r2c, 1 = c2r */
    int n, howmany, istride, idist, ostride, odist;
    double *rbuf;   /* real side */
    double *cbuf;   /* complex side, interleaved re/im */
    double *cosv, *sinv; /* n twiddles */
};

static struct fftw_plan_s *make_plan(int kind, int n, int howmany, int istride,
                                     int idist, int ostride, int odist) {
    struct fftw_plan_s *p = calloc(1, sizeof(*p));
    p->kind = kind;
    p->n = n;
    p->howmany = howmany;
    p->istride = istride;
    p->idist = idist;
    p->ostride = ostride;
    p->odist = odist;
    p->cosv = malloc(sizeof(double) * (size_t)n);
    p->sinv = malloc(sizeof(double) * (size_t)n);
    for (int m = 0; m < n; m++) {
        const long double ang = 2.0L * 3.14159265358979323846264338327950288L * (long double)m / (long double)n;
        p->cosv[m] = (double)cosl(ang);
        p->sinv[m] = (double)sinl(ang);
    }
    return p;
}

fftw_plan fftw_plan_many_dft_r2c(int rank, const int *n, int howmany, double *in,
                                 const int *inembed, int istride, int idist,
                                 fftw_complex *out, const int *onembed,
                                 int ostride, int odist, unsigned flags) {
    (void)inembed; (void)onembed; (void)flags;
    if (rank != 1) return NULL;
    struct fftw_plan_s *p = make_plan(0, n[0], howmany, istride, idist, ostride, odist);
    p->rbuf = in;
    p->cbuf = (double *)out;
    return p;
}

fftw_plan fftw_plan_many_dft_c2r(int rank, const int *n, int howmany,
                                 fftw_complex *in, const int *inembed,
                                 int istride, int idist, double *out,
                                 const int *onembed, int ostride, int odist,
                                 unsigned flags) {
    (void)inembed; (void)onembed; (void)flags;
    if (rank != 1) return NULL;
    struct fftw_plan_s *p = make_plan(1, n[0], howmany, istride, idist, ostride, odist);
    p->cbuf = (double *)in;
    p->rbuf = out;
    return p;
}

static void exec_r2c(const struct fftw_plan_s *p) {
    const int n = p->n, nc = n / 2 + 1;
    double *tmp = malloc(sizeof(double) * (size_t)n);
    for (int b = 0; b < p->howmany; b++) {
        const double *x = p->rbuf + (size_t)b * p->idist;
        double *y = p->cbuf + 2 * (size_t)b * p->odist;
        for (int j = 0; j < n; j++) tmp[j] = x[(size_t)j * p->istride];
        for (int k = 0; k < nc; k++) {
            long double re = 0, im = 0;
            for (int j = 0; j < n; j++) {
                const int m = (int)(((long)j * k) % n);
                re += (long double)tmp[j] * p->cosv[m];
                im -= (long double)tmp[j] * p->sinv[m];
            }
            y[2 * (size_t)k * p->ostride] = (double)re;
            y[2 * (size_t)k * p->ostride + 1] = (double)im;
        }
    }
    free(tmp);
}

static void exec_c2r(const struct fftw_plan_s *p) {
    const int n = p->n, nc = n / 2 + 1;
    double *re_in = malloc(sizeof(double) * (size_t)nc);
    double *im_in = malloc(sizeof(double) * (size_t)nc);
    for (int b = 0; b < p->howmany; b++) {
        const double *y = p->cbuf + 2 * (size_t)b * p->idist;
        double *x = p->rbuf + (size_t)b * p->odist;
        for (int k = 0; k < nc; k++) {
            re_in[k] = y[2 * (size_t)k * p->istride];
            im_in[k] = y[2 * (size_t)k * p->istride + 1];
        }
        for (int j = 0; j < n; j++) {
            long double acc = re_in[0];
            for (int k = 1; k < nc; k++) {
                const int m = (int)(((long)j * k) % n);
                const long double term = (long double)re_in[k] * p->cosv[m] - (long double)im_in[k] * p->sinv[m];
                /* interior modes appear twice (k and n-k); Nyquist once */
                acc += (2 * k == n) ? term : 2 * term;
            }
            if (n % 2 == 0) {
                /* Nyquist imaginary part is ignored by definition; the loop
                 * above used only re*cos there, and sin(pi j) == 0 exactly
                 * in the twiddle table up to rounding: recompute exactly. */
                const int k = n / 2;
                const int m = (int)(((long)j * k) % n);
                acc -= (long double)re_in[k] * p->cosv[m] - (long double)im_in[k] * p->sinv[m];
                acc += (j % 2 ? -1.0L : 1.0L) * re_in[k];
            }
            x[(size_t)j * p->ostride] = (double)acc;
        }
    }
    free(re_in);
    free(im_in);
}

void fftw_execute(const fftw_plan p) {
    if (!p) return;
    if (p->kind == 0) exec_r2c(p);
    else exec_c2r(p);
}

void fftw_destroy_plan(fftw_plan p) {
    if (!p) return;
    free(p->cosv);
    free(p->sinv);
    free(p);
}

void *fftw_malloc(size_t n) { return malloc(n); }

void fftw_free(void *p) { free(p); }
