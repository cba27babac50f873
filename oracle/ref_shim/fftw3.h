/*
 * Stand-in for the subset of the FFTW3 API that the reference uses, so that
 * its unmodified sources compile into the test oracle (oracle/_ref).  FFTW3
 * itself is not installed in this image.  The implementation
 * (oracle/ref_shim/fftw_subset.c) is a plain O(n^2) real DFT with FFTW's
 * documented conventions: unnormalised transforms, r2c writes n/2+1 outputs,
 * c2r reads n/2+1 inputs and assumes Hermitian symmetry, strided "many"
 * layout with stride/dist as given.  Used at simulation/organic_hmc.c:317-322
 * and simulation/organic_bosons.c:66-177.
 *
 * fftw_complex follows FFTW's own rule: it is the C99 complex type when
 * <complex.h> was included first, otherwise double[2].
 */
#ifndef EPHMC_ORACLE_FFTW3_SHIM_H
#define EPHMC_ORACLE_FFTW3_SHIM_H

#include <stddef.h>

#if defined(complex) && defined(I)
typedef double _Complex fftw_complex;
#else
typedef double fftw_complex[2];
#endif

typedef struct fftw_plan_s *fftw_plan;

#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)

fftw_plan fftw_plan_many_dft_r2c(int rank, const int *n, int howmany,
                                 double *in, const int *inembed, int istride,
                                 int idist, fftw_complex *out,
                                 const int *onembed, int ostride, int odist,
                                 unsigned flags);
fftw_plan fftw_plan_many_dft_c2r(int rank, const int *n, int howmany,
                                 fftw_complex *in, const int *inembed,
                                 int istride, int idist, double *out,
                                 const int *onembed, int ostride, int odist,
                                 unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);
void *fftw_malloc(size_t n);
void fftw_free(void *p);

#endif
