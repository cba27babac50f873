/*
 * Declaration-only stand-in for <cblas.h>, used ONLY to compile the
 * unmodified reference sources into the test oracle (oracle/_ref).  The
 * definition of cblas_dgemm comes from the OpenBLAS shared library linked by
 * oracle/Makefile.  Prototype per the public CBLAS interface; the reference
 * calls it at simulation/organic_dense_matrix.c:601-602 (Schur branch only).
 */
#ifndef EPHMC_ORACLE_CBLAS_SHIM_H
#define EPHMC_ORACLE_CBLAS_SHIM_H

enum CBLAS_ORDER { CblasRowMajor = 101, CblasColMajor = 102 };
enum CBLAS_TRANSPOSE { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 };

void cblas_dgemm(enum CBLAS_ORDER order, enum CBLAS_TRANSPOSE transa,
                 enum CBLAS_TRANSPOSE transb, int m, int n, int k,
                 double alpha, const double *a, int lda, const double *b,
                 int ldb, double beta, double *c, int ldc);

#endif
