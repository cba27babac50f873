/*
 * Declaration-only stand-in for <lapacke.h>, used ONLY to compile the
 * unmodified reference sources into the test oracle (oracle/_ref).  The
 * definitions come from an OpenBLAS shared library that exports the standard
 * LAPACKE symbols (see oracle/Makefile).  Prototypes follow the public
 * LAPACKE C interface (LAPACK 3.x); only the routines the reference calls
 * are declared:
 *   dgetrf / dgetri  simulation/organic_dense_matrix.c:580,595
 *   dgees            simulation/organic_dense_matrix.c:560
 *   dsyev            simulation/organic_trans_loc.c:40
 * This file is test infrastructure, not part of the shipped library.
 */
#ifndef EPHMC_ORACLE_LAPACKE_SHIM_H
#define EPHMC_ORACLE_LAPACKE_SHIM_H

#define LAPACK_ROW_MAJOR 101
#define LAPACK_COL_MAJOR 102

typedef int lapack_int;
typedef int lapack_logical;
typedef lapack_logical (*LAPACK_D_SELECT2)(const double *, const double *);

lapack_int LAPACKE_dgetrf(int matrix_layout, lapack_int m, lapack_int n,
                          double *a, lapack_int lda, lapack_int *ipiv);
lapack_int LAPACKE_dgetri(int matrix_layout, lapack_int n, double *a,
                          lapack_int lda, const lapack_int *ipiv);
lapack_int LAPACKE_dgees(int matrix_layout, char jobvs, char sort,
                         LAPACK_D_SELECT2 select, lapack_int n, double *a,
                         lapack_int lda, lapack_int *sdim, double *wr,
                         double *wi, double *vs, lapack_int ldvs);
lapack_int LAPACKE_dsyev(int matrix_layout, char jobz, char uplo,
                         lapack_int n, double *a, lapack_int lda, double *w);

#endif
