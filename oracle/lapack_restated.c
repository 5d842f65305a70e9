/*
 * ORACLE — test infrastructure only.  Nothing in the shipped library links
 * or calls this file; it is the checker the GPU results are compared with.
 *
 * CPU restatement of the two LAPACK routines the reference's kriging weights
 * call: DPOTRF('U') and DPOTRS('U') from CLAPACK 3.1.1.1 (reference LAPACK
 * 3.1.1 translated by f2c, linked with CLAPACK's own f2c'd reference BLAS;
 * SConstruct:16-19 links lapack, f2c, tmglib and blas from that tree).
 * CLAPACK is not vendored in the reference, so this is written from the
 * published LAPACK/BLAS algorithms:
 *
 *   DPOTRF: ILAENV gives NB = 64 for DPOTRF, and for N <= NB the routine runs
 *   the unblocked DPOTF2.  DPOTF2 (upper) walks columns j = 1..N:
 *       ajj = A(j,j) - DDOT(j-1, A(1,j), A(1,j))
 *       if ajj <= 0 or ajj is NaN: A(j,j) = ajj, INFO = j, stop
 *       A(j,j) = sqrt(ajj)
 *       A(j,j+1:N) += -1 * A(1:j-1,j+1:N)^T A(1:j-1,j)   (DGEMV 'T', beta 1)
 *       A(j,j+1:N) *= (1 / ajj)                          (DSCAL)
 *   Reference DDOT and DGEMV accumulate their dot products left to right from
 *   0; DSCAL multiplies by the precomputed reciprocal.
 *
 *   DPOTRS (upper): DTRSM('L','U','T','N') then DTRSM('L','U','N','N').
 *   The transposed solve is the dot-product form
 *       x_i = (b_i - sum_{k<i} A(k,i) x_k) / A(i,i)   (k ascending),
 *   the non-transposed one is the column (axpy) form
 *       for k = N..1: if b_k != 0: b_k /= A(k,k); b_i -= b_k A(i,k), i < k.
 *
 * Only N <= 64 is restated; larger N (the blocked DPOTRF path) returns
 * INFO = -1000.  Build with -ffp-contract=off so that every a*b+c stays two
 * roundings, as in the f2c'd C.
 */
#include <math.h>
#include <stdio.h>

#define A_(i, j) a[(i) + (long)(j) * lda]

int oracle_dpotf2_upper(int n, double *a, int lda)
{
    for (int j = 0; j < n; ++j) {
        double dot = 0.0;
        for (int i = 0; i < j; ++i) dot = dot + A_(i, j) * A_(i, j);
        double ajj = A_(j, j) - dot;
        if (ajj <= 0.0 || ajj != ajj) {
            A_(j, j) = ajj;
            return j + 1;
        }
        ajj = sqrt(ajj);
        A_(j, j) = ajj;
        if (j < n - 1) {
            if (j > 0) {
                for (int k = j + 1; k < n; ++k) {
                    double temp = 0.0;
                    for (int i = 0; i < j; ++i) temp = temp + A_(i, k) * A_(i, j);
                    A_(j, k) = A_(j, k) + (-1.0 * temp);
                }
            }
            double r = 1.0 / ajj;
            for (int k = j + 1; k < n; ++k) A_(j, k) = r * A_(j, k);
        }
    }
    return 0;
}

void oracle_dpotrs_upper(int n, int nrhs, const double *a, int lda, double *b, int ldb)
{
    if (n == 0 || nrhs == 0) return;
    for (int c = 0; c < nrhs; ++c) {
        double *x = b + (long)c * ldb;
        for (int i = 0; i < n; ++i) {
            double temp = x[i];
            for (int k = 0; k < i; ++k) temp = temp - A_(k, i) * x[k];
            temp = temp / A_(i, i);
            x[i] = temp;
        }
        for (int k = n - 1; k >= 0; --k) {
            if (x[k] != 0.0) {
                x[k] = x[k] / A_(k, k);
                for (int i = 0; i < k; ++i) x[i] = x[i] - x[k] * A_(i, k);
            }
        }
    }
}

/* Fortran-ABI entry points with the CLAPACK signatures, for building the
   reference's own sources (my_kriging_weights.h:93,100,200,210-211). */
int dpotrf_(char *uplo, int *n, double *a, int *lda, int *info)
{
    if (!(*uplo == 'U' || *uplo == 'u')) { *info = -1; return 0; }
    if (*n < 0) { *info = -2; return 0; }
    if (*n > 64) {
        fprintf(stderr, "oracle dpotrf_: N=%d > 64 is not restated\n", *n);
        *info = -1000;
        return 0;
    }
    *info = oracle_dpotf2_upper(*n, a, *lda);
    return 0;
}

int dpotrs_(char *uplo, int *n, int *nrhs, double *a, int *lda, double *b, int *ldb, int *info)
{
    *info = 0;
    if (!(*uplo == 'U' || *uplo == 'u')) { *info = -1; return 0; }
    if (*n < 0) { *info = -2; return 0; }
    if (*nrhs < 0) { *info = -3; return 0; }
    oracle_dpotrs_upper(*n, *nrhs, a, *lda, b, *ldb);
    return 0;
}
