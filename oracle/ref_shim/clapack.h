/* Test-infrastructure shim: prototypes of the two CLAPACK 3.1.1.1 routines
   the reference's weight code calls (my_kriging_weights.h:93,100,200,210).
   Their bodies are the oracle's restatement in oracle/lapack_restated.c. */
#ifndef ORACLE_SHIM_CLAPACK_H
#define ORACLE_SHIM_CLAPACK_H
int dpotrf_(char *uplo, integer *n, doublereal *a, integer *lda, integer *info);
int dpotrs_(char *uplo, integer *n, integer *nrhs, doublereal *a, integer *lda,
            doublereal *b, integer *ldb, integer *info);
#endif
