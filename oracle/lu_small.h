/*
 * lu_small.h -- TEST INFRASTRUCTURE (oracle). Not part of the product.
 *
 * Small dense LU with partial pivoting and Cholesky, written from the published
 * LAPACK algorithms (dgetf2 + dgetrs for dgesv, dpotf2 + dpotrs for dposv).
 * The reference solver calls LAPACK dgesv on 3x3 systems (dbs.c:282 in
 * semismooth_newton, dbs.c:318 in projected_newton, dbs.c:432 in riglnk) and
 * dposv on bilateral constraints (dbs.c:334,349,399). No LAPACK library is
 * installed here, so both the compiled reference (oracle/_ref) and the C
 * restatement (oracle/) link these routines; that gives them identical
 * rounding on the 3x3 solves.
 */
#ifndef ORC_LU_SMALL_H
#define ORC_LU_SMALL_H

/* Solve A x = b for one right-hand side; A is n x n column-major (lda = n),
 * overwritten by its LU factors; b is overwritten by x. Returns LAPACK's info:
 * 0 on success, k > 0 when U(k,k) is exactly zero (b is then left untouched). */
int orc_dgesv (int n, double *a, int *ipiv, double *b);

/* Cholesky solve of a symmetric positive definite system (upper triangle of A
 * used), LAPACK dposv('U') semantics; returns info as LAPACK does. */
int orc_dposv (int n, double *a, double *b);

#endif
