/*
 * paco_oracle.h -- TEST INFRASTRUCTURE ONLY (the parity checker).
 *
 * CPU restatement, in FP64, of the paco-svd hot path:
 *   stage 1: one-sided Golub-Kahan Householder upper bidiagonalization
 *            (upper_bidiagonalization.cpp:83-120, 182-218, 426-563, 774-893)
 *   stage 2: bidiagonal divide-and-conquer with 3-column leaves and
 *            bottom-up pairwise merges (svd.cpp:134-195, 225-975, 977-1596,
 *            1596-1864, 1866-1981; leaf partition svd_tiling.cpp:83-130).
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg may
 * load this library, and only as the checker: the product path is the CUDA
 * library under paco-svd_b200/ and never calls into the oracle.
 *
 * Parity is pinned against LAPACK (dgesdd sigma, dgebrd |d|,|e|, dlasd4
 * roots) through golden fixtures generated by tests/golden/make_golden.py.
 */
#ifndef PACO_ORACLE_H
#define PACO_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Leaf partition of an N-column bidiagonal, as svd_tiling.cpp:83-130 builds it
 * (leaves of 3 columns, remainder cases for N%3).  Returns the leaf count;
 * starts/ends must hold N/3+1 entries.  N<=2 gives the single leaf [0,N). */
int oracle_leaf_partition(int N, int *starts, int *ends);

/* Stage 1.  A (M x N row-major, in/out) is overwritten with the Householder
 * vectors; d[N], e[N-1], tauq[N], taup[N-1] are written; U (M x M) and
 * Vt (N x N) are formed explicitly, so that A_in = U * B * Vt. */
int oracle_bidiag(int M, int N, double *A, double *U, double *Vt,
                  double *d, double *e, double *tauq, double *taup);

/* Stage 2.  d[N] (in: diagonal, out: sigma descending), e[N-1] (consumed),
 * U (M x M, in/out: first N columns are rotated), Vt (N x N, in/out).
 * stats (optional, 4 ints): [0]=merges, [1]=total deflated, [2]=max secular
 * iterations, [3]=secular non-convergence count. */
int oracle_bdc(int M, int N, double *d, double *e, double *U, double *Vt, int *stats);

/* Both stages on an FP32 input (what the reference's svd_main runs). */
int oracle_svd(int M, int N, const float *A, double *sigma, double *U, double *Vt);

/* One secular-equation root (the solver used inside oracle_bdc):
 * dsig[0..k-1] ascending with dsig[0]=0 < dsig[1] < ..., z[0..k-1].
 * Root i lies in (dsig[i], dsig[i+1]) (or above dsig[k-1] for i=k-1).
 * Writes sigma_i and diff[j] = dsig[j]^2 - sigma_i^2 (j<k).  Returns the
 * iteration count, or -1 if the iteration limit was reached. */
int oracle_secular_root(int k, const double *dsig, const double *z, int i,
                        double *sigma, double *diff);

#ifdef __cplusplus
}
#endif
#endif
