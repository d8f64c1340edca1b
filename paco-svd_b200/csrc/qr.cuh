// QR-first reduction of tall matrices (qr.cu): blocked Householder QR with
// the blocks factored on one thread-block cluster, and the formation of
// U = Q blockdiag(U_R, I) after the SVD of R.
#pragma once

#include "bidiag.cuh"

constexpr int QB = 64;  // columns per QR block

// Set-up of the cluster kernel (once per device, outside stream capture).
void qr_init();
// True when the cluster kernel can hold an M-row block of QB columns.
bool qr_fits(int M, int N);
// W of the stage-1 workspace w (M x ldw, holding A) <- R in its upper
// triangle and the Householder vectors below the diagonal; tau[N] the
// scalars.  Enqueued on s.
// qb: columns per block, 64 (QB, also for 0) or 32.
int qr_factor(const BdWs &w, int M, int N, float *tau, cudaStream_t s, int qb = 0);
// QR of one block of nb <= QB columns at column q0 of W (ld ldw), rows
// [q0, M): R on and above the diagonal, the reflectors below it, their
// scalars in tau[0, nb).  PACO_ERR_UNSUPPORTED when the rows do not fit.
// small: a cluster of fewer CTAs (down to one) for panels of few rows.
int qr_panel(float *W, long ldw, int M, int q0, int nb, float *tau, cudaStream_t s, bool small = false);
// R (N x N, ld N) <- the upper triangle of W[0:N, 0:N].
void qr_extract_r_launch(const BdWs &w, int N, float *R, cudaStream_t s);
// U (M x uc, ld uc) <- the first uc columns of Q blockdiag(UR, I) with Q from
// qr_factor and UR N x N (ld N; null: the identity, so U = Q); uc = M (0
// means M), or N for the thin U.
// nbf: reflectors per block update, 128 (NBF, also for 0) or 64.
int qr_form_u(const BdWs &w, int M, int N, const float *tau, const float *UR, float *U, cudaStream_t s, int uc = 0,
              int nbf = 0);
