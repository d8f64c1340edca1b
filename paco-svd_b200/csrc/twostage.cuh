// Two-stage reduction to bidiagonal form (twostage.cu): A -> upper band of
// bandwidth b by blocked Householder QR / LQ panels, band -> bidiagonal by
// bulge chasing on one thread-block cluster, and the back-transformation of
// U and V by the chasing reflectors.
#pragma once

#include "bidiag.cuh"

namespace ts {
// Storage of the chasing reflectors: task (sweep s, step j) at
// ((s * jmax + j) * b) floats, tau first, then v[1..L) (v[0] = 1 implicit).
inline int jmax(int N, int b) { return (N - 2 + b) / b; }  // ceil((N - 1) / b)
inline size_t refl_floats(int N, int b) { return (size_t)N * jmax(N, b) * b; }
inline size_t band_floats(int N, int b) { return (size_t)N * 3 * b; }
}  // namespace ts

// Set-up of the chasing kernel (once per device, outside stream capture).
void ts_init();
// True when the chasing kernel's cluster holds the N x 3b band (b = 32 or 64).
bool ts_fits(int N, int b);
// W of w (M x ldw, holding A) <- the upper band B (bandwidth b) with the QR
// reflectors below the diagonal (tauq) and the LQ reflectors right of the band
// (row r: v[r + b] = 1 implicit, entries from column r + b + 1; taup).
int ts_band_reduce(const BdWs &w, int M, int N, int b, float *tauq, float *taup, cudaStream_t s);
// band (N x 3b) <- B from W; chases B to bidiagonal form: d[N], e[N - 1], the
// left (refl_l) and right (refl_r) reflectors of every task.
int ts_chase(const BdWs &w, int N, int b, float *band, float *refl_l, float *refl_r, float *d, float *e,
             cudaStream_t s);
// Vt (N x N) <- P1^T, P1 = blockdiag(I_b, F) from the LQ reflectors in W; uses
// w.Vtmp and Q (at least (N - b)^2 floats) as scratch.
int ts_form_p1t(const BdWs &w, int N, int b, const float *taup, float *Q, float *Vt, cudaStream_t s);
// X <- the chasing reflectors of refl applied in sweep order: trans = 0: X
// (N x N, ld N) <- G_K ... G_1 X (left, columns independent); trans = 1: the
// first N columns of the ncols x ld matrix X <- X[:, :N] H_1 ... H_K.
int ts_apply(float *X, long ld, int N, int ncols, int trans, int b, const float *refl, DevStatus *st,
             cudaStream_t s);
