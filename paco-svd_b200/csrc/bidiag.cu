// Stage 1: one-sided Golub-Kahan Householder upper bidiagonalization of a
// row-major M x N FP32 matrix (M >= N), blocked in panels of NB columns,
// followed by the explicit formation of U (M x M) and Vt (N x N).
//
// Reference: upper_bidiagonalization.cpp (DEAVEN-MITCH/paco-svd).  The
// reflector convention is the reference's (:182-218): sigma = |x[1:]|^2,
// mu = +sqrt(x0^2 + sigma), v0 = x0 - mu (x0 <= 0) else -sigma/(x0 + mu),
// tau = 2 v0^2/(sigma + v0^2), v = x/v0 with v[0] = 1 implicit, d or e = mu;
// sigma == 0 (or a length-1 vector) gives tau = 0 and keeps x.  The
// reference applies each reflector to the whole trailing matrix at once
// (:426-563, two read+write sweeps per column step); here the updates are
// deferred within a panel (A <- A - V Y^T - X U^T, dlabrd-style blocking), so
// each column step only reads the trailing matrix:
//
//   row pass (RP, row-parallel)  one TMA-staged read of every trailing row
//       finishes X(:, i-1) = taup*(A u - corrections)   [previous row reflector]
//       updates column i and accumulates A^T x          [this column reflector]
//       -- the two GEMVs of a step share that single read.
//   column pass (CP, column-parallel)
//       reduces the A^T x partials into Y(:, i), updates row i, and
//       accumulates the row reflector's norm and panel dot products.
//
// Cross-block reductions (norms, panel dots) are finished by the last block
// to arrive (ticket counter), summing the per-block partials in block order,
// so results are bitwise reproducible.  After each panel one GEMM applies
// the rank-2*NB update to the trailing matrix.
#include <cstdlib>
#include <vector>

#include "bidiag.cuh"
#include "gemm.cuh"
#include "qr.cuh"
#include "tma.cuh"

using namespace bd;

// ------------------------------------------------------------ small kernels

__global__ void bd_copy_in(const float *__restrict__ a, float *__restrict__ W, int M, int N, long ldw,
                           DevStatus *st)
{
    long total = (long)M * ldw;
    bool bad = false;
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < total; t += (long)gridDim.x * blockDim.x) {
        long r = t / ldw, c = t % ldw;
        float v = 0.f;
        if (c < N) {
            v = a[r * N + c];
            if (!isfinite(v)) { // reported, and replaced so every later step stays finite
                bad = true;
                v = 0.f;
            }
        }
        W[t] = v;
    }
    if (bad) dev_fail(st, PACO_ERR_NONFINITE, 0);
}

// a <- Householder vectors with d on the diagonal and e on the superdiagonal
__global__ void bd_copy_out(float *__restrict__ a, const float *__restrict__ W, int M, int N, long ldw,
                            const float *d, const float *e)
{
    long total = (long)M * N;
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < total; t += (long)gridDim.x * blockDim.x) {
        long r = t / N, c = t % N;
        float v = W[r * ldw + c];
        if (r == c) v = d[r];
        else if (c == r + 1) v = e[r];
        a[t] = v;
    }
}

__global__ void bd_set_identity(float *Q, long n, long ld)
{
    long total = n * n;
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < total; t += (long)gridDim.x * blockDim.x) {
        long r = t / n, c = t % n;
        Q[r * ld + c] = (r == c) ? 1.f : 0.f;
    }
}

// Q (rows x cols, ld cols) <- the rows x cols block of the identity
__global__ void bd_set_eye(float *Q, long rows, long cols)
{
    long total = rows * cols;
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < total; t += (long)gridDim.x * blockDim.x)
        Q[t] = (t / cols == t % cols) ? 1.f : 0.f;
}

__global__ void bd_transpose(const float *__restrict__ src, float *__restrict__ dst, int n)
{
    __shared__ float tile[32][33];
    int bx = blockIdx.x * 32, by = blockIdx.y * 32;
    for (int y = threadIdx.y; y < 32; y += blockDim.y) {
        int r = by + y, c = bx + threadIdx.x;
        if (r < n && c < n) tile[y][threadIdx.x] = src[(long)r * n + c];
    }
    __syncthreads();
    for (int y = threadIdx.y; y < 32; y += blockDim.y) {
        int r = bx + y, c = by + threadIdx.x;
        if (r < n && c < n) dst[(long)r * n + c] = tile[threadIdx.x][y];
    }
}

// scales the stored entries of the last column reflector (rows >= N)
__global__ void bd_scale_last_col(float *W, long ldw, int M, int N, const float *inv_v0c)
{
    float s = inv_v0c[N - 1];
    for (int r = N + blockIdx.x * blockDim.x + threadIdx.x; r < M; r += gridDim.x * blockDim.x)
        W[(long)r * ldw + N - 1] *= s;
}

// ------------------------------------------------------------- row pass

// mode bits
#define RP_DO_X 1      // finish X(:, i-1-p0) for the row reflector of row i-1
#define RP_DO_COL 2    // column step i: update column i, accumulate A^T x
#define RP_PANEL_END 4 // materialize the implicit 1 of row i-1 at column i

template <int CPT>
__global__ void __launch_bounds__(RP_THREADS, 1) bd_row_pass(BdArgs a, int i, int p0, int mode, int R)
{
    extern __shared__ __align__(128) float tiles[];
    __shared__ __align__(8) uint64_t bars[2];
    __shared__ float red[RP_THREADS / 32][RMAX];
    __shared__ float xs[RMAX];
    __shared__ float s_t3[NB + 1], s_t4[NB], s_ycol[NB], s_wcol[NB];
    __shared__ float s_part[RMAX][PR];
    __shared__ float s_red[PR];
    __shared__ int s_flag;
    __shared__ float s_v0;

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int M = a.M, N = a.N;
    const long ldw = a.ldw;
    const bool doX = (mode & RP_DO_X) != 0, doCol = (mode & RP_DO_COL) != 0;
    const int ii = i - p0;  // panel columns before column i
    const int iip = ii - 1; // local index of the previous row reflector
    const int L = (int)(ldw - p0);
    const int G = gridDim.x;
    const int nrows = M - i;
    const int rpb = (nrows + G - 1) / G;
    const int r0 = i + blockIdx.x * rpb;
    const int r1 = min(M, r0 + rpb);
    DevStatus *st = a.st;

    // row reflector i-1 (columns i..N-1, implicit 1 at column i)
    const float invr = doX ? a.inv_v0r[i - 1] : 0.f;
    const float taup_prev = doX ? a.taup[i - 1] : 0.f;
    const float invc = (ii >= 1) ? a.inv_v0c[i - 1] : 1.f;

    float4 u4[CPT], acc4[CPT];
#pragma unroll
    for (int k = 0; k < CPT; k++) {
        int c = p0 + 4 * (tid + k * RP_THREADS);
        float uv[4];
#pragma unroll
        for (int e = 0; e < 4; e++) {
            int j = c + e;
            float v = 0.f;
            if (doX) {
                if (j == i) v = 1.f;
                else if (j > i && j < N) v = a.rowbuf[j] * invr;
            }
            uv[e] = v;
        }
        u4[k] = make_float4(uv[0], uv[1], uv[2], uv[3]);
        acc4[k] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    if (tid <= NB) s_t3[tid] = (doX && tid <= iip) ? a.sc->t3[tid] : 0.f;
    if (tid < NB) {
        s_t4[tid] = (doX && tid < iip) ? a.sc->t4[tid] : 0.f;
        s_ycol[tid] = (doCol && tid < ii) ? a.Yt[(long)tid * ldw + i] : 0.f;
        s_wcol[tid] = (doCol && tid < ii) ? ((tid == ii - 1) ? 1.f : a.W[(long)(p0 + tid) * ldw + i]) : 0.f;
    }
    for (int t = tid; t < RMAX * PR; t += RP_THREADS) (&s_part[0][0])[t] = 0.f;

    // block 0 stores the scaled row reflector i-1 into row i-1 of W
    if (doX && blockIdx.x == 0) {
        for (int j = i + 1 + tid; j < N; j += RP_THREADS) a.W[(long)(i - 1) * ldw + j] = a.rowbuf[j] * invr;
        if ((mode & RP_PANEL_END) && tid == 0) a.W[(long)(i - 1) * ldw + i] = 1.f;
    }

    if (tid == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        mbar_init_fence();
    }
    __syncthreads();

    const int nbatch = (r1 > r0) ? (r1 - r0 + R - 1) / R : 0;
    auto issue = [&](int b, int stage) {
        int rb = r0 + b * R;
        int nr = min(R, r1 - rb);
        mbar_expect_tx(&bars[stage], (uint32_t)nr * L * 4u);
        for (int rr = 0; rr < nr; rr++)
            tma_load_1d(tiles + ((long)stage * R + rr) * L, a.W + (long)(rb + rr) * ldw + p0, (uint32_t)L * 4u,
                        &bars[stage]);
    };
    if (tid == 0) {
        if (nbatch > 0) issue(0, 0);
        if (nbatch > 1) issue(1, 1);
    }
    uint32_t phase0 = 0, phase1 = 0;
    float w_ss = 0.f, w_g1 = 0.f, w_g2 = 0.f;
    bool failed = false;

    for (int b = 0; b < nbatch; b++) {
        const int stage = b & 1;
        const int rb = r0 + b * R;
        const int nr = min(R, r1 - rb);
        bool ok = mbar_wait_bounded(&bars[stage], stage ? phase1 : phase0, st, 100 + i);
        if (stage) phase1 ^= 1; else phase0 ^= 1;
        if (__syncthreads_or(!ok)) { failed = true; break; }
        const float *T = tiles + (long)stage * R * L;

        // (1) A u partial dot products, one per staged row
        if (doX) {
            float pd[RMAX];
#pragma unroll
            for (int rr = 0; rr < RMAX; rr++) pd[rr] = 0.f;
#pragma unroll
            for (int rr = 0; rr < RMAX; rr++) {
                if (rr < nr) {
#pragma unroll
                    for (int k = 0; k < CPT; k++) {
                        int c4 = tid + k * RP_THREADS;
                        if (4 * c4 < L) {
                            float4 v = *reinterpret_cast<const float4 *>(T + (long)rr * L + 4 * c4);
                            pd[rr] += v.x * u4[k].x + v.y * u4[k].y + v.z * u4[k].z + v.w * u4[k].w;
                        }
                    }
                }
            }
#pragma unroll
            for (int rr = 0; rr < RMAX; rr++) {
                if (rr < nr) {
                    float v = warp_sum(pd[rr]);
                    if (lane == 0) red[warp][rr] = v;
                }
            }
            __syncthreads();
        }
        // (2) per-row panel work: warp rr handles staged row rr
        if (warp < nr) {
            const int rr = warp, r = rb + rr;
            const float *trow = T + (long)rr * L;
            float aq = (lane < ii) ? trow[lane] : 0.f;
            if (lane == ii - 1) {
                aq *= invc;
                a.W[(long)r * ldw + (i - 1)] = aq;
            }
            float xq = (doX && lane < iip) ? a.X[(long)r * NB + lane] : 0.f;
            float Xn = 0.f;
            if (doX) {
                float dot = 0.f;
#pragma unroll
                for (int w2 = 0; w2 < RP_THREADS / 32; w2++) dot += red[w2][rr];
                float s = ((lane <= iip) ? aq * s_t3[lane] : 0.f) + ((lane < iip) ? xq * s_t4[lane] : 0.f);
                float corr = warp_sum(s);
                Xn = taup_prev * (dot - corr);
                if (lane == 0) a.X[(long)r * NB + iip] = Xn;
            }
            if (doCol) {
                float xrq = (lane < ii - 1) ? xq : ((lane == ii - 1) ? Xn : 0.f);
                float s = (lane < ii) ? (aq * s_ycol[lane] + xrq * s_wcol[lane]) : 0.f;
                float xr = trow[ii] - warp_sum(s);
                if (lane == 0) {
                    a.W[(long)r * ldw + i] = xr;
                    xs[rr] = xr;
                    if (r == i) a.sc->x0col = xr;
                }
                if (r > i) {
                    if (lane == 0) w_ss += xr * xr;
                    if (lane < ii) {
                        w_g1 += aq * xr;
                        w_g2 += xrq * xr;
                    }
                }
            }
        }
        __syncthreads();
        // (3) A^T x accumulation over the staged rows below the pivot
        if (doCol) {
#pragma unroll
            for (int rr = 0; rr < RMAX; rr++) {
                if (rr < nr && rb + rr > i) {
                    float xr = xs[rr];
#pragma unroll
                    for (int k = 0; k < CPT; k++) {
                        int c4 = tid + k * RP_THREADS;
                        if (4 * c4 < L) {
                            float4 v = *reinterpret_cast<const float4 *>(T + (long)rr * L + 4 * c4);
                            acc4[k].x += v.x * xr; acc4[k].y += v.y * xr;
                            acc4[k].z += v.z * xr; acc4[k].w += v.w * xr;
                        }
                    }
                }
            }
        }
        __syncthreads();
        if (tid == 0 && b + 2 < nbatch) {
            proxy_async_fence();
            issue(b + 2, stage);
        }
    }
    if (failed || !doCol) return;

    // block partials: A^T x (all tile columns), |x|^2, panel dots
#pragma unroll
    for (int k = 0; k < CPT; k++) {
        int c4 = tid + k * RP_THREADS;
        if (4 * c4 < L) *reinterpret_cast<float4 *>(a.ypart + (long)blockIdx.x * ldw + p0 + 4 * c4) = acc4[k];
    }
    if (warp < RMAX) {
        if (lane == 0) s_part[warp][0] = w_ss;
        s_part[warp][1 + lane] = w_g1;
        s_part[warp][1 + NB + lane] = w_g2;
    }
    __syncthreads();
    for (int t = tid; t < PR; t += RP_THREADS) {
        float v = 0.f;
        for (int w = 0; w < RMAX; w++) v += s_part[w][t];
        a.tpart[(long)t * PCAP + blockIdx.x] = v;
    }
    if (!last_block_ticket(&st->counters[0], G, &s_flag)) return;

    // last block: finish the column reflector and t1 = V^T v, t2 = X^T v
    {
        reduce_records(a.tpart, G, 1 + 2 * NB, s_red);
        if (tid == 0) {
            float x0 = __ldcg(&a.sc->x0col);
            float beta, tau, v0;
            make_reflector(x0, s_red[0], M - i, &beta, &tau, &v0);
            a.d[i] = beta;
            a.tauq[i] = tau;
            a.inv_v0c[i] = 1.f / v0;
            s_v0 = v0;
        }
        __syncthreads();
        if (tid < ii) {
            float inv = 1.f / s_v0;
            a.sc->t1[tid] = __ldcg(&a.W[(long)i * ldw + p0 + tid]) + s_red[1 + tid] * inv;
            a.sc->t2[tid] = __ldcg(&a.X[(long)i * NB + tid]) + s_red[1 + NB + tid] * inv;
        }
    }
}

// ----------------------------------------------------------- column pass

__global__ void __launch_bounds__(CP_THREADS) bd_col_pass(BdArgs a, int i, int p0, int Gr)
{
    __shared__ float red[CP_THREADS / 32][32];
    __shared__ float sA[CP_THREADS / 32][32], sB[CP_THREADS / 32][32];
    __shared__ float s_t1[NB], s_t2[NB], s_ai[NB], s_xi[NB];
    __shared__ float s_part[PR];
    __shared__ float s_red[PR];
    __shared__ int s_flag;
    __shared__ float s_v0;

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int N = a.N;
    const long ldw = a.ldw;
    const int ii = i - p0;
    const int j = i + 1 + blockIdx.x * 32 + lane;
    const bool valid = j < N;
    DevStatus *st = a.st;

    // (1) sum the row-pass partials of A^T x for this column
    float yv[RB_CAP / (CP_THREADS / 32)];
#pragma unroll
    for (int k = 0; k < RB_CAP / (CP_THREADS / 32); k++) {
        int bb = warp + (CP_THREADS / 32) * k;
        yv[k] = (valid && bb < Gr) ? __ldcg(&a.ypart[(long)bb * ldw + j]) : 0.f;
    }
    float ys = 0.f;
#pragma unroll
    for (int k = 0; k < RB_CAP / (CP_THREADS / 32); k++) ys += yv[k];
    red[warp][lane] = ys;
    for (int t = tid; t < PR; t += CP_THREADS) s_part[t] = 0.f;
    if (tid < NB) {
        bool q = tid < ii;
        s_t1[tid] = q ? a.sc->t1[tid] : 0.f;
        s_t2[tid] = q ? a.sc->t2[tid] : 0.f;
        s_ai[tid] = q ? a.W[(long)i * ldw + p0 + tid] : 0.f;
        s_xi[tid] = q ? a.X[(long)i * NB + tid] : 0.f;
    }
    __syncthreads();

    // (2) warp w owns panel indices q in [4w, 4w+4)
    float Yq[4], Wq[4];
    float pa = 0.f, pb = 0.f;
#pragma unroll
    for (int e = 0; e < 4; e++) {
        int q = 4 * warp + e;
        bool use = valid && q < ii;
        Yq[e] = use ? a.Yt[(long)q * ldw + j] : 0.f;
        Wq[e] = use ? a.W[(long)(p0 + q) * ldw + j] : 0.f;
        if (q < NB) {
            pa += Yq[e] * s_t1[q] + Wq[e] * s_t2[q];
            pb += Yq[e] * s_ai[q] + Wq[e] * s_xi[q];
        }
    }
    sA[warp][lane] = pa;
    sB[warp][lane] = pb;
    __syncthreads();

    // (3) Y(j, ii) and the updated row entry a_j (every warp, same values)
    float y = 0.f, sa = 0.f, sb = 0.f;
#pragma unroll
    for (int w = 0; w < CP_THREADS / 32; w++) { y += red[w][lane]; sa += sA[w][lane]; sb += sB[w][lane]; }
    float Ynew = 0.f, aj = 0.f;
    if (valid) {
        float wij = a.W[(long)i * ldw + j];
        float yj = wij + y * a.inv_v0c[i];
        Ynew = a.tauq[i] * (yj - sa);
        aj = wij - Ynew - sb;
        if (warp == 0) {
            a.Yt[(long)ii * ldw + j] = Ynew;
            a.rowbuf[j] = aj;
            if (j == i + 1) a.sc->x0row = aj;
        }
    }
    // (4) partials of the row reflector: |a|^2, Y^T a, U a (entries j >= i+2)
    float m = (valid && j >= i + 2) ? aj : 0.f;
#pragma unroll
    for (int e = 0; e < 4; e++) {
        int q = 4 * warp + e;
        if (q < ii) {
            float g3 = warp_sum(Yq[e] * m);
            float g4 = warp_sum(Wq[e] * m);
            if (lane == 0) { s_part[1 + q] = g3; s_part[NB + 2 + q] = g4; }
        }
    }
    if (warp == 0) {
        float ss = warp_sum(m * m);
        float g3 = warp_sum(Ynew * m);
        if (lane == 0) { s_part[0] = ss; s_part[1 + ii] = g3; }
    }
    __syncthreads();
    for (int t = tid; t < PR; t += CP_THREADS) a.cpart[(long)t * PCAP + blockIdx.x] = s_part[t];
    if (!last_block_ticket(&st->counters[1], gridDim.x, &s_flag)) return;

    // last block: row reflector of row i and t3 = Y^T u, t4 = U u
    {
        reduce_records(a.cpart, gridDim.x, 2 * NB + 2, s_red);
        if (tid == 0) {
            float x0 = __ldcg(&a.sc->x0row);
            float beta, tau, v0;
            make_reflector(x0, s_red[0], N - i - 1, &beta, &tau, &v0);
            a.e[i] = beta;
            a.taup[i] = tau;
            a.inv_v0r[i] = 1.f / v0;
            s_v0 = v0;
        }
        __syncthreads();
        float inv = 1.f / s_v0;
        if (tid <= ii) a.sc->t3[tid] = __ldcg(&a.Yt[(long)tid * ldw + i + 1]) + s_red[1 + tid] * inv;
        if (tid < ii) a.sc->t4[tid] = __ldcg(&a.W[(long)(p0 + tid) * ldw + i + 1]) + s_red[NB + 2 + tid] * inv;
    }
}

// ---------------------------------------------- compact-WY formation of U, V

// Vp (Lp x NBF, ld NBF): explicit block of nbp reflectors with unit diagonal.
//   column reflectors (U): Vp[r][q] = W[p0+r][p0+q]        (r > q)
//   row reflectors    (V): Vp[r][q] = W[p0+q][p0+1+r]      (r > q)
__global__ void bd_panel_vectors(const float *W, long ldw, int p0, int nbp, int Lp, int rowref, float *Vp)
{
    long total = (long)Lp * NBF;
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < total; t += (long)gridDim.x * blockDim.x) {
        int r = (int)(t / NBF), q = (int)(t % NBF);
        float v = 0.f;
        if (q < nbp) {
            if (r == q) v = 1.f;
            else if (r > q) v = rowref ? W[(long)(p0 + q) * ldw + p0 + 1 + r] : W[(long)(p0 + r) * ldw + p0 + q];
        }
        Vp[t] = v;
    }
}

// T (NBF x NBF, upper triangular) of the forward block reflector
// H_0 ... H_{nbp-1} = I - Vp T Vp^T, from the Gram matrix G = Vp^T Vp:
//   T[q][q] = tau_q,  T[0:q, q] = -tau_q T[0:q, 0:q] G[0:q, q]
// (the recurrence of LAPACK's larft).  Row r of T only needs its own earlier
// entries and G, so every row is computed independently: one warp per row
// (8 rows per CTA), lane l holding T[r][l + 32 j], each new entry a warp dot
// product against column q of G, read as row q (G is symmetric, and the
// GEMM that forms it computes both halves with the same summation order).
// The rows of G a CTA reads are staged in shared memory first.
__global__ void __launch_bounds__(256) bd_build_t(const float *gram, int nbp, const float *tau, float *T)
{
    extern __shared__ float sm_t[];  // rows r0 .. nbp-1 of G
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int r0 = blockIdx.x * 8;
    const int r = r0 + warp;
    for (int t = threadIdx.x; t < (nbp - r0) * NBF; t += blockDim.x)
        sm_t[t] = gram[(long)r0 * NBF + t];
    __syncthreads();
    constexpr int J = NBF / 32;
    float t[J];
#pragma unroll
    for (int j = 0; j < J; j++) t[j] = 0.f;
    if (r < nbp) {
        const float tr = tau[r];
#pragma unroll
        for (int j = 0; j < J; j++)
            if (lane + 32 * j == r) t[j] = tr;
        for (int q = r + 1; q < nbp; q++) {
            const float *g = sm_t + (long)(q - r0) * NBF;
            float p = 0.f;
#pragma unroll
            for (int j = 0; j < J; j++) {
                const int bb = lane + 32 * j;
                if (bb >= r && bb < q) p = fmaf(t[j], g[bb], p);
            }
            p = warp_sum(p);
            const float v = -tau[q] * p;
#pragma unroll
            for (int j = 0; j < J; j++)
                if (lane + 32 * j == q) t[j] = v;
        }
    }
#pragma unroll
    for (int j = 0; j < J; j++) T[(long)r * NBF + lane + 32 * j] = t[j];
}

// Q_sub <- (I - Vp T' Vp^T) Q_sub for Q_sub = Q[ro:ro+Lr, co:co+Lc] (ld ldq),
// T' = T (forward block reflector H_0 ... H_{nbp-1}) or its transpose (the
// transposed product, as a QR factorization applies to its trailing columns).
// Vp (Lr x NBF) must hold the block's reflectors.
cudaError_t apply_block_reflector_ex(const BdWs &w, float *Q, long ldq, long ro, int Lr, long co, int Lc, int nbp,
                                     const float *tau, bool transT, cudaStream_t s)
{
    const int splits = std::max(1, std::min(SPLITS, ceil_div(Lr, 512)));
    // G = Vp^T Vp: one 128 x 128 tile, so the long k = Lr dimension is split
    // finely (64 rows per CTA, as many splits as the partial buffer holds)
    // (the partial buffer holds SPLITS * NBF * max(M, N) >= SPLITS * NBF * ldq floats)
    const int gsplits = (int)std::max(1L, std::min({(long)ceil_div(Lr, 64), 64L, (long)SPLITS * ldq / NBF}));
    cudaError_t err = gemm_run(nbp, nbp, Lr, 1.f, gop(w.Vp, 1, NBF), gop(w.Vp, NBF, 1), 0.f, w.gram, NBF, gsplits,
                               w.gscr, s);
    if (err) return err;
    paco_count_launch(), bd_build_t<<<NBF / 8, 256, (size_t)NBF * NBF * sizeof(float), s>>>(w.gram, nbp, tau, w.T);
    float *Qs = Q + ro * ldq + co;
    // G1 = Vp^T Q_sub  (nbp x Lc)
    err = gemm_any(nbp, Lc, Lr, 1.f, gop(w.Vp, 1, NBF), gop(Qs, ldq, 1), 0.f, w.G1, Lc, splits, w.gscr, w.tcs,
                   w.tcs_floats, w.st, s);
    if (err) return err;
    // G2 = T' G1 (128 x Lc x 128: small, but on the SIMT engine it runs on
    // only Lc / 128 CTAs, so it goes to the tensor cores from Lc = 256 on)
    const GemmOp Top = transT ? gop(w.T, 1, NBF) : gop(w.T, NBF, 1);
    if (w.tcs && gemm_tc_enabled() && Lc >= 256 && gemm_tc_scratch_floats(nbp, Lc, nbp) <= w.tcs_floats)
        err = gemm_tc_run(nbp, Lc, nbp, 1.f, Top, gop(w.G1, Lc, 1), 0.f, w.G2, Lc, w.tcs, w.st, s);
    else
        err = gemm_any(nbp, Lc, nbp, 1.f, Top, gop(w.G1, Lc, 1), 0.f, w.G2, Lc, 1, nullptr, w.tcs, w.tcs_floats,
                       w.st, s);
    if (err) return err;
    // Q_sub -= Vp G2
    return gemm_any(Lr, Lc, nbp, -1.f, gop(w.Vp, NBF, 1), gop(w.G2, Lc, 1), 1.f, Qs, ldq, 1, nullptr, w.tcs,
                    w.tcs_floats, w.st, s);
}

cudaError_t apply_block_reflector_right(const BdWs &w, float *X, long ldx, long ro, int Lr, long co, int Lc, int nbp,
                                        const float *tau, cudaStream_t s)
{
    const int gsplits = (int)std::max(1L, std::min({(long)ceil_div(Lc, 64), 64L, (long)SPLITS * ldx / NBF}));
    cudaError_t err = gemm_run(nbp, nbp, Lc, 1.f, gop(w.Vp, 1, NBF), gop(w.Vp, NBF, 1), 0.f, w.gram, NBF, gsplits,
                               w.gscr, s);
    if (err) return err;
    paco_count_launch(), bd_build_t<<<NBF / 8, 256, (size_t)NBF * NBF * sizeof(float), s>>>(w.gram, nbp, tau, w.T);
    float *Xs = X + ro * ldx + co;
    // G1 = X_sub Vp  (Lr x nbp, k = Lc)
    const int splits = std::max(1, std::min(SPLITS, ceil_div(Lc, 512)));
    err = gemm_any(Lr, nbp, Lc, 1.f, gop(Xs, ldx, 1), gop(w.Vp, NBF, 1), 0.f, w.G1, nbp, splits, w.gscr, w.tcs,
                   w.tcs_floats, w.st, s);
    if (err) return err;
    // G2 = G1 T  (Lr x nbp)
    err = gemm_any(Lr, nbp, nbp, 1.f, gop(w.G1, nbp, 1), gop(w.T, NBF, 1), 0.f, w.G2, nbp, 1, nullptr, w.tcs,
                   w.tcs_floats, w.st, s);
    if (err) return err;
    // X_sub -= G2 Vp^T
    return gemm_any(Lr, Lc, nbp, -1.f, gop(w.G2, nbp, 1), gop(w.Vp, 1, NBF), 1.f, Xs, ldx, 1, nullptr, w.tcs,
                    w.tcs_floats, w.st, s);
}

// Q_sub <- (I - Vp T Vp^T) Q_sub for Q_sub = Q[off:off+Lp, off:off+Lp] (ld ldq)
static cudaError_t apply_block_reflector(const BdWs &w, float *Q, long ldq, long off, int Lp, int nbp,
                                         const float *tau, cudaStream_t s)
{
    return apply_block_reflector_ex(w, Q, ldq, off, Lp, off, Lp, nbp, tau, false, s);
}

// Vp (Lp x NBF) <- the explicit reflectors of column block [p0, p0 + nbp) of W
// (column vectors below the diagonal, unit diagonal)
void bd_column_vectors(const float *W, long ldw, int p0, int nbp, int Lp, float *Vp, cudaStream_t s)
{
    paco_count_launch(), bd_panel_vectors<<<std::min(4096, ceil_div((long)Lp * NBF, 256)), 256, 0, s>>>(
        W, ldw, p0, nbp, Lp, 0, Vp);
}

void bd_copy_in_launch(const float *a, float *W, int M, int N, long ldw, DevStatus *st, cudaStream_t s)
{
    paco_count_launch(), bd_copy_in<<<std::min(4096, ceil_div((long)M * ldw, 256)), 256, 0, s>>>(a, W, M, N, ldw, st);
}

// ------------------------------------------------------------ host driver

size_t bd_workspace_bytes(int M, int N)
{
    BdWs w;
    return bd_carve(nullptr, M, N, &w);
}

static int pick_R(int L)
{
    long budget = 192 * 1024;
    int R = (int)(budget / (2L * L * 4));
    return std::max(1, std::min(RMAX, R));
}

template <int CPT>
static void launch_rp(const BdArgs &a, int i, int p0, int mode, int G, int R, int L, cudaStream_t s)
{
    size_t smem = (size_t)2 * R * L * 4;
    paco_count_launch(), bd_row_pass<CPT><<<G, RP_THREADS, smem, s>>>(a, i, p0, mode, R);
}

static void rp_launch(const BdArgs &a, int i, int p0, int mode, int G, cudaStream_t s);

// ---------------------------------------------------------- kernel timing
// Optional CUDA-event timing of every row-pass launch (the stage's dominant
// kernel), recorded on the launching stream.  The events of one stage-1 run
// form a "run"; a run issued directly is read once, a run captured into a CUDA
// graph is re-recorded by every replay of that graph (read after each replay).
namespace {
struct ProfRun {
    std::vector<cudaEvent_t> ev; // start/end pairs
    std::vector<double> bytes;   // bytes each launch had to read
};
struct RpProfile {
    bool on = false;
    bool capturing = false;
    std::vector<cudaEvent_t> free_ev;
    ProfRun cur;
    std::vector<ProfRun> graph_runs;          // owned by captured graphs
    std::vector<std::pair<int, bool>> pending; // (run id, direct?) awaiting a read
    std::vector<ProfRun> direct_runs;
    double ms = 0, launches = 0, bytes = 0;
    int kind = 0; // dominant stage-1 kernel timed: 0 row pass, 1 persistent panel kernel
} g_prof;

cudaEvent_t prof_event()
{
    if (!g_prof.free_ev.empty()) {
        cudaEvent_t e = g_prof.free_ev.back();
        g_prof.free_ev.pop_back();
        return e;
    }
    cudaEvent_t e;
    cudaEventCreate(&e);
    return e;
}

void prof_record(cudaEvent_t e, cudaStream_t s)
{
    if (g_prof.capturing) cudaEventRecordWithFlags(e, s, cudaEventRecordExternal);
    else cudaEventRecord(e, s);
}
}  // namespace

void bd_profile_enable(int on)
{
    g_prof.on = on != 0;
    g_prof.ms = g_prof.launches = g_prof.bytes = 0;
    for (auto &p : g_prof.pending)
        if (p.second)
            for (cudaEvent_t e : g_prof.direct_runs[p.first].ev) g_prof.free_ev.push_back(e);
    g_prof.pending.clear();
    g_prof.direct_runs.clear();
}

// opens a stage-1 run (called by bd_run)
static void prof_begin(cudaStream_t s)
{
    g_prof.cur = ProfRun();
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaStreamIsCapturing(s, &cs);
    g_prof.capturing = (cs == cudaStreamCaptureStatusActive);
}

// closes the run: a captured run is kept for its graph, a direct run is queued
static void prof_end()
{
    if (!g_prof.on) return;
    if (g_prof.capturing) {
        g_prof.graph_runs.push_back(std::move(g_prof.cur));
    } else {
        g_prof.direct_runs.push_back(std::move(g_prof.cur));
        g_prof.pending.push_back({(int)g_prof.direct_runs.size() - 1, true});
    }
    g_prof.capturing = false;
}

// id of the run captured last (-1 if none), for the graph cache
int bd_profile_last_graph_run() { return (int)g_prof.graph_runs.size() - 1; }

// a replay of a graph holding run `id` was launched
void bd_profile_replayed(int id)
{
    if (g_prof.on && id >= 0) g_prof.pending.push_back({id, false});
}

// totals since the last enable: [0] ms in the timed kernel, [1] launches,
// [2] bytes, [3] which kernel (0 row pass, 1 persistent panel kernel)
void bd_profile_read(double out[4])
{
    for (auto &p : g_prof.pending) {
        ProfRun &r = p.second ? g_prof.direct_runs[p.first] : g_prof.graph_runs[p.first];
        for (size_t t = 0; t + 1 < r.ev.size(); t += 2) {
            float x = 0.f;
            cudaEventSynchronize(r.ev[t + 1]);
            cudaEventElapsedTime(&x, r.ev[t], r.ev[t + 1]);
            g_prof.ms += x;
        }
        for (double v : r.bytes) g_prof.bytes += v;
        g_prof.launches += (double)(r.ev.size() / 2);
        if (p.second) {
            for (cudaEvent_t e : r.ev) g_prof.free_ev.push_back(e);
            r.ev.clear();
        }
    }
    g_prof.pending.clear();
    out[0] = g_prof.ms;
    out[1] = g_prof.launches;
    out[2] = g_prof.bytes;
    out[3] = g_prof.kind;
}

// Bytes one persistent panel launch must read from memory: the live row
// segments [p0, N) of rows [p0, M) once if they stay resident in shared memory,
// else those of rows [i, M) at every step i of the panel (and the X pass).
static double pk_alg_bytes(int M, int N, int p0, int p1, int G, long ldw)
{
    const long L = ldw - p0;
    const long own = (M - p0 + G - 1) / G;
    if (own * L * 4 <= 200L * 1024) return 4.0 * (double)(M - p0) * (double)(N - p0);
    double b = 0;
    const int last = (p1 < N) ? p1 : p1 - 1;
    for (int i = p0; i <= last; i++) b += 4.0 * (double)(M - i) * (double)(N - p0);
    return b;
}

static void rp(const BdArgs &a, int i, int p0, int mode, int G, cudaStream_t s)
{
    const bool prof = g_prof.on;
    if (prof) {
        cudaEvent_t e = prof_event();
        prof_record(e, s);
        g_prof.cur.ev.push_back(e);
        // bytes the pass must read: the live segment [p0, N) of every active row
        g_prof.cur.bytes.push_back(4.0 * (double)(a.M - i) * (double)(a.N - p0));
    }
    rp_launch(a, i, p0, mode, G, s);
    if (prof) {
        cudaEvent_t e = prof_event();
        prof_record(e, s);
        g_prof.cur.ev.push_back(e);
    }
}

static void rp_launch(const BdArgs &a, int i, int p0, int mode, int G, cudaStream_t s)
{
    int L = (int)(a.ldw - p0);
    int R = pick_R(L);
    int chunks = ceil_div(L, 4 * RP_THREADS);
    if (chunks <= 1) launch_rp<1>(a, i, p0, mode, G, R, L, s);
    else if (chunks == 2) launch_rp<2>(a, i, p0, mode, G, R, L, s);
    else launch_rp<4>(a, i, p0, mode, G, R, L, s);
}

static bool rp_attrs_set[PACO_MAX_DEVICES] = {};
void bd_init_attrs()
{
    const int dev = paco_device();
    if (rp_attrs_set[dev]) return;
    int maxs = 200 * 1024;
    cudaFuncSetAttribute(bd_row_pass<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, maxs);
    cudaFuncSetAttribute(bd_row_pass<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, maxs);
    cudaFuncSetAttribute(bd_row_pass<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, maxs);
    cudaFuncSetAttribute(bd_build_t, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(NBF * NBF * sizeof(float)));
    gemm_tc_init_attrs();
    bd_tail_init();
    qr_init();
    bd_fork_events();
    rp_attrs_set[dev] = true;
}

// Stage 1 of k matrices of one shape (jobs[0..k)): set-up, the panels in
// lockstep (one persistent panel launch serves every matrix, G = num_sms / k
// CTAs each; the last columns of every matrix on its own cluster launch, on
// side[j] when k > 1), the trailing updates, the formation of U and V.
int bd_run_multi(int k, const BdJob *jobs, cudaStream_t s0, cudaStream_t *side, int num_sms)
{
    cudaStream_t s = s0;
    if (k < 1 || k > PK_KMAX) return PACO_ERR_INVALID_ARG;
    const int M = jobs[0].M, N = jobs[0].N;
    for (int j = 1; j < k; j++)
        if (jobs[j].M != M || jobs[j].N != N) return PACO_ERR_INVALID_ARG;
    bd_init_attrs();
    const PacoTune tune = paco_tune_for(M, N);
    prof_begin(s);
    // PACO_PK_TRACE=<p0>: phase timestamps of the panel starting at column p0
    static int trace_env = -2;
    if (trace_env == -2) {
        const char *v = getenv("PACO_PK_TRACE");
        trace_env = v ? atoi(v) : -1;
    }
    BdWs w[PK_KMAX];
    BdArgs a[PK_KMAX];
    PkCtl *ctl[PK_KMAX];
    unsigned pk_cnt[PK_KMAX]; // arrivals on each matrix's barrier counter so far
    for (int j = 0; j < k; j++) {
        const BdJob &J = jobs[j];
        bd_carve(J.workspace, M, N, &w[j]);
        if (!tune.tc) w[j].tcs = nullptr;  // the large products stay on the SIMT engine
        BdArgs &x = a[j];
        x.M = M; x.N = N; x.ldw = w[j].ldw; x.st = w[j].st;
        x.W = w[j].W; x.Yt = w[j].Yt; x.X = w[j].X; x.ypart = w[j].ypart; x.tpart = w[j].tpart;
        x.cpart = w[j].cpart; x.rowbuf = w[j].rowbuf; x.inv_v0c = w[j].inv_v0c; x.inv_v0r = w[j].inv_v0r;
        x.sc = w[j].sc;
        x.d = J.d; x.e = J.e; x.tauq = J.tauq; x.taup = J.taup;
        x.bcA = w[j].bcA; x.bcB = w[j].bcB;
        x.trace = (trace_env >= 0 && j == 0) ? w[j].trace : nullptr;
        x.trace_p0 = trace_env;
        ctl[j] = w[j].ctl;
        pk_cnt[j] = 0;
    }

    const int gmax = std::max(1, std::min(RB_CAP, num_sms / k));
    const int rpc = std::max(1, tune.rows_per_cta);
    auto grid_rows = [&](int rows) { return std::max(1, std::min(gmax, ceil_div(rows, rpc))); };
    bd_pk_init_attrs();
    // the persistent panel kernel needs every CTA co-resident (one per SM)
    static int use_pk_env = -1;
    if (use_pk_env < 0) {
        const char *v = getenv("PACO_PERSISTENT");
        use_pk_env = !(v && v[0] == '0');
    }
    const bool use_pk = use_pk_env != 0 && tune.persistent;
    for (int j = 0; j < k; j++) {
        cudaMemsetAsync(w[j].st->counters, 0, sizeof(w[j].st->counters), s);
        cudaMemsetAsync(w[j].ctl, 0, sizeof(PkCtl), s);
        cudaMemsetAsync(w[j].Yt, 0, sizeof(float) * NB * w[j].ldw, s);
        cudaMemsetAsync(w[j].X, 0, sizeof(float) * (size_t)M * NB, s);
        paco_count_launch(), bd_copy_in<<<std::min(4096, ceil_div((long)M * w[j].ldw, 256)), 256, 0, s>>>(
            jobs[j].a_in, w[j].W, M, N, w[j].ldw, w[j].st);
    }
    // fork / join of the side streams (k > 1)
    cudaEvent_t *fe = bd_fork_events();
    auto fork = [&]() {
        cudaEventRecord(fe[0], s);
        for (int j = 0; j < k; j++) cudaStreamWaitEvent(side[j], fe[0], 0);
    };
    auto join = [&]() {
        for (int j = 0; j < k; j++) {
            cudaEventRecord(fe[1 + j], side[j]);
            cudaStreamWaitEvent(s, fe[1 + j], 0);
        }
    };

    // the last columns, once their block fits in a cluster's shared memory,
    // go to the cluster kernel in one launch per matrix
    const int tail_p = (use_pk && !tune.no_tail) ? bd_tail_start(M, N) : N;
    for (int p0 = 0; p0 < N; p0 += NB) {
        if (p0 == tail_p) {
            cudaEvent_t e0 = nullptr, e1 = nullptr;
            if (g_prof.on) prof_record(e0 = prof_event(), s);
            int ran = 0;
            if (k == 1) {
                ran = bd_tail_launch(a[0], p0, s) ? 1 : 0;
            } else {
                fork();
                for (int j = 0; j < k; j++) ran += bd_tail_launch(a[j], p0, side[j]) ? 1 : 0;
                join();
            }
            const bool done = ran == k;
            if (g_prof.on) {
                prof_record(e1 = prof_event(), s);
                g_prof.cur.ev.push_back(e0);
                g_prof.cur.ev.push_back(e1);
                g_prof.cur.bytes.push_back(done ? 4.0 * k * (double)(M - p0) * (double)(N - p0) : 0.0);
            }
            if (done) break;
            // a cluster launch that could not run leaves its matrix untouched, so
            // when none ran the panels simply go on; some but not all cannot
            // happen for one shape unless a launch failed
            if (ran > 0) return PACO_ERR_CUDA;
        }
        const int p1 = std::min(N, p0 + NB), nbp = p1 - p0;
        const int Gp = grid_rows(M - p0);
        bool pk = false;
        if (use_pk) {
            cudaEvent_t e0 = nullptr, e1 = nullptr;
            if (g_prof.on) prof_record(e0 = prof_event(), s);
            pk = bd_panel_pk_launch_multi(k, a, ctl, p0, p1, Gp, pk_cnt, s);
            if (g_prof.on) {
                prof_record(e1 = prof_event(), s);
                g_prof.cur.ev.push_back(e0);
                g_prof.cur.ev.push_back(e1);
                g_prof.cur.bytes.push_back(k * pk_alg_bytes(M, N, p0, p1, Gp, w[0].ldw));
                g_prof.kind = 1;
            }
        }
        for (int j = 0; j < k; j++) {
            if (!pk) {
                for (int i = p0; i < p1; i++) {
                    int G = grid_rows(M - i);
                    int mode = RP_DO_COL | ((i > p0) ? RP_DO_X : 0);
                    rp(a[j], i, p0, mode, G, s);
                    if (i < N - 1)
                        paco_count_launch(), bd_col_pass<<<ceil_div(N - i - 1, 32), CP_THREADS, 0, s>>>(a[j], i, p0, G);
                }
            }
            if (p1 < N) {
                if (!pk) rp(a[j], p1, p0, RP_DO_X | RP_PANEL_END, grid_rows(M - p1), s);
                // A[p1:, p1:] -= [V | X] [Y^T ; U]
                const BdWs &x = w[j];
                GemmOp A = gop(x.W + (long)p1 * x.ldw + p0, x.ldw, 1);
                A.p2 = x.X + (long)p1 * NB; A.rs2 = NB; A.cs2 = 1; A.ksplit = nbp;
                GemmOp B = gop(x.Yt + p1, x.ldw, 1);
                B.p2 = x.W + (long)p0 * x.ldw + p1; B.rs2 = x.ldw; B.cs2 = 1; B.ksplit = nbp;
                gemm_any(M - p1, N - p1, 2 * nbp, -1.f, A, B, 1.f, x.W + (long)p1 * x.ldw + p1, x.ldw, 1, nullptr,
                         x.tcs, x.tcs_floats, x.st, s);
            } else if (M > N) {
                paco_count_launch(), bd_scale_last_col<<<std::min(1024, ceil_div(M - N, 256)), 256, 0, s>>>(
                    w[j].W, w[j].ldw, M, N, w[j].inv_v0c);
            }
        }
    }

    // the formation of U and V (nbf reflectors per block update): each matrix
    // on its own side stream (k > 1)
    const int nbf = tune.wy == 64 ? 64 : NBF;
    if (k > 1) fork();
    for (int j = 0; j < k; j++) {
        const BdWs &x = w[j];
        const BdJob &J = jobs[j];
        cudaStream_t s = (k > 1) ? side[j] : s0;
        // U = H_0 ... H_{N-1} (backward accumulation of the column reflectors,
        // NBF reflectors per block update)
        const int uc = J.thin ? N : M;  // columns of U formed
        paco_count_launch(), bd_set_eye<<<std::min(8192, ceil_div((long)M * uc, 256)), 256, 0, s>>>(J.u, M, uc);
        for (int p0 = ((N - 1) / nbf) * nbf; p0 >= 0; p0 -= nbf) {
            int nbp = std::min(N, p0 + nbf) - p0, Lp = M - p0;
            paco_count_launch(), bd_panel_vectors<<<std::min(4096, ceil_div((long)Lp * NBF, 256)), 256, 0, s>>>(
                x.W, x.ldw, p0, nbp, Lp, 0, x.Vp);
            // columns < p0 of [I; 0] have no entries in rows >= p0: the block leaves them
            apply_block_reflector_ex(x, J.u, uc, p0, Lp, p0, uc - p0, nbp, J.tauq + p0, false, s);
        }
        // V = G_0 ... G_{N-2} (row reflectors), then Vt = V^T
        paco_count_launch(), bd_set_identity<<<std::min(8192, ceil_div((long)N * N, 256)), 256, 0, s>>>(x.Vtmp, N, N);
        for (int p0 = ((N - 1) / nbf) * nbf; p0 >= 0; p0 -= nbf) {
            int nbp = std::min(N - 1, p0 + nbf) - p0, Lp = N - p0 - 1;
            if (nbp <= 0 || Lp <= 0) continue;
            paco_count_launch(), bd_panel_vectors<<<std::min(4096, ceil_div((long)Lp * NBF, 256)), 256, 0, s>>>(
                x.W, x.ldw, p0, nbp, Lp, 1, x.Vp);
            apply_block_reflector(x, x.Vtmp, N, p0 + 1, Lp, nbp, J.taup + p0, s);
        }
        paco_count_launch(), bd_transpose<<<dim3(ceil_div(N, 32), ceil_div(N, 32)), dim3(32, 8), 0, s>>>(x.Vtmp, J.vt, N);
        paco_count_launch(), bd_copy_out<<<std::min(4096, ceil_div((long)M * N, 256)), 256, 0, s>>>(
            J.a_out, x.W, M, N, x.ldw, J.d, J.e);
    }
    if (k > 1) join();
    prof_end();
    return cudaGetLastError() == cudaSuccess ? PACO_OK : PACO_ERR_CUDA;
}

int bd_run(int M, int N, const float *a_in, float *a_out, float *u, float *vt, float *d, float *e, float *tauq,
           float *taup, void *workspace, cudaStream_t s, int num_sms)
{
    BdJob job = {M, N, a_in, a_out, u, vt, d, e, tauq, taup, workspace, 0};
    return bd_run_multi(1, &job, s, nullptr, num_sms);
}

// Events of the fork / join of the side streams: created once (outside any
// stream capture, by bd_init_attrs), reused by every call.
cudaEvent_t *bd_fork_events()
{
    static cudaEvent_t ev[1 + PK_KMAX] = {};
    if (!ev[0])
        for (auto &e : ev) cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
    return ev;
}
