// Batched SVD of many small matrices (1 <= N <= M <= 2048): three persistent
// launches, each with a work queue over the matrices (largest first), so the
// whole batch takes three kernels whatever its size:
//   1. bt_bidiag_k (512 threads per matrix)  Golub-Kahan Householder
//      bidiagonalization, unblocked, with the reflector convention of
//      upper_bidiagonalization.cpp:182-218.  One fused sweep per column step:
//      each warp owns whole rows (held in registers, lane l has columns l,
//      l+32, ... of the active chunks; rows wider than 512 columns go in
//      segments, in two passes), applies the left reflector H_i and the
//      right reflector G_i to them, and in the same sweep accumulates the
//      column norm and the products S_j = sum_r x_r a_rj that the next step's
//      left reflector needs (w_j = a_ij + S_j / v0), so the trailing block is
//      read and written once per step.
//   2. bt_bdc_k (256 threads per matrix, two CTAs per SM)  bidiagonal divide
//      and conquer with the device bodies of bdc_dev.cuh (the code the level
//      kernels of the large path run): levels in sequence, every phase spread
//      over the CTA's threads or warps (a secular root per thread for small
//      merges, per warp for large ones), back-transform products through
//      64x64 shared-memory tiles.
//   3. bt_apply_k (512 threads per matrix)  U = H_0 ... H_{N-1} blockdiag(Q, I)
//      and V = G_0 ... G_{N-2} W applied to the divide-and-conquer vectors in
//      compact-WY blocks of 32 reflectors, last block first; this replaces
//      the formation of U, V and the two final products of svd.cpp:1911-1981.
// Each matrix keeps its Householder vectors, d/e/tau and Q^T/W^T in its own
// area of the workspace between the launches; the divide-and-conquer and
// back-transform scratch lives in one slot per CTA.
#include <algorithm>
#include <cstring>
#include <mutex>
#include <vector>

#include "batched.cuh"

// reflector of upper_bidiagonalization.cpp:182-218 from x0 and sigma = |x[1:]|^2
static __device__ __forceinline__ void bt_reflector(float x0, float sigma, int len, float *beta, float *tau,
                                                    float *v0)
{
    if (len <= 1 || sigma == 0.f) {
        *beta = x0; *tau = 0.f; *v0 = 1.f;
        return;
    }
    float mu = sqrtf(x0 * x0 + sigma);
    float v = (x0 <= 0.f) ? x0 - mu : -sigma / (x0 + mu);
    *v0 = v;
    *tau = 2.f * v * v / (sigma + v * v);
    *beta = mu;
}

// shared memory of the sweep kernels (1 and 3), carved from dynamic shared
// memory for rows of at most maxc columns
struct BtSweepSh {
    float *part;  // W_SWEEP x maxc per-warp partial column sums
    float *wv;    // maxc: w of the current left reflector
    float *uv;    // maxc: current right reflector (u_{i+1} = 1)
    float *rv;    // maxc: pivot row after its left update
    float *ssig;  // W_SWEEP
    int *item, *bad;
    int maxc;
};

__host__ __device__ static size_t bt_sweep_smem(int maxc)
{
    return sizeof(float) * ((size_t)(bt::W_SWEEP + 3) * maxc + bt::W_SWEEP) + 4 * sizeof(int);
}

static __device__ BtSweepSh bt_sweep_sh(unsigned char *raw, int maxc)
{
    BtSweepSh sh;
    float *f = reinterpret_cast<float *>(raw);
    sh.maxc = maxc;
    sh.part = f;
    sh.wv = f + (size_t)bt::W_SWEEP * maxc;
    sh.uv = sh.wv + maxc;
    sh.rv = sh.uv + maxc;
    sh.ssig = sh.rv + maxc;
    sh.item = reinterpret_cast<int *>(sh.ssig + bt::W_SWEEP);
    sh.bad = sh.item + 1;
    return sh;
}

// rows in flight per warp for NA active 32-column chunks (<= 48 row values
// per lane in registers)
template <int NA>
struct BtRows {
    static constexpr int RB = 48 / NA > 8 ? 8 : (48 / NA < 2 ? 2 : 48 / NA);
};

// the persistent work queue: the next matrix for this CTA, or -1
static __device__ __forceinline__ int bt_next(unsigned *queue, int count, int *s_item)
{
    __syncthreads();
    if (threadIdx.x == 0) *s_item = (int)atomicAdd(queue, 1u);
    __syncthreads();
    const int b = *s_item;
    return b < count ? b : -1;
}

// ---------------------------------------------------------------- kernel 1

// Sweep of the rows r in [r0, M) over the column chunks q0 .. q0+NA-1 (lane l
// holds column 32 (q0 + j) + l): the left update (H_ci) and the right update
// (G_ci) of the columns > ci, then the accumulation for the next column
// reflector (column cn = ci + 1, rows > cn):  ssig += a_r,cn^2,
// part[c] += a_r,cn * a_rc  (c > cn).  MODE 0 copies the rows in from A
// instead (NaN/Inf -> 0, flagged) and does no update.  Each warp has RB rows
// in flight (rows base + rb * W_SWEEP + warp).  Column ci lies in chunk q0.
template <int MODE, int NA>
static __device__ void bt_sweep(const BtSweepSh &sh, const float *A, float *W, long ldw, int M, int N, int r0, int ci,
                                int q0, float inv_v0, float tq, float tp, int *bad)
{
    using namespace bt;
    constexpr int RBn = BtRows<NA>::RB;
    constexpr int NW = W_SWEEP;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int cn = ci + 1;  // next column (MODE 0: ci = -1, cn = 0)
    const int c0 = 32 * q0 + lane;
    const bool cn_hi = (cn >> 5) > q0;  // column cn in the second active chunk
    float acc[NA];
#pragma unroll
    for (int j = 0; j < NA; j++) acc[j] = 0.f;
    float ssig = 0.f;
    for (int base = r0; base < M; base += NW * RBn) {
        float a[RBn][NA];
#pragma unroll
        for (int rb = 0; rb < RBn; rb++) {
            const int r = base + rb * NW + warp;
            const float *src = (MODE == 0) ? A + (long)r * N : W + (long)r * ldw;
#pragma unroll
            for (int j = 0; j < NA; j++) {
                const int c = c0 + 32 * j;
                a[rb][j] = (r < M && c >= ci && c < N) ? src[c] : 0.f;
            }
        }
#pragma unroll
        for (int rb = 0; rb < RBn; rb++) {
            const int r = base + rb * NW + warp;
            if (r >= M) break;
            float *row = W + (long)r * ldw;
            if (MODE == 0) {
#pragma unroll
                for (int j = 0; j < NA; j++) {
                    const int c = c0 + 32 * j;
                    if (!isfinite(a[rb][j])) { a[rb][j] = 0.f; *bad = 1; }
                    if (c < N) row[c] = a[rb][j];
                }
            } else {
                // Householder vector entry of column ci (chunk q0)
                const float x = __shfl_sync(0xffffffffu, a[rb][0], ci & 31);
                const float vr = x * inv_v0;
                if (lane == (ci & 31)) row[ci] = vr;
                const float lf = tq * vr;
                float dot = 0.f;
#pragma unroll
                for (int j = 0; j < NA; j++) {
                    const int c = c0 + 32 * j;
                    if (c > ci && c < N) {
                        a[rb][j] -= lf * sh.wv[c];
                        dot += a[rb][j] * sh.uv[c];
                    }
                }
                dot = warp_sum(dot) * tp;
#pragma unroll
                for (int j = 0; j < NA; j++) {
                    const int c = c0 + 32 * j;
                    if (c > ci && c < N) {
                        a[rb][j] -= dot * sh.uv[c];
                        row[c] = a[rb][j];
                    }
                }
            }
            if (cn < N && r > cn) {
                float xs = a[rb][0];
                if (NA > 1 && cn_hi) xs = a[rb][NA > 1 ? 1 : 0];
                const float xn = __shfl_sync(0xffffffffu, xs, cn & 31);
                ssig += xn * xn;
#pragma unroll
                for (int j = 0; j < NA; j++) {
                    const int c = c0 + 32 * j;
                    if (c > cn) acc[j] += xn * a[rb][j];
                }
            }
        }
    }
#pragma unroll
    for (int j = 0; j < NA; j++) {
        const int c = c0 + 32 * j;
        if (c < N) sh.part[warp * sh.maxc + c] = acc[j];
    }
    if (lane == 0) sh.ssig[warp] = ssig;
}

// bt_sweep for rows wider than 16 chunks: each warp takes RW rows at a time,
// in segments of 512 columns and two passes (left update and the dot with
// the right reflector, then the right update and the sums for the next
// column reflector, which go straight into the warp's row of part).
template <int MODE>
static __device__ void bt_sweep_wide(const BtSweepSh &sh, const float *A, float *W, long ldw, int M, int N, int r0,
                                     int ci, float inv_v0, float tq, float tp, int *bad)
{
    using namespace bt;
    constexpr int SEG = 16, NW = W_SWEEP, RW = 2;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int cn = ci + 1;
    const int q0 = ci < 0 ? 0 : ci >> 5;
    const int cbeg = 32 * q0;
    float *mypart = sh.part + warp * sh.maxc;
    for (int c = cbeg + lane; c < N; c += 32) mypart[c] = 0.f;
    float ssig = 0.f;
    for (int base = r0 + warp * RW; base < M; base += NW * RW) {
        const int nr = min(RW, M - base);
        float xn[RW];
#pragma unroll
        for (int w = 0; w < RW; w++) xn[w] = 0.f;
        if (MODE == 0) {
            for (int s0 = cbeg; s0 < N; s0 += 32 * SEG) {
                float a[RW][SEG];
#pragma unroll
                for (int w = 0; w < RW; w++) {
                    const float *src = A + (long)(base + w) * N;
#pragma unroll
                    for (int j = 0; j < SEG; j++) {
                        const int c = s0 + 32 * j + lane;
                        a[w][j] = (w < nr && c < N) ? src[c] : 0.f;
                    }
                }
#pragma unroll
                for (int w = 0; w < RW; w++) {
                    if (w >= nr) break;
                    const int r = base + w;
                    float *row = W + (long)r * ldw;
#pragma unroll
                    for (int j = 0; j < SEG; j++) {
                        const int c = s0 + 32 * j + lane;
                        if (!isfinite(a[w][j])) { a[w][j] = 0.f; *bad = 1; }
                        if (c < N) row[c] = a[w][j];
                    }
                    if (s0 == cbeg) xn[w] = __shfl_sync(0xffffffffu, a[w][0], 0);
                    if (r > cn) {
#pragma unroll
                        for (int j = 0; j < SEG; j++) {
                            const int c = s0 + 32 * j + lane;
                            if (c > cn && c < N) mypart[c] += xn[w] * a[w][j];
                        }
                    }
                }
            }
        } else {
            float vr[RW], dot[RW];
#pragma unroll
            for (int w = 0; w < RW; w++) { vr[w] = 0.f; dot[w] = 0.f; }
            for (int s0 = cbeg; s0 < N; s0 += 32 * SEG) {
                float a[RW][SEG];
#pragma unroll
                for (int w = 0; w < RW; w++) {
                    const float *row = W + (long)(base + w) * ldw;
#pragma unroll
                    for (int j = 0; j < SEG; j++) {
                        const int c = s0 + 32 * j + lane;
                        a[w][j] = (w < nr && c >= ci && c < N) ? row[c] : 0.f;
                    }
                }
#pragma unroll
                for (int w = 0; w < RW; w++) {
                    if (w >= nr) break;
                    float *row = W + (long)(base + w) * ldw;
                    if (s0 == cbeg) {
                        vr[w] = __shfl_sync(0xffffffffu, a[w][0], ci & 31) * inv_v0;
                        if (lane == (ci & 31)) row[ci] = vr[w];
                    }
                    const float lf = tq * vr[w];
#pragma unroll
                    for (int j = 0; j < SEG; j++) {
                        const int c = s0 + 32 * j + lane;
                        if (c > ci && c < N) {
                            a[w][j] -= lf * sh.wv[c];
                            dot[w] += a[w][j] * sh.uv[c];
                            row[c] = a[w][j];
                        }
                    }
                }
            }
#pragma unroll
            for (int w = 0; w < RW; w++) dot[w] = warp_sum(dot[w]) * tp;
            for (int s0 = cbeg; s0 < N; s0 += 32 * SEG) {
                float a[RW][SEG];
#pragma unroll
                for (int w = 0; w < RW; w++) {
                    const float *row = W + (long)(base + w) * ldw;
#pragma unroll
                    for (int j = 0; j < SEG; j++) {
                        const int c = s0 + 32 * j + lane;
                        a[w][j] = (w < nr && c > ci && c < N) ? row[c] : 0.f;
                    }
                }
#pragma unroll
                for (int w = 0; w < RW; w++) {
                    if (w >= nr) break;
                    const int r = base + w;
                    float *row = W + (long)r * ldw;
#pragma unroll
                    for (int j = 0; j < SEG; j++) {
                        const int c = s0 + 32 * j + lane;
                        if (c > ci && c < N) {
                            a[w][j] -= dot[w] * sh.uv[c];
                            row[c] = a[w][j];
                        }
                    }
                    if (s0 == cbeg) {
                        const float xs = ((cn >> 5) > q0) ? a[w][1] : a[w][0];
                        xn[w] = __shfl_sync(0xffffffffu, xs, cn & 31);
                    }
                    if (cn < N && r > cn) {
#pragma unroll
                        for (int j = 0; j < SEG; j++) {
                            const int c = s0 + 32 * j + lane;
                            if (c > cn && c < N) mypart[c] += xn[w] * a[w][j];
                        }
                    }
                }
            }
        }
#pragma unroll
        for (int w = 0; w < RW; w++)
            if (w < nr && cn < N && base + w > cn) ssig += xn[w] * xn[w];
    }
    if (lane == 0) sh.ssig[warp] = ssig;
}

// bt_sweep over the chunks q0 .. (N-1)/32
template <int MODE>
static __device__ void bt_sweep_any(const BtSweepSh &sh, const float *A, float *W, long ldw, int M, int N, int r0,
                                    int ci, float inv_v0, float tq, float tp, int *bad)
{
    const int q0 = ci < 0 ? 0 : ci >> 5;
    const int na = ((N - 1) >> 5) - q0 + 1;
#define BT_SWEEP_CASE(K) \
    case K: bt_sweep<MODE, K>(sh, A, W, ldw, M, N, r0, ci, q0, inv_v0, tq, tp, bad); break;
    if (na > 16) {
        bt_sweep_wide<MODE>(sh, A, W, ldw, M, N, r0, ci, inv_v0, tq, tp, bad);
        return;
    }
    switch (na) {
        BT_SWEEP_CASE(1) BT_SWEEP_CASE(2) BT_SWEEP_CASE(3) BT_SWEEP_CASE(4)
        BT_SWEEP_CASE(5) BT_SWEEP_CASE(6) BT_SWEEP_CASE(7) BT_SWEEP_CASE(8)
        BT_SWEEP_CASE(9) BT_SWEEP_CASE(10) BT_SWEEP_CASE(11) BT_SWEEP_CASE(12)
        BT_SWEEP_CASE(13) BT_SWEEP_CASE(14) BT_SWEEP_CASE(15) BT_SWEEP_CASE(16)
        default: break;
    }
#undef BT_SWEEP_CASE
}

// Stage 1 for one matrix: d, e, tauq, taup and the Householder vectors in W.
static __device__ void bt_bidiag(const BtSweepSh &sh, const float *A, const BtMat &m, int M, int N)
{
    using namespace bt;
    constexpr int NT = T_SWEEP, NW = W_SWEEP;
    const int tid = threadIdx.x;
    float *W = m.W;
    const long ldw = m.ldw;
    bt_sweep_any<0>(sh, A, W, ldw, M, N, 0, -1, 0.f, 0.f, 0.f, sh.bad);
    __syncthreads();
    for (int i = 0; i < N; i++) {
        // column reflector i from the sums of the previous sweep (every
        // thread computes the same scalars, in the same order)
        float sig = 0.f;
#pragma unroll
        for (int w = 0; w < NW; w++) sig += sh.ssig[w];
        const float x0 = W[(long)i * ldw + i];
        float beta, tq, v0;
        bt_reflector(x0, sig, M - i, &beta, &tq, &v0);
        const float inv_v0 = 1.f / v0;
        // w_j = a_ij + S_j / v0 and the left update of the pivot row
        for (int c = i + 1 + tid; c < N; c += NT) {
            float S = 0.f;
#pragma unroll
            for (int w = 0; w < NW; w++) S += sh.part[w * sh.maxc + c];
            const float aic = W[(long)i * ldw + c];
            const float wj = aic + inv_v0 * S;
            sh.wv[c] = wj;
            sh.rv[c] = aic - tq * wj;
        }
        __syncthreads();
        if (tid == 0) {  // after every thread has read x0
            m.d[i] = beta;
            m.tauq[i] = tq;
            W[(long)i * ldw + i] = beta;
        }
        // row reflector i on the pivot row's columns > i (every warp sums the
        // same values in the same order)
        float tp = 0.f;
        if (i < N - 1) {
            float rs = 0.f;
            for (int c = i + 2 + (tid & 31); c < N; c += 32) rs += sh.rv[c] * sh.rv[c];
            rs = warp_sum(rs);
            float eb, v0r;
            bt_reflector(sh.rv[i + 1], rs, N - i - 1, &eb, &tp, &v0r);
            const float inv_r = 1.f / v0r;
            for (int c = i + 1 + tid; c < N; c += NT) {
                const float u = (c == i + 1) ? 1.f : sh.rv[c] * inv_r;
                sh.uv[c] = u;
                W[(long)i * ldw + c] = (c == i + 1) ? eb : u;
            }
            if (tid == 0) {
                m.e[i] = eb;
                m.taup[i] = tp;
            }
        }
        __syncthreads();
        bt_sweep_any<1>(sh, nullptr, W, ldw, M, N, i + 1, i, inv_v0, tq, tp, nullptr);
        __syncthreads();
    }
}

// prof[0]: SM cycles of kernel 1 per matrix, summed
__global__ void __launch_bounds__(bt::T_SWEEP, 1) bt_bidiag_k(const BtItem *items, int count, unsigned *queue,
                                                              char *arena, int maxc, unsigned long long *prof)
{
    extern __shared__ __align__(16) unsigned char bt_sm1[];
    const BtSweepSh sh = bt_sweep_sh(bt_sm1, maxc);
    for (;;) {
        const int b = bt_next(queue, count, sh.item);
        if (b < 0) break;
        const BtItem it = items[b];
        BtMat m;
        bt_mat_carve(arena + it.moff, it.M, it.N, &m);
        if (threadIdx.x == 0) *sh.bad = 0;
        __syncthreads();
        const long long t0 = clock64();
        bt_bidiag(sh, it.A, m, it.M, it.N);
        if (threadIdx.x == 0) {
            *m.code = *sh.bad ? PACO_ERR_NONFINITE : 0;
            atomicAdd(&prof[0], (unsigned long long)(clock64() - t0));
        }
    }
}

// ---------------------------------------------------------------- kernel 2

// C (M x Nc) = X (M x K) Y (K x Nc), all row-major with the given leading
// dimensions: 64 x 64 output tiles, 16-deep k slices staged in shared memory,
// a 4 x 4 block of outputs per thread.  All 256 threads of the CTA call it.
static __device__ void bt_gemm64(int M, int Nc, int K, const float *X, long ldx, const float *Y, long ldy, float *C,
                                 long ldc)
{
    __shared__ __align__(16) float Xs[16][68];
    __shared__ __align__(16) float Ys[16][68];
    const int tid = threadIdx.x, ty = tid >> 4, tx = tid & 15;
    for (int m0 = 0; m0 < M; m0 += 64)
        for (int n0 = 0; n0 < Nc; n0 += 64) {
            float acc[4][4];
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) acc[i][j] = 0.f;
            for (int k0 = 0; k0 < K; k0 += 16) {
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    const int e = tid + 256 * q;
                    const int r = e >> 4, kk = e & 15;
                    const int gm = m0 + r, gk = k0 + kk;
                    Xs[kk][r] = (gm < M && gk < K) ? X[(long)gm * ldx + gk] : 0.f;
                    const int kr = e >> 6, c = e & 63;
                    const int gk2 = k0 + kr, gn = n0 + c;
                    Ys[kr][c] = (gk2 < K && gn < Nc) ? Y[(long)gk2 * ldy + gn] : 0.f;
                }
                __syncthreads();
#pragma unroll
                for (int kk = 0; kk < 16; kk++) {
                    const float4 a = *reinterpret_cast<const float4 *>(&Xs[kk][ty * 4]);
                    const float4 b = *reinterpret_cast<const float4 *>(&Ys[kk][tx * 4]);
                    const float av[4] = {a.x, a.y, a.z, a.w}, bv[4] = {b.x, b.y, b.z, b.w};
#pragma unroll
                    for (int i = 0; i < 4; i++)
#pragma unroll
                        for (int j = 0; j < 4; j++) acc[i][j] = fmaf(av[i], bv[j], acc[i][j]);
                }
                __syncthreads();
            }
#pragma unroll
            for (int i = 0; i < 4; i++) {
                const int gm = m0 + ty * 4 + i;
                if (gm >= M) continue;
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    const int gn = n0 + tx * 4 + j;
                    if (gn < Nc) C[(long)gm * ldc + gn] = acc[i][j];
                }
            }
        }
}

// qt/wt rows [0, k) of a merge = Us / Vs times st / gt
static __device__ void bt_btgemm(const LevelArgs &A, int mg)
{
    const int s = A.w.mg_s[A.off + mg];
    const MergeMeta mm = A.w.meta[s];
    const int N = A.N;
    const long off = (long)s * N + s;
    bt_gemm64(mm.k, mm.n, mm.k, A.w.Us + off, N, A.ST + off, N, A.QT + off, N);
    bt_gemm64(mm.k, mm.nc, mm.k, A.w.Vs + off, N, A.GT + off, N, A.WT + off, N);
}

// Stage 2 for one matrix.  prof[6..11]: cycles of set-up and leaves,
// prepare, rotate + gather, secular roots, Loewner z + vectors + copy-back,
// back-transform products + finalize (thread 0's clock).
static __device__ void bt_bdc(const BtMat &m, const BtBdcSlot &sl, int N, unsigned char *dyn, int *lv_off,
                              int *lv_nm, int *s_nlev, unsigned long long *prof)
{
    using namespace bt;
    constexpr int NT = T_BDC, NW = T_BDC / 32;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    long long tc = clock64();
    auto lap = [&](int k) {
        if (tid == 0) {
            const long long t = clock64();
            atomicAdd(&prof[k], (unsigned long long)(t - tc));
            tc = t;
        }
    };
    LevelArgs A;
    A.N = N; A.off = 0; A.d_e = m.e; A.d = m.d;
    A.QT = m.QT; A.ST = sl.ST; A.WT = m.WT; A.GT = sl.GT;
    int *ib = sl.idx;
    A.idxq = ib; A.f = (float *)(ib + N); A.l = (float *)(ib + 2 * N); A.dsig = (float *)(ib + 3 * N);
    A.zhat = (float *)(ib + 4 * N); A.srow = ib + 5 * N;
    A.diff = sl.diff;
    A.w = sl.bw;
    A.w.perm = m.perm;
    A.w.sig = m.sig;
    if (tid == 0) *s_nlev = bdc_schedule_dev(N, nullptr, A.w, lv_off, lv_nm);
    for (long t = tid; t < (long)N * N; t += NT) {
        const float v = (t / N == t % N) ? 1.f : 0.f;
        m.QT[t] = v;
        m.WT[t] = v;
    }
    __syncthreads();
    const int nleaf = leaf_partition(N, nullptr, nullptr);
    for (int t = tid; t < nleaf; t += NT) bdc_leaf_dev(t, N, A.w, m.d, m.e, A.QT, A.WT, A.idxq, A.f, A.l);
    __syncthreads();
    const int nlev = min(*s_nlev, BDC_MAX_LEVELS);
    lap(6);
    for (int lv = 0; lv < nlev; lv++) {
        A.off = lv_off[lv];
        const int nm = lv_nm[lv];
        for (int mg = 0; mg < nm; mg++) bdc_prepare_dev(A, mg, dyn);
        lap(7);
        for (int mg = 0; mg < nm; mg++)
            for (int c = tid; c < N; c += NT) bdc_rotate_dev(A, mg, c);
        __syncthreads();
        for (int mg = 0; mg < nm; mg++) {
            const int nc = A.w.meta[A.w.mg_s[A.off + mg]].nc;
            for (int x = tid; x < nc * nc; x += NT) bdc_gather_dev(A, mg, x % nc, x / nc, x / nc + 1);
        }
        __syncthreads();
        lap(8);
        // roots of small merges one per thread, of large merges one per warp
        for (int g = tid; g < N; g += NT) bdc_secular_dev<1>(A, nm, g, 0, 0, KSMALL);
        for (int g = warp; g < N; g += NW) bdc_secular_dev<32>(A, nm, g, lane, KSMALL, 0x7fffffff);
        __syncthreads();
        lap(9);
        for (int g = tid; g < N; g += NT) bdc_lowner_dev<1>(A, nm, g, 0, 0, KSMALL);
        for (int g = warp; g < N; g += NW) bdc_lowner_dev<32>(A, nm, g, lane, KSMALL, 0x7fffffff);
        __syncthreads();
        for (int g = tid; g < N; g += NT) bdc_vectors_dev<1>(A, nm, g, 0, 0, KSMALL);
        for (int g = warp; g < N; g += NW) bdc_vectors_dev<32>(A, nm, g, lane, KSMALL, 0x7fffffff);
        __syncthreads();
        for (int mg = 0; mg < nm; mg++) {
            const int nc = A.w.meta[A.w.mg_s[A.off + mg]].nc;
            for (int x = tid; x < nc * nc; x += NT) bdc_copyback_dev(A, mg, x % nc, x / nc, x / nc + 1);
        }
        __syncthreads();
        lap(10);
        for (int mg = 0; mg < nm; mg++) bt_btgemm(A, mg);
        __syncthreads();
        for (int mg = 0; mg < nm; mg++) bdc_finalize_dev(A, mg);
        lap(11);
    }
    for (int base = 0; base < N; base += NT) bdc_rank_desc_dev(N, m.d, m.perm, m.sig, base);
    __syncthreads();
}

// prof[1]: SM cycles of kernel 2 per matrix, summed
__global__ void __launch_bounds__(bt::T_BDC, 2) bt_bdc_k(const BtItem *items, int count, unsigned *queue,
                                                         char *arena, char *slots, size_t slot_bytes,
                                                         unsigned long long *prof)
{
    extern __shared__ __align__(16) unsigned char bt_dyn[];  // bdc_prepare scratch
    __shared__ int s_item, s_nlev;
    __shared__ int lv_off[BDC_MAX_LEVELS], lv_nm[BDC_MAX_LEVELS];
    char *slot = slots + (size_t)blockIdx.x * slot_bytes;
    for (;;) {
        const int b = bt_next(queue, count, &s_item);
        if (b < 0) break;
        const BtItem it = items[b];
        BtMat m;
        bt_mat_carve(arena + it.moff, it.M, it.N, &m);
        BtBdcSlot sl;
        bt_bdc_carve(slot, it.N, &sl);
        if (threadIdx.x == 0) {
            sl.bw.st->code = 0;
            sl.bw.st->secular_nonconv = 0;
        }
        __syncthreads();
        const long long t0 = clock64();
        bt_bdc(m, sl, it.N, bt_dyn, lv_off, lv_nm, &s_nlev, prof);
        __syncthreads();
        if (threadIdx.x == 0) {
            int code = *m.code;
            if (!code) code = sl.bw.st->code;
            if (!code && sl.bw.st->secular_nonconv) code = PACO_ERR_NONCONVERGENCE;
            *m.code = code;
            atomicAdd(&prof[1], (unsigned long long)(clock64() - t0));
        }
    }
}

// ---------------------------------------------------------------- kernel 3

// entry r of column reflector k (below the diagonal of W) / row reflector k
// (right of the superdiagonal); kRowMajorK: the entries of consecutive
// reflectors for one r are adjacent in memory
struct BtColVec {
    static constexpr bool kRowMajorK = true;
    const float *W;
    long ldw;
    __device__ float operator()(int k, int r) const { return W[(long)r * ldw + k]; }
};
struct BtRowVec {
    static constexpr bool kRowMajorK = false;
    const float *W;
    long ldw;
    __device__ float operator()(int k, int r) const { return W[(long)k * ldw + r]; }
};

namespace bt {
constexpr int ANB = 32;   // reflectors per block of the blocked application
constexpr int ARCH = 128; // rows of V staged at a time
}  // namespace bt

__host__ __device__ static size_t bt_apply_smem()
{
    using namespace bt;
    return sizeof(float) * ((size_t)ARCH * (ANB + 1) + 2 * ANB * (ANB + 1) + (size_t)T_SWEEP * ANB) + 16;
}

// Y (R x C, ld ldy) <- H_0 H_1 ... H_k1 Y, reflector k acting on rows >= p_k =
// k + sh_off with v_k(p_k) = 1 and v_k(r) = vec(k, r) below.  Blocks of ANB
// consecutive reflectors are applied as I - V T V^T (compact WY, T upper
// triangular from the Gram matrix V^T V by the larft recurrence), last block
// first: Z = V^T Y, Z' = T Z, Y -= V Z'.  Every thread owns one column of a
// strip of at most 512 columns; narrow strips split the rows over groups of
// threads.  V is staged through shared memory ARCH rows at a time.
template <typename Vec>
static __device__ void bt_apply_blocked(float *sm, float *Y, long ldy, int R, int C, int k1, int sh_off,
                                        const float *tau, Vec vec)
{
    using namespace bt;
    constexpr int NT = T_SWEEP, NB = ANB, LD = ANB + 1;
    if (k1 < 0) return;
    float *Vs = sm;                  // ARCH x LD
    float *Ts = Vs + ARCH * LD;      // NB x LD
    float *Gs = Ts + NB * LD;        // NB x LD
    float *Zs = Gs + NB * LD;        // NT x NB partial sums
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    for (int kb = (k1 / NB) * NB; kb >= 0; kb -= NB) {
        const int nb = min(k1 + 1, kb + NB) - kb;
        const int pb = kb + sh_off;  // first row of the block's reflectors
        auto stage = [&](int r0, int nr) {
            __syncthreads();
            for (int x = tid; x < nr * NB; x += NT) {
                int rr, jj;
                if (Vec::kRowMajorK) { rr = x / NB; jj = x % NB; }
                else { jj = x / nr; rr = x % nr; }
                const int r = r0 + rr, k = kb + jj, p = k + sh_off;
                float v = 0.f;
                if (jj < nb && r >= p) v = (r == p) ? 1.f : vec(k, r);
                Vs[rr * LD + jj] = v;
            }
            __syncthreads();
        };
        // Gram matrix of the block's vectors: entries (e / NB, e % NB), e = tid, tid + NT
        float g0 = 0.f, g1 = 0.f;
        for (int r0 = pb; r0 < R; r0 += ARCH) {
            const int nr = min(ARCH, R - r0);
            stage(r0, nr);
            const int i0 = tid / NB, i1 = (tid + NT) / NB, j = tid % NB;
            for (int rr = 0; rr < nr; rr++) {
                const float vj = Vs[rr * LD + j];
                g0 = fmaf(Vs[rr * LD + i0], vj, g0);
                g1 = fmaf(Vs[rr * LD + i1], vj, g1);
            }
        }
        Gs[(tid / NB) * LD + tid % NB] = g0;
        Gs[((tid + NT) / NB) * LD + tid % NB] = g1;
        __syncthreads();
        // T: one warp per row i, lane l holds T[i][l]:  T[i][i] = tau,
        // T[i][j] = -tau_j sum_{b=i}^{j-1} T[i][b] G[b][j]
        for (int i = warp; i < NB; i += NT / 32) {
            float t = (lane == i && i < nb) ? tau[kb + i] : 0.f;
            if (i < nb) {
                for (int j = i + 1; j < nb; j++) {
                    float p = (lane >= i && lane < j) ? t * Gs[lane * LD + j] : 0.f;
                    p = warp_sum(p);
                    if (lane == j) t = -tau[kb + j] * p;
                }
            }
            Ts[i * LD + lane] = t;
        }
        __syncthreads();
        for (int c0 = 0; c0 < C; c0 += NT) {
            const int Cs = min(NT, C - c0);
            const int S = max(1, NT / Cs);
            const int c = tid % Cs, g = tid / Cs;
            const bool act = g < S;
            float z[NB];
#pragma unroll
            for (int jj = 0; jj < NB; jj++) z[jj] = 0.f;
            // Z = V^T Y (each group of threads over its share of the rows)
            for (int r0 = pb; r0 < R; r0 += ARCH) {
                const int nr = min(ARCH, R - r0);
                stage(r0, nr);
                if (act) {
                    // four rows' loads in flight before their products
                    int rr = g;
                    for (; rr + 3 * S < nr; rr += 4 * S) {
                        float y[4];
#pragma unroll
                        for (int u = 0; u < 4; u++) y[u] = Y[(long)(r0 + rr + u * S) * ldy + c0 + c];
#pragma unroll
                        for (int u = 0; u < 4; u++)
#pragma unroll
                            for (int jj = 0; jj < NB; jj++) z[jj] = fmaf(Vs[(rr + u * S) * LD + jj], y[u], z[jj]);
                    }
                    for (; rr < nr; rr += S) {
                        const float y = Y[(long)(r0 + rr) * ldy + c0 + c];
#pragma unroll
                        for (int jj = 0; jj < NB; jj++) z[jj] = fmaf(Vs[rr * LD + jj], y, z[jj]);
                    }
                }
            }
            if (act) {
#pragma unroll
                for (int jj = 0; jj < NB; jj++) Zs[(g * NB + jj) * Cs + c] = z[jj];
            }
            __syncthreads();
            if (act && g == 0) {
                // sum the groups, then Z' = T Z for this column
#pragma unroll
                for (int jj = 0; jj < NB; jj++) {
                    float v = z[jj];
                    for (int h = 1; h < S; h++) v += Zs[(h * NB + jj) * Cs + c];
                    z[jj] = v;
                }
#pragma unroll
                for (int i = 0; i < NB; i++) {
                    float v = 0.f;
#pragma unroll
                    for (int jj = 0; jj < NB; jj++)
                        if (jj >= i) v = fmaf(Ts[i * LD + jj], z[jj], v);
                    Zs[i * Cs + c] = v;  // group 0's slots: read back by every group below
                }
            }
            __syncthreads();
            if (act) {
#pragma unroll
                for (int jj = 0; jj < NB; jj++) z[jj] = Zs[jj * Cs + c];
            }
            // Y -= V Z'
            for (int r0 = pb; r0 < R; r0 += ARCH) {
                const int nr = min(ARCH, R - r0);
                stage(r0, nr);
                if (act) {
                    int rr = g;
                    for (; rr + 3 * S < nr; rr += 4 * S) {
                        float v[4];
#pragma unroll
                        for (int u = 0; u < 4; u++) v[u] = Y[(long)(r0 + rr + u * S) * ldy + c0 + c];
#pragma unroll
                        for (int u = 0; u < 4; u++) {
#pragma unroll
                            for (int jj = 0; jj < NB; jj++) v[u] = fmaf(-Vs[(rr + u * S) * LD + jj], z[jj], v[u]);
                            Y[(long)(r0 + rr + u * S) * ldy + c0 + c] = v[u];
                        }
                    }
                    for (; rr < nr; rr += S) {
                        float *y = Y + (long)(r0 + rr) * ldy + c0 + c;
                        float v = *y;
#pragma unroll
                        for (int jj = 0; jj < NB; jj++) v = fmaf(-Vs[rr * LD + jj], z[jj], v);
                        *y = v;
                    }
                }
            }
            __syncthreads();
        }
    }
    __syncthreads();
}

// prof[2..5]: SM cycles of the U/X set-up, the U sweeps, the V sweeps and
// the outputs; matrices finished
__global__ void __launch_bounds__(bt::T_SWEEP, 1) bt_apply_k(const BtItem *items, int count, unsigned *queue,
                                                             char *arena, float *xslots, size_t xslot_floats,
                                                             int *status, unsigned long long *prof)
{
    using namespace bt;
    constexpr int NT = T_SWEEP;
    extern __shared__ __align__(16) float bt_sm3[];
    int *s_item = reinterpret_cast<int *>(reinterpret_cast<unsigned char *>(bt_sm3) + bt_apply_smem() - 16);
    const int tid = threadIdx.x;
    float *X = xslots + (size_t)blockIdx.x * xslot_floats;
    for (;;) {
        const int b = bt_next(queue, count, s_item);
        if (b < 0) break;
        const BtItem it = items[b];
        const int M = it.M, N = it.N;
        BtMat m;
        bt_mat_carve(arena + it.moff, M, N, &m);
        const long long t0 = clock64();
        // U = H blockdiag(Q, I): Q(:, r) = qt row perm[r]
        for (long t = tid; t < (long)M * M; t += NT) {
            const int row = (int)(t / M), col = (int)(t % M);
            float v;
            if (col < N) v = (row < N) ? m.QT[(long)m.perm[col] * N + row] : 0.f;
            else v = (row == col) ? 1.f : 0.f;
            it.U[t] = v;
        }
        // X = W: W(:, r) = wt row perm[r]
        for (long t = tid; t < (long)N * N; t += NT) {
            const int row = (int)(t / N), col = (int)(t % N);
            X[t] = m.WT[(long)m.perm[col] * N + row];
        }
        __syncthreads();
        const long long t1 = clock64();
        bt_apply_blocked(bt_sm3, it.U, M, M, M, N - 1, 0, m.tauq, BtColVec{m.W, m.ldw});
        const long long t2 = clock64();
        bt_apply_blocked(bt_sm3, X, N, N, N, N - 2, 1, m.taup, BtRowVec{m.W, m.ldw});
        for (long t = tid; t < (long)N * N; t += NT) {
            const int r = (int)(t / N), j = (int)(t % N);
            it.Vt[t] = X[(long)j * N + r];
        }
        for (int t = tid; t < N; t += NT) it.sigma[t] = m.sig[t];
        __syncthreads();
        if (tid == 0) {
            const long long t3 = clock64();
            atomicAdd(&prof[2], (unsigned long long)(t1 - t0));
            atomicAdd(&prof[3], (unsigned long long)(t2 - t1));
            atomicAdd(&prof[4], (unsigned long long)(t3 - t2));
            atomicAdd(&prof[5], 1ull);
            if (status) status[it.index] = *m.code;
        }
    }
}

// ---------------------------------------------------------------- host

static size_t bt_dyn_smem(int maxN) { return (size_t)20 * std::max(1, maxN) + 64; }

struct BtPlan {
    int Mx, Nx, slots1, slots2, slots3, maxc1, maxc3;
    size_t items_off, arena_off, arena_bytes, bdc_off, bdc_slot, x_off, x_slot, total;
    std::vector<size_t> moff;
};

static int bt_occupancy(const void *fn, int threads, size_t dyn)
{
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, threads, dyn) != cudaSuccess || n < 1) {
        cudaGetLastError();
        n = 1;
    }
    return n;
}

static bool bt_plan(int count, const int *M, const int *N, BtPlan *p)
{
    if (count <= 0 || !M || !N) return false;
    int Mx = 1, Nx = 1;
    for (int b = 0; b < count; b++) {
        if (N[b] < 1 || M[b] < N[b] || M[b] > PACO_BATCH_MAX_M) return false;
        Mx = std::max(Mx, M[b]);
        Nx = std::max(Nx, N[b]);
    }
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
        cudaGetLastError();
        sms = 148;
    }
    static bool attr[PACO_MAX_DEVICES] = {};
    if (!attr[paco_device()]) {
        cudaFuncSetAttribute(bt_bdc_k, cudaFuncAttributeMaxDynamicSharedMemorySize, 48 * 1024);
        const int big = (int)bt_sweep_smem(PACO_BATCH_MAX_M);
        cudaFuncSetAttribute(bt_bidiag_k, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
        cudaFuncSetAttribute(bt_apply_k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bt_apply_smem());
        cudaGetLastError();
        attr[paco_device()] = true;
    }
    p->maxc1 = (Nx + 31) & ~31;
    p->maxc3 = (Mx + 31) & ~31;
    p->Mx = Mx;
    p->Nx = Nx;
    p->items_off = 256;
    p->arena_off = (p->items_off + sizeof(BtItem) * (size_t)count + 255) & ~(size_t)255;
    p->moff.resize(count);
    size_t a = 0;
    for (int b = 0; b < count; b++) {
        BtMat m;
        p->moff[b] = a;
        a += bt_mat_carve(nullptr, M[b], N[b], &m);
    }
    p->arena_bytes = a;
    BtBdcSlot sl;
    p->bdc_slot = bt_bdc_carve(nullptr, Nx, &sl);
    p->x_slot = (size_t)Nx * Nx;
    p->slots1 = std::min(count, sms * bt_occupancy((const void *)bt_bidiag_k, bt::T_SWEEP, bt_sweep_smem(p->maxc1)));
    p->slots2 = std::min(count, sms * bt_occupancy((const void *)bt_bdc_k, bt::T_BDC, bt_dyn_smem(Nx)));
    // divide-and-conquer scratch is N^2-sized per CTA: at most about 4 GiB of it
    p->slots2 = std::max(1, std::min(p->slots2, (int)std::max<size_t>(sms / 4, ((size_t)4 << 30) / p->bdc_slot)));
    p->slots3 = std::min(count, sms * bt_occupancy((const void *)bt_apply_k, bt::T_SWEEP, bt_apply_smem()));
    p->bdc_off = p->arena_off + a;
    p->x_off = p->bdc_off + p->bdc_slot * p->slots2;
    p->total = p->x_off + ((sizeof(float) * p->x_slot * p->slots3 + 255) & ~(size_t)255);
    return true;
}

// Test hook (not in the public header): the cycle counters of the last batched
// call on this workspace (synchronizes the device).  out[0] stage 1, out[1]
// stage 2, out[2..4] set-up, U sweeps, V sweeps + outputs, out[5] matrices,
// out[6..11] the stage-2 phases.
extern "C" int paco_debug_batched_phases(const void *workspace, double out[12])
{
    unsigned long long v[12];
    if (!workspace || cudaDeviceSynchronize() != cudaSuccess ||
        cudaMemcpy(v, (const char *)workspace + 64, sizeof(v), cudaMemcpyDeviceToHost) != cudaSuccess)
        return PACO_ERR_CUDA;
    for (int k = 0; k < 12; k++) out[k] = (double)v[k];
    return PACO_OK;
}

// Test hook (not in the public header): while enabled, the three launches of
// each batched call are bracketed by CUDA events on the call's stream;
// paco_debug_batched_times waits for the last call and returns the three
// kernels' durations in milliseconds.
static bool g_bt_timing = false;
static cudaEvent_t g_bt_ev[4];

// Sets this unit's secular iteration limit (a test hook; synchronous).
void bt_set_sec_maxit(int n)
{
    cudaMemcpyToSymbol(g_sec_maxit, &n, sizeof(int));
}

extern "C" void paco_debug_batched_timing(int on)
{
    if (on && !g_bt_timing)
        for (auto &e : g_bt_ev) cudaEventCreate(&e);
    g_bt_timing = on != 0;
}

extern "C" int paco_debug_batched_times(float out[3])
{
    if (!g_bt_timing || cudaEventSynchronize(g_bt_ev[3]) != cudaSuccess) return PACO_ERR_CUDA;
    for (int k = 0; k < 3; k++) cudaEventElapsedTime(&out[k], g_bt_ev[k], g_bt_ev[k + 1]);
    return PACO_OK;
}

// Pinned host staging for the work-queue descriptors: a copy from pageable
// memory would first wait for the stream's earlier work, which serializes a
// serving loop that enqueues batch after batch.  A buffer is reused once the
// event recorded after its copy has completed; the pool grows with the number
// of calls in flight.
namespace {
struct BtStaging {
    void *p;
    size_t cap;
    cudaEvent_t done;
};
std::mutex g_bt_staging_mu;
std::vector<BtStaging> g_bt_staging;
}  // namespace

static cudaError_t bt_copy_items(void *dst, const void *src, size_t bytes, cudaStream_t s)
{
    std::lock_guard<std::mutex> lock(g_bt_staging_mu);
    BtStaging *slot = nullptr;
    for (auto &b : g_bt_staging)
        if (b.cap >= bytes && cudaEventQuery(b.done) == cudaSuccess) { slot = &b; break; }
    cudaGetLastError();  // a not-ready query is not an error of this call
    if (!slot) {
        BtStaging b;
        b.cap = std::max(bytes, (size_t)1 << 20);
        if (cudaMallocHost(&b.p, b.cap) != cudaSuccess) return cudaErrorMemoryAllocation;
        if (cudaEventCreateWithFlags(&b.done, cudaEventDisableTiming) != cudaSuccess) return cudaErrorUnknown;
        g_bt_staging.push_back(b);
        slot = &g_bt_staging.back();
    }
    memcpy(slot->p, src, bytes);
    cudaError_t err = cudaMemcpyAsync(dst, slot->p, bytes, cudaMemcpyHostToDevice, s);
    if (err == cudaSuccess) err = cudaEventRecord(slot->done, s);
    return err;
}

// Matrices larger than PACO_BATCH_MAX_M go to the multi-matrix form
// (paco_svd_multi), which takes one shape: true when every matrix of the list
// has the shape of the first and it is larger than that limit.
static bool bt_route_multi(int count, const int *M, const int *N)
{
    if (count < 1 || !M || !N || M[0] <= PACO_BATCH_MAX_M) return false;
    for (int b = 1; b < count; b++)
        if (M[b] != M[0] || N[b] != N[0]) return false;
    return true;
}

size_t paco_batched_workspace_size(int count, const int *M, const int *N)
{
    if (bt_route_multi(count, M, N)) return paco_svd_multi_workspace_size(count, M[0], N[0]);
    BtPlan p;
    return bt_plan(count, M, N, &p) ? p.total : 0;
}

int paco_svd_batched(int count, const int *M, const int *N, const float *const *A, float *const *U,
                     float *const *Vt, float *const *sigma, int *status, void *workspace, size_t ws_bytes,
                     void *stream)
{
    if (bt_route_multi(count, M, N))
        return paco_svd_multi(count, M[0], N[0], A, U, Vt, sigma, status, workspace, ws_bytes, stream);
    BtPlan p;
    if (!bt_plan(count, M, N, &p)) {
        for (int b = 0; b < count && M && N; b++)
            if (N[b] >= 1 && M[b] >= N[b] && M[b] > PACO_BATCH_MAX_M) return PACO_ERR_UNSUPPORTED;
        return PACO_ERR_INVALID_ARG;
    }
    if (!A || !U || !Vt || !sigma || !workspace || ws_bytes < p.total) return PACO_ERR_INVALID_ARG;
    for (int b = 0; b < count; b++)
        if (!A[b] || !U[b] || !Vt[b] || !sigma[b]) return PACO_ERR_INVALID_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    // work queue: largest matrices first (cost ~ M^2 N + M N^2)
    std::vector<BtItem> items(count);
    for (int b = 0; b < count; b++) {
        BtItem &it = items[b];
        it.M = M[b]; it.N = N[b]; it.index = b; it.pad = 0;
        it.A = A[b]; it.U = U[b]; it.Vt = Vt[b]; it.sigma = sigma[b];
        it.moff = p.moff[b];
    }
    std::stable_sort(items.begin(), items.end(), [](const BtItem &x, const BtItem &y) {
        const double cx = (double)x.M * x.M * x.N + (double)x.M * x.N * x.N;
        const double cy = (double)y.M * y.M * y.N + (double)y.M * y.N * y.N;
        return cx > cy;
    });
    char *ws = (char *)workspace;
    unsigned *queues = (unsigned *)ws;  // one counter per kernel
    unsigned long long *prof = (unsigned long long *)(ws + 64);
    const BtItem *dit = (const BtItem *)(ws + p.items_off);
    if (cudaMemsetAsync(ws, 0, 256, s) != cudaSuccess) return PACO_ERR_CUDA;
    if (bt_copy_items(ws + p.items_off, items.data(), sizeof(BtItem) * count, s) != cudaSuccess)
        return PACO_ERR_CUDA;
    char *arena = ws + p.arena_off;
    if (g_bt_timing) cudaEventRecord(g_bt_ev[0], s);
    paco_count_launch(), bt_bidiag_k<<<p.slots1, bt::T_SWEEP, bt_sweep_smem(p.maxc1), s>>>(dit, count, queues + 0,
                                                                                           arena, p.maxc1, prof);
    if (g_bt_timing) cudaEventRecord(g_bt_ev[1], s);
    paco_count_launch(), bt_bdc_k<<<p.slots2, bt::T_BDC, bt_dyn_smem(p.Nx), s>>>(
                             dit, count, queues + 1, arena, ws + p.bdc_off, p.bdc_slot, prof);
    if (g_bt_timing) cudaEventRecord(g_bt_ev[2], s);
    paco_count_launch(), bt_apply_k<<<p.slots3, bt::T_SWEEP, bt_apply_smem(), s>>>(
                             dit, count, queues + 2, arena, (float *)(ws + p.x_off), p.x_slot, status, prof);
    if (g_bt_timing) cudaEventRecord(g_bt_ev[3], s);
    return cudaGetLastError() == cudaSuccess ? PACO_OK : PACO_ERR_CUDA;
}
