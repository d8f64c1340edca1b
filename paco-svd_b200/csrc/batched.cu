// Batched SVD of many small matrices (1 <= N <= M <= 512) in one persistent
// launch.  Every CTA (256 threads) takes the next matrix from a work queue
// (matrices sorted by cost, largest first) and runs the whole pipeline of
// the single-matrix path for it:
//   1. Golub-Kahan Householder bidiagonalization, unblocked, with the reflector
//      convention of upper_bidiagonalization.cpp:182-218.  One fused sweep per
//      column step: each warp owns whole rows (held in registers, lane l has
//      columns l, l+32, ...), applies the left reflector H_i and the right
//      reflector G_i to them, and in the same sweep accumulates the column
//      norm and the products  S_j = sum_r x_r a_rj  that the next step's left
//      reflector needs (w_j = a_ij + S_j / v0), so the trailing block is read
//      and written once per step.
//   2. Bidiagonal divide and conquer with the device bodies of bdc_dev.cuh
//      (the same code the level kernels of the large path run), levels in
//      sequence, merges of a level one after another, every phase spread over
//      the CTA's threads or warps.
//   3. U = H_0 ... H_{N-1} blockdiag(Q, I) and V = G_0 ... G_{N-2} W, applied
//      backward to the divide-and-conquer vectors with one fused sweep per
//      reflector (apply H_i, accumulate the w of H_{i-1}), which replaces the
//      formation of U, V and the two final products of svd.cpp:1911-1981.
// Per-matrix scratch lives in one slot per CTA, carved for the matrix at hand.
#include <algorithm>
#include <cstring>
#include <vector>

#include "batched.cuh"
#include "bdc_dev.cuh"

namespace bt {
constexpr int THREADS = 256;
constexpr int WARPS = THREADS / 32;
constexpr int VPL = PACO_BATCH_MAX_M / 32;  // row values per lane
}  // namespace bt

struct BtItem {
    int M, N, index, pad;
    const float *A;
    float *U, *Vt, *sigma;
};

struct BtSlot {
    float *W;       // M x ldw  working copy of A, then the Householder vectors
    long ldw;
    float *d, *e, *tauq, *taup;
    float *qt, *wt; // 2 N^2 each: Q^T / st and W^T / gt of the divide and conquer
    int *idx;       // 16 N
    float *diff;    // N x N  d_j^2 - sigma_i^2 of the secular roots
    float *X;       // N x N  V W before the transpose into Vt
    BdcWs bw;
};

__host__ __device__ static size_t bt_carve(char *base, int M, int N, BtSlot *s)
{
    size_t off = 0;
    auto take = [&](size_t bytes) -> char * {
        off = (off + 255) & ~(size_t)255;
        char *p = base ? base + off : nullptr;
        off += bytes;
        return p;
    };
    const size_t nn = (size_t)N * N;
    const int nleaf = N / 3 + 2;
    s->ldw = (N + 3) & ~3;
    s->W = (float *)take(sizeof(float) * (size_t)M * s->ldw);
    s->d = (float *)take(sizeof(float) * N);
    s->e = (float *)take(sizeof(float) * N);
    s->tauq = (float *)take(sizeof(float) * N);
    s->taup = (float *)take(sizeof(float) * N);
    s->qt = (float *)take(sizeof(float) * 2 * nn);
    s->wt = (float *)take(sizeof(float) * 2 * nn);
    s->idx = (int *)take(sizeof(int) * 16 * (size_t)N);
    s->diff = (float *)take(sizeof(float) * nn);
    s->X = (float *)take(sizeof(float) * nn);
    BdcWs &w = s->bw;
    w.st = (DevStatus *)take(sizeof(DevStatus));
    w.Us = (float *)take(sizeof(float) * nn);
    w.Vs = (float *)take(sizeof(float) * nn);
    w.zsec = (double *)take(sizeof(double) * N);
    w.rot = (RotEntry *)take(sizeof(RotEntry) * N);
    w.meta = (MergeMeta *)take(sizeof(MergeMeta) * N);
    w.leaf_s = (int *)take(sizeof(int) * nleaf);
    w.leaf_e = (int *)take(sizeof(int) * nleaf);
    w.mg_s = (int *)take(sizeof(int) * nleaf);
    w.mg_m = (int *)take(sizeof(int) * nleaf);
    w.mg_e = (int *)take(sizeof(int) * nleaf);
    w.perm = (int *)take(sizeof(int) * N);
    w.sig = (float *)take(sizeof(float) * N);
    w.tcs = nullptr;
    w.tcs_floats = 0;
    return (off + 255) & ~(size_t)255;
}

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

struct BtShared {
    float part[bt::WARPS][PACO_BATCH_MAX_M]; // per-warp partial column sums
    float wv[PACO_BATCH_MAX_M];              // w of the current left reflector
    float uv[PACO_BATCH_MAX_M];              // current right reflector (u_{i+1} = 1)
    float rv[PACO_BATCH_MAX_M];              // pivot row after its left update
    float ssig[bt::WARPS];
    int lv_off[BDC_MAX_LEVELS], lv_nm[BDC_MAX_LEVELS];
    int nlev, item, bad;
};

// ---------------------------------------------------------------- stage 1

// a[q] for a run-time q without indexing the register array dynamically
static __device__ __forceinline__ float bt_pick(const float (&a)[bt::VPL], int q)
{
    float x = 0.f;
#pragma unroll
    for (int j = 0; j < bt::VPL; j++)
        if (j == q) x = a[j];
    return x;
}

// Sweep of the rows r in [r0, M): optional left/right updates of columns
// >= c0, then the accumulation for the next column reflector (column cn,
// rows > cn):  ssig += a_r,cn^2,  part[c] += a_r,cn * a_rc  (c > cn).
// mode 0: copy-in from A (NaN/Inf -> 0, flagged), no updates.
template <int MODE>
static __device__ void bt_sweep(BtShared &sh, const float *A, float *W, long ldw, int M, int N, int r0, int ci,
                                float inv_v0, float tq, float tp, int *bad)
{
    using namespace bt;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int cn = ci + 1;  // next column (MODE 0: ci = -1, cn = 0)
    float acc[VPL];
#pragma unroll
    for (int q = 0; q < VPL; q++) acc[q] = 0.f;
    float ssig = 0.f;
    for (int r = r0 + warp; r < M; r += WARPS) {
        float a[VPL];
        float *row = W + (long)r * ldw;
        if (MODE == 0) {
            const float *src = A + (long)r * N;
#pragma unroll
            for (int q = 0; q < VPL; q++) {
                const int c = lane + 32 * q;
                float x = (c < N) ? src[c] : 0.f;
                if (!isfinite(x)) { x = 0.f; *bad = 1; }
                a[q] = x;
                if (c < N) row[c] = x;
            }
        } else {
#pragma unroll
            for (int q = 0; q < VPL; q++) {
                const int c = lane + 32 * q;
                a[q] = (c >= ci && c < N) ? row[c] : 0.f;
            }
            // Householder vector entry of column ci
            const float x = __shfl_sync(0xffffffffu, bt_pick(a, ci >> 5), ci & 31);
            const float vr = x * inv_v0;
            if (lane == (ci & 31)) row[ci] = vr;
            // left update (H_ci) then right update (G_ci) of columns > ci
            const float lf = tq * vr;
            float dot = 0.f;
#pragma unroll
            for (int q = 0; q < VPL; q++) {
                const int c = lane + 32 * q;
                if (c > ci && c < N) {
                    a[q] -= lf * sh.wv[c];
                    dot += a[q] * sh.uv[c];
                }
            }
            dot = warp_sum(dot) * tp;
#pragma unroll
            for (int q = 0; q < VPL; q++) {
                const int c = lane + 32 * q;
                if (c > ci && c < N) {
                    a[q] -= dot * sh.uv[c];
                    row[c] = a[q];
                }
            }
        }
        if (cn < N && r > cn) {
            const float xn = __shfl_sync(0xffffffffu, bt_pick(a, cn >> 5), cn & 31);
            ssig += xn * xn;
#pragma unroll
            for (int q = 0; q < VPL; q++) {
                const int c = lane + 32 * q;
                if (c > cn) acc[q] += xn * a[q];
            }
        }
    }
#pragma unroll
    for (int q = 0; q < VPL; q++) {
        const int c = lane + 32 * q;
        if (c < N) sh.part[warp][c] = acc[q];
    }
    if (lane == 0) sh.ssig[warp] = ssig;
}

// Stage 1 for one matrix: d, e, tauq, taup and the Householder vectors in W.
static __device__ void bt_bidiag(BtShared &sh, const float *A, const BtSlot &s, int M, int N)
{
    using namespace bt;
    const int tid = threadIdx.x;
    float *W = s.W;
    const long ldw = s.ldw;
    bt_sweep<0>(sh, A, W, ldw, M, N, 0, -1, 0.f, 0.f, 0.f, &sh.bad);
    __syncthreads();
    for (int i = 0; i < N; i++) {
        // column reflector i from the sums of the previous sweep (every
        // thread computes the same scalars, in the same order)
        float sig = 0.f;
#pragma unroll
        for (int w = 0; w < WARPS; w++) sig += sh.ssig[w];
        const float x0 = W[(long)i * ldw + i];
        float beta, tq, v0;
        bt_reflector(x0, sig, M - i, &beta, &tq, &v0);
        const float inv_v0 = 1.f / v0;
        // w_j = a_ij + S_j / v0 and the left update of the pivot row
        for (int c = tid; c < N; c += THREADS) {
            if (c > i) {
                float S = 0.f;
#pragma unroll
                for (int w = 0; w < WARPS; w++) S += sh.part[w][c];
                const float wj = W[(long)i * ldw + c] + inv_v0 * S;
                sh.wv[c] = wj;
                sh.rv[c] = W[(long)i * ldw + c] - tq * wj;
            }
        }
        __syncthreads();
        if (tid == 0) {  // after every thread has read x0
            s.d[i] = beta;
            s.tauq[i] = tq;
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
            for (int c = tid; c < N; c += THREADS) {
                if (c == i + 1) {
                    sh.uv[c] = 1.f;
                    W[(long)i * ldw + c] = eb;
                } else if (c > i + 1) {
                    const float u = sh.rv[c] * inv_r;
                    sh.uv[c] = u;
                    W[(long)i * ldw + c] = u;
                }
            }
            if (tid == 0) {
                s.e[i] = eb;
                s.taup[i] = tp;
            }
        }
        __syncthreads();
        bt_sweep<1>(sh, nullptr, W, ldw, M, N, i + 1, i, inv_v0, tq, tp, nullptr);
        __syncthreads();
    }
}

// ---------------------------------------------------------------- stage 2

static __device__ void bt_bdc(BtShared &sh, const BtSlot &s, int N, unsigned char *dyn)
{
    using namespace bt;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    LevelArgs A;
    A.N = N; A.off = 0; A.d_e = s.e; A.d = s.d;
    A.QT = s.qt; A.ST = s.qt + (size_t)N * N; A.WT = s.wt; A.GT = s.wt + (size_t)N * N;
    int *ib = s.idx;
    A.idxq = ib; A.f = (float *)(ib + N); A.l = (float *)(ib + 2 * N); A.dsig = (float *)(ib + 3 * N);
    A.zhat = (float *)(ib + 4 * N); A.srow = ib + 5 * N;
    A.diff = s.diff;
    A.w = s.bw;
    if (tid == 0) sh.nlev = bdc_schedule_dev(N, nullptr, s.bw, sh.lv_off, sh.lv_nm);
    for (long t = tid; t < (long)N * N; t += THREADS) {
        const float v = (t / N == t % N) ? 1.f : 0.f;
        s.qt[t] = v;
        s.wt[t] = v;
    }
    __syncthreads();
    const int nleaf = leaf_partition(N, nullptr, nullptr);
    for (int t = tid; t < nleaf; t += THREADS)
        bdc_leaf_dev(t, N, s.bw, s.d, s.e, A.QT, A.WT, A.idxq, A.f, A.l);
    __syncthreads();
    const int nlev = min(sh.nlev, BDC_MAX_LEVELS);
    for (int lv = 0; lv < nlev; lv++) {
        A.off = sh.lv_off[lv];
        const int nm = sh.lv_nm[lv];
        for (int mg = 0; mg < nm; mg++) bdc_prepare_dev(A, mg, dyn);
        for (int mg = 0; mg < nm; mg++)
            for (int c = tid; c < N; c += THREADS) bdc_rotate_dev(A, mg, c);
        __syncthreads();
        for (int mg = 0; mg < nm; mg++)
            for (int c = tid; c < N; c += THREADS) bdc_gather_dev(A, mg, c, 0, N);
        __syncthreads();
        for (int g = warp; g < N; g += WARPS) bdc_secular_dev(A, nm, g, lane);
        __syncthreads();
        for (int g = warp; g < N; g += WARPS) bdc_lowner_dev(A, nm, g, lane);
        __syncthreads();
        for (int g = warp; g < N; g += WARPS) bdc_vectors_dev(A, nm, g, lane);
        __syncthreads();
        for (int mg = 0; mg < nm; mg++)
            for (int c = tid; c < N; c += THREADS) bdc_copyback_dev(A, mg, c, 0, N);
        __syncthreads();
        for (int mg = 0; mg < nm; mg++) {
            const MergeMeta mm = A.w.meta[A.w.mg_s[A.off + mg]];
            for (int which = 0; which < 2; which++) {
                const int ncols = which ? mm.nc : mm.n;
                for (int tm = 0; tm * 128 < mm.k; tm++)
                    for (int tn = 0; tn * 128 < ncols; tn++) bdc_btgemm_dev(A, mg, which, tm, tn);
            }
        }
        __syncthreads();
        for (int mg = 0; mg < nm; mg++) bdc_finalize_dev(A, mg);
    }
    for (int base = 0; base < N; base += THREADS) bdc_rank_desc_dev(N, s.d, s.bw.perm, s.bw.sig, base);
    __syncthreads();
}

// ---------------------------------------------------------------- stage 3

// Backward application of reflectors k = k1, k1-1, ..., 0 to the rows of Y
// (R rows, C <= 512 columns, ld ldy): reflector k acts on rows >= k + sh_off
// with v_{k+sh_off} = 1 and v_r = vec(k, r) for r > k + sh_off.  Each sweep
// applies reflector k and accumulates the w of reflector k-1.
template <typename Vec>
static __device__ void bt_apply_back(BtShared &sh, float *Y, long ldy, int R, int C, int k1, int sh_off,
                                     const float *tau, Vec vec)
{
    using namespace bt;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (k1 < 0) return;
    // w of reflector k1
    {
        const int p = k1 + sh_off;
        float acc[VPL];
#pragma unroll
        for (int q = 0; q < VPL; q++) acc[q] = 0.f;
        for (int r = p + warp; r < R; r += WARPS) {
            const float vr = (r == p) ? 1.f : vec(k1, r);
            const float *row = Y + (long)r * ldy;
#pragma unroll
            for (int q = 0; q < VPL; q++) {
                const int c = lane + 32 * q;
                if (c < C) acc[q] += vr * row[c];
            }
        }
#pragma unroll
        for (int q = 0; q < VPL; q++) {
            const int c = lane + 32 * q;
            if (c < C) sh.part[warp][c] = acc[q];
        }
        __syncthreads();
        for (int c = tid; c < C; c += THREADS) {
            float w = 0.f;
#pragma unroll
            for (int x = 0; x < WARPS; x++) w += sh.part[x][c];
            sh.wv[c] = w;
        }
        __syncthreads();
    }
    for (int k = k1; k >= 0; k--) {
        const int p = k + sh_off;
        const float tk = tau[k];
        const bool nxt = k > 0;
        float acc[VPL];
#pragma unroll
        for (int q = 0; q < VPL; q++) acc[q] = 0.f;
        for (int r = p + warp; r < R; r += WARPS) {
            const float vr = (r == p) ? 1.f : vec(k, r);
            const float vn = nxt ? vec(k - 1, r) : 0.f;  // r > p - 1: entry of reflector k-1
            const float f = tk * vr;
            float *row = Y + (long)r * ldy;
#pragma unroll
            for (int q = 0; q < VPL; q++) {
                const int c = lane + 32 * q;
                if (c < C) {
                    const float y = row[c] - f * sh.wv[c];
                    row[c] = y;
                    acc[q] += vn * y;
                }
            }
        }
        if (!nxt) break;
#pragma unroll
        for (int q = 0; q < VPL; q++) {
            const int c = lane + 32 * q;
            if (c < C) sh.part[warp][c] = acc[q];
        }
        __syncthreads();
        // row p - 1 is untouched by reflector k: w' = Y[p-1] + sum of the partials
        for (int c = tid; c < C; c += THREADS) {
            float w = Y[(long)(p - 1) * ldy + c];
#pragma unroll
            for (int x = 0; x < WARPS; x++) w += sh.part[x][c];
            sh.wv[c] = w;
        }
        __syncthreads();
    }
    __syncthreads();
}

// entry r of column reflector k (below the diagonal of W) / row reflector k
// (right of the superdiagonal)
struct BtColVec {
    const float *W;
    long ldw;
    __device__ float operator()(int k, int r) const { return W[(long)r * ldw + k]; }
};
struct BtRowVec {
    const float *W;
    long ldw;
    __device__ float operator()(int k, int r) const { return W[(long)k * ldw + r]; }
};

// ---------------------------------------------------------------- kernel

__global__ void __launch_bounds__(bt::THREADS) bt_svd(const BtItem *items, int count, unsigned *queue,
                                                      int *status, char *slots, size_t slot_bytes)
{
    using namespace bt;
    extern __shared__ __align__(16) unsigned char bt_dyn[];  // bdc_prepare scratch
    __shared__ BtShared sh;
    const int tid = threadIdx.x;
    char *slot = slots + (size_t)blockIdx.x * slot_bytes;
    for (;;) {
        if (tid == 0) sh.item = (int)atomicAdd(queue, 1u);
        __syncthreads();
        const int b = sh.item;
        if (b >= count) break;
        const BtItem it = items[b];
        const int M = it.M, N = it.N;
        BtSlot s;
        bt_carve(slot, M, N, &s);
        if (tid == 0) {
            sh.bad = 0;
            s.bw.st->code = 0;
            s.bw.st->secular_nonconv = 0;
        }
        __syncthreads();
        bt_bidiag(sh, it.A, s, M, N);
        bt_bdc(sh, s, N, bt_dyn);
        // U = H blockdiag(Q, I): Q(:, r) = qt row perm[r]
        const int *perm = s.bw.perm;
        for (long t = tid; t < (long)M * M; t += THREADS) {
            const int row = (int)(t / M), col = (int)(t % M);
            float v;
            if (col < N) v = (row < N) ? s.qt[(long)perm[col] * N + row] : 0.f;
            else v = (row == col) ? 1.f : 0.f;
            it.U[t] = v;
        }
        // X = W: W(:, r) = wt row perm[r]
        for (long t = tid; t < (long)N * N; t += THREADS) {
            const int row = (int)(t / N), col = (int)(t % N);
            s.X[t] = s.wt[(long)perm[col] * N + row];
        }
        __syncthreads();
        bt_apply_back(sh, it.U, M, M, M, N - 1, 0, s.tauq, BtColVec{s.W, s.ldw});
        bt_apply_back(sh, s.X, N, N, N, N - 2, 1, s.taup, BtRowVec{s.W, s.ldw});
        for (long t = tid; t < (long)N * N; t += THREADS) {
            const int r = (int)(t / N), j = (int)(t % N);
            it.Vt[t] = s.X[(long)j * N + r];
        }
        for (int t = tid; t < N; t += THREADS) it.sigma[t] = s.bw.sig[t];
        __syncthreads();
        if (tid == 0 && status) {
            int code = s.bw.st->code;
            if (!code && sh.bad) code = PACO_ERR_NONFINITE;
            if (!code && s.bw.st->secular_nonconv) code = PACO_ERR_NONCONVERGENCE;
            status[it.index] = code;
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------- host

static size_t bt_dyn_smem(int maxN) { return (size_t)20 * std::max(1, maxN) + 64; }

struct BtPlan {
    int Mx, Nx, slots;
    size_t slot_bytes, items_off, slots_off, total;
};

static int bt_blocks_per_sm(size_t dyn)
{
    static int cached = -1;
    static size_t cached_dyn = 0;
    if (cached < 0 || cached_dyn != dyn) {
        cudaFuncSetAttribute(bt_svd, cudaFuncAttributeMaxDynamicSharedMemorySize, 48 * 1024);
        int n = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, bt_svd, bt::THREADS, dyn) != cudaSuccess || n < 1)
            n = 1;
        cached = n;
        cached_dyn = dyn;
    }
    return cached;
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
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    BtSlot s;
    p->Mx = Mx;
    p->Nx = Nx;
    p->slot_bytes = bt_carve(nullptr, Mx, Nx, &s);
    p->slots = std::min(count, sms * bt_blocks_per_sm(bt_dyn_smem(Nx)));
    p->items_off = 256;
    p->slots_off = (p->items_off + sizeof(BtItem) * (size_t)count + 255) & ~(size_t)255;
    p->total = p->slots_off + p->slot_bytes * p->slots;
    return true;
}

size_t paco_batched_workspace_size(int count, const int *M, const int *N)
{
    BtPlan p;
    return bt_plan(count, M, N, &p) ? p.total : 0;
}

int paco_svd_batched(int count, const int *M, const int *N, const float *const *A, float *const *U,
                     float *const *Vt, float *const *sigma, int *status, void *workspace, size_t ws_bytes,
                     void *stream)
{
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
    }
    std::stable_sort(items.begin(), items.end(), [](const BtItem &x, const BtItem &y) {
        const double cx = (double)x.M * x.M * x.N + (double)x.M * x.N * x.N;
        const double cy = (double)y.M * y.M * y.N + (double)y.M * y.N * y.N;
        return cx > cy;
    });
    char *ws = (char *)workspace;
    const size_t dyn = bt_dyn_smem(p.Nx);
    if (cudaMemsetAsync(ws, 0, 256, s) != cudaSuccess) return PACO_ERR_CUDA;
    if (cudaMemcpyAsync(ws + p.items_off, items.data(), sizeof(BtItem) * count, cudaMemcpyHostToDevice, s) !=
        cudaSuccess)
        return PACO_ERR_CUDA;
    paco_count_launch();
    bt_svd<<<p.slots, bt::THREADS, dyn, s>>>((const BtItem *)(ws + p.items_off), count, (unsigned *)ws, status,
                                             ws + p.slots_off, p.slot_bytes);
    return cudaGetLastError() == cudaSuccess ? PACO_OK : PACO_ERR_CUDA;
}
