// Two-stage reduction to bidiagonal form.  The reference names it as future
// work ("use aic to apply householder transformation", README.md:23); its
// one-stage kernel is upper_bidiagonalization.cpp.
//
// Stage 1, dense -> upper band of bandwidth b (ts_band_reduce): for each
// panel of b columns, the QR of the column panel (the QR block kernel of
// qr.cu on one thread-block cluster) and its block reflector applied to the
// trailing columns, then the LQ of the row panel W[k:k+b, k+b:N] (the panel
// transposed, factored by the same kernel, transposed back) and its block
// reflector applied from the right to the rows below.  Every step is a
// panel factorization or a block-reflector product; no column-by-column
// pass streams the trailing matrix.
//
// Stage 2, band -> bidiagonal by bulge chasing (ts_chase_k): sweep s
// annihilates row s beyond the superdiagonal with a right reflector on
// columns [s+1, s+b], which fills the b x b block below the diagonal; a left
// reflector on rows [s+1, s+b] clears its first column and fills row s+1
// beyond the band; step j of the sweep repeats this b columns further on
// (right reflector on columns c0 = s+1+jb .. c0+b-1 from row c0-b, left
// reflector on rows c0 .. c0+b-1 from column c0), until the matrix ends.
// Task (s, j) touches rows [c0-b, c0+b) only, and needs (s, j-1) and
// (s-1, j+2) done, so super-step t runs task j = t - 3s of every sweep s at
// once: the concurrent tasks are 3b - 1 rows apart and never share a row.
// The band lives in the shared memory of one 16-CTA cluster (contiguous
// row ranges, row r stored at columns r - b .. r + 2b - 1), each task runs
// on a team of four warps of the CTA owning its row c0 through distributed
// shared memory, and the super-steps are separated by cluster barriers.
//
// Back-transformation: U = Q1 blockdiag(Q2 U_B, I), V = P1 P2 V_B with Q1, P1
// from stage 1 (formed explicitly by the compact-WY products of qr.cu) and
// Q2, P2 the products of the chasing reflectors.  ts_apply_k applies the
// chasing reflectors of every sweep, in sweep order, to U[:, :N] from the
// right and to Vt from the left; it splits the matrix into chunks of 8 (or
// 4) independent columns (rows of U) held in shared memory, and stages the
// reflectors of the sweeps ahead by cp.async while a sweep is applied.
#include <cooperative_groups.h>

#include "qr.cuh"
#include "tma.cuh"
#include "twostage.cuh"

namespace {
namespace cg = cooperative_groups;

constexpr int CT = 512, CTEAM = 128, NTEAM = CT / CTEAM;  // chasing kernel: threads, threads per task, teams
constexpr int AT = 256;                    // back-transformation kernel threads

// dst[c * ldd + r] = src[r * lds + c] for r < rows, c < cols
__global__ void ts_transpose(const float *__restrict__ src, long lds, int rows, int cols, float *__restrict__ dst,
                             long ldd)
{
    __shared__ float tile[32][33];
    const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
    for (int y = threadIdx.y; y < 32; y += blockDim.y) {
        const int r = r0 + y, c = c0 + threadIdx.x;
        if (r < rows && c < cols) tile[y][threadIdx.x] = src[(long)r * lds + c];
    }
    __syncthreads();
    for (int y = threadIdx.y; y < 32; y += blockDim.y) {
        const int c = c0 + y, r = r0 + threadIdx.x;
        if (r < rows && c < cols) dst[(long)c * ldd + r] = tile[threadIdx.x][y];
    }
}

void transpose_launch(const float *src, long lds, int rows, int cols, float *dst, long ldd, cudaStream_t s)
{
    if (rows <= 0 || cols <= 0) return;
    paco_count_launch(), ts_transpose<<<dim3(ceil_div(cols, 32), ceil_div(rows, 32)), dim3(32, 8), 0, s>>>(
                             src, lds, rows, cols, dst, ldd);
}

// band[i * 3b + o] <- B[i, i + o - b] for the band (o - b in [0, b]), 0 elsewhere
__global__ void ts_band_from_w(const float *__restrict__ W, long ldw, int N, int b, float *__restrict__ band)
{
    const long total = (long)N * 3 * b;
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < total; t += (long)gridDim.x * blockDim.x) {
        const int i = (int)(t / (3 * b)), o = (int)(t % (3 * b));
        const int c = i + o - b;
        band[t] = (o >= b && o <= 2 * b && c < N) ? W[(long)i * ldw + c] : 0.f;
    }
}

// Vt <- blockdiag(I_b, F^T), F ((N - b) x (N - b), ld N - b)
__global__ void ts_p1t(const float *__restrict__ F, int N, int b, float *__restrict__ Vt)
{
    const long total = (long)N * N;
    const int n = N - b;
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < total; t += (long)gridDim.x * blockDim.x) {
        const int i = (int)(t / N), j = (int)(t % N);
        Vt[t] = (i < b || j < b) ? (i == j ? 1.f : 0.f) : F[(long)(j - b) * n + (i - b)];
    }
}

struct ChaseArgs {
    const float *band;  // N x 3b (global copy of B)
    float *refl_l, *refl_r, *d, *e;
    int N, rpc, jmax, T;
};

__device__ __forceinline__ void cluster_fence() { asm volatile("fence.acq_rel.cluster;" ::: "memory"); }

// Per-team shared state of a chasing task.
template <int B>
struct ChaseTeam {
    float vb[B];     // the current reflector, v[0] = 1, zero beyond its length
    float *rowp[B];  // rowp[l] = address of band element (c0 + l, c0)
    float tau;
};

__device__ __forceinline__ void team_sync(int team)
{
    asm volatile("bar.sync %0, %1;" ::"r"(team + 1), "r"(CTEAM) : "memory");
}

// One chasing task (sweep s, step j) on a team of CTEAM threads (4 warps).
// rows_of[o] is the generic address of CTA o's band rows; element (r, c) of
// the band is entry c - r + B of row r's storage.  The team's first warp forms
// the two reflectors; the updates split each row (then each column) into
// B/16 segments of 16 entries, one thread per segment, the segment sums of a
// row added by shuffles between neighbouring lanes.
template <int B>
__device__ void chase_task(const ChaseArgs &a, int s, int j, int team, ChaseTeam<B> &ts, float *const *rows_of,
                           int rpc)
{
    constexpr int NL = B / 32, OFF = B, LDB = 3 * B, GS = B / 16, SEG = 16;
    constexpr int STRIDE = CTEAM / GS;  // rows (columns) one pass of the team covers
    const int tid = threadIdx.x % CTEAM, lane = threadIdx.x & 31, N = a.N;
    const bool lead = tid < 32;  // the team's first warp
    auto at = [&](int r, int c) -> float * {
        const int o = r / rpc;
        return rows_of[o] + (long)(r - o * rpc) * LDB + (c - r + OFF);
    };
    const int c0 = s + 1 + j * B;
    const int c1 = min(c0 + B - 1, N - 1), L = c1 - c0 + 1;
    const int rp = (j == 0) ? s : c0 - B;
    const bool remote = (rp / rpc != c1 / rpc);  // rows of another CTA are touched
    const int g = tid % GS, gi = tid / GS;       // segment, row (column) slot
    // ---- right reflector on columns [c0, c1] from row rp (first warp)
    if (lead) {
        float *prow = at(rp, c0);
        float x[NL];
#pragma unroll
        for (int k = 0; k < NL; k++) {
            const int l = lane + 32 * k;
            x[k] = (l < L) ? prow[l] : 0.f;
        }
        float sg = 0.f;
#pragma unroll
        for (int k = 0; k < NL; k++)
            if (lane + 32 * k >= 1) sg += x[k] * x[k];
        sg = warp_sum(sg);
        const float x0 = __shfl_sync(0xffffffffu, x[0], 0);
        float beta, tau, v0;
        make_reflector(x0, sg, L, &beta, &tau, &v0);
        const float inv = 1.f / v0;
        float *rr = a.refl_r + ((long)s * a.jmax + j) * B;
#pragma unroll
        for (int k = 0; k < NL; k++) {
            const int l = lane + 32 * k;
            const float v = (l == 0) ? 1.f : (l < L ? x[k] * inv : 0.f);
            ts.vb[l] = v;
            rr[l] = (l == 0) ? tau : v;
            if (l < L) prow[l] = (l == 0) ? beta : 0.f;
        }
        if (lane == 0) ts.tau = tau;
    }
    team_sync(team);
    float tau = ts.tau;
    if (tau != 0.f) {
        // rows rp+1 .. c1, GS threads per row
        for (int base = 0; base < 2 * B - 1; base += STRIDE) {
            const int r = rp + 1 + base + gi;
            const bool act = r <= c1;
            float *p = act ? at(r, c0) + SEG * g : nullptr;
            float seg[SEG];
            float w = 0.f;
#pragma unroll
            for (int l = 0; l < SEG; l++) {
                const int lc = SEG * g + l;
                seg[l] = (act && lc < L) ? p[l] : 0.f;
                w += seg[l] * ts.vb[lc];
            }
#pragma unroll
            for (int o = 1; o < GS; o <<= 1) w += __shfl_xor_sync(0xffffffffu, w, o);
            w *= tau;
            if (act) {
#pragma unroll
                for (int l = 0; l < SEG; l++)
                    if (SEG * g + l < L) p[l] = seg[l] - w * ts.vb[SEG * g + l];
            }
        }
    }
    // the row updates are read from here on, by other threads
    if (remote) cluster_fence();
    team_sync(team);
    // ---- left reflector on rows [c0, c1] from column c0 (first warp)
    if (lead) {
        float *rp_[NL];
#pragma unroll
        for (int k = 0; k < NL; k++) {
            const int l = lane + 32 * k;
            rp_[k] = (l < L) ? at(c0 + l, c0) : nullptr;
            if (l < L) ts.rowp[l] = rp_[k];
        }
        float y[NL];
#pragma unroll
        for (int k = 0; k < NL; k++) y[k] = rp_[k] ? *rp_[k] : 0.f;
        float sg = 0.f;
#pragma unroll
        for (int k = 0; k < NL; k++)
            if (lane + 32 * k >= 1) sg += y[k] * y[k];
        sg = warp_sum(sg);
        const float y0 = __shfl_sync(0xffffffffu, y[0], 0);
        float beta, tl, v0;
        make_reflector(y0, sg, L, &beta, &tl, &v0);
        const float inv = 1.f / v0;
        float *rl = a.refl_l + ((long)s * a.jmax + j) * B;
#pragma unroll
        for (int k = 0; k < NL; k++) {
            const int l = lane + 32 * k;
            const float v = (l == 0) ? 1.f : (l < L ? y[k] * inv : 0.f);
            ts.vb[l] = v;
            rl[l] = (l == 0) ? tl : v;
            if (l < L) *rp_[k] = (l == 0) ? beta : 0.f;
        }
        if (lane == 0) ts.tau = tl;
    }
    team_sync(team);
    tau = ts.tau;
    if (tau != 0.f) {
        // columns c0+1 .. e1 of rows [c0, c1], GS threads per column
        const int e1 = min(c0 + 2 * B - 1, N - 1);
        for (int base = 0; base < 2 * B - 1; base += STRIDE) {
            const int c = c0 + 1 + base + gi;
            const bool act = c <= e1;
            float seg[SEG];
            float w = 0.f;
#pragma unroll
            for (int l = 0; l < SEG; l++) {
                const int lr = SEG * g + l;
                seg[l] = (act && lr < L) ? ts.rowp[lr][c - c0] : 0.f;
                w += ts.vb[lr] * seg[l];
            }
#pragma unroll
            for (int o = 1; o < GS; o <<= 1) w += __shfl_xor_sync(0xffffffffu, w, o);
            w *= tau;
            if (act) {
#pragma unroll
                for (int l = 0; l < SEG; l++) {
                    const int lr = SEG * g + l;
                    if (lr < L) ts.rowp[lr][c - c0] = seg[l] - w * ts.vb[lr];
                }
            }
        }
    }
    team_sync(team);  // vb and rowp are free for the team's next task (its rows are disjoint)
}

template <int B>
__global__ void __launch_bounds__(CT, 1) ts_chase_k(ChaseArgs a)
{
    extern __shared__ float sb[];  // this CTA's rows of the band, 3B floats each
    __shared__ ChaseTeam<B> teams[NTEAM];
    __shared__ float *rows_of[16];
    constexpr int LDB = 3 * B;
    cg::cluster_group cl = cg::this_cluster();
    const int rank = (int)cl.block_rank(), CS = (int)cl.num_blocks();
    const int N = a.N, rpc = a.rpc;
    const int r0 = rank * rpc, r1 = min(N, r0 + rpc);
    const int team = threadIdx.x / CTEAM;
    for (long t = threadIdx.x; t < (long)max(0, r1 - r0) * LDB; t += CT) sb[t] = a.band[(long)r0 * LDB + t];
    // own rows through the CTA's shared window, the others' through the cluster's
    if (threadIdx.x < CS)
        rows_of[threadIdx.x] = ((int)threadIdx.x == rank) ? sb : cl.map_shared_rank(sb, (int)threadIdx.x);
    cl.sync();
    const long den = 3L * B - 1;
    for (int t = 0; t < a.T; t++) {
        // sweeps whose step j = t - 3s starts at c0 = 1 + tB - s(3B - 1) in [r0, r1)
        const long num = 1L + (long)t * B;
        long s_hi = min((long)t / 3, (long)N - 2);
        s_hi = (num - r0 >= 0) ? min(s_hi, (num - r0) / den) : -1;
        const long s_lo = (num - r1 >= 0) ? (num - r1) / den + 1 : 0;
        for (long s = s_lo + team; s <= s_hi; s += NTEAM)
            chase_task<B>(a, (int)s, (int)(t - 3 * s), team, teams[team], rows_of, rpc);
        cl.sync();
    }
    for (int r = r0 + (int)threadIdx.x; r < r1; r += CT) {
        a.d[r] = sb[(long)(r - r0) * LDB + B];
        if (r < N - 1) a.e[r] = sb[(long)(r - r0) * LDB + B + 1];
    }
}

__device__ __forceinline__ void cp_async16(void *dst, const void *src)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}

// Applies the chasing reflectors of every sweep, in sweep order, to CW
// columns of X held in shared memory (row r at r + r/32, so the rows that
// the reflectors of one warp start at fall into different banks).  A
// reflector's work on 4 columns (a float4 column group, G = CW / 4 of them)
// is split over P = B / 8 neighbouring lanes, 8 interleaved rows each, kept
// in registers between the dot product (summed over the P lanes by
// shuffles) and the update; the reflectors of the sweeps ahead are staged
// by cp.async (row stride B + 4 floats) while sweep s is applied.
template <int CW, int B, int NS>
__global__ void __launch_bounds__(AT, 1) ts_apply_k(float *X, long ld, int N, int ncols, int trans, int jmax,
                                                   const float *__restrict__ refl)
{
    constexpr int G = CW / 4, RS = B + 4, P = B / 8, JSTEP = AT / (P * G);
    extern __shared__ __align__(16) float sm[];
    const int rows_p = N + N / 32 + 1;
    float *Xs = sm;
    float *Rb = Xs + (long)rows_p * CW;  // NS stages of jmax reflectors, RS floats each
    const long rb = (long)jmax * RS;
    const int cbase = blockIdx.x * CW, ncw = min(CW, ncols - cbase);
    auto ri = [](int r) { return r + (r >> 5); };
    if (trans) {
        for (long t = threadIdx.x; t < (long)CW * N; t += AT) {
            const int c = (int)(t / N), r = (int)(t % N);
            Xs[ri(r) * CW + c] = (c < ncw) ? X[(long)(cbase + c) * ld + r] : 0.f;
        }
    } else {
        for (long t = threadIdx.x; t < (long)N * CW; t += AT) {
            const int r = (int)(t / CW), c = (int)(t % CW);
            Xs[ri(r) * CW + c] = (c < ncw) ? X[(long)r * ld + cbase + c] : 0.f;
        }
    }
    auto stage = [&](int s, float *dst) {
        const int J = (N - 2 - s + B) / B;
        const float *src = refl + (long)s * jmax * B;
        for (int i = threadIdx.x; i < J * (B / 4); i += AT) {
            const int j = i / (B / 4), q = i % (B / 4);
            cp_async16(dst + j * RS + 4 * q, src + (long)j * B + 4 * q);
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
    };
    const int q = threadIdx.x % P, g = (threadIdx.x / P) % G, js = threadIdx.x / (P * G);
    // the reflectors of sweeps s .. s + NS - 2 are in flight while sweep s is
    // applied (one commit group per sweep, empty ones past the last sweep)
    for (int q = 0; q < NS - 1; q++) {
        if (q <= N - 2)
            stage(q, Rb + q * rb);
        else
            asm volatile("cp.async.commit_group;" ::: "memory");
    }
    for (int s = 0; s <= N - 2; s++) {
        const float *R = Rb + (s % NS) * rb;
        const int sn = s + NS - 1;
        if (sn <= N - 2)
            stage(sn, Rb + (sn % NS) * rb);
        else
            asm volatile("cp.async.commit_group;" ::: "memory");
        asm volatile("cp.async.wait_group %0;" ::"n"(NS - 1) : "memory");
        __syncthreads();
        const int J = (N - 2 - s + B) / B;
        // thread: part q (rows q, q + P, q + 2P, ... of the reflector: the 8
        // lanes of a quarter-warp reach 8 different banks), column group g,
        // reflector slot js; the P parts of a reflector are neighbouring lanes
        for (int jb = 0; jb < J; jb += JSTEP) {
            const int jj = jb + js;
            const float *v = R + jj * RS;
            const float tau = (jj < J) ? v[0] : 0.f;
            const int c0 = s + 1 + jj * B, L = min(B, N - c0);
            float4 seg[8];
            float4 w = make_float4(0.f, 0.f, 0.f, 0.f);
            if (tau != 0.f) {
#pragma unroll
                for (int l = 0; l < 8; l++) {
                    const int lr = q + P * l;
                    if (lr < L) {
                        seg[l] = *reinterpret_cast<const float4 *>(Xs + ri(c0 + lr) * CW + 4 * g);
                        const float vl = lr ? v[lr] : 1.f;
                        w.x += vl * seg[l].x; w.y += vl * seg[l].y; w.z += vl * seg[l].z; w.w += vl * seg[l].w;
                    }
                }
            }
#pragma unroll
            for (int o = 1; o < P; o <<= 1) {
                w.x += __shfl_xor_sync(0xffffffffu, w.x, o);
                w.y += __shfl_xor_sync(0xffffffffu, w.y, o);
                w.z += __shfl_xor_sync(0xffffffffu, w.z, o);
                w.w += __shfl_xor_sync(0xffffffffu, w.w, o);
            }
            if (tau != 0.f) {
                w.x *= tau; w.y *= tau; w.z *= tau; w.w *= tau;
#pragma unroll
                for (int l = 0; l < 8; l++) {
                    const int lr = q + P * l;
                    if (lr < L) {
                        const float vl = lr ? v[lr] : 1.f;
                        *reinterpret_cast<float4 *>(Xs + ri(c0 + lr) * CW + 4 * g) =
                            make_float4(seg[l].x - vl * w.x, seg[l].y - vl * w.y, seg[l].z - vl * w.z,
                                        seg[l].w - vl * w.w);
                    }
                }
            }
        }
        __syncthreads();  // the stage of sweep s is free for sweep s + NS
    }
    if (trans) {
        for (long t = threadIdx.x; t < (long)ncw * N; t += AT) {
            const int c = (int)(t / N), r = (int)(t % N);
            X[(long)(cbase + c) * ld + r] = Xs[ri(r) * CW + c];
        }
    } else {
        for (long t = threadIdx.x; t < (long)N * CW; t += AT) {
            const int r = (int)(t / CW), c = (int)(t % CW);
            if (c < ncw) X[(long)r * ld + cbase + c] = Xs[ri(r) * CW + c];
        }
    }
}

struct TsCfg {
    int cs = 0;        // cluster size of the chasing kernel (0: unavailable)
    int max_smem = 0;  // dynamic shared memory per CTA
};

size_t chase_smem(int N, int b, int cs) { return sizeof(float) * (size_t)((N + cs - 1) / cs) * 3 * b; }

TsCfg ts_cfg_probe()
{
    TsCfg cfg;
    int dev = 0, optin = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess) {
        cudaGetLastError();
        return cfg;
    }
    const int smem = optin - 8192;  // room for the static shared memory
    bool ok = true;
    for (auto f : {(const void *)ts_chase_k<32>, (const void *)ts_chase_k<64>}) {
        ok = ok && cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) == cudaSuccess &&
             cudaFuncSetAttribute(f, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) == cudaSuccess;
    }
    for (auto f : {(const void *)ts_apply_k<8, 32, 4>, (const void *)ts_apply_k<4, 32, 4>,
                   (const void *)ts_apply_k<8, 64, 4>, (const void *)ts_apply_k<4, 64, 4>,
                   (const void *)ts_apply_k<8, 32, 2>, (const void *)ts_apply_k<4, 32, 2>,
                   (const void *)ts_apply_k<8, 64, 2>, (const void *)ts_apply_k<4, 64, 2>})
        ok = ok && cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, optin) == cudaSuccess;
    if (!ok) {
        cudaGetLastError();
        return cfg;
    }
    for (int cs : {16, 8}) {
        cudaLaunchConfig_t lc = {};
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = cs;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        lc.gridDim = dim3(cs);
        lc.blockDim = dim3(CT);
        lc.dynamicSmemBytes = smem;
        lc.attrs = at;
        lc.numAttrs = 1;
        int n = 0;
        if (cudaOccupancyMaxActiveClusters(&n, (const void *)ts_chase_k<64>, &lc) == cudaSuccess && n >= 1) {
            cfg.cs = cs;
            cfg.max_smem = smem;
            break;
        }
        cudaGetLastError();
    }
    return cfg;
}

TsCfg g_ts_cfg[PACO_MAX_DEVICES];
bool g_ts_done[PACO_MAX_DEVICES];

TsCfg ts_cfg()
{
    const int dev = paco_device();
    if (!g_ts_done[dev]) {
        g_ts_cfg[dev] = ts_cfg_probe();
        g_ts_done[dev] = true;
    }
    return g_ts_cfg[dev];
}


size_t apply_smem(int N, int b, int cw, int ns)
{
    return sizeof(float) * ((size_t)(N + N / 32 + 1) * cw + (size_t)ns * ts::jmax(N, b) * (b + 4));
}

int optin_smem()
{
    int dev = 0, optin = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    return optin;
}

// Columns per CTA and reflector stages of the back-transformation: the first
// of (8, 4), (8, 2), (4, 4), (4, 2) that lets two CTAs share an SM (16 warps
// to hide the shared-memory latency), else the first that fits one CTA.
struct ApplyCfg {
    int cw, ns;
};

ApplyCfg apply_cfg(int N, int b)
{
    const ApplyCfg c[4] = {{8, 4}, {8, 2}, {4, 4}, {4, 2}};
    const size_t optin = (size_t)optin_smem(), two = 113 * 1024;
    for (const ApplyCfg &x : c)
        if (apply_smem(N, b, x.cw, x.ns) <= two) return x;
    for (const ApplyCfg &x : c)
        if (apply_smem(N, b, x.cw, x.ns) <= optin) return x;
    return {0, 0};
}

}  // namespace

void ts_init() { (void)ts_cfg(); }

bool ts_fits(int N, int b)
{
    const TsCfg c = ts_cfg();
    if (c.cs <= 0 || (b != 32 && b != 64) || N <= b || c.cs > 16) return false;
    return chase_smem(N, b, c.cs) <= (size_t)c.max_smem && apply_cfg(N, b).cw > 0 && qr_fits(N, b);
}

int ts_band_reduce(const BdWs &w, int M, int N, int b, float *tauq, float *taup, cudaStream_t s)
{
    cudaMemsetAsync(taup, 0, sizeof(float) * N, s);
    float *P = w.Vtmp;  // the transposed row panel, L x b
    for (int k = 0; k < N; k += b) {
        const int kb = std::min(b, N - k), k1 = k + kb;
        int rc = qr_panel(w.W, w.ldw, M, k, kb, tauq + k, s, true);
        if (rc) return rc;
        if (k1 < N) {
            bd_column_vectors(w.W, w.ldw, k, kb, M - k, w.Vp, s);
            if (apply_block_reflector_ex(w, w.W, w.ldw, k, M - k, k1, N - k1, kb, tauq + k, true, s) != cudaSuccess)
                return PACO_ERR_CUDA;
        }
        const int L = N - k - b;  // columns right of the band of the row panel
        if (L <= 0) continue;
        const int nr = std::min(kb, L);  // rows of the panel with a reflector
        float *Wr = w.W + (long)k * w.ldw + k + b;
        transpose_launch(Wr, w.ldw, kb, L, P, b, s);
        // all kb columns of P: with L < kb the reflectors of the first L rows
        // still apply to the panel's other rows (their own taus come out 0)
        rc = qr_panel(P, b, L, 0, kb, taup + k, s, true);
        if (rc) return rc;
        transpose_launch(P, b, L, kb, Wr, w.ldw, s);
        if (k1 < M) {
            bd_column_vectors(P, b, 0, nr, L, w.Vp, s);
            if (apply_block_reflector_right(w, w.W, w.ldw, k1, M - k1, k + b, L, nr, taup + k, s) != cudaSuccess)
                return PACO_ERR_CUDA;
        }
    }
    return cudaGetLastError() == cudaSuccess ? PACO_OK : PACO_ERR_CUDA;
}

int ts_chase(const BdWs &w, int N, int b, float *band, float *refl_l, float *refl_r, float *d, float *e,
             cudaStream_t s)
{
    const TsCfg cfg = ts_cfg();
    if (!ts_fits(N, b)) return PACO_ERR_UNSUPPORTED;
    paco_count_launch(), ts_band_from_w<<<std::min(4096, ceil_div((long)N * 3 * b, 256)), 256, 0, s>>>(
                             w.W, w.ldw, N, b, band);
    ChaseArgs a;
    a.band = band;
    a.refl_l = refl_l;
    a.refl_r = refl_r;
    a.d = d;
    a.e = e;
    a.N = N;
    a.rpc = ceil_div(N, cfg.cs);
    a.jmax = ts::jmax(N, b);
    a.T = 3 * (N - 2) + 1;
    cudaLaunchConfig_t lc = {};
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = cfg.cs;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    lc.gridDim = dim3(cfg.cs);
    lc.blockDim = dim3(CT);
    lc.dynamicSmemBytes = chase_smem(N, b, cfg.cs);
    lc.stream = s;
    lc.attrs = at;
    lc.numAttrs = 1;
    paco_count_launch();
    const cudaError_t err =
        b == 32 ? cudaLaunchKernelEx(&lc, ts_chase_k<32>, a) : cudaLaunchKernelEx(&lc, ts_chase_k<64>, a);
    if (err != cudaSuccess) {
        cudaGetLastError();
        return PACO_ERR_CUDA;
    }
    return PACO_OK;
}

int ts_form_p1t(const BdWs &w, int N, int b, const float *taup, float *Q, float *Vt, cudaStream_t s)
{
    const int n = N - b;
    // column r of Wt holds the LQ reflector of row r (unit entry at row r)
    transpose_launch(w.W + b, w.ldw, n, n, w.Vtmp, n, s);
    BdWs wt = w;
    wt.W = w.Vtmp;
    wt.ldw = n;
    const int rc = qr_form_u(wt, n, n, taup, nullptr, Q, s, n, 0);
    if (rc) return rc;
    paco_count_launch(), ts_p1t<<<std::min(8192, ceil_div((long)N * N, 256)), 256, 0, s>>>(Q, N, b, Vt);
    return cudaGetLastError() == cudaSuccess ? PACO_OK : PACO_ERR_CUDA;
}

int ts_apply(float *X, long ld, int N, int ncols, int trans, int b, const float *refl, DevStatus *st, cudaStream_t s)
{
    (void)st;
    if (N < 2 || ncols <= 0) return PACO_OK;
    const ApplyCfg ac = apply_cfg(N, b);
    const int cw = ac.cw, ns = ac.ns;
    if (cw == 0) return PACO_ERR_UNSUPPORTED;
    const int jm = ts::jmax(N, b);
    const int grid = ceil_div(ncols, cw);
    paco_count_launch();
    using K = void (*)(float *, long, int, int, int, int, const float *);
    K k = ns == 4 ? (cw == 8 ? (b == 32 ? ts_apply_k<8, 32, 4> : ts_apply_k<8, 64, 4>)
                             : (b == 32 ? ts_apply_k<4, 32, 4> : ts_apply_k<4, 64, 4>))
                  : (cw == 8 ? (b == 32 ? ts_apply_k<8, 32, 2> : ts_apply_k<8, 64, 2>)
                             : (b == 32 ? ts_apply_k<4, 32, 2> : ts_apply_k<4, 64, 2>));
    k<<<grid, AT, apply_smem(N, b, cw, ns), s>>>(X, ld, N, ncols, trans, jm, refl);
    return cudaGetLastError() == cudaSuccess ? PACO_OK : PACO_ERR_CUDA;
}
