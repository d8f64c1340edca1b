// QR-first reduction for tall matrices (M >= 1.6 N by default): A = Q R by
// blocked Householder QR, then the SVD pipeline runs on the N x N factor R
// and U = Q * blockdiag(U_R, I).  The reference lists this as future work
// ("3 step bidiagonalization", README.md:22); it cuts the bandwidth-bound
// column steps of stage 1 from an M x N to an N x N trailing matrix.
//
// qr_block_k   QR of a block of QB = 64 columns, rows [q0, M), in place in
//              W: one thread-block cluster holds the block's rows in the
//              shared memory of its CTAs (contiguous chunks, row stride
//              QB + 1 floats); column by column it forms the reflector of
//              make_reflector's convention (upper_bidiagonalization.cpp:
//              182-218: mu = +sqrt, Parlett v0, tau = 2 v0^2/(sigma + v0^2),
//              implicit v[0] = 1) and applies it to the block's remaining
//              columns.  The CTAs' partial sums (the column norm, then
//              v^T A for the remaining columns) are pushed into every CTA's
//              shared memory through distributed shared memory and added in
//              rank order, so each CTA forms the same reflector; one cluster
//              barrier per column (the next column's sums are formed right
//              after a column's update, v^T A from unscaled x: see the kernel).
// trailing     A[q0:, q1:N] <- (I - V T^T V^T) A[q0:, q1:N] through the
//              block-reflector products of stage 1 (Gram on the SIMT engine,
//              T, then V^T A, T^T G1, A -= V G2 on the tensor cores).
// U            blockdiag(U_R, I) is written into U, then the reflectors are
//              applied to it backward in blocks of NBF = 128 (all M columns).
#include "qr.cuh"
#include "tma.cuh"

namespace {

constexpr int QT = 512, QW = QT / 32;  // threads and warps per CTA
constexpr int QCS_MAX = 16;            // largest cluster

struct QrArgs {
    float *W;
    long ldw;
    int M, q0, nb, rpc;
    float *tau;
};

__device__ __forceinline__ void q_cluster_sync()
{
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}

__device__ __forceinline__ uint32_t q_dsmem(const void *local, int rank)
{
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(smem_u32(local)), "r"(rank));
    return r;
}

__device__ __forceinline__ unsigned q_rank()
{
    unsigned r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}

__device__ __forceinline__ unsigned q_nrank()
{
    unsigned r;
    asm volatile("mov.u32 %0, %%cluster_nctarank;" : "=r"(r));
    return r;
}

// Sum over the CTA of one value per thread (all threads call it).
__device__ __forceinline__ float q_block_sum(float v, float *red)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    v = warp_sum(v);
    __syncthreads();
    if (lane == 0) red[warp] = v;
    __syncthreads();
    float t = 0.f;
#pragma unroll
    for (int w = 0; w < QW; w++) t += red[w];
    return t;
}

__device__ __forceinline__ void q_st(uint32_t addr, float v)
{
    asm volatile("st.shared::cluster.f32 [%0], %1;" ::"r"(addr), "f"(v) : "memory");
}

// Every CTA pushes its partial sums into a slot of its own in every CTA of
// the cluster (remote stores), so after the cluster barrier each CTA adds the
// slots from its own shared memory, in rank order.  One cluster barrier per
// column: right after a column's update each CTA publishes, for the next
// column x (pivot row p), |x below p|^2 and S_k = sum_{r > p} x_r A[r, k]
// for the columns k right of it, and the owner of row p publishes that row;
// with v = x / v0 below the pivot (v_p = 1) the reflector's v^T A is then
// A[p, k] + S_k / v0, formed by every CTA after the barrier.  The slots
// alternate between two sets (column parity).
__global__ void __launch_bounds__(QT, 1) qr_block_k(QrArgs a)
{
    extern __shared__ float qrows[];          // rpc x (QB + 1): this CTA's rows of the block
    __shared__ float s_sig[2][QCS_MAX];       // partial |x below the pivot|^2, by parity and CTA
    __shared__ float s_S[2][QCS_MAX][QB];     // partial S_k, by parity and CTA
    __shared__ float s_prow[2][QB];           // the pivot row, from its owner
    __shared__ float wpart[QW][QB];           // per-warp partials
    __shared__ float red[QW];
    __shared__ float s_wsum[QB];              // tau v^T A[:, k] of the current column
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int rank = (int)q_rank(), CS = (int)q_nrank();
    const int LD = QB + 1, nb = a.nb;
    const int r0 = a.q0 + rank * a.rpc;
    const int nr = max(0, min(a.rpc, a.M - r0));
    for (int t = tid; t < nr * nb; t += QT) {
        const int i = t / nb, k = t % nb;
        qrows[i * LD + k] = a.W[(long)(r0 + i) * a.ldw + a.q0 + k];
    }
    // slots read for columns past the last row (no owner, no rows below) hold 0
    for (int t = tid; t < 2 * QB; t += QT) (&s_prow[0][0])[t] = 0.f;
    for (int t = tid; t < 2 * QCS_MAX * QB; t += QT) (&s_S[0][0][0])[t] = 0.f;
    if (tid < 2 * QCS_MAX) (&s_sig[0][0])[tid] = 0.f;
    q_cluster_sync();  // every CTA of the cluster runs (and has cleared its slots) before the first remote store
    // this CTA's partials of column col into slot set par of every CTA
    auto publish = [&](int col, int par) {
        const int pr = a.q0 + col;
        float accs = 0.f, acc0 = 0.f, acc1 = 0.f;
        for (int i = warp; i < nr; i += QW) {
            const int r = r0 + i;
            if (r <= pr) continue;
            const float x = qrows[i * LD + col];
            if (lane == 0) accs += x * x;
            const int k0 = col + 1 + lane, k1 = col + 33 + lane;
            if (k0 < nb) acc0 += x * qrows[i * LD + k0];
            if (k1 < nb) acc1 += x * qrows[i * LD + k1];
        }
        wpart[warp][lane] = acc0;
        wpart[warp][lane + 32] = acc1;
        const float sig = q_block_sum(accs, red);  // its barriers also publish wpart
        const int kn = nb - col - 1;
        if (tid < kn) {
            float t = 0.f;
#pragma unroll
            for (int w = 0; w < QW; w++) t += wpart[w][tid];
            for (int c = 0; c < CS; c++) q_st(q_dsmem(&s_S[par][rank][col + 1 + tid], c), t);
        }
        if (tid < CS) q_st(q_dsmem(&s_sig[par][rank], tid), sig);
        if (pr >= r0 && pr < r0 + nr) {
            const int i = pr - r0, w = nb - col;
            for (int t = tid; t < w * CS; t += QT) {
                const int k = col + t % w, c = t / w;
                q_st(q_dsmem(&s_prow[par][k], c), qrows[i * LD + k]);
            }
        }
    };
    publish(0, 0);
    for (int j = 0; j < nb; j++) {
        const int par = j & 1, pr = a.q0 + j;  // pivot row
        q_cluster_sync();                      // every CTA's partials of column j are in place
        float sig = 0.f;
#pragma unroll
        for (int c = 0; c < QCS_MAX; c++) sig += (c < CS) ? s_sig[par][c] : 0.f;
        float beta, tau, v0;
        make_reflector(s_prow[par][j], sig, a.M - pr, &beta, &tau, &v0);
        const float inv = 1.f / v0;
        const int kn = nb - j - 1;
        if (tid < kn) {
            const int k = j + 1 + tid;
            float S = 0.f;
#pragma unroll
            for (int c = 0; c < QCS_MAX; c++) S += (c < CS) ? s_S[par][c][k] : 0.f;
            s_wsum[k] = tau * (s_prow[par][k] + S * inv);
        }
        if (tid == 0 && rank == 0) a.tau[j] = tau;  // tau of the block's column j
        __syncthreads();
        // A[r, k] -= tau v_r w_k for the remaining columns, v stored in column j
        for (int i = warp; i < nr; i += QW) {
            const int r = r0 + i;
            if (r < pr) continue;
            const float v = (r == pr) ? 1.f : qrows[i * LD + j] * inv;
            const int k0 = j + 1 + lane, k1 = j + 33 + lane;
            if (k0 < nb) qrows[i * LD + k0] -= v * s_wsum[k0];
            if (k1 < nb) qrows[i * LD + k1] -= v * s_wsum[k1];
            __syncwarp();
            if (lane == 0) qrows[i * LD + j] = (r == pr) ? beta : v;
        }
        __syncthreads();
        if (j + 1 < nb) publish(j + 1, par ^ 1);
    }
    __syncthreads();
    for (int t = tid; t < nr * nb; t += QT) {
        const int i = t / nb, k = t % nb;
        a.W[(long)(r0 + i) * a.ldw + a.q0 + k] = qrows[i * LD + k];
    }
    q_cluster_sync();  // no CTA leaves while another may still write into its shared memory
}

// R (N x N, ld N) <- the upper triangle of W[0:N, 0:N]
__global__ void qr_extract_r(const float *__restrict__ W, long ldw, int N, float *__restrict__ R)
{
    const long total = (long)N * N;
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < total; t += (long)gridDim.x * blockDim.x) {
        const long r = t / N, c = t % N;
        R[t] = (c >= r) ? W[r * ldw + c] : 0.f;
    }
}

// U (M x uc, ld uc) <- the first uc columns of blockdiag(UR (N x N, ld N), I)
__global__ void qr_blockdiag(const float *__restrict__ UR, int N, int M, int uc, float *__restrict__ U)
{
    const long total = (long)M * uc;
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < total; t += (long)gridDim.x * blockDim.x) {
        const long r = t / uc, c = t % uc;
        float v;
        if (UR && r < N && c < N) v = UR[r * N + c];
        else v = (r == c) ? 1.f : 0.f;
        U[t] = v;
    }
}

struct QrCfg {
    int cs = 0;        // cluster size that can run (16, 8) or 0
    int max_smem = 0;  // dynamic shared memory the kernel may use
};

QrCfg qr_cfg()
{
    static QrCfg cfgs[PACO_MAX_DEVICES];
    static bool done[PACO_MAX_DEVICES] = {};
    const int devi = paco_device();
    QrCfg &cfg = cfgs[devi];
    if (done[devi]) return cfg;
    done[devi] = true;
    int dev = 0, optin = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess) {
        cudaGetLastError();
        return cfg;
    }
    const int smem = optin - 16384;  // room for the static shared memory
    if (cudaFuncSetAttribute(qr_block_k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess ||
        cudaFuncSetAttribute(qr_block_k, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) {
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
        lc.blockDim = dim3(QT);
        lc.dynamicSmemBytes = smem;
        lc.attrs = at;
        lc.numAttrs = 1;
        int n = 0;
        if (cudaOccupancyMaxActiveClusters(&n, qr_block_k, &lc) == cudaSuccess && n >= 1) {
            cfg.cs = cs;
            cfg.max_smem = smem;
            break;
        }
        cudaGetLastError();
    }
    return cfg;
}

size_t qr_smem_bytes(int rows, int cs)
{
    const int rpc = (rows + cs - 1) / cs;
    return sizeof(float) * (size_t)rpc * (QB + 1);
}

}  // namespace

void qr_init() { (void)qr_cfg(); }

bool qr_fits(int M, int N)
{
    const QrCfg cfg = qr_cfg();
    return cfg.cs > 0 && N >= 1 && M >= N && qr_smem_bytes(M, cfg.cs) <= (size_t)cfg.max_smem;
}

// QR of the block of nb <= QB columns at q0 of W, rows [q0, M), in place
// (R on and above the diagonal, the reflectors below); tau[0, nb) its scalars.
int qr_panel(float *W, long ldw, int M, int q0, int nb, float *tau, cudaStream_t s, bool small)
{
    const QrCfg cfg = qr_cfg();
    const int rows = M - q0;
    if (cfg.cs <= 0 || nb < 1 || nb > QB || rows < 1 || qr_smem_bytes(rows, cfg.cs) > (size_t)cfg.max_smem)
        return PACO_ERR_UNSUPPORTED;
    // small: the smallest cluster (down to one CTA) that keeps at most 256
    // rows per CTA; fewer CTAs make the two cluster barriers per column cheaper
    int cs = cfg.cs;
    while (small && cs > 1 && rows <= (cs / 2) * 256) cs /= 2;
    QrArgs a;
    a.W = W; a.ldw = ldw; a.M = M; a.q0 = q0; a.nb = nb;
    a.rpc = (rows + cs - 1) / cs;
    a.tau = tau;
    cudaLaunchConfig_t lc = {};
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = cs;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    lc.gridDim = dim3(cs);
    lc.blockDim = dim3(QT);
    lc.dynamicSmemBytes = qr_smem_bytes(rows, cs);
    lc.stream = s;
    lc.attrs = at;
    lc.numAttrs = 1;
    paco_count_launch();
    if (cudaLaunchKernelEx(&lc, qr_block_k, a) != cudaSuccess) {
        cudaGetLastError();
        return PACO_ERR_CUDA;
    }
    return PACO_OK;
}

// The columns of W (M x ldw, already holding A) become R (upper triangle) and
// the Householder vectors (below the diagonal); tau[N] receives the scalars.
int qr_factor(const BdWs &w, int M, int N, float *tau, cudaStream_t s, int qb)
{
    if (!qr_fits(M, N)) return PACO_ERR_UNSUPPORTED;
    qb = (qb == 32) ? 32 : QB;
    for (int q0 = 0; q0 < N; q0 += qb) {
        const int nb = std::min(qb, N - q0), rows = M - q0;
        const int rc = qr_panel(w.W, w.ldw, M, q0, nb, tau + q0, s);
        if (rc) return rc;
        const int q1 = q0 + nb;
        if (q1 < N) {
            bd_column_vectors(w.W, w.ldw, q0, nb, rows, w.Vp, s);
            if (apply_block_reflector_ex(w, w.W, w.ldw, q0, rows, q1, N - q1, nb, tau + q0, true, s) != cudaSuccess)
                return PACO_ERR_CUDA;
        }
    }
    return cudaGetLastError() == cudaSuccess ? PACO_OK : PACO_ERR_CUDA;
}

void qr_extract_r_launch(const BdWs &w, int N, float *R, cudaStream_t s)
{
    paco_count_launch(), qr_extract_r<<<std::min(8192, ceil_div((long)N * N, 256)), 256, 0, s>>>(w.W, w.ldw, N, R);
}

// U (M x uc, ld uc; uc = M, or N for the thin U) <- the first uc columns of
// Q blockdiag(UR, I), Q = H_0 ... H_{N-1} from qr_factor
int qr_form_u(const BdWs &w, int M, int N, const float *tau, const float *UR, float *U, cudaStream_t s, int uc,
              int nbf)
{
    if (uc <= 0) uc = M;
    nbf = (nbf == 64) ? 64 : bd::NBF;
    paco_count_launch(), qr_blockdiag<<<std::min(8192, ceil_div((long)M * uc, 256)), 256, 0, s>>>(UR, N, M, uc, U);
    for (int p0 = ((N - 1) / nbf) * nbf; p0 >= 0; p0 -= nbf) {
        const int nbp = std::min(N, p0 + nbf) - p0, Lp = M - p0;
        bd_column_vectors(w.W, w.ldw, p0, nbp, Lp, w.Vp, s);
        if (apply_block_reflector_ex(w, U, uc, p0, Lp, 0, uc, nbp, tau + p0, false, s) != cudaSuccess)
            return PACO_ERR_CUDA;
    }
    return cudaGetLastError() == cudaSuccess ? PACO_OK : PACO_ERR_CUDA;
}
