// Tail of the stage-1 bidiagonalization on one thread-block cluster.
//
// Once the trailing block A[p:, p:] (m = M - p rows, w = N - p columns) fits
// in the shared memory of a cluster of CS CTAs, its column steps no longer
// need the whole GPU: the cluster runs them unblocked, as the reference loop
// does (upper_bidiagonalization.cpp:182-218, reflectors of :189-216), with one
// cluster barrier per step instead of two grid barriers.  Tail row r lives in
// the shared memory of CTA r % CS for all remaining steps.  Step i:
//   every CTA  reads through distributed shared memory the CTAs' sums of the
//              previous sweep (sigma = |x[1:]|^2 and S_c = sum_r x_r a_rc over
//              the rows r > i, x = column i) and the pivot row i from its
//              owner, and forms the column reflector (beta, tauq, v0),
//              w_c = a_ic + S_c / v0, the left-updated pivot row
//              r_c = a_ic - tauq w_c and its row reflector (e, taup, u): the
//              same inputs in the same order in every CTA
//   sweep      each warp takes whole rows r > i (lane l holds columns
//              l + 32 j): v_r = a_ri / v0 goes to W as the column reflector's
//              entry, a_rc -= tauq v_r w_c, a_rc -= taup (a_r . u) u_c, and the
//              sums of the next step are accumulated (x_r = a_r,i+1, r > i+1)
// A CTA adds its warps' sums in a fixed order into a double-buffered partial
// that the next step's barrier publishes.  W receives the reflectors in the
// layout of the panel path (column vectors below the diagonal, row vectors
// right of the superdiagonal, implicit ones not stored), d/e/tauq/taup and
// 1/v0 of every reflector.
#include "bidiag.cuh"
#include "tma.cuh"

using namespace bd;

namespace {

constexpr int TT = 512, TW = TT / 32;  // threads and warps per CTA
constexpr int TAIL_NA = 24;            // 32-column chunks a lane can hold: w <= 768

struct TailArgs {
    float *W;  // the working matrix (tail origin at W + p * ldw + p)
    long ldw;
    int p, m, w, w4, own_max;
    float *d, *e, *tauq, *taup, *inv_v0c, *inv_v0r;
};

struct TailSh {
    float *rows;   // own_max x w4: this CTA's rows (tail columns 0 .. w-1)
    float *wpart;  // TW x w4: per-warp sums of the current sweep
    float *part;   // 2 x w4: the CTA's sums, by step parity
    float *wv, *uv, *rv;
};

__host__ __device__ inline size_t tail_smem_floats(int own_max, int w4) { return (size_t)(own_max + TW + 5) * w4; }

// All threads of all CTAs of the cluster; called with converged warps.
__device__ __forceinline__ void cluster_sync_all()
{
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}

// The same shared-memory word in CTA `rank` of the cluster.
__device__ __forceinline__ uint32_t dsmem_addr(const void *local, int rank)
{
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(smem_u32(local)), "r"(rank));
    return r;
}

// Ordered after the cluster barrier by that barrier's own memory clobber;
// independent loads stay free to overlap.
__device__ __forceinline__ float ld_dsmem(uint32_t addr)
{
    float v;
    asm volatile("ld.shared::cluster.f32 %0, [%1];" : "=f"(v) : "r"(addr));
    return v;
}

__device__ __forceinline__ void tail_reflector(float x0, float sigma, int len, float *beta, float *tau, float *v0)
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

// Sweep of this CTA's rows r > max(ci, -1) over the chunks q0 .. q0+NA-1.
// UPDATE: apply the step-ci reflectors first (column ci lies in chunk q0).
// Then accumulate the next step's sums (column cn = ci + 1, rows r > cn)
// into the warp's row of wpart (columns > cn) and ssig_w.
template <bool UPDATE, int NA>
__device__ void tail_sweep(const TailSh &sh, const TailArgs &t, int rank, int CS, int ci, float inv_v0, float tq,
                           float tp, float *ssig_w)
{
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int q0 = ci < 0 ? 0 : ci >> 5;
    const int cn = ci + 1;
    const int w = t.w;
    const bool cn_hi = (cn >> 5) > q0;
    float acc[NA];
#pragma unroll
    for (int j = 0; j < NA; j++) acc[j] = 0.f;
    float ssig = 0.f;
    // local rows k with tail row rank + k*CS > ci
    const int kfirst = (ci >= rank) ? (ci - rank) / CS + 1 : 0;
    int own = (t.m - rank + CS - 1) / CS;
    if (own < 0) own = 0;
    float *Wt = t.W + (long)t.p * t.ldw + t.p;
    for (int k = kfirst + warp; k < own; k += TW) {
        const int rl = rank + k * CS;
        float *row = sh.rows + (long)k * t.w4;
        float a[NA];
#pragma unroll
        for (int j = 0; j < NA; j++) {
            const int c = 32 * (q0 + j) + lane;
            a[j] = (c >= ci && c < w) ? row[c] : 0.f;
        }
        if (UPDATE) {
            const float x = __shfl_sync(0xffffffffu, a[0], ci & 31);
            const float vr = x * inv_v0;
            if (lane == (ci & 31)) Wt[(long)rl * t.ldw + ci] = vr;
            const float lf = tq * vr;
            float dot = 0.f;
#pragma unroll
            for (int j = 0; j < NA; j++) {
                const int c = 32 * (q0 + j) + lane;
                if (c > ci && c < w) {
                    a[j] -= lf * sh.wv[c];
                    dot += a[j] * sh.uv[c];
                }
            }
            dot = warp_sum(dot) * tp;
#pragma unroll
            for (int j = 0; j < NA; j++) {
                const int c = 32 * (q0 + j) + lane;
                if (c > ci && c < w) {
                    a[j] -= dot * sh.uv[c];
                    row[c] = a[j];
                }
            }
        }
        if (cn < w && rl > cn) {
            float xs = a[0];
            if (NA > 1 && cn_hi) xs = a[NA > 1 ? 1 : 0];
            const float xn = __shfl_sync(0xffffffffu, xs, cn & 31);
            ssig += xn * xn;
#pragma unroll
            for (int j = 0; j < NA; j++) {
                const int c = 32 * (q0 + j) + lane;
                if (c > cn) acc[j] += xn * a[j];
            }
        }
    }
#pragma unroll
    for (int j = 0; j < NA; j++) {
        const int c = 32 * (q0 + j) + lane;
        if (c < w) sh.wpart[warp * t.w4 + c] = acc[j];
    }
    if (lane == 0) ssig_w[warp] = ssig;
}

template <bool UPDATE>
__device__ void tail_sweep_any(const TailSh &sh, const TailArgs &t, int rank, int CS, int ci, float inv_v0, float tq,
                               float tp, float *ssig_w)
{
    const int q0 = ci < 0 ? 0 : ci >> 5;
    const int na = ((t.w - 1) >> 5) - q0 + 1;
#define TAIL_CASE(K) \
    case K: tail_sweep<UPDATE, K>(sh, t, rank, CS, ci, inv_v0, tq, tp, ssig_w); break;
    switch (na) {
        TAIL_CASE(1) TAIL_CASE(2) TAIL_CASE(3) TAIL_CASE(4) TAIL_CASE(5) TAIL_CASE(6)
        TAIL_CASE(7) TAIL_CASE(8) TAIL_CASE(9) TAIL_CASE(10) TAIL_CASE(11) TAIL_CASE(12)
        TAIL_CASE(13) TAIL_CASE(14) TAIL_CASE(15) TAIL_CASE(16) TAIL_CASE(17) TAIL_CASE(18)
        TAIL_CASE(19) TAIL_CASE(20) TAIL_CASE(21) TAIL_CASE(22) TAIL_CASE(23) TAIL_CASE(24)
        default: break;
    }
#undef TAIL_CASE
}

// The CTA's sums of the sweep just done (columns > cn) into part[par].
__device__ __forceinline__ void tail_reduce(const TailSh &sh, const TailArgs &t, int cn, int par, const float *ssig_w,
                                            float *sig_cta)
{
    for (int c = cn + 1 + (int)threadIdx.x; c < t.w; c += TT) {
        float s = 0.f;
#pragma unroll
        for (int q = 0; q < TW; q++) s += sh.wpart[q * t.w4 + c];
        sh.part[par * t.w4 + c] = s;
    }
    if (threadIdx.x == 0) {
        float s = 0.f;
#pragma unroll
        for (int q = 0; q < TW; q++) s += ssig_w[q];
        sig_cta[par] = s;
    }
}

}  // namespace

__global__ void __launch_bounds__(TT, 1) bd_tail_k(TailArgs t, int CS)
{
    extern __shared__ __align__(16) float tail_sm[];
    __shared__ float ssig_w[TW], sig_cta[2], s_sig[32], s_x0;
    const int tid = threadIdx.x, lane = tid & 31;
    const int rank = blockIdx.x;  // the grid is one cluster
    TailSh sh;
    sh.rows = tail_sm;
    sh.wpart = sh.rows + (size_t)t.own_max * t.w4;
    sh.part = sh.wpart + (size_t)TW * t.w4;
    sh.wv = sh.part + 2 * (size_t)t.w4;
    sh.uv = sh.wv + t.w4;
    sh.rv = sh.uv + t.w4;
    const int w = t.w, m = t.m;
    float *Wt = t.W + (long)t.p * t.ldw + t.p;

    // this CTA's rows, in from W
    const int own = max(0, (m - rank + CS - 1) / CS);
    for (long q = tid; q < (long)own * t.w4; q += TT) {
        const int k = (int)(q / t.w4), c = (int)(q % t.w4);
        sh.rows[q] = (c < w) ? Wt[(long)(rank + k * CS) * t.ldw + c] : 0.f;
    }
    __syncthreads();
    tail_sweep_any<false>(sh, t, rank, CS, -1, 0.f, 0.f, 0.f, ssig_w);
    __syncthreads();
    tail_reduce(sh, t, 0, 0, ssig_w, sig_cta);

    for (int i = 0; i < w; i++) {
        const int par = i & 1;
        __syncthreads();     // converged warps for the aligned cluster barrier
        cluster_sync_all();  // every CTA's sums of column i and the pivot row i are in place
        const int owner = i % CS;
        const float *prow = sh.rows + (long)(i / CS) * t.w4;  // pivot row in its owner
        if (tid < CS) s_sig[tid] = ld_dsmem(dsmem_addr(&sig_cta[par], tid));
        if (tid == 32) s_x0 = ld_dsmem(dsmem_addr(prow + i, owner));
        __syncthreads();
        float sig = 0.f;
        for (int q = 0; q < CS; q++) sig += s_sig[q];
        const float x0 = s_x0;
        float beta, tq, v0;
        tail_reflector(x0, sig, m - i, &beta, &tq, &v0);
        const float inv_v0 = 1.f / v0;
        for (int c = i + 1 + tid; c < w; c += TT) {
            // all remote loads in flight before the first add
            float v[16];
#pragma unroll
            for (int q = 0; q < 16; q++) v[q] = (q < CS) ? ld_dsmem(dsmem_addr(sh.part + par * t.w4 + c, q)) : 0.f;
            const float aic = ld_dsmem(dsmem_addr(prow + c, owner));
            float S = 0.f;
#pragma unroll
            for (int q = 0; q < 16; q++) S += v[q];
            const float wj = aic + inv_v0 * S;
            sh.wv[c] = wj;
            sh.rv[c] = aic - tq * wj;
        }
        __syncthreads();
        if (rank == 0 && tid == 0) {
            t.d[t.p + i] = beta;
            t.tauq[t.p + i] = tq;
            t.inv_v0c[t.p + i] = inv_v0;
            Wt[(long)i * t.ldw + i] = beta;
        }
        float tp = 0.f;
        if (i < w - 1) {
            // every warp sums the same values in the same order
            float rs = 0.f;
            for (int c = i + 2 + lane; c < w; c += 32) rs += sh.rv[c] * sh.rv[c];
            rs = warp_sum(rs);
            float eb, v0r;
            tail_reflector(sh.rv[i + 1], rs, w - i - 1, &eb, &tp, &v0r);
            const float inv_r = 1.f / v0r;
            for (int c = i + 1 + tid; c < w; c += TT) {
                const float u = (c == i + 1) ? 1.f : sh.rv[c] * inv_r;
                sh.uv[c] = u;
                if (rank == 0) Wt[(long)i * t.ldw + c] = (c == i + 1) ? eb : u;
            }
            if (rank == 0 && tid == 0) {
                t.e[t.p + i] = eb;
                t.taup[t.p + i] = tp;
                t.inv_v0r[t.p + i] = inv_r;
            }
        }
        __syncthreads();
        tail_sweep_any<true>(sh, t, rank, CS, i, inv_v0, tq, tp, ssig_w);
        __syncthreads();
        tail_reduce(sh, t, i + 1, par ^ 1, ssig_w, sig_cta);
    }
    // no CTA leaves while another may still read its shared memory
    __syncthreads();
    cluster_sync_all();
}

// ------------------------------------------------------------------ host

namespace {
struct TailCfg {
    int cs = 0;        // cluster size that can run (16, 8) or 0
    int max_smem = 0;  // dynamic shared memory the kernel may use
};

TailCfg tail_cfg()
{
    static TailCfg cfgs[PACO_MAX_DEVICES];
    static bool done[PACO_MAX_DEVICES] = {};
    const int devi = paco_device();
    TailCfg &cfg = cfgs[devi];
    if (done[devi]) return cfg;
    done[devi] = true;
    int dev = 0, optin = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess) {
        cudaGetLastError();
        return cfg;
    }
    const int smem = optin - 2048;  // room for the static shared memory
    if (cudaFuncSetAttribute(bd_tail_k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess ||
        cudaFuncSetAttribute(bd_tail_k, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) {
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
        lc.blockDim = dim3(TT);
        lc.dynamicSmemBytes = smem;
        lc.attrs = at;
        lc.numAttrs = 1;
        int n = 0;
        if (cudaOccupancyMaxActiveClusters(&n, bd_tail_k, &lc) == cudaSuccess && n >= 1) {
            cfg.cs = cs;
            cfg.max_smem = smem;
            break;
        }
        cudaGetLastError();
    }
    return cfg;
}

bool tail_fits(const TailCfg &cfg, int m, int w)
{
    if (cfg.cs == 0 || w < 1 || w > 32 * TAIL_NA) return false;
    const int w4 = (w + 3) & ~3;
    const int own_max = (m + cfg.cs - 1) / cfg.cs;
    return tail_smem_floats(own_max, w4) * sizeof(float) <= (size_t)cfg.max_smem;
}
}  // namespace

// Called outside stream capture first (the set-up queries the device).
void bd_tail_init() { (void)tail_cfg(); }

int bd_tail_start(int M, int N)
{
    static int env = -1;
    if (env < 0) {
        const char *v = getenv("PACO_TAIL");
        env = (v && v[0] == '0') ? 0 : 1;
    }
    if (!env) return N;
    const TailCfg cfg = tail_cfg();
    // the first panel boundary from which the rest fits in the cluster
    for (int p = 0; p < N; p += NB)
        if (tail_fits(cfg, M - p, N - p)) return p;
    return N;
}

bool bd_tail_launch(const BdArgs &a, int p, cudaStream_t s)
{
    const TailCfg cfg = tail_cfg();
    const int m = a.M - p, w = a.N - p;
    if (!tail_fits(cfg, m, w)) return false;
    TailArgs t;
    t.W = a.W;
    t.ldw = a.ldw;
    t.p = p;
    t.m = m;
    t.w = w;
    t.w4 = (w + 3) & ~3;
    t.own_max = (m + cfg.cs - 1) / cfg.cs;
    t.d = a.d; t.e = a.e; t.tauq = a.tauq; t.taup = a.taup;
    t.inv_v0c = a.inv_v0c; t.inv_v0r = a.inv_v0r;
    cudaLaunchConfig_t lc = {};
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = cfg.cs;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    lc.gridDim = dim3(cfg.cs);
    lc.blockDim = dim3(TT);
    lc.dynamicSmemBytes = tail_smem_floats(t.own_max, t.w4) * sizeof(float);
    lc.stream = s;
    lc.attrs = at;
    lc.numAttrs = 1;
    paco_count_launch();
    if (cudaLaunchKernelEx(&lc, bd_tail_k, t, cfg.cs) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return true;
}
