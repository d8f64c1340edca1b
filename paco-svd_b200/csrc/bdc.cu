// Stage 2: bidiagonal divide and conquer (BDC) of the N x N upper bidiagonal
// (d, e) produced by stage 1, then U[:, :N] <- U[:, :N] Q and Vt <- W^T Vt.
//
// Reference: svd.cpp (DEAVEN-MITCH/paco-svd), a LAPACK sbdsdc/slasd1-4 style
// solver that runs on one vector core: 3-column leaves (svd.cpp:1596-1864,
// partition svd_tiling.cpp:83-130), bottom-up pairwise merges with the odd
// tail carried (svd.cpp:168-189), each merge = scale (:225-323), deflation
// (:325-975), secular roots (:977-1336), Loewner z and vectors
// (:1337-1496), back-transform matmul (:1498-1521), idxq sort (:1523-1590);
// then a descending sort (:1866-1909) and the U/Vt update (:1911-1981).
//
// Here every merge of a tree level is processed at once, one kernel per
// phase:
//   prepare   (CTA per merge)  scale, z, merge of the two sorted runs,
//                              FP64 deflation scan -> rotation list
//   rotate    (column-parallel) Givens rotations of the qt/wt rows
//   gather    (2-D)            permuted copies into st/gt
//   secular   (warp per root)  FP64 bracketed rational iteration
//   lowner    (thread per z)   Gu-Eisenstat z recomputed in FP64
//   vectors   (warp per root)  normalized singular vectors of the secular problem
//   copyback  (2-D)            deflated rows back into qt/wt
//   btgemm    (128x128 tiles)  qt[0:k] = Us st[0:k], wt[0:k] = Vs gt[0:k]
//   finalize  (CTA per merge)  f/l, idxq (merge of two sorted runs), unscale
// Fixes relative to the reference (kept in the CPU restatement too): leaves
// are solved with sign-consistent rotations, k == 2 takes the general
// secular path, the all-deflated case keeps d sorted, orgnrm == 0 skips the
// scaling, and the final order is a full descending sort.
#include <vector>

#include "bdc_dev.cuh"

// merges at least this large take their back-transform on the tensor cores
#define BDC_TC_MIN_N 256

// --------------------------------------------------------------- kernels

__global__ void bdc_schedule(int N, const uint8_t *tiling, BdcWs w)
{
    if (threadIdx.x == 0 && blockIdx.x == 0) bdc_schedule_dev(N, tiling, w, nullptr, nullptr);
}

struct HostMerge {
    int s, n, nc;
};

struct HostLevel {
    int off, nm, max_n, max_nc;
    std::vector<HostMerge> merges;
};

static int host_schedule(int N, std::vector<HostLevel> &lv)
{
    int nleaf = leaf_partition(N, nullptr, nullptr);
    std::vector<int> s(nleaf), e(nleaf);
    leaf_partition(N, s.data(), e.data());
    int cnt = nleaf, out = 0;
    while (cnt > 1) {
        HostLevel L{out, 0, 0, 0, {}};
        int wpos = 0, r = 0;
        while (r < cnt - 1) {
            int ms = s[r], me = e[r + 1];
            int sq = (me == N);
            int n = me - ms - 1 + sq, nc = me - ms;
            L.nm++; L.max_n = std::max(L.max_n, n); L.max_nc = std::max(L.max_nc, nc);
            L.merges.push_back({ms, n, nc});
            out++;
            s[wpos] = ms; e[wpos] = me; wpos++;
            r += 2;
        }
        if (r == cnt - 1) { s[wpos] = s[r]; e[wpos] = e[r]; wpos++; }
        cnt = wpos;
        lv.push_back(L);
    }
    return nleaf;
}

// one thread per leaf
__global__ void bdc_leaves(int N, int nleaf, BdcWs w, float *d, const float *e, float *QT, float *WT, int *idxq,
                           float *fv, float *lv)
{
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < nleaf) bdc_leaf_dev(t, N, w, d, e, QT, WT, idxq, fv, lv);
}

__global__ void __launch_bounds__(256) bdc_prepare(LevelArgs A)
{
    extern __shared__ __align__(16) unsigned char sm[];
    bdc_prepare_dev(A, blockIdx.x, sm);
}

__global__ void bdc_rotate(LevelArgs A)
{
    bdc_rotate_dev(A, blockIdx.y, blockIdx.x * blockDim.x + threadIdx.x);
}

__global__ void bdc_gather(LevelArgs A)
{
    bdc_gather_dev(A, blockIdx.z, blockIdx.x * blockDim.x + threadIdx.x, blockIdx.y * GATHER_ROWS,
                   (blockIdx.y + 1) * GATHER_ROWS);
}

__global__ void bdc_copyback(LevelArgs A)
{
    bdc_copyback_dev(A, blockIdx.z, blockIdx.x * blockDim.x + threadIdx.x, blockIdx.y * GATHER_ROWS,
                     (blockIdx.y + 1) * GATHER_ROWS);
}

__global__ void __launch_bounds__(256) bdc_secular(LevelArgs A, int nm)
{
    bdc_secular_dev<32>(A, nm, (blockIdx.x * blockDim.x + threadIdx.x) >> 5, threadIdx.x & 31, 0, 0x7fffffff);
}

__global__ void __launch_bounds__(256) bdc_lowner(LevelArgs A, int nm)
{
    bdc_lowner_dev<32>(A, nm, (blockIdx.x * blockDim.x + threadIdx.x) >> 5, threadIdx.x & 31, 0, 0x7fffffff);
}

__global__ void __launch_bounds__(256) bdc_vectors(LevelArgs A, int nm)
{
    bdc_vectors_dev<32>(A, nm, (blockIdx.x * blockDim.x + threadIdx.x) >> 5, threadIdx.x & 31, 0, 0x7fffffff);
}

// merges with n >= skip_n are multiplied on the tensor cores instead
__global__ void __launch_bounds__(256) bdc_btgemm(LevelArgs A, int tiles_n, int skip_n)
{
    if (A.w.meta[A.w.mg_s[A.off + blockIdx.z]].n >= skip_n) return;
    bdc_btgemm_dev(A, blockIdx.z, blockIdx.y, blockIdx.x / tiles_n, blockIdx.x % tiles_n);
}

__global__ void __launch_bounds__(256) bdc_finalize(LevelArgs A)
{
    bdc_finalize_dev(A, blockIdx.x);
}

// ------------------------------------------------------------ final stage

__global__ void __launch_bounds__(256) bdc_sort_desc(int N, const float *d, int *perm, float *sig)
{
    bdc_rank_desc_dev(N, d, perm, sig, blockIdx.x * blockDim.x);
}

__global__ void bdc_init_qw(float *QT, float *WT, int N)
{
    long total = (long)N * N;
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < total; t += (long)gridDim.x * blockDim.x) {
        float v = (t / N == t % N) ? 1.f : 0.f;
        QT[t] = v;
        WT[t] = v;
    }
}

__global__ void bdc_copy_cols(const float *src, long lds, float *dst, long ldd, int rows, int cols)
{
    long total = (long)rows * cols;
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < total; t += (long)gridDim.x * blockDim.x) {
        long r = t / cols, c = t % cols;
        dst[r * ldd + c] = src[r * lds + c];
    }
}

__global__ void bdc_copy_vec(const float *src, float *dst, int n)
{
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) dst[t] = src[t];
}

// ------------------------------------------------------------- host driver

size_t bdc_workspace_bytes(int M, int N)
{
    BdcWs w;
    return bdc_carve(nullptr, M, N, &w);
}

static bool bdc_attrs_set[PACO_MAX_DEVICES] = {};

// Sets this unit's secular iteration limit (a test hook; synchronous).
void bdc_set_sec_maxit(int n)
{
    cudaMemcpyToSymbol(g_sec_maxit, &n, sizeof(int));
}

void bdc_init_attrs()
{
    const int dev = paco_device();
    if (!bdc_attrs_set[dev]) {
        cudaFuncSetAttribute(bdc_prepare, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
        gemm_tc_init_attrs();
        bdc_attrs_set[dev] = true;
    }
}

int bdc_run(int M, int N, float *a, float *u, float *vt, float *d, float *e, float *qt, float *wt, uint32_t *idx,
            void *workspace, const uint8_t *tiling, cudaStream_t s, long ldu)
{
    const long lu = ldu > 0 ? ldu : M;
    BdcWs w;
    bdc_carve(workspace, M, N, &w);
    bdc_init_attrs();
    if (!paco_tune_for(M, N).tc) w.tcs = nullptr;
    std::vector<HostLevel> lv;
    const int nleaf = host_schedule(N, lv);
    LevelArgs A;
    A.N = N; A.off = 0; A.d_e = e; A.d = d;
    A.QT = qt; A.ST = qt + (size_t)N * N; A.WT = wt; A.GT = wt + (size_t)N * N;
    int *ib = (int *)idx;
    A.idxq = ib; A.f = (float *)(ib + N); A.l = (float *)(ib + 2 * N); A.dsig = (float *)(ib + 3 * N);
    A.zhat = (float *)(ib + 4 * N); A.srow = ib + 5 * N;
    A.diff = a;
    A.w = w;

    paco_count_launch(), bdc_schedule<<<1, 32, 0, s>>>(N, tiling, w);
    paco_count_launch(), bdc_init_qw<<<std::min(8192, ceil_div((long)N * N, 256)), 256, 0, s>>>(qt, wt, N);
    paco_count_launch(), bdc_leaves<<<ceil_div(nleaf, 128), 128, 0, s>>>(N, nleaf, w, d, e, A.QT, A.WT, A.idxq, A.f, A.l);
    for (const HostLevel &L : lv) {
        A.off = L.off;
        const int dn = L.max_n - 1;
        size_t smem = (size_t)dn * (8 + 4 + 4 + 4) + 64;
        paco_count_launch(), bdc_prepare<<<L.nm, 256, smem, s>>>(A);
        paco_count_launch(), bdc_rotate<<<dim3(ceil_div(L.max_nc, 128), L.nm), 128, 0, s>>>(A);
        dim3 g2(ceil_div(L.max_nc, 128), ceil_div(L.max_nc, GATHER_ROWS), L.nm);
        paco_count_launch(), bdc_gather<<<g2, 128, 0, s>>>(A);
        paco_count_launch(), bdc_secular<<<ceil_div((long)N * 32, 256), 256, 0, s>>>(A, L.nm);
        paco_count_launch(), bdc_lowner<<<ceil_div((long)N * 32, 256), 256, 0, s>>>(A, L.nm);
        paco_count_launch(), bdc_vectors<<<ceil_div((long)N * 32, 256), 256, 0, s>>>(A, L.nm);
        paco_count_launch(), bdc_copyback<<<g2, 128, 0, s>>>(A);
        int tiles_n = ceil_div(L.max_nc, 128);
        // back-transforms of large merges on the tensor cores, limited on the
        // device to the merge's k (rows beyond k hold deflated vectors)
        int skip_n = 0x7fffffff;
        if (w.tcs && L.max_n >= BDC_TC_MIN_N) {
            bool fits = true;
            for (const HostMerge &g : L.merges)
                if (g.n >= BDC_TC_MIN_N && gemm_tc_scratch_floats(g.n, g.nc, g.n) > w.tcs_floats) fits = false;
            if (fits) skip_n = BDC_TC_MIN_N;
        }
        paco_count_launch(), bdc_btgemm<<<dim3(tiles_n * ceil_div(L.max_n, 128), 2, L.nm), 256, 0, s>>>(A, tiles_n,
                                                                                                      skip_n);
        if (skip_n != 0x7fffffff) {
            for (const HostMerge &g : L.merges) {
                if (g.n < skip_n) continue;
                const long off = (long)g.s * N + g.s;
                const int *kd = &w.meta[g.s].k;
                gemm_tc_run(g.n, g.n, g.n, 1.f, gop(w.Us + off, N, 1), gop(A.ST + off, N, 1), 0.f, A.QT + off, N,
                            w.tcs, w.st, s, kd);
                gemm_tc_run(g.n, g.nc, g.n, 1.f, gop(w.Vs + off, N, 1), gop(A.GT + off, N, 1), 0.f, A.WT + off, N,
                            w.tcs, w.st, s, kd);
            }
        }
        paco_count_launch(), bdc_finalize<<<L.nm, 256, 0, s>>>(A);
    }
    paco_count_launch(), bdc_sort_desc<<<ceil_div(N, 256), 256, 0, s>>>(N, d, w.perm, w.sig);
    // U[:, :N] <- U[:, :N] Q with Q(:, r) = qt row perm[r]; result staged in a (M x N)
    gemm_any(M, N, N, 1.f, gop(u, lu, 1), gop(qt, 1, N, w.perm), 0.f, a, N, 1, nullptr, w.tcs, w.tcs_floats, w.st, s);
    paco_count_launch(), bdc_copy_cols<<<std::min(8192, ceil_div((long)M * N, 256)), 256, 0, s>>>(a, N, u, lu, M, N);
    // Vt <- W^T Vt with W^T row r = wt row perm[r]; staged in Us
    gemm_any(N, N, N, 1.f, gop(wt, N, 1, w.perm), gop(vt, N, 1), 0.f, w.Us, N, 1, nullptr, w.tcs, w.tcs_floats, w.st,
             s);
    paco_count_launch(), bdc_copy_cols<<<std::min(8192, ceil_div((long)N * N, 256)), 256, 0, s>>>(w.Us, N, vt, N, N, N);
    paco_count_launch(), bdc_copy_vec<<<ceil_div(N, 256), 256, 0, s>>>(w.sig, d, N);
    return cudaGetLastError() == cudaSuccess ? PACO_OK : PACO_ERR_CUDA;
}
