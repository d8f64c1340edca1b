// FP32 GEMM on the 5th-generation tensor cores (tcgen05, sm_100a), accurate
// to about FP32 through a 3xTF32 split:  x = x_hi + x_lo with x_hi, x_lo TF32,
//     A*B ~= A_lo*B_hi + A_hi*B_lo + A_hi*B_hi      (FP32 accumulation in TMEM)
//
// tc_pack  rounds one operand into its hi/lo TF32 parts and writes them as
//          ready-made shared-memory tile images: 128 rows x 32 k, K-major,
//          128-byte swizzle (16-byte chunk c of row r stored at chunk
//          c ^ (r & 7)), so the GEMM kernel moves whole tiles with 1-D bulk
//          copies.  One CTA per image, transposed through shared memory so
//          both the reads and the writes are coalesced.
// tc_gemm  one CTA per 128x128 tile of C (and per k-range with split-K):
//          thread 0 runs a 2-stage pipeline of bulk copies (mbarrier
//          complete_tx) and issues the MMAs (tcgen05.mma.cta_group::1
//          .kind::tf32, M=128, N=128, K=8) into a TMEM accumulator; a
//          tcgen05.commit per stage releases the stage.  The split's k range
//          runs in chains of KCHAIN images: the 4 warps add each finished
//          chain into FP32 sums in TMEM (round-to-nearest; the tensor cores
//          round their own accumulation toward zero).  The C tile is
//          bulk-copied into shared memory while the products run (beta != 0);
//          the 4 warps then read the accumulator with tcgen05.ld, combine it
//          with C in shared memory and the tile leaves by bulk stores, one
//          per row (plain coalesced stores when rows are not 16-byte aligned).
// Every wait is bounded; a wait that gives up records PACO_ERR_TIMEOUT, the
// copies still in flight are waited for (again bounded), the CTA frees its
// tensor memory and returns.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>

#include "gemm_tc.cuh"
#include "tma.cuh"

namespace {

constexpr int TM = 128, TN = 128, TK = 32;  // tile of C; k per image (128 bytes of TF32)
constexpr int IMG = TM * TK;                // floats per tile image (16 KB)
constexpr int STAGES = 2;
constexpr int MAX_SPLITS = 8;
constexpr int KCHAIN = 4;              // k images (of 32) per accumulation chain of a skinny product
constexpr int MAX_CHAIN_SPLITS = 128;
constexpr uint32_t IDESC = (1u << 4)             // D format F32
                           | (2u << 7)           // A format TF32
                           | (2u << 10)          // B format TF32 (both K-major: bits 15, 16 clear)
                           | ((TN >> 3) << 17)   // N >> 3
                           | ((TM >> 4) << 24);  // M >> 4

__device__ __forceinline__ float tf32_round(float x)
{
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}

// Shared-memory matrix descriptor for a K-major, 128-byte-swizzled tile whose
// 8-row groups are 1024 bytes apart (start address 1024-aligned for k = 0).
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr)
{
    uint64_t d = 0;
    d |= (uint64_t)((saddr & 0x3FFFF) >> 4);  // start address >> 4
    d |= (uint64_t)1 << 16;                   // leading byte offset (not used by this layout)
    d |= (uint64_t)(1024 >> 4) << 32;         // stride byte offset >> 4
    d |= (uint64_t)1 << 46;                   // descriptor version 1
    d |= (uint64_t)2 << 61;                   // 128-byte swizzle
    return d;
}

__device__ __forceinline__ void mma_tf32(uint32_t tmem, uint64_t ad, uint64_t bd, uint32_t accum)
{
    const uint32_t z = 0;
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n}\n" ::"r"(tmem),
        "l"(ad), "l"(bd), "r"(IDESC), "r"(accum), "r"(z));
}

__device__ __forceinline__ void mma_commit(uint64_t *bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&v)[32])
{
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
          "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]),
          "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]),
          "=r"(v[30]), "=r"(v[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_st32(uint32_t taddr, const uint32_t (&v)[32])
{
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,"
        "%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31,%32};" ::"r"(taddr),
        "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7]), "r"(v[8]),
        "r"(v[9]), "r"(v[10]), "r"(v[11]), "r"(v[12]), "r"(v[13]), "r"(v[14]), "r"(v[15]), "r"(v[16]),
        "r"(v[17]), "r"(v[18]), "r"(v[19]), "r"(v[20]), "r"(v[21]), "r"(v[22]), "r"(v[23]), "r"(v[24]),
        "r"(v[25]), "r"(v[26]), "r"(v[27]), "r"(v[28]), "r"(v[29]), "r"(v[30]), "r"(v[31])
        : "memory");
    asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
}

struct TcGeom {
    int MT, NT, KT, splits;
};

TcGeom tc_geom(int M, int N, int K)
{
    TcGeom g;
    g.MT = ceil_div(M, TM);
    g.NT = ceil_div(N, TN);
    g.KT = ceil_div(K, TK);
    // as many CTAs as fit one wave on the SMs (a second, partial wave would
    // double the time), at least 4 images of k per split
    const int tiles = g.MT * g.NT, fill = std::max(1, 148 / tiles);
    g.splits = std::max(1, std::min({MAX_SPLITS, fill, g.KT / 4}));
    // The tensor cores round each accumulation into TMEM toward zero, so a
    // long k chain would lose about one ulp of the running sum per MMA: both
    // kernels run a split's k range in chains of KCHAIN (KCP) images whose
    // sums are added in FP32 with round-to-nearest.  Skinny products (one or
    // two row tiles, e.g. V^T Q with k = the matrix height) take more splits,
    // to fill the SMs, as long as the partial sums stay small.
    if (g.MT <= 2) {
        const long budget = 32L << 20;  // floats of partial sums
        const long cap = std::max(1L, std::min((long)MAX_CHAIN_SPLITS, budget / std::max(1L, (long)M * N)));
        g.splits = (int)std::max(1L, std::min({cap, (long)fill, (long)std::max(1, g.KT / KCHAIN)}));
    }
    return g;
}

}  // namespace

// ------------------------------------------------------------------ packing

// Operand X with R rows and K columns, element (r, k) = opA(r, k) (or opB(k, r)
// when `transposed`); writes hi and lo images, image (rt, kt) at
// (rt * KT + kt) * IMG floats.  One CTA of 256 threads per image.
// With lim, k >= *lim (and, for A, rows >= *lim) read as 0.
__device__ __forceinline__ void tc_pack_image(GemmOp X, int transposed, int R, int K, int KT, float *hi, float *lo,
                                              const int *lim, int img)
{
    __shared__ float tile[TM][TK + 1];
    const int rt = img / KT, kt = img % KT;
    const int t = threadIdx.x;
    if (lim) {
        const int l = *lim;
        K = min(K, l);
        if (!transposed) R = min(R, l);
    }
    const bool kfast = transposed ? (X.rs == 1) : (X.cs == 1);
#pragma unroll 4
    for (int i = 0; i < 16; i++) {
        int r, k;
        if (kfast) { r = i * 8 + (t >> 5); k = t & 31; }
        else { r = t & 127; k = i * 2 + (t >> 7); }
        const int gr = rt * TM + r, gk = kt * TK + k;
        float v = 0.f;
        if (gr < R && gk < K) v = transposed ? gop_b(X, gk, gr) : gop_a(X, gr, gk);
        tile[r][k] = v;
    }
    __syncthreads();
    const long base = (long)img * IMG;
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const int chunk = i * 256 + t;         // 16-byte chunk of the image
        const int r = chunk >> 3, pos = chunk & 7;
        const int k0 = (pos ^ (r & 7)) << 2;   // logical k of that chunk
        float4 h, l;
        float v;
        v = tile[r][k0 + 0]; h.x = tf32_round(v); l.x = tf32_round(v - h.x);
        v = tile[r][k0 + 1]; h.y = tf32_round(v); l.y = tf32_round(v - h.y);
        v = tile[r][k0 + 2]; h.z = tf32_round(v); l.z = tf32_round(v - h.z);
        v = tile[r][k0 + 3]; h.w = tf32_round(v); l.w = tf32_round(v - h.w);
        reinterpret_cast<float4 *>(hi + base)[chunk] = h;
        reinterpret_cast<float4 *>(lo + base)[chunk] = l;
    }
}

// Both operands of a product in one launch: CTAs [0, nA) pack the images of
// A (R = M), the others those of B (transposed, R = N), one image each.
__global__ void __launch_bounds__(256) tc_pack(GemmOp A, int M, float *Ahi, float *Alo, int nA, GemmOp B, int N,
                                               float *Bhi, float *Blo, int K, int KT, const int *lim)
{
    const int img = blockIdx.x;
    if (img < nA)
        tc_pack_image(A, 0, M, K, KT, Ahi, Alo, lim, img);
    else
        tc_pack_image(B, 1, N, K, KT, Bhi, Blo, lim, img - nA);
}

// ------------------------------------------------------------------ GEMM

// Direct B: when Bd.p is set, B is not pre-packed: it is a plain row-major
// operand (B(k, n) = Bd.p[k * Bd.rs + n]) that all 128 threads read from
// global memory one 32 x 128 tile at a time (the next tile's loads in flight
// while the current tile's MMAs run), split into TF32 hi and lo parts and
// store into the stage's images in the swizzled K-major layout tc_pack writes.
// A stays pre-packed (bulk copies).  Kdim is K (rows of B beyond it read 0).
__global__ void __launch_bounds__(128, 1)
    tc_gemm(int M, int N, int KT, int kper, float alpha, const float *Ahi, const float *Alo, const float *Bhi,
            const float *Blo, float beta, float *C, long ldc, float *part, int ctma, const int *lim, DevStatus *st,
            GemmOp Bd, int Kdim)
{
    if (lim) M = min(M, *lim);  // rows at or beyond the limit are left as they are
    extern __shared__ __align__(1024) unsigned char tc_smem_raw[];
    __shared__ __align__(8) uint64_t full[STAGES], empty[STAGES], done, cbar, chbar;
    __shared__ uint32_t s_tmem;
    __shared__ int s_fail;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int nt = blockIdx.x, mt = blockIdx.y, z = blockIdx.z;
    const int kb0 = z * kper, kb1 = min(KT, kb0 + kper);
    const int nk = max(0, kb1 - kb0);
    const int m0 = mt * TM, n0 = nt * TN;
    const int nrows = min(TM, M - m0), ncols = min(TN, N - n0);
    // stage buffers [stage][Ahi, Alo, Bhi, Blo][IMG], 1024-byte aligned for the
    // swizzle, then the C tile (TM x TN, row-major) for the bulk-copy epilogue
    float *stage = (float *)(tc_smem_raw + ((1024u - (smem_u32(tc_smem_raw) & 1023u)) & 1023u));
    float *Csm = stage + (long)STAGES * 4 * IMG;
    // destination of this CTA: C, or its split-K partial buffer
    float *Cd = C;
    long ld = ldc;
    float al = alpha, be = beta;
    if (part) {
        Cd = part + (long)z * M * N;
        ld = N;
        al = 1.f;
        be = 0.f;
    }
    const bool cload = ctma && be != 0.f && nrows > 0;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                     "r"(2 * TN)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        for (int s = 0; s < STAGES; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        mbar_init(&done, 1);
        mbar_init(&cbar, 1);
        mbar_init(&chbar, 1);
        mbar_init_fence();
        s_fail = 0;
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = s_tmem;
    // The split's k range runs in chains of KCHAIN images: each finished
    // chain's accumulator (TMEM columns 0..TN-1) is added by the four warps
    // into FP32 sums (columns TN..2TN-1, round-to-nearest) before the next
    // chain overwrites it.  Returns false (in every thread) when a wait gave up.
    const int nch = (nk + KCHAIN - 1) / KCHAIN;
    const bool chained = nch > 1;
    const uint32_t tq = tmem + ((uint32_t)(warp * 32) << 16);
    auto fold = [&](int c, bool fail) -> bool {
        if (__syncthreads_or(fail)) return false;
        const bool okw = mbar_wait_bounded(&chbar, c & 1, st, 508);
        if (__syncthreads_or(!okw)) return false;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll 1
        for (int cb = 0; cb < TN; cb += 32) {
            uint32_t v[32], w[32];
            tmem_ld32(tq + (uint32_t)cb, v);
            if (c > 0) {
                tmem_ld32(tq + (uint32_t)(TN + cb), w);
#pragma unroll
                for (int q = 0; q < 32; q++) v[q] = __float_as_uint(__uint_as_float(v[q]) + __uint_as_float(w[q]));
            }
            tmem_st32(tq + (uint32_t)(TN + cb), v);
        }
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        return true;
    };

    if (tid == 0 && cload) {
        // the C tile streams in while the products run
        mbar_expect_tx(&cbar, (uint32_t)(nrows * ncols * 4));
        for (int r = 0; r < nrows; r++)
            tma_load_1d(Csm + r * TN, Cd + (long)(m0 + r) * ld + n0, (uint32_t)(ncols * 4), &cbar);
    }
    if (Bd.p) {
        // thread (warp w, lane l): k chunks c = w, w + 4 (4 k each) of image
        // rows n = l + 32 j, j < 4; two images of B in flight in registers
        // (even images in rb0, odd ones in rb1) while one is converted
        const long abase = (long)mt * KT * IMG;
        using Reg = float[2][4][4];
        Reg rb0, rb1;
        auto load_b = [&](Reg &rb, int j) {
            const int kbase = (kb0 + j) * TK;
#pragma unroll
            for (int cc = 0; cc < 2; cc++)
#pragma unroll
                for (int i = 0; i < 4; i++) {
                    const int gk = kbase + 4 * (warp + 4 * cc) + i;
#pragma unroll
                    for (int q = 0; q < 4; q++) {
                        const int gn = n0 + lane + 32 * q;
                        rb[cc][i][q] = (gk < Kdim && gn < N) ? __ldg(Bd.p + (long)gk * Bd.rs + gn) : 0.f;
                    }
                }
        };
        if (nk > 0) load_b(rb0, 0);
        if (nk > 1) load_b(rb1, 1);
        bool ok = true;
        int issued = 0, consumed = 0;
        // one k-block: its B image from rb into the stage, rb refilled with
        // image kb + 2, the MMAs; false when the loop has to stop
        auto step = [&](int kb, Reg &rb) -> bool {
            const int s = kb % STAGES;
            // the stage's previous MMAs are done before it is refilled
            if (tid == 0 && kb >= STAGES && ok && !mbar_wait_bounded(&empty[s], ((kb / STAGES) - 1) & 1, st, 505))
                ok = false;
            if (__syncthreads_or(tid == 0 && !ok)) return false;
            float *dst = stage + (long)s * 4 * IMG;
            if (tid == 0) {
                mbar_expect_tx(&full[s], 2u * IMG * 4u);
                tma_load_1d(dst + 0 * IMG, Ahi + abase + (long)(kb0 + kb) * IMG, IMG * 4u, &full[s]);
                tma_load_1d(dst + 1 * IMG, Alo + abase + (long)(kb0 + kb) * IMG, IMG * 4u, &full[s]);
                issued = kb + 1;
            }
#pragma unroll
            for (int cc = 0; cc < 2; cc++) {
                const int c = warp + 4 * cc;
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    const int r = lane + 32 * q;
                    float4 h, l;
                    h.x = tf32_round(rb[cc][0][q]); l.x = tf32_round(rb[cc][0][q] - h.x);
                    h.y = tf32_round(rb[cc][1][q]); l.y = tf32_round(rb[cc][1][q] - h.y);
                    h.z = tf32_round(rb[cc][2][q]); l.z = tf32_round(rb[cc][2][q] - h.z);
                    h.w = tf32_round(rb[cc][3][q]); l.w = tf32_round(rb[cc][3][q] - h.w);
                    const int off = r * TK + ((c ^ (r & 7)) << 2);
                    *reinterpret_cast<float4 *>(dst + 2 * IMG + off) = h;
                    *reinterpret_cast<float4 *>(dst + 3 * IMG + off) = l;
                }
            }
            if (kb + 2 < nk) load_b(rb, kb + 2);
            proxy_async_fence();  // the images written here, visible to the tensor cores
            __syncthreads();
            if (tid == 0 && ok) {
                if (!mbar_wait_bounded(&full[s], (kb / STAGES) & 1, st, 506)) {
                    ok = false;
                } else {
                    consumed = kb + 1;
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                    const uint32_t base = smem_u32(dst);
                    const uint64_t ahi = smem_desc(base), alo = smem_desc(base + IMG * 4);
                    const uint64_t bhi = smem_desc(base + 2 * IMG * 4), blo = smem_desc(base + 3 * IMG * 4);
#pragma unroll
                    for (int j = 0; j < TK / 8; j++) {
                        const uint64_t dk = (uint64_t)(j * 32 >> 4);
                        mma_tf32(tmem, alo + dk, bhi + dk, ((kb % KCHAIN) | j) ? 1u : 0u);
                        mma_tf32(tmem, ahi + dk, blo + dk, 1u);
                        mma_tf32(tmem, ahi + dk, bhi + dk, 1u);
                    }
                    mma_commit(&empty[s]);
                }
            }
            if (chained && (kb % KCHAIN == KCHAIN - 1 || kb + 1 == nk)) {
                if (tid == 0 && ok) mma_commit(&chbar);
                if (!fold(kb / KCHAIN, tid == 0 && !ok)) {
                    if (tid == 0) ok = false;
                    return false;
                }
            }
            return true;
        };
        for (int kb = 0; kb < nk; kb += 2) {
            if (!step(kb, rb0)) break;
            if (kb + 1 < nk && !step(kb + 1, rb1)) break;
        }
        if (tid == 0) {
            if (!ok) {
                s_fail = 1;
                for (int j = consumed; j < issued; j++)
                    mbar_wait_bounded(&full[j % STAGES], (j / STAGES) & 1, st, 507, 1000000000LL);
            }
            mma_commit(&done);
        }
    } else {
        // packed B: thread 0 issues the copies and the MMAs; every thread
        // joins the chain folds
        const long abase = (long)mt * KT * IMG, bbase = (long)nt * KT * IMG;
        auto produce = [&](int j) {  // k-block j of this split into stage j % STAGES
            float *dst = stage + (long)(j % STAGES) * 4 * IMG;
            uint64_t *bar = &full[j % STAGES];
            const long ko = (long)(kb0 + j) * IMG;
            mbar_expect_tx(bar, 4u * IMG * 4u);
            tma_load_1d(dst + 0 * IMG, Ahi + abase + ko, IMG * 4u, bar);
            tma_load_1d(dst + 1 * IMG, Alo + abase + ko, IMG * 4u, bar);
            tma_load_1d(dst + 2 * IMG, Bhi + bbase + ko, IMG * 4u, bar);
            tma_load_1d(dst + 3 * IMG, Blo + bbase + ko, IMG * 4u, bar);
        };
        int issued = 0, consumed = 0;
        if (tid == 0)
            for (; issued < nk && issued < STAGES; issued++) produce(issued);
        bool ok = true;
        for (int kb = 0; kb < nk; kb++) {
            if (tid == 0 && ok) {
                const int s = kb % STAGES;
                if (!mbar_wait_bounded(&full[s], (kb / STAGES) & 1, st, 500)) {
                    ok = false;
                } else {
                    consumed = kb + 1;
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                    const uint32_t base = smem_u32(stage + (long)s * 4 * IMG);
                    const uint64_t ahi = smem_desc(base), alo = smem_desc(base + IMG * 4);
                    const uint64_t bhi = smem_desc(base + 2 * IMG * 4), blo = smem_desc(base + 3 * IMG * 4);
#pragma unroll
                    for (int j = 0; j < TK / 8; j++) {
                        const uint64_t dk = (uint64_t)(j * 32 >> 4);  // 8 TF32 = 32 bytes along k
                        mma_tf32(tmem, alo + dk, bhi + dk, ((kb % KCHAIN) | j) ? 1u : 0u);
                        mma_tf32(tmem, ahi + dk, blo + dk, 1u);
                        mma_tf32(tmem, ahi + dk, bhi + dk, 1u);
                    }
                    mma_commit(&empty[s]);
                    // refill the stage the previous k-block used once its MMAs are done
                    if (kb >= 1 && issued < nk) {
                        const int pk = kb - 1;
                        if (!mbar_wait_bounded(&empty[pk % STAGES], (pk / STAGES) & 1, st, 501))
                            ok = false;
                        else
                            produce(issued++);
                    }
                }
            }
            if (chained && (kb % KCHAIN == KCHAIN - 1 || kb + 1 == nk)) {
                if (tid == 0 && ok) mma_commit(&chbar);
                if (!fold(kb / KCHAIN, tid == 0 && !ok)) {
                    if (tid == 0) ok = false;
                    break;
                }
            } else if (!chained && tid == 0 && !ok) {
                break;
            }
        }
        if (tid == 0) {
            if (!ok) {
                s_fail = 1;
                // copies still in flight land before the CTA may exit
                for (int j = consumed; j < issued; j++)
                    mbar_wait_bounded(&full[j % STAGES], (j / STAGES) & 1, st, 503, 1000000000LL);
            }
            mma_commit(&done);  // arrives when every MMA issued above has completed
        }
    }
    __syncthreads();
    bool ok = mbar_wait_bounded(&done, 0, st, 502);
    if (cload) ok = mbar_wait_bounded(&cbar, 0, st, 504) && ok;
    if (!ok) s_fail = 1;
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");

    if (!s_fail) {
        const bool empty_k = (nk == 0);  // the accumulator was never written: the product is 0
        // warp w owns TMEM lanes 32w..32w+31 (rows of the tile); each 32x32
        // block is transposed through shared memory so that the lanes then
        // walk the columns of one row
        float(*sb)[33] = reinterpret_cast<float(*)[33]>(stage + warp * 32 * 33);
        const uint32_t taddr = tq + (chained ? (uint32_t)TN : 0u);  // the sums, or the one chain's accumulator
#pragma unroll 1
        for (int c0 = 0; c0 < TN; c0 += 32) {
            uint32_t v[32];
            tmem_ld32(taddr + (uint32_t)c0, v);
#pragma unroll
            for (int q = 0; q < 32; q++) sb[lane][q] = __uint_as_float(v[q]);
            __syncwarp();
            const int cl = c0 + lane;
            if (cl < ncols) {
                if (ctma) {
#pragma unroll 4
                    for (int rr = 0; rr < 32; rr++) {
                        const int rl = warp * 32 + rr;
                        if (rl >= nrows) break;
                        float x = empty_k ? 0.f : al * sb[rr][lane];
                        if (cload) x = fmaf(be, Csm[rl * TN + cl], x);
                        Csm[rl * TN + cl] = x;
                    }
                } else {
#pragma unroll 4
                    for (int rr = 0; rr < 32; rr++) {
                        const int m = m0 + warp * 32 + rr;
                        if (m >= M) break;
                        float *c = Cd + (long)m * ld + n0 + cl;
                        float x = empty_k ? 0.f : al * sb[rr][lane];
                        if (be != 0.f) x = fmaf(be, *c, x);
                        *c = x;
                    }
                }
            }
            __syncwarp();
        }
        if (ctma) {
            proxy_async_fence();
            __syncthreads();
            // one bulk store per row of the tile, spread over warp 0's lanes
            if (warp == 0) {
                for (int r = lane; r < nrows; r += 32)
                    tma_store_1d(Cd + (long)(m0 + r) * ld + n0, Csm + r * TN, (uint32_t)(ncols * 4));
                tma_store_commit_and_drain();
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * TN) : "memory");
}

// ------------------------------------------------------------------ persistent GEMM

// Persistent, warp-specialized form of tc_gemm for products without split-K:
// CTA b takes tiles b, b + gridDim.x, ... (6 warps).  Warp 0 issues the copies
// (operand stages; the C tile when beta != 0), warp 1 issues the MMAs, warps
// 2-5 run the epilogue.  A tile's k range runs in chains of KCP images, chain
// g into TMEM accumulator g & 1: with one chain per tile the epilogue writes
// tile t out of its accumulator while the MMAs of tile t+1 fill the other;
// with several, the epilogue adds each finished chain into FP32 sums (TMEM
// columns 2TN..3TN-1) while the next chain accumulates, and writes the tile
// out of the sums.
// With a tensor map for C (C rows 16-byte aligned, no row limit) the C tile
// moves in two halves of 64 columns, each with one 2-D TMA load and one TMA
// store: the load of a half of the next tile starts as soon as the store of
// that half of this tile has read the buffer, so C streams continuously.
// Otherwise (plain mode) the epilogue reads and writes C in global memory.
// Barriers:
//   full/empty[s]    operand stage s loaded / consumed by the MMAs
//   accf/acce[a]     accumulator a complete / read out by the epilogue
//   cfull/cempty[h]  C half h loaded / written back (its buffer free)
// Every wait is bounded; a role that gives up raises s_abort, the others stop
// at their next check or time out, copies in flight and issued MMAs are
// waited for (bounded) and the tensor memory is freed.
constexpr int PT_THREADS = 192;
constexpr int KCP = 4;  // k images per accumulation chain of the persistent kernel
constexpr int CH = TN / 2;  // columns of a C half

__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *tm, int x, int y, uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
            smem_u32(dst)),
        "l"(tm), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void tma_store_2d(const CUtensorMap *tm, int x, int y, const void *src)
{
    asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.bulk_group [%0, {%1, %2}], [%3];" ::"l"(tm), "r"(x),
                 "r"(y), "r"(smem_u32(src))
                 : "memory");
}

__global__ void __launch_bounds__(PT_THREADS, 1)
    tc_gemm_p(int M, int N, int KT, int NTt, int ntiles, float alpha, const float *Ahi, const float *Alo,
              const float *Bhi, const float *Blo, float beta, float *C, long ldc, int use_tm,
              const __grid_constant__ CUtensorMap tmC, const int *lim, DevStatus *st)
{
    if (lim) M = min(M, *lim);
    extern __shared__ __align__(1024) unsigned char tc_smem_raw[];
    __shared__ __align__(8) uint64_t full[STAGES], empty[STAGES], accf[2], acce[2], cfull[2], cempty[2], done;
    __shared__ uint32_t s_tmem;
    __shared__ volatile int s_abort;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    float *stage = (float *)(tc_smem_raw + ((1024u - (smem_u32(tc_smem_raw) & 1023u)) & 1023u));
    float *Cbuf = stage + (long)STAGES * 4 * IMG;  // [2][TM][CH]: the two C halves
    float *sbuf = Cbuf + TM * TN;                  // 4 x 32 x 33 epilogue staging
    const bool cload = use_tm && beta != 0.f;
    const int ntl = (ntiles - (int)blockIdx.x + (int)gridDim.x - 1) / (int)gridDim.x;  // tiles of this CTA

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                     "r"(4 * TN)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        for (int k = 0; k < STAGES; k++) {
            mbar_init(&full[k], 1);
            mbar_init(&empty[k], 1);
        }
        for (int k = 0; k < 2; k++) {
            mbar_init(&accf[k], 1);
            mbar_init(&acce[k], 1);
            mbar_init(&cfull[k], 1);
            mbar_init(&cempty[k], 1);
        }
        mbar_init(&done, 1);
        mbar_init_fence();
        s_abort = 0;
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = s_tmem;

    if (warp == 0 && lane == 0) {
        // ------------------------------------------------ producer
        int it = 0, cl = 0;  // stage uses issued, C tiles issued
        for (int lt = 0; lt < ntl && !s_abort; lt++) {
            const int t = blockIdx.x + lt * gridDim.x, mt = t / NTt, nt = t % NTt;
            const long abase = (long)mt * KT * IMG, bbase = (long)nt * KT * IMG;
            bool ok = true;
            for (int kb = 0; kb < KT; kb++, it++) {
                const int sidx = it % STAGES;
                if (it >= STAGES && !mbar_wait_bounded(&empty[sidx], ((it / STAGES) - 1) & 1, st, 611)) {
                    ok = false;
                    break;
                }
                float *dst = stage + (long)sidx * 4 * IMG;
                const long ko = (long)kb * IMG;
                mbar_expect_tx(&full[sidx], 4u * IMG * 4u);
                tma_load_1d(dst + 0 * IMG, Ahi + abase + ko, IMG * 4u, &full[sidx]);
                tma_load_1d(dst + 1 * IMG, Alo + abase + ko, IMG * 4u, &full[sidx]);
                tma_load_1d(dst + 2 * IMG, Bhi + bbase + ko, IMG * 4u, &full[sidx]);
                tma_load_1d(dst + 3 * IMG, Blo + bbase + ko, IMG * 4u, &full[sidx]);
            }
            if (!ok) { s_abort = 1; break; }
            // the C halves of this tile, each once the epilogue has written the
            // same half of the previous tile back (the box always moves its
            // full size: rows and columns outside C read as zero)
            if (cload) {
                for (int h = 0; h < 2 && ok; h++) {
                    if (lt > 0 && !mbar_wait_bounded(&cempty[h], (lt - 1) & 1, st, 610)) { ok = false; break; }
                    mbar_expect_tx(&cfull[h], (uint32_t)(TM * CH * 4));
                    tma_load_2d(Cbuf + h * TM * CH, &tmC, nt * TN + h * CH, mt * TM, &cfull[h]);
                }
                if (!ok) { s_abort = 1; break; }
                cl++;
            }
        }
        // copies in flight land before the CTA exits: the last use of each stage
        for (int j = max(0, it - STAGES); j < it; j++)
            mbar_wait_bounded(&full[j % STAGES], (j / STAGES) & 1, st, 612, 1000000000LL);
        if (cl > 0)
            for (int h = 0; h < 2; h++) mbar_wait_bounded(&cfull[h], (cl - 1) & 1, st, 613, 1000000000LL);
    } else if (warp == 1 && lane == 0) {
        // ------------------------------------------------ MMA issuer
        // each tile's k range in chains of KCP images, one TMEM accumulator
        // per chain, alternating (the epilogue folds a finished chain into
        // its FP32 sums while the next one accumulates)
        int it = 0, g = 0;
        for (int lt = 0; lt < ntl && !s_abort; lt++) {
            bool ok = true;
            for (int c0 = 0; c0 < KT && ok; c0 += KCP, g++) {
                const int ab = g & 1;
                if (g >= 2 && !mbar_wait_bounded(&acce[ab], ((g >> 1) - 1) & 1, st, 620)) { ok = false; break; }
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t acc = tmem + (uint32_t)(ab * TN);
                const int c1 = min(KT, c0 + KCP);
                for (int kb = c0; kb < c1; kb++, it++) {
                    const int sidx = it % STAGES;
                    if (!mbar_wait_bounded(&full[sidx], (it / STAGES) & 1, st, 621)) { ok = false; break; }
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                    const uint32_t base = smem_u32(stage + (long)sidx * 4 * IMG);
                    const uint64_t ahi = smem_desc(base), alo = smem_desc(base + IMG * 4);
                    const uint64_t bhi = smem_desc(base + 2 * IMG * 4), blo = smem_desc(base + 3 * IMG * 4);
#pragma unroll
                    for (int j = 0; j < TK / 8; j++) {
                        const uint64_t dk = (uint64_t)(j * 32 >> 4);
                        mma_tf32(acc, alo + dk, bhi + dk, ((kb - c0) | j) ? 1u : 0u);
                        mma_tf32(acc, ahi + dk, blo + dk, 1u);
                        mma_tf32(acc, ahi + dk, bhi + dk, 1u);
                    }
                    mma_commit(&empty[sidx]);
                }
                if (ok) mma_commit(&accf[ab]);
            }
            if (!ok) { s_abort = 1; break; }
        }
        mma_commit(&done);  // every MMA issued above has completed when this arrives
        mbar_wait_bounded(&done, 0, st, 622);
    } else if (warp >= 2) {
        // ------------------------------------------------ epilogue (warps 2-5)
        const int q = warp & 3;  // TMEM lane quarter of this warp: rows 32q..32q+31
        const int ew = warp - 2;
        float(*sb)[33] = reinterpret_cast<float(*)[33]>(sbuf + ew * 32 * 33);
        const int nch = (KT + KCP - 1) / KCP;
        // with more than one chain, the chains of a tile are summed in FP32
        // (round-to-nearest) into TMEM columns 2TN..3TN-1, which only the
        // epilogue touches; a single chain is read straight from its accumulator
        const bool chained = nch > 1;
        const uint32_t lq = (uint32_t)(q * 32) << 16;
        const uint32_t tsum = tmem + (uint32_t)(2 * TN) + lq;
        int g = 0;
        for (int lt = 0; lt < ntl; lt++) {
            bool abort = false;
            uint32_t tout = tsum;
            int ab = 0;
            for (int c = 0; c < nch; c++, g++) {
                ab = g & 1;
                const bool ok = mbar_wait_bounded(&accf[ab], (g >> 1) & 1, st, 630);
                if (bar_or(1, 128, !ok || s_abort)) { abort = true; break; }  // the same decision in every warp
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t tacc = tmem + (uint32_t)(ab * TN) + lq;
                if (!chained) {  // released after the write-out below
                    tout = tacc;
                    g++;
                    break;
                }
#pragma unroll 1
                for (int cb = 0; cb < TN; cb += 32) {
                    uint32_t v[32], w[32];
                    tmem_ld32(tacc + (uint32_t)cb, v);
                    if (c > 0) {
                        tmem_ld32(tsum + (uint32_t)cb, w);
#pragma unroll
                        for (int k = 0; k < 32; k++) v[k] = __float_as_uint(__uint_as_float(v[k]) + __uint_as_float(w[k]));
                    }
                    tmem_st32(tsum + (uint32_t)cb, v);
                }
                // the accumulator is read out: the MMAs of chain g + 2 may use it
                asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
                bar_or(1, 128, false);
                if (ew == 0 && lane == 0) mbar_arrive(&acce[ab]);
            }
            if (abort) { s_abort = 1; break; }
            const int t = blockIdx.x + lt * gridDim.x, mt = t / NTt, nt = t % NTt;
            const int m0 = mt * TM, n0 = nt * TN;
            const int nrows = min(TM, M - m0), ncols = min(TN, N - n0);
#pragma unroll
            for (int h = 0; h < 2; h++) {
                float *Ch = Cbuf + h * TM * CH;
                if (use_tm) {
                    bool okc = true;
                    if (cload) okc = mbar_wait_bounded(&cfull[h], lt & 1, st, 631);
                    if (bar_or(1, 128, !okc || s_abort)) { abort = true; break; }
                }
#pragma unroll 1
                for (int c0 = h * CH; c0 < (h + 1) * CH; c0 += 32) {
                    uint32_t v[32];
                    tmem_ld32(tout + (uint32_t)c0, v);
#pragma unroll
                    for (int k = 0; k < 32; k++) sb[lane][k] = __uint_as_float(v[k]);
                    __syncwarp();
                    const int cl = c0 + lane;
                    if (use_tm) {
                        // the whole box goes back; TMA drops what lies outside C
                        const int cc = cl - h * CH;
#pragma unroll 4
                        for (int rr = 0; rr < 32; rr++) {
                            const int rl = q * 32 + rr;
                            float x = alpha * sb[rr][lane];
                            if (cload) x = fmaf(beta, Ch[rl * CH + cc], x);
                            Ch[rl * CH + cc] = x;
                        }
                    } else if (cl < ncols) {
#pragma unroll 4
                        for (int rr = 0; rr < 32; rr++) {
                            const int rl = q * 32 + rr;
                            if (rl >= nrows) break;
                            float *cp = C + (long)(m0 + rl) * ldc + n0 + cl;
                            float x = alpha * sb[rr][lane];
                            if (beta != 0.f) x = fmaf(beta, *cp, x);
                            *cp = x;
                        }
                    }
                    __syncwarp();
                }
                if (h == 1 && !chained) {
                    // the accumulator is read out: the MMAs of chain g + 1 may use it
                    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
                    bar_or(1, 128, false);
                    if (ew == 0 && lane == 0) mbar_arrive(&acce[ab]);
                }
                if (use_tm) {
                    proxy_async_fence();  // the half's writes visible to the TMA store
                    bar_or(1, 128, false);
                    if (ew == 0 && lane == 0) {
                        tma_store_2d(&tmC, n0 + h * CH, m0, Ch);
                        tma_store_commit_and_drain();  // the store has read the buffer
                    }
                    bar_or(1, 128, false);
                    if (cload && ew == 0 && lane == 0) mbar_arrive(&cempty[h]);
                }
            }
            if (abort) { s_abort = 1; break; }
        }
        // the last stores complete before the CTA exits
        if (use_tm && ew == 0 && lane == 0) asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        __syncwarp();
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(4 * TN) : "memory");
    }
}

// ------------------------------------------------------------------ host

// stages, the C tile, and slack for the 1024-byte alignment
static size_t tc_smem_bytes() { return (size_t)(STAGES * 4 * IMG + TM * TN) * sizeof(float) + 1024; }
// the persistent kernel adds the epilogue staging of its four epilogue warps
static size_t tc_p_smem_bytes() { return tc_smem_bytes() + 4 * 32 * 33 * sizeof(float); }

static int tc_sms()
{
    static int sms[PACO_MAX_DEVICES] = {};
    const int dev = paco_device();
    if (!sms[dev]) {
        int n = 0;
        if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n < 1) n = 148;
        sms[dev] = n;
    }
    return sms[dev];
}

// Tensor map of C (FP32, M rows of N columns, row stride ldc floats) with a
// box of one C half (TM rows x CH columns); false when the driver entry point
// is not available or the encoding is refused.
static bool encode_c_map(CUtensorMap *tm, float *C, int M, int N, long ldc)
{
    static PFN_cuTensorMapEncodeTiled_v12000 enc = nullptr;
    static int tried = 0;
    if (!tried) {
        tried = 1;
        void *fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            enc = (PFN_cuTensorMapEncodeTiled_v12000)fn;
        cudaGetLastError();
    }
    if (!enc) return false;
    const cuuint64_t dims[2] = {(cuuint64_t)N, (cuuint64_t)M};
    const cuuint64_t strides[1] = {(cuuint64_t)ldc * sizeof(float)};
    const cuuint32_t box[2] = {(cuuint32_t)CH, (cuuint32_t)TM};
    const cuuint32_t estr[2] = {1, 1};
    return enc(tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, (void *)C, dims, strides, box, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// PACO_TC_PERSISTENT=0 keeps every product on the one-tile-per-CTA kernel
static int g_tc_persistent = -1;
// PACO_TC_DIRECT_B=0 packs B in a separate pass for the one-tile kernel too
static const bool g_tc_direct_b = [] {
    const char *e = getenv("PACO_TC_DIRECT_B");
    return !(e && e[0] == '0');
}();

static bool tc_persistent()
{
    if (g_tc_persistent < 0) {
        const char *e = getenv("PACO_TC_PERSISTENT");
        g_tc_persistent = (e && e[0] == '0') ? 0 : 1;
    }
    return g_tc_persistent == 1;
}

// Test hook: one CTA holds tensor memory while thread 0 waits on an mbarrier
// nothing arrives at; the wait gives up after max_cycles and records
// PACO_ERR_TIMEOUT, then the tensor memory is freed (the path every tcgen05
// kernel here takes when a wait gives up).
__global__ void __launch_bounds__(128) tc_dbg_wait_timeout(DevStatus *st, long long max_cycles)
{
    __shared__ __align__(8) uint64_t bar;
    __shared__ uint32_t s_tmem;
    const int warp = threadIdx.x >> 5;
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                     "r"(32)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        mbar_init_fence();
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = s_tmem;
    if (threadIdx.x == 0) mbar_wait_bounded(&bar, 0, st, 998, max_cycles);
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(32) : "memory");
}

bool gemm_tc_debug_timeout(DevStatus *st, long long max_cycles, cudaStream_t s)
{
    paco_count_launch();
    tc_dbg_wait_timeout<<<1, 128, 0, s>>>(st, max_cycles);
    return cudaGetLastError() == cudaSuccess;
}

int gemm_tc_set_persistent(int on)
{
    const int prev = tc_persistent() ? 1 : 0;
    g_tc_persistent = on ? 1 : 0;
    return prev;
}

size_t gemm_tc_scratch_floats(int M, int N, int K)
{
    if (M <= 0 || N <= 0 || K <= 0) return 0;
    const TcGeom g = tc_geom(M, N, K);
    size_t f = (size_t)2 * (g.MT + g.NT) * g.KT * IMG;
    if (g.splits > 1) f += (size_t)g.splits * M * N;
    return f;
}

bool gemm_tc_enabled()
{
    static int on = -1;
    if (on < 0) {
        const char *e = getenv("PACO_TC");
        on = (e && e[0] == '0') ? 0 : 1;
    }
    return on == 1;
}

void gemm_tc_init_attrs()
{
    cudaFuncSetAttribute(tc_gemm, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tc_smem_bytes());
    cudaFuncSetAttribute(tc_gemm_p, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tc_p_smem_bytes());
}

cudaError_t gemm_tc_run(int M, int N, int K, float alpha, GemmOp A, GemmOp B, float beta, float *C, long ldc,
                        float *scratch, DevStatus *st, cudaStream_t s, const int *lim)
{
    if (M <= 0 || N <= 0) return cudaSuccess;
    K = std::max(K, 1);
    TcGeom g = tc_geom(M, N, K);
    if (lim) g.splits = 1;
    float *Ahi = scratch, *Alo = Ahi + (size_t)g.MT * g.KT * IMG;
    float *Bhi = Alo + (size_t)g.MT * g.KT * IMG, *Blo = Bhi + (size_t)g.NT * g.KT * IMG;
    float *part = g.splits > 1 ? Blo + (size_t)g.NT * g.KT * IMG : nullptr;
    const int kper = ceil_div(g.KT, g.splits);
    const bool persistent = !part && tc_persistent();
    // the one-tile kernel reads a plain row-major B itself (no packing pass)
    const bool bdirect = !persistent && !lim && g_tc_direct_b && B.cs == 1 && !B.gather && !B.p2;
    const int nA = g.MT * g.KT, nB = bdirect ? 0 : g.NT * g.KT;
    paco_count_launch(), tc_pack<<<nA + nB, 256, 0, s>>>(A, M, Ahi, Alo, nA, B, N, Bhi, Blo, K, g.KT, lim);
    // bulk-copy epilogue when every row segment of the destination is 16-byte aligned
    const float *dst = part ? part : C;
    const long dld = part ? (long)N : ldc;
    const int ctma = ((((uintptr_t)dst) & 15) == 0 && (dld % 4) == 0 && (N % 4) == 0) ? 1 : 0;
    if (persistent) {
        const int ntiles = g.MT * g.NT;
        const int grid = std::min(ntiles, tc_sms());
        CUtensorMap tm;
        const int use_tm = (ctma && !lim && encode_c_map(&tm, C, M, N, ldc)) ? 1 : 0;
        if (!use_tm) memset(&tm, 0, sizeof(tm));
        paco_count_launch(), tc_gemm_p<<<grid, PT_THREADS, tc_p_smem_bytes(), s>>>(
                                 M, N, g.KT, g.NT, ntiles, alpha, Ahi, Alo, Bhi, Blo, beta, C, ldc, use_tm, tm, lim, st);
        return cudaGetLastError();
    }
    GemmOp Bd = gop(nullptr, 0, 0);
    if (bdirect) Bd = B;
    paco_count_launch(), tc_gemm<<<dim3(g.NT, g.MT, g.splits), 128, tc_smem_bytes(), s>>>(
                             M, N, g.KT, kper, alpha, Ahi, Alo, Bhi, Blo, beta, C, ldc, part, ctma, lim, st, Bd, K);
    if (part) {
        if (lim) return cudaErrorInvalidValue;  // a limited product is never split (see gemm_tc_scratch_floats)
        return gemm_splitk_reduce_run(M, N, g.splits, alpha, part, beta, C, ldc, s);
    }
    return cudaGetLastError();
}

// Products below this many multiply-adds stay on the SIMT engine: the packing
// passes and the 3 MMAs per k-step do not pay for themselves there.
static constexpr double TC_MIN_MACS = (double)(1 << 24);

static bool tc_shape_ok(int M, int N, int K)
{
    return M >= 64 && N >= 64 && K >= 32 && (double)M * N * K >= TC_MIN_MACS;
}

cudaError_t gemm_any(int M, int N, int K, float alpha, GemmOp A, GemmOp B, float beta, float *C, long ldc,
                     int splits, float *simt_scratch, float *tc_scratch, size_t tc_floats, DevStatus *st,
                     cudaStream_t s)
{
    if (tc_scratch && gemm_tc_enabled() && tc_shape_ok(M, N, K) && gemm_tc_scratch_floats(M, N, K) <= tc_floats)
        return gemm_tc_run(M, N, K, alpha, A, B, beta, C, ldc, tc_scratch, st, s);
    return gemm_run(M, N, K, alpha, A, B, beta, C, ldc, splits, simt_scratch, s);
}

size_t gemm_tc_scratch_for(const int (*shapes)[3], int n)
{
    size_t f = 0;
    for (int i = 0; i < n; i++)
        if (tc_shape_ok(shapes[i][0], shapes[i][1], shapes[i][2]))
            f = std::max(f, gemm_tc_scratch_floats(shapes[i][0], shapes[i][1], shapes[i][2]));
    return f;
}
