// FP32 GEMM tile engine (SIMT FMA, FP32 accumulate) used by every matrix
// product of the pipeline: the panel trailing update of stage 1, the
// compact-WY formation of U and V, the merge back-transforms and the final
// U*Q, W^T*Vt products of stage 2.
//
// One CTA of 256 threads computes a 128x128 tile of
//     C = alpha * opA * opB + beta * C      (beta == 0: C is not read)
// with operands addressed through strides, so transposes and row gathers
// need no copies:
//     opA(m, k) = A.p[row(m) * A.rs + k * A.cs],  row(m) = A.gather ? A.gather[m] : m
//     opB(k, n) = B.p[k * B.rs + col(n) * B.cs],  col(n) = B.gather ? B.gather[n] : n
#pragma once

#include "common.cuh"

struct GemmOp {
    const float *p;
    long rs, cs;
    const int *gather;
    // Optional second operand concatenated along k: for k >= ksplit the
    // element comes from p2 at (k - ksplit) with strides rs2, cs2.  Lets one
    // launch compute A1*B1 + A2*B2 (the rank-2nb panel update).
    const float *p2;
    long rs2, cs2;
    int ksplit;
};

__host__ __device__ static inline GemmOp gop(const float *p, long rs, long cs, const int *gather = nullptr)
{
    GemmOp o;
    o.p = p; o.rs = rs; o.cs = cs; o.gather = gather;
    o.p2 = nullptr; o.rs2 = 0; o.cs2 = 0; o.ksplit = 0x7fffffff;
    return o;
}

namespace gemm_cfg {
constexpr int BM = 128, BN = 128, BK = 8, THREADS = 256;
}

__device__ __forceinline__ float gop_a(const GemmOp &A, int m, int k)
{
    long r = A.gather ? (long)A.gather[m] : (long)m;
    if (k >= A.ksplit) return A.p2[r * A.rs2 + (long)(k - A.ksplit) * A.cs2];
    return A.p[r * A.rs + (long)k * A.cs];
}
__device__ __forceinline__ float gop_b(const GemmOp &B, int k, int n)
{
    long c = B.gather ? (long)B.gather[n] : (long)n;
    if (k >= B.ksplit) return B.p2[(long)(k - B.ksplit) * B.rs2 + c * B.cs2];
    return B.p[(long)k * B.rs + c * B.cs];
}

// Loads the A (BM x BK) and B (BK x BN) slices starting at k0 into registers,
// choosing the thread mapping that keeps global reads coalesced.
__device__ __forceinline__ void gemm_load(const GemmOp &A, const GemmOp &B, int M, int N, int kend,
                                          int m0, int n0, int k0, float ra[4], float rb[4])
{
    using namespace gemm_cfg;
    const int t = threadIdx.x;
    const bool a_kfast = (A.cs == 1);
    const bool b_nfast = (B.cs == 1 && B.gather == nullptr);
#pragma unroll
    for (int i = 0; i < 4; i++) {
        int m, k;
        if (a_kfast) { k = t & 7; m = (t >> 3) + 32 * i; }
        else { m = t & 127; k = (t >> 7) + 2 * i; }
        int gm = m0 + m, gk = k0 + k;
        ra[i] = (gm < M && gk < kend) ? gop_a(A, gm, gk) : 0.f;
    }
#pragma unroll
    for (int i = 0; i < 4; i++) {
        int n, k;
        if (b_nfast) { n = t & 127; k = (t >> 7) + 2 * i; }
        else { k = t & 7; n = (t >> 3) + 32 * i; }
        int gn = n0 + n, gk = k0 + k;
        rb[i] = (gn < N && gk < kend) ? gop_b(B, gk, gn) : 0.f;
    }
}

__device__ __forceinline__ void gemm_store_smem(const GemmOp &A, const GemmOp &B, float (*As)[gemm_cfg::BM],
                                                float (*Bs)[gemm_cfg::BN], const float ra[4], const float rb[4])
{
    const int t = threadIdx.x;
    const bool a_kfast = (A.cs == 1);
    const bool b_nfast = (B.cs == 1 && B.gather == nullptr);
#pragma unroll
    for (int i = 0; i < 4; i++) {
        int m, k;
        if (a_kfast) { k = t & 7; m = (t >> 3) + 32 * i; }
        else { m = t & 127; k = (t >> 7) + 2 * i; }
        As[k][m] = ra[i];
    }
#pragma unroll
    for (int i = 0; i < 4; i++) {
        int n, k;
        if (b_nfast) { n = t & 127; k = (t >> 7) + 2 * i; }
        else { k = t & 7; n = (t >> 3) + 32 * i; }
        Bs[k][n] = rb[i];
    }
}

// Computes C[m0:m0+128, n0:n0+128] over k in [kbeg, kend).  C(m, n) is at
// C[m * ldc + n].  All 256 threads of the CTA must call it.
static __device__ __noinline__ void gemm_tile(int M, int N, int kbeg, int kend, float alpha, GemmOp A, GemmOp B,
                          float beta, float *C, long ldc, int m0, int n0)
{
    using namespace gemm_cfg;
    __shared__ __align__(16) float As[2][BK][BM];
    __shared__ __align__(16) float Bs[2][BK][BN];
    const int t = threadIdx.x;
    const int ty = t >> 4, tx = t & 15;
    float acc[8][8];
#pragma unroll
    for (int i = 0; i < 8; i++)
#pragma unroll
        for (int j = 0; j < 8; j++) acc[i][j] = 0.f;

    float ra[4], rb[4];
    int buf = 0;
    if (kbeg < kend) {
        gemm_load(A, B, M, N, kend, m0, n0, kbeg, ra, rb);
        gemm_store_smem(A, B, As[0], Bs[0], ra, rb);
    }
    __syncthreads();
    for (int k0 = kbeg; k0 < kend; k0 += BK) {
        const bool more = (k0 + BK < kend);
        if (more) gemm_load(A, B, M, N, kend, m0, n0, k0 + BK, ra, rb);
#pragma unroll
        for (int kk = 0; kk < BK; kk++) {
            float4 a0 = *reinterpret_cast<const float4 *>(&As[buf][kk][ty * 4]);
            float4 a1 = *reinterpret_cast<const float4 *>(&As[buf][kk][64 + ty * 4]);
            float4 b0 = *reinterpret_cast<const float4 *>(&Bs[buf][kk][tx * 4]);
            float4 b1 = *reinterpret_cast<const float4 *>(&Bs[buf][kk][64 + tx * 4]);
            float av[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
            float bv[8] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
#pragma unroll
            for (int i = 0; i < 8; i++)
#pragma unroll
                for (int j = 0; j < 8; j++) acc[i][j] = fmaf(av[i], bv[j], acc[i][j]);
        }
        if (more) {
            gemm_store_smem(A, B, As[buf ^ 1], Bs[buf ^ 1], ra, rb);
            buf ^= 1;
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 8; i++) {
        int m = m0 + ((i < 4) ? ty * 4 + i : 64 + ty * 4 + (i - 4));
        if (m >= M) continue;
#pragma unroll
        for (int j = 0; j < 8; j++) {
            int n = n0 + ((j < 4) ? tx * 4 + j : 64 + tx * 4 + (j - 4));
            if (n >= N) continue;
            float *c = C + (long)m * ldc + n;
            float v = alpha * acc[i][j];
            if (beta != 0.f) v = fmaf(beta, *c, v);
            *c = v;
        }
    }
}

// Fast path of gemm_tile for the common layout: opA k-contiguous and opB
// n-contiguous, no gathers or split operands, row strides multiples of 4
// floats and 16-byte aligned bases (checked on the host).  float4 loads, a
// 16-deep k slice per stage.
static __device__ __noinline__ void gemm_tile_fast(int M, int N, int kbeg, int kend, float alpha, GemmOp A,
                                                  GemmOp B, float beta, float *C, long ldc, int m0, int n0)
{
    constexpr int BM = 128, BN = 128, BK = 16;
    __shared__ __align__(16) float As[2][BK][BM];
    __shared__ __align__(16) float Bs[2][BK][BN];
    const int t = threadIdx.x;
    const int ty = t >> 4, tx = t & 15;
    float acc[8][8];
#pragma unroll
    for (int i = 0; i < 8; i++)
#pragma unroll
        for (int j = 0; j < 8; j++) acc[i][j] = 0.f;
    float4 ra[2], rb[2];
    auto load = [&](int k0) {
#pragma unroll
        for (int q = 0; q < 2; q++) {
            int idx = t + 256 * q;
            int row = idx >> 2, kq = idx & 3;
            int gm = m0 + row, gk = k0 + 4 * kq;
            float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
            if (gm < M) {
                const float *src = A.p + (long)gm * A.rs + gk;
                if (gk + 3 < kend) v = *reinterpret_cast<const float4 *>(src);
                else {
                    if (gk < kend) v.x = src[0];
                    if (gk + 1 < kend) v.y = src[1];
                    if (gk + 2 < kend) v.z = src[2];
                }
            }
            ra[q] = v;
            int krow = idx >> 5, nq = idx & 31;
            int gn = n0 + 4 * nq, gk2 = k0 + krow;
            float4 w = make_float4(0.f, 0.f, 0.f, 0.f);
            if (gk2 < kend) {
                const float *src = B.p + (long)gk2 * B.rs + gn;
                if (gn + 3 < N) w = *reinterpret_cast<const float4 *>(src);
                else {
                    if (gn < N) w.x = src[0];
                    if (gn + 1 < N) w.y = src[1];
                    if (gn + 2 < N) w.z = src[2];
                }
            }
            rb[q] = w;
        }
    };
    auto store = [&](int buf) {
#pragma unroll
        for (int q = 0; q < 2; q++) {
            int idx = t + 256 * q;
            int row = idx >> 2, kq = idx & 3;
            As[buf][4 * kq + 0][row] = ra[q].x;
            As[buf][4 * kq + 1][row] = ra[q].y;
            As[buf][4 * kq + 2][row] = ra[q].z;
            As[buf][4 * kq + 3][row] = ra[q].w;
            int krow = idx >> 5, nq = idx & 31;
            *reinterpret_cast<float4 *>(&Bs[buf][krow][4 * nq]) = rb[q];
        }
    };
    int buf = 0;
    if (kbeg < kend) {
        load(kbeg);
        store(0);
    }
    __syncthreads();
    for (int k0 = kbeg; k0 < kend; k0 += BK) {
        const bool more = (k0 + BK < kend);
        if (more) load(k0 + BK);
#pragma unroll
        for (int kk = 0; kk < BK; kk++) {
            float4 a0 = *reinterpret_cast<const float4 *>(&As[buf][kk][ty * 4]);
            float4 a1 = *reinterpret_cast<const float4 *>(&As[buf][kk][64 + ty * 4]);
            float4 b0 = *reinterpret_cast<const float4 *>(&Bs[buf][kk][tx * 4]);
            float4 b1 = *reinterpret_cast<const float4 *>(&Bs[buf][kk][64 + tx * 4]);
            float av[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
            float bv[8] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
#pragma unroll
            for (int i = 0; i < 8; i++)
#pragma unroll
                for (int j = 0; j < 8; j++) acc[i][j] = fmaf(av[i], bv[j], acc[i][j]);
        }
        if (more) {
            store(buf ^ 1);
            buf ^= 1;
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 8; i++) {
        int m = m0 + ((i < 4) ? ty * 4 + i : 64 + ty * 4 + (i - 4));
        if (m >= M) continue;
#pragma unroll
        for (int h = 0; h < 2; h++) {
            int n = n0 + h * 64 + tx * 4;
            float *c = C + (long)m * ldc + n;
            float v[4];
#pragma unroll
            for (int j = 0; j < 4; j++) v[j] = alpha * acc[i][h * 4 + j];
            if (n + 3 < N && (((uintptr_t)c) & 15) == 0) {
                if (beta != 0.f) {
                    float4 o = *reinterpret_cast<const float4 *>(c);
                    v[0] = fmaf(beta, o.x, v[0]); v[1] = fmaf(beta, o.y, v[1]);
                    v[2] = fmaf(beta, o.z, v[2]); v[3] = fmaf(beta, o.w, v[3]);
                }
                *reinterpret_cast<float4 *>(c) = make_float4(v[0], v[1], v[2], v[3]);
            } else {
                for (int j = 0; j < 4; j++)
                    if (n + j < N) c[j] = (beta != 0.f) ? fmaf(beta, c[j], v[j]) : v[j];
            }
        }
    }
}

// True when gemm_tile_fast applies to (A, B).
static inline bool gemm_fast_ok(const GemmOp &A, const GemmOp &B)
{
    auto plain = [](const GemmOp &o) {
        return o.cs == 1 && o.gather == nullptr && o.p2 == nullptr && (o.rs % 4) == 0 &&
               (((uintptr_t)o.p) & 15) == 0;
    };
    return plain(A) && plain(B);
}

// Host-side launcher for a single (optionally split-K) product; defined in gemm.cu.
// With splits > 1 the partial tiles go to `scratch` (splits * M * N floats) and a
// deterministic second pass sums them in split order.
cudaError_t gemm_run(int M, int N, int K, float alpha, GemmOp A, GemmOp B, float beta, float *C,
                     long ldc, int splits, float *scratch, cudaStream_t s);

// C = alpha * sum_z scratch[z] + beta * C over `splits` partial M x N products
// (row-major, ld N), summed in split order.
cudaError_t gemm_splitk_reduce_run(int M, int N, int splits, float alpha, const float *scratch, float beta,
                                   float *C, long ldc, cudaStream_t s);
