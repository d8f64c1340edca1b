// Launchers for the FP32 tile engine of gemm.cuh.
#include "gemm.cuh"

__global__ void __launch_bounds__(256) gemm_kernel(int M, int N, int K, float alpha, GemmOp A, GemmOp B,
                                                   float beta, float *C, long ldc, int splits, float *scratch,
                                                   int fast)
{
    using namespace gemm_cfg;
    const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
    int kb = 0, ke = K;
    float al = alpha, be = beta;
    float *Cd = C;
    long ld = ldc;
    if (splits > 1) {
        const int z = blockIdx.z;
        int kchunk = ((K + splits - 1) / splits + 15) / 16 * 16;
        kb = min(K, z * kchunk);
        ke = min(K, kb + kchunk);
        al = 1.f; be = 0.f; Cd = scratch + (long)z * M * N; ld = N;
    }
    if (fast) gemm_tile_fast(M, N, kb, ke, al, A, B, be, Cd, ld, m0, n0);
    else gemm_tile(M, N, kb, ke, al, A, B, be, Cd, ld, m0, n0);
}

__global__ void gemm_splitk_reduce(int M, int N, int splits, float alpha, const float *scratch, float beta,
                                   float *C, long ldc)
{
    long total = (long)M * N;
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < total; t += (long)gridDim.x * blockDim.x) {
        float s = 0.f;
        for (int z = 0; z < splits; z++) s += scratch[(long)z * total + t];
        long m = t / N, n = t % N;
        float *c = C + m * ldc + n;
        float v = alpha * s;
        if (beta != 0.f) v = fmaf(beta, *c, v);
        *c = v;
    }
}

cudaError_t gemm_splitk_reduce_run(int M, int N, int splits, float alpha, const float *scratch, float beta,
                                   float *C, long ldc, cudaStream_t s)
{
    long total = (long)M * N;
    int blocks = (int)std::min<long>(4096, (total + 255) / 256);
    paco_count_launch(), gemm_splitk_reduce<<<blocks, 256, 0, s>>>(M, N, splits, alpha, scratch, beta, C, ldc);
    return cudaGetLastError();
}

cudaError_t gemm_run(int M, int N, int K, float alpha, GemmOp A, GemmOp B, float beta, float *C, long ldc,
                     int splits, float *scratch, cudaStream_t s)
{
    using namespace gemm_cfg;
    if (M <= 0 || N <= 0) return cudaSuccess;
    if (splits < 1 || !scratch) splits = 1;
    dim3 grid(ceil_div(N, BN), ceil_div(M, BM), splits);
    const int fast = gemm_fast_ok(A, B) ? 1 : 0;
    paco_count_launch(), gemm_kernel<<<grid, THREADS, 0, s>>>(M, N, K, alpha, A, B, beta, C, ldc, splits, scratch, fast);
    if (splits > 1) return gemm_splitk_reduce_run(M, N, splits, alpha, scratch, beta, C, ldc, s);
    return cudaGetLastError();
}
