"""The tensor-core (tcgen05, 3xTF32) product against a float64 product and the
SIMT engine, on the operand layouts the SVD pipeline uses: row-major and
transposed operands, partial 128-tiles, split-K, beta = 0 and beta = 1, on
both the persistent kernel (several tiles per CTA) and the one-tile-per-CTA
kernel.  Called through the library's test hook paco_debug_gemm."""
import ctypes

import numpy as np
import pytest

import pacosvd as P

pytestmark = pytest.mark.gpu


def _hook():
    L = P.lib()
    if not hasattr(L, "_gemm_hook"):
        vp, i, lg, f = ctypes.c_void_p, ctypes.c_int, ctypes.c_long, ctypes.c_float
        L.paco_debug_gemm_ws_bytes.argtypes = [i, i, i]
        L.paco_debug_gemm_ws_bytes.restype = ctypes.c_size_t
        L.paco_debug_gemm.argtypes = [i, i, i, f, vp, lg, lg, vp, lg, lg, f, vp, lg, i, vp, ctypes.c_size_t, vp]
        L.paco_debug_gemm.restype = i
        L._gemm_hook = True
    return L


def run_gemm(A, B, C, alpha, beta, mode, a_trans=False, b_trans=False):
    """C (M x N, torch cuda) <- alpha op(A) op(B) + beta C; op = transpose when *_trans."""
    import torch
    L = _hook()
    M, N = C.shape
    K = A.shape[0] if a_trans else A.shape[1]
    a_rs, a_cs = (1, A.stride(0)) if a_trans else (A.stride(0), 1)
    b_rs, b_cs = (1, B.stride(0)) if b_trans else (B.stride(0), 1)
    nbytes = L.paco_debug_gemm_ws_bytes(M, N, K)
    ws = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    rc = L.paco_debug_gemm(M, N, K, alpha, A.data_ptr(), a_rs, a_cs, B.data_ptr(), b_rs, b_cs, beta,
                           C.data_ptr(), C.stride(0), mode, ws.data_ptr(), nbytes, None)
    torch.cuda.synchronize()
    assert rc == P.PACO_OK, rc


SHAPES = [
    (128, 128, 32, False, False),
    (256, 384, 256, False, False),
    (200, 130, 70, False, False),      # partial tiles in m, n, k
    (128, 4096, 4096, True, False),    # G1 = Vp^T Q: one m-tile, split-K
    (1000, 1100, 64, False, False),    # trailing update shape
    (517, 517, 517, False, True),      # W^T-like transposed B
    (96, 64, 1300, True, True),
    (2048, 2048, 64, False, False),    # 256 tiles: the persistent kernel walks 2 per CTA
    (4100, 1030, 96, False, False),    # 297 tiles, partial in m and n, N % 4 != 0 (plain stores)
    (4096, 4096, 64, False, True),     # 1024 tiles, 7 per CTA
]


@pytest.mark.parametrize("M,N,K,at,bt", SHAPES)
@pytest.mark.parametrize("beta", [0.0, 1.0])
def test_tensor_core_product_matches_float64(M, N, K, at, bt, beta):
    import torch
    g = torch.Generator().manual_seed(M * 7 + N * 3 + K)
    A64 = torch.randn((K, M) if at else (M, K), generator=g, dtype=torch.float64)
    B64 = torch.randn((N, K) if bt else (K, N), generator=g, dtype=torch.float64)
    C64 = torch.randn((M, N), generator=g, dtype=torch.float64)
    A, B = A64.float().cuda(), B64.float().cuda()
    opA = (A64.float().double().T if at else A64.float().double())
    opB = (B64.float().double().T if bt else B64.float().double())
    ref = -1.0 * (opA @ opB) + beta * C64.float().double()
    scale = (opA.abs() @ opB.abs()).max().item() + beta * C64.abs().max().item()
    for mode in (1, 2, 0):
        C = C64.float().cuda()
        run_gemm(A, B, C, -1.0, beta, mode, at, bt)
        err = (C.double().cpu() - ref).abs().max().item()
        # 3xTF32 keeps about FP32 accuracy: well under 1e-5 of the |A||B| scale
        assert err <= 1e-5 * scale, (mode, err, scale)


def test_tensor_core_product_is_deterministic():
    import torch
    g = torch.Generator().manual_seed(5)
    A = torch.randn(128, 3000, generator=g).cuda()
    B = torch.randn(3000, 640, generator=g).cuda()
    outs = []
    for _ in range(2):
        C = torch.zeros(128, 640, device="cuda")
        run_gemm(A, B, C, 1.0, 0.0, 1)
        outs.append(C.cpu())
    assert torch.equal(outs[0], outs[1])


@pytest.mark.parametrize("M,N,K", [(2048, 2048, 64), (1000, 1100, 64), (600, 700, 128)])
def test_persistent_and_per_tile_kernels_agree_bitwise(M, N, K):
    # k <= 4 images is one accumulation chain in both kernels: same products,
    # same accumulation order within a tile, identical bits
    import torch
    g = torch.Generator().manual_seed(M + N + K)
    A = torch.randn(M, K, generator=g).cuda()
    B = torch.randn(K, N, generator=g).cuda()
    C0 = torch.randn(M, N, generator=g).cuda()
    outs = []
    for mode in (1, 2):
        C = C0.clone()
        run_gemm(A, B, C, -1.0, 1.0, mode)
        outs.append(C.cpu())
    assert torch.equal(outs[0], outs[1])


def test_long_k_products_sum_their_chains():
    # 2048 x 2048 (256 tiles: no split-K, the persistent kernel) and the
    # one-tile kernel (mode 2, one CTA per tile and split of k), k = 4096.
    # The tensor cores round every accumulation into TMEM toward zero; both
    # kernels fold chains of 4 images into FP32 sums with round-to-nearest, so
    # neither carries that bias through 1536 MMAs: both stay within 1e-6 of
    # the |A||B| scale, with RMS errors of the same size.
    import torch
    M = N = 2048
    K = 4096
    g = torch.Generator().manual_seed(77)
    A64 = torch.randn(M, K, generator=g, dtype=torch.float64).float().double()
    B64 = torch.randn(K, N, generator=g, dtype=torch.float64).float().double()
    ref = A64 @ B64
    scale = (A64.abs() @ B64.abs()).max().item()
    err = {}
    for mode in (1, 2):
        C = torch.zeros(M, N, device="cuda")
        run_gemm(A64.float().cuda(), B64.float().cuda(), C, 1.0, 0.0, mode)
        d = C.double().cpu() - ref
        err[mode] = (d.abs().max().item(), d.pow(2).mean().sqrt().item())
    for mode in (1, 2):
        assert err[mode][0] <= 1e-6 * scale, (err, scale)
    assert 0.5 <= err[1][1] / err[2][1] <= 2.0, err


def test_skinny_product_with_few_splits_is_accurate():
    # one row tile (128 x 2048), k = 16384: a few splits of 128 images, each
    # folding 32 chains in the kernel
    import torch
    g = torch.Generator().manual_seed(78)
    A64 = torch.randn(128, 16384, generator=g, dtype=torch.float64).float().double()
    B64 = torch.randn(16384, 2048, generator=g, dtype=torch.float64).float().double()
    ref = A64 @ B64
    scale = (A64.abs() @ B64.abs()).max().item()
    C = torch.zeros(128, 2048, device="cuda")
    run_gemm(A64.float().cuda(), B64.float().cuda(), C, 1.0, 0.0, 2)
    assert (C.double().cpu() - ref).abs().max().item() <= 1e-6 * scale
