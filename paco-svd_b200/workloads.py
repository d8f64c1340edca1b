"""Seeded synthetic inputs of the benchmark configurations (no public dataset
is involved): the single-matrix generators (uniform, N(0,1), graded and
clustered spectra built as Q1 diag(sigma) Q2^T with Haar-random Q1, Q2) and
the batched form's shape list.  Shared by bench.py and the tests so that both
run the same matrices for the same seed.
"""
from __future__ import annotations

import numpy as np

WORKLOADS = {
    "cfg2a": dict(M=4096, N=4096, gen="normal"),
    "cfg2b": dict(M=4096, N=4096, gen="graded"),
    "cfg1": dict(M=64, N=32, gen="uniform"),
    "cfg3": dict(M=8192, N=4096, gen="clustered"),
    # batched form: 10,000 matrices, M uniform on [32, 512], N uniform on [16, M], iid N(0,1)
    "cfg4": dict(kind="batched", count=10000, Mlo=32, Mhi=512, Nlo=16, gen="normal"),
    # multi-matrix form: 8 matrices of the precision-form configuration per call
    "cfg3x8": dict(kind="multi", M=8192, N=4096, count=8, gen="clustered"),
    # serving form: Poisson requests at 2,000/s for 60 s, 90% M log-uniform on [16, 256], 10% on
    # [256, 2048], N uniform on [M/4, M], 20% graded spectra, 64 GB device working-set cap
    "cfg5": dict(kind="serving", rate=2000.0, seconds=60.0, cap_gb=64),
}


def make_matrix(wl, seed=1234, with_sigma=False):
    """The workload's seeded matrix; with_sigma also returns its exact
    singular values (descending) for the generators that construct them."""
    M, N, gen = wl["M"], wl["N"], wl["gen"]
    rng = np.random.default_rng(seed)
    if gen == "uniform":
        A = rng.uniform(-1, 1, (M, N)).astype(np.float32)
        return (A, None) if with_sigma else A
    if gen == "normal":
        A = rng.standard_normal((M, N), dtype=np.float32)
        return (A, None) if with_sigma else A

    def haar(n, m):
        Q, R = np.linalg.qr(rng.standard_normal((n, m)))
        return Q * np.sign(np.diag(R))[None, :]

    if gen == "graded":
        sig = 10.0 ** (-6 * np.arange(N) / (N - 1))
    else:  # 512 clusters of 8, centres log-uniform in [1e-4, 1], spacing 1e-7
        centres = 10.0 ** rng.uniform(-4, 0, N // 8)
        sig = np.sort((centres[:, None] * (1 + 1e-7 * np.arange(8))[None, :]).ravel())[::-1]
    A = ((haar(M, N) * sig[None, :]) @ haar(N, N).T).astype(np.float32)
    return (A, np.sort(sig)[::-1].copy()) if with_sigma else A


def batched_shapes(wl, seed):
    """(M, N) of every matrix of the batched workload: M uniform on
    [Mlo, Mhi], N uniform on [Nlo, M]."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(wl["count"]):
        M = int(rng.integers(wl["Mlo"], wl["Mhi"] + 1))
        out.append((M, int(rng.integers(wl["Nlo"], M + 1))))
    return out


def make_clustered_device(M, N, seed, device="cuda"):
    """The clustered-spectrum generator of make_matrix on the GPU (torch, FP64
    QR of seeded Gaussians, cast to FP32), for workloads that need many such
    matrices: 512 clusters of 8 (for N = 4096), centres log-uniform in
    [1e-4, 1], relative spacing 1e-7.  Returns (A, exact sigma descending)."""
    import torch
    g = torch.Generator(device=device)
    g.manual_seed(seed)

    def haar(n, m):
        Q, R = torch.linalg.qr(torch.randn(n, m, generator=g, device=device, dtype=torch.float64))
        return Q * torch.sign(torch.diagonal(R))[None, :]

    centres = 10.0 ** (4.0 * torch.rand(N // 8, generator=g, device=device, dtype=torch.float64) - 4.0)
    steps = 1.0 + 1e-7 * torch.arange(8, device=device, dtype=torch.float64)
    sig = torch.sort((centres[:, None] * steps[None, :]).reshape(-1), descending=True).values
    A = ((haar(M, N) * sig[None, :]) @ haar(N, N).T).float()
    return A, sig.cpu().numpy()
