"""Generates the golden fixtures in this directory from LAPACK (scipy's
OpenBLAS), the goldens the reference's own verifiers use:

* ``scripts/verify_svd.py:89``  -- sigma from ``np.linalg.svd`` (FP32 -> sgesdd);
  tightened here to FP64 ``dgesdd`` of the FP32 input cast to FP64.
* ``scripts/bidiag_gen.f90:122`` -- ``sgebrd``; the FP64 ``dgebrd`` |d|, |e| are
  stored (B is unique up to the signs of its rows/columns, and the reference's
  reflector convention differs from LAPACK's by a sign).
* secular-equation roots from ``dlasd4`` (the routine the reference's
  ``SecularEquationSolver``, ``svd.cpp:977-1336``, restates).

Inputs are seeded synthetic matrices (``numpy.random.default_rng``); no
public dataset is involved.  Run:  ``python tests/golden/make_golden.py``.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "oracle"))
import oracle as O  # noqa: E402


def haar(rng, n, m=None):
    """Haar-random orthonormal n x m (QR of a Gaussian with sign fix)."""
    m = n if m is None else m
    Q, R = np.linalg.qr(rng.standard_normal((n, m)))
    return Q * np.sign(np.diag(R))[None, :]


def small_cases():
    rng = np.random.default_rng(20240531)
    cases = {}
    shapes = [(1, 1), (2, 1), (2, 2), (3, 2), (3, 3), (4, 4), (5, 4), (7, 7), (8, 8),
              (9, 8), (10, 10), (16, 5), (32, 32), (33, 31), (48, 17), (64, 32)]
    for (M, N) in shapes:
        cases[f"u{M}x{N}"] = rng.uniform(-1, 1, (M, N)).astype(np.float32)
    # the reference's own generator draws U[-10, 10) (bidiag_gen.f90:83-85)
    cases["ref32x32"] = rng.uniform(-10, 10, (32, 32)).astype(np.float32)
    cases["zeros12x9"] = np.zeros((12, 9), np.float32)
    cases["negeye8"] = -np.eye(8, dtype=np.float32)
    cases["diag11"] = np.diag(np.float32([3, 3, 3, 2, 2, 1, 1, 1, 0, 0, 5]))
    cases["rank2_20x13"] = (rng.standard_normal((20, 2)) @ rng.standard_normal((2, 13))).astype(np.float32)
    cases["ones16"] = np.ones((16, 16), np.float32)
    n = 64
    cases["graded64"] = (haar(rng, n) @ np.diag(10.0 ** (-6 * np.arange(n) / (n - 1))) @ haar(rng, n).T).astype(np.float32)
    cl = np.repeat(np.logspace(-4, 0, 16), 4) * (1 + 1e-7 * np.tile(np.arange(4), 16))
    cases["clustered64"] = (haar(rng, 96, 64) @ np.diag(cl) @ haar(rng, 64).T).astype(np.float32)
    return cases


def cfg1():
    """64 x 32, iid U[-1, 1) from a seed (the plain CPU-runnable case)."""
    rng = np.random.default_rng(1)
    return rng.uniform(-1, 1, (64, 32)).astype(np.float32)


def main():
    out = {}
    for name, A in {"cfg1": cfg1(), **small_cases()}.items():
        M, N = A.shape
        out[f"{name}/A"] = A
        out[f"{name}/sigma_d"] = O.lapack_dgesdd_sigma(A)
        out[f"{name}/sigma_s"] = np.linalg.svd(A, compute_uv=False).astype(np.float32)
        d, e = O.lapack_gebrd(A)
        out[f"{name}/absd"] = np.abs(d)
        out[f"{name}/abse"] = np.abs(e)
    np.savez_compressed(os.path.join(HERE, "svd_golden.npz"), **out)

    rng = np.random.default_rng(7)
    sec = {}
    for t, k in enumerate([2, 3, 4, 7, 16, 33, 100]):
        d = np.sort(rng.uniform(0, 1, k)); d[0] = 0.0
        z = rng.standard_normal(k); z /= np.linalg.norm(z) * rng.uniform(0.3, 3.0)
        roots = np.array([O.lapack_dlasd4(d, z, i)[0] for i in range(k)])
        sec[f"p{t}/d"] = d; sec[f"p{t}/z"] = z; sec[f"p{t}/roots"] = roots
    np.savez_compressed(os.path.join(HERE, "secular_golden.npz"), **sec)
    print("wrote", len(out) // 5, "svd cases and", len(sec) // 3, "secular problems")


if __name__ == "__main__":
    main()
