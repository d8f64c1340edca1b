#!/usr/bin/env python
"""Golden-file CLI: the LAPACK goldens the reference's checkers read, in its
file layout (raw little-endian FP32, row-major, no headers).

    python golden_files.py [--root DIR] [--generate] [--seed S]

DIR (default: the parent of the working directory, as main.cpp's "../"
paths are) holds args.txt ("M N").  With --generate the input matrix
DIR/input/A_gm.bin is written first, entries uniform on [-10, 10) from a
seed (the distribution of scripts/bidiag_gen.f90:84-85, whose own RNG is
unseeded); otherwise the existing A_gm.bin is read.  Then, with LAPACK from
scipy's bundled OpenBLAS (through its LAPACKE interface; the reference
compiles scripts/bidiag_gen.f90 against system LAPACK, which needs a Fortran
compiler this project does not assume):

  DIR/output/U_golden.bin      M x M   sorgbr('Q') after sgebrd
  DIR/output/B_golden.bin      M x N   d on the diagonal, e on the superdiagonal
  DIR/output/Vt_golden.bin     N x N   sorgbr('P') after sgebrd
  DIR/output/sigma_golden.bin  N       FP64 dgesdd singular values, descending,
                                       stored as FP32

as scripts/bidiag_gen.f90:120-159 and scripts/gen_data.py:160-182 produce
them (sgebrd's sign convention: B equals this library's bidiagonal up to the
signs of its entries).  scripts/verify_result.py compares a run's U.bin,
B.bin, Vt.bin (svd_main --stage1) with A; scripts/verify_svd.py compares
sigma.bin, U.bin, Vt.bin (svd_main) with LAPACK.
"""
from __future__ import annotations

import argparse
import ctypes
import glob
import os
import sys

import numpy as np

_LAPACK = None
ROW_MAJOR = 101


def lapack():
    """scipy's bundled OpenBLAS, opened with ctypes (its LAPACKE symbols carry
    a scipy_ prefix)."""
    global _LAPACK
    if _LAPACK is None:
        import scipy
        libs = glob.glob(os.path.join(os.path.dirname(scipy.__file__), "..", "scipy.libs", "*openblas*"))
        if not libs:
            raise RuntimeError("scipy's bundled OpenBLAS was not found")
        _LAPACK = ctypes.CDLL(libs[0])
    return _LAPACK


def _fp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def sgebrd_sorgbr(A: np.ndarray):
    """FP32 LAPACK stage 1 of a row-major M x N matrix (M >= N): returns
    (U M x M, d, e, Vt N x N) with A = U B Vt."""
    L = lapack()
    M, N = A.shape
    a = np.ascontiguousarray(A, dtype=np.float32).copy()
    d = np.zeros(N, np.float32)
    e = np.zeros(max(N - 1, 1), np.float32)
    tq = np.zeros(N, np.float32)
    tp = np.zeros(N, np.float32)
    f = L.scipy_LAPACKE_sgebrd
    f.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_float), ctypes.c_int] + \
        [ctypes.POINTER(ctypes.c_float)] * 4
    f.restype = ctypes.c_int
    info = f(ROW_MAJOR, M, N, _fp(a), N, _fp(d), _fp(e), _fp(tq), _fp(tp))
    if info != 0:
        raise RuntimeError(f"sgebrd info={info}")
    g = L.scipy_LAPACKE_sorgbr
    g.argtypes = [ctypes.c_int, ctypes.c_char, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                  ctypes.POINTER(ctypes.c_float), ctypes.c_int, ctypes.POINTER(ctypes.c_float)]
    g.restype = ctypes.c_int
    U = np.zeros((M, M), np.float32)
    U[:, :N] = a
    info = g(ROW_MAJOR, b"Q", M, M, N, _fp(U), M, _fp(tq))
    if info != 0:
        raise RuntimeError(f"sorgbr(Q) info={info}")
    Vt = np.ascontiguousarray(a[:N, :N]).copy()
    info = g(ROW_MAJOR, b"P", N, N, M, _fp(Vt), N, _fp(tp))
    if info != 0:
        raise RuntimeError(f"sorgbr(P) info={info}")
    return U, d, e[: N - 1], Vt


def bidiagonal(M: int, N: int, d, e) -> np.ndarray:
    B = np.zeros((M, N), np.float32)
    B[np.arange(N), np.arange(N)] = d
    if N > 1:
        B[np.arange(N - 1), np.arange(1, N)] = e
    return B


def write_goldens(root: str, generate: bool = False, seed: int = 0) -> dict:
    with open(os.path.join(root, "args.txt")) as f:
        M, N = (int(x) for x in f.read().split()[:2])
    if M < N:
        raise SystemExit("M must be greater than N")
    a_path = os.path.join(root, "input", "A_gm.bin")
    if generate:
        os.makedirs(os.path.dirname(a_path), exist_ok=True)
        A = np.random.default_rng(seed).uniform(-10.0, 10.0, (M, N)).astype(np.float32)
        A.tofile(a_path)
    else:
        A = np.fromfile(a_path, np.float32, count=M * N)
        if A.size != M * N:
            raise SystemExit(f"{a_path} holds {A.size} floats, expected {M * N}")
        A = A.reshape(M, N)
    U, d, e, Vt = sgebrd_sorgbr(A)
    import scipy.linalg
    sigma = scipy.linalg.svd(A.astype(np.float64), compute_uv=False, lapack_driver="gesdd")
    out = os.path.join(root, "output")
    os.makedirs(out, exist_ok=True)
    files = {"U_golden.bin": U, "B_golden.bin": bidiagonal(M, N, d, e), "Vt_golden.bin": Vt,
             "sigma_golden.bin": sigma.astype(np.float32)}
    for name, arr in files.items():
        np.ascontiguousarray(arr, dtype=np.float32).tofile(os.path.join(out, name))
    return {"M": M, "N": N, "files": sorted(files)}


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--root", default="..", help="directory holding args.txt, input/ and output/")
    ap.add_argument("--generate", action="store_true", help="write a seeded input/A_gm.bin first")
    ap.add_argument("--seed", type=int, default=0)
    args = ap.parse_args(argv)
    r = write_goldens(args.root, args.generate, args.seed)
    print(f"wrote {', '.join(r['files'])} for M={r['M']} N={r['N']}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
