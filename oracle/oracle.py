"""Python side of the oracle -- TEST INFRASTRUCTURE ONLY.

Loads ``liboracle.so`` (the FP64 C restatement in ``paco_oracle.c``) with
ctypes, and wraps the LAPACK routines the reference's own verifiers use as
goldens (``scripts/verify_svd.py:89`` compares against ``np.linalg.svd``;
``scripts/bidiag_gen.f90:122-151`` calls ``sgebrd``/``sorgbr``).  Only the
tests, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg import
this module; the product path never does.
"""
from __future__ import annotations

import ctypes
import glob
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None
_LAPACK = None


def build() -> str:
    """Compile liboracle.so in place (gcc); returns its path."""
    subprocess.run(["make", "-s", "-C", _HERE, "liboracle.so"], check=True)
    return os.path.join(_HERE, "liboracle.so")


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        src = os.path.join(_HERE, "paco_oracle.c")
        if not os.path.exists(path) or os.path.getmtime(path) < os.path.getmtime(src):
            build()
        L = ctypes.CDLL(path)
        dp = ctypes.POINTER(ctypes.c_double)
        ip = ctypes.POINTER(ctypes.c_int)
        L.oracle_leaf_partition.argtypes = [ctypes.c_int, ip, ip]
        L.oracle_bidiag.argtypes = [ctypes.c_int, ctypes.c_int] + [dp] * 7
        L.oracle_bdc.argtypes = [ctypes.c_int, ctypes.c_int, dp, dp, dp, dp, ip]
        L.oracle_svd.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_float), dp, dp, dp]
        L.oracle_secular_root.argtypes = [ctypes.c_int, dp, dp, ctypes.c_int, dp, dp]
        _LIB = L
    return _LIB


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _ip(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


def leaf_partition(N: int):
    s = np.zeros(N // 3 + 2, np.int32)
    e = np.zeros(N // 3 + 2, np.int32)
    n = lib().oracle_leaf_partition(N, _ip(s), _ip(e))
    return [(int(s[i]), int(e[i])) for i in range(n)]


def bidiag(A: np.ndarray):
    """Stage 1 on A (M x N, any float dtype).  Returns dict of FP64 outputs."""
    M, N = A.shape
    a = np.ascontiguousarray(A, dtype=np.float64).copy()
    U = np.zeros((M, M)); Vt = np.zeros((N, N))
    d = np.zeros(N); e = np.zeros(max(N - 1, 1)); tq = np.zeros(N); tp = np.zeros(max(N - 1, 1))
    rc = lib().oracle_bidiag(M, N, _dp(a), _dp(U), _dp(Vt), _dp(d), _dp(e), _dp(tq), _dp(tp))
    if rc:
        raise ValueError(f"oracle_bidiag rejected M={M} N={N}")
    return dict(A=a, U=U, Vt=Vt, d=d, e=e[: N - 1], tauq=tq, taup=tp[: N - 1])


def bdc(M: int, d, e, U=None, Vt=None):
    """Stage 2 on (d, e); U (M x M) / Vt (N x N) default to identity."""
    N = len(d)
    d = np.array(d, dtype=np.float64)
    e2 = np.zeros(max(N, 1)); e2[: N - 1] = e[: N - 1]
    U = np.eye(M) if U is None else np.array(U, dtype=np.float64)
    Vt = np.eye(N) if Vt is None else np.array(Vt, dtype=np.float64)
    st = np.zeros(4, np.int32)
    rc = lib().oracle_bdc(M, N, _dp(d), _dp(e2), _dp(U), _dp(Vt), _ip(st))
    if rc:
        raise ValueError("oracle_bdc rejected its input")
    return dict(sigma=d, U=U, Vt=Vt, merges=int(st[0]), deflated=int(st[1]),
                maxit=int(st[2]), nonconv=int(st[3]))


def svd(A: np.ndarray):
    """Both stages on an FP32 matrix; returns (sigma, U, Vt) in FP64."""
    A = np.ascontiguousarray(A, dtype=np.float32)
    M, N = A.shape
    s = np.zeros(N); U = np.zeros((M, M)); Vt = np.zeros((N, N))
    rc = lib().oracle_svd(M, N, A.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), _dp(s), _dp(U), _dp(Vt))
    if rc:
        raise ValueError(f"oracle_svd rejected M={M} N={N}")
    return s, U, Vt


def secular_root(dsig, z, i):
    k = len(dsig)
    ds = np.ascontiguousarray(dsig, dtype=np.float64)
    zz = np.ascontiguousarray(z, dtype=np.float64)
    sig = np.zeros(1); diff = np.zeros(k)
    it = lib().oracle_secular_root(k, _dp(ds), _dp(zz), i, _dp(sig), _dp(diff))
    return float(sig[0]), diff, int(it)


# --------------------------------------------------------------------- LAPACK


def lapack():
    """scipy's bundled OpenBLAS (LAPACK 3.x), opened with ctypes."""
    global _LAPACK
    if _LAPACK is None:
        import scipy
        libs = glob.glob(os.path.join(os.path.dirname(scipy.__file__), "..", "scipy.libs", "*openblas*"))
        _LAPACK = ctypes.CDLL(libs[0])
    return _LAPACK


def lapack_gebrd(A: np.ndarray):
    """LAPACKE_dgebrd on an FP64 copy of A (row-major): returns (d, e)."""
    L = lapack()
    M, N = A.shape
    a = np.ascontiguousarray(A, dtype=np.float64).copy()
    d = np.zeros(N); e = np.zeros(max(N - 1, 1)); tq = np.zeros(N); tp = np.zeros(N)
    f = L.scipy_LAPACKE_dgebrd
    f.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double), ctypes.c_int] + \
        [ctypes.POINTER(ctypes.c_double)] * 4
    info = f(101, M, N, _dp(a), N, _dp(d), _dp(e), _dp(tq), _dp(tp))
    if info != 0:
        raise RuntimeError(f"dgebrd info={info}")
    return d, e[: N - 1]


def lapack_dgesdd_sigma(A: np.ndarray):
    import scipy.linalg
    return scipy.linalg.svd(np.asarray(A, dtype=np.float64), compute_uv=False, lapack_driver="gesdd")


def lapack_dlasd4(dsig, z, i):
    """dlasd4 root i (0-based) of 1 + sum z_j^2/(d_j^2 - s^2)."""
    import scipy.linalg.lapack as LL
    n = len(dsig)
    out = LL.dlasd4(i, np.asarray(dsig, np.float64), np.asarray(z, np.float64), rho=1.0)
    # scipy returns (delta, sigma, work, info)
    delta, sigma, work, info = out
    return float(sigma), int(info)


# ------------------------------------------------------------------ metrics


def sigma_err(s, s_ref):
    """max_i |s_i - s_ref_i| / s_ref_1 (the tolerance's metric)."""
    s = np.asarray(s, np.float64); s_ref = np.asarray(s_ref, np.float64)
    return float(np.max(np.abs(s - s_ref)) / max(s_ref[0], np.finfo(float).tiny))


def residual(A, U, s, Vt):
    """||A - U[:, :N] diag(s) Vt||_F / ||A||_F."""
    A = np.asarray(A, np.float64)
    N = A.shape[1]
    R = A - (np.asarray(U, np.float64)[:, :N] * np.asarray(s, np.float64)[None, :]) @ np.asarray(Vt, np.float64)
    return float(np.linalg.norm(R) / max(np.linalg.norm(A), np.finfo(float).tiny))


def orth_err(Q):
    """||Q^T Q - I||_F."""
    Q = np.asarray(Q, np.float64)
    return float(np.linalg.norm(Q.T @ Q - np.eye(Q.shape[1])))
