"""Python binding of libpacosvd.so (the B200 SVD library) through its C ABI.

Mirrors the reference's operator surface (DEAVEN-MITCH/paco-svd): the two
device kernels ``upper_bidiagonalization`` (upper_bidiagonalization.cpp:967)
and ``svd_DC`` (svd.cpp:2105), the tiling helpers ``getTilingSize`` /
``GenerateTiling`` (svd_tiling.cpp:67, 83), and the whole ``svd_main`` flow
(main.cpp) as :func:`svd`.  PyTorch supplies device memory and streams only;
every computation is a kernel of libpacosvd.so.  There is no CPU fallback:
without the library or a GPU these functions raise.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libpacosvd.so")

PACO_OK = 0
PACO_ERR_INVALID_ARG = 1
PACO_ERR_UNSUPPORTED = 2
PACO_ERR_CUDA = 3
PACO_ERR_DEVICE = 4
PACO_ERR_NONCONVERGENCE = 5
PACO_ERR_TIMEOUT = 6
PACO_ERR_BAD_TILING = 7
PACO_ERR_NONFINITE = 8
PACO_MAX_N = 8192

_STATUS_NAMES = {
    0: "OK", 1: "invalid argument", 2: "unsupported shape", 3: "CUDA error", 4: "device error",
    5: "secular non-convergence", 6: "device wait timeout", 7: "tiling blob does not match N",
    8: "non-finite input",
}


class PacoError(RuntimeError):
    def __init__(self, code: int, what: str):
        self.code = code
        super().__init__(f"{what}: status {code} ({_STATUS_NAMES.get(code, '?')})")


_lib = None


def build() -> str:
    """Compiles libpacosvd.so and svd_main in place (nvcc, sm_100a)."""
    import subprocess
    subprocess.run(["make", "-s", "-C", _HERE, "-j8"], check=True)
    return LIB_PATH


def lib():
    """Loads libpacosvd.so; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: run `make -C {_HERE}` (the CUDA library is required)")
        L = ctypes.CDLL(LIB_PATH)
        vp, i, f32p, u8p = ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p
        L.getTilingSize.argtypes = [i, i]; L.getTilingSize.restype = i
        L.GenerateTiling.argtypes = [i, i, u8p]; L.GenerateTiling.restype = None
        L.paco_buffer_sizes.argtypes = [i, i, ctypes.POINTER(ctypes.c_size_t)]; L.paco_buffer_sizes.restype = None
        L.paco_workspace_size.argtypes = [i, i]; L.paco_workspace_size.restype = ctypes.c_size_t
        L.upper_bidiagonalization.argtypes = [i, i] + [f32p] * 7 + [vp, vp]
        L.upper_bidiagonalization.restype = i
        L.svd_DC.argtypes = [i, i] + [f32p] * 7 + [vp, vp, u8p, vp]
        L.svd_DC.restype = i
        L.paco_sync_status.argtypes = [vp, vp, ctypes.POINTER(ctypes.c_int)]; L.paco_sync_status.restype = i
        L.paco_svd_workspace_size.argtypes = [i, i]; L.paco_svd_workspace_size.restype = ctypes.c_size_t
        L.paco_svd.argtypes = [i, i, f32p, f32p, f32p, f32p, vp, ctypes.c_size_t, vp]; L.paco_svd.restype = i
        L.paco_ctx_create.argtypes = [i, i, ctypes.POINTER(vp)]; L.paco_ctx_create.restype = i
        L.paco_ctx_svd_host.argtypes = [vp, vp, vp, vp, vp]; L.paco_ctx_svd_host.restype = i
        L.paco_ctx_destroy.argtypes = [vp]; L.paco_ctx_destroy.restype = None
        L.paco_version.argtypes = []; L.paco_version.restype = ctypes.c_char_p
        ip = ctypes.POINTER(ctypes.c_int)
        L.paco_autotune.argtypes = [i, i, vp, ctypes.POINTER(ctypes.c_double)]; L.paco_autotune.restype = i
        L.paco_tune_get.argtypes = [i, i, ip]; L.paco_tune_get.restype = i
        L.paco_tune_set.argtypes = [i, i, ip]; L.paco_tune_set.restype = i
        L.paco_batched_workspace_size.argtypes = [i, ip, ip]
        L.paco_batched_workspace_size.restype = ctypes.c_size_t
        L.paco_svd_batched.argtypes = [i, ip, ip, ctypes.POINTER(vp), ctypes.POINTER(vp), ctypes.POINTER(vp),
                                       ctypes.POINTER(vp), vp, vp, ctypes.c_size_t, vp]
        L.paco_svd_batched.restype = i
        L.paco_svd_multi_workspace_size.argtypes = [i, i, i]
        L.paco_svd_multi_workspace_size.restype = ctypes.c_size_t
        L.paco_svd_multi.argtypes = [i, i, i, ctypes.POINTER(vp), ctypes.POINTER(vp), ctypes.POINTER(vp),
                                     ctypes.POINTER(vp), vp, vp, ctypes.c_size_t, vp]
        L.paco_svd_multi.restype = i
        L.paco_svd_thin.argtypes = [i, i, f32p, f32p, f32p, f32p, vp, ctypes.c_size_t, vp]
        L.paco_svd_thin.restype = i
        L.paco_tune_qr.argtypes = [i, i, i]
        L.paco_tune_qr.restype = i
        L.paco_tune_param.argtypes = [i, i, i, i]
        L.paco_tune_param.restype = i
        L.paco_autotune_multi.argtypes = [i, i, i, vp, ctypes.POINTER(ctypes.c_double)]
        L.paco_autotune_multi.restype = i
        L.paco_multi_group.argtypes = [i]
        L.paco_multi_group.restype = i
        _lib = L
    return _lib


def _check(code: int, what: str):
    if code != PACO_OK:
        raise PacoError(code, what)


# ------------------------------------------------------------- host helpers


def tiling_size(N: int) -> int:
    return lib().getTilingSize(N, 1)


def generate_tiling(N: int) -> bytes:
    """Host tiling blob (leaf partition of svd_tiling.cpp:83-130)."""
    buf = (ctypes.c_uint8 * tiling_size(N))()
    lib().GenerateTiling(N, 1, buf)
    return bytes(buf)


def buffer_sizes(M: int, N: int):
    out = (ctypes.c_size_t * 12)()
    lib().paco_buffer_sizes(M, N, out)
    keys = ["U", "A", "Vt", "d", "e", "tauq", "taup", "qt", "wt", "tiling", "idx", "workspace"]
    return dict(zip(keys, [int(v) for v in out]))


def workspace_size(M: int, N: int) -> int:
    return int(lib().paco_workspace_size(M, N))


# ----------------------------------------------------------- device helpers


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("pacosvd needs a CUDA device (no CPU fallback)")
    return torch


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def _stream(stream=None):
    torch = _torch()
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)


def sync_status(workspace, stream=None):
    """Synchronizes and returns (status, info) from the device status block."""
    info = ctypes.c_int(0)
    rc = lib().paco_sync_status(_ptr(workspace), _stream(stream), ctypes.byref(info))
    return rc, info.value


def _check_matrix(A):
    torch = _torch()
    if A.dim() != 2 or A.dtype != torch.float32 or not A.is_cuda:
        raise ValueError("A must be a 2-D float32 CUDA tensor")
    return A.contiguous()


def bidiag(A, check=True):
    """Stage 1 on a copy of A.  Returns dict(A=householder vectors, U, Vt, d, e, tauq, taup)."""
    torch = _torch()
    A = _check_matrix(A).clone()
    M, N = A.shape
    dev = A.device
    U = torch.empty(M, M, device=dev); Vt = torch.empty(N, N, device=dev)
    d = torch.empty(N, device=dev); e = torch.zeros(max(N - 1, 1), device=dev)
    tq = torch.empty(N, device=dev); tp = torch.zeros(max(N - 1, 1), device=dev)
    ws = torch.empty(max(workspace_size(M, N), 256), dtype=torch.uint8, device=dev)
    rc = lib().upper_bidiagonalization(M, N, _ptr(A), _ptr(U), _ptr(Vt), _ptr(d), _ptr(e), _ptr(tq), _ptr(tp),
                                       _ptr(ws), _stream())
    _check(rc, "upper_bidiagonalization")
    if check:
        rc, info = sync_status(ws)
        _check(rc, f"upper_bidiagonalization (device, info={info})")
    return dict(A=A, U=U, Vt=Vt, d=d, e=e[: N - 1], tauq=tq, taup=tp[: N - 1], workspace=ws)


def svd_dc(M, d, e, U, Vt, tiling=None, workspace=None, check=True):
    """Stage 2 on (d, e) with U (M x M) and Vt (N x N) updated in place.
    Returns (sigma, U, Vt).  `tiling` is a host blob (bytes) or None for the
    canonical partition."""
    torch = _torch()
    N = d.numel()
    dev = d.device
    d = d.clone(); e2 = torch.zeros(max(N, 1), device=dev); e2[: N - 1] = e[: N - 1]
    a = torch.empty(M, N, device=dev)
    qt = torch.empty(2 * N * N, device=dev); wt = torch.empty(2 * N * N, device=dev)
    idx = torch.empty(16 * N, dtype=torch.int32, device=dev)
    ws = workspace if workspace is not None else torch.zeros(max(workspace_size(M, N), 256), dtype=torch.uint8,
                                                            device=dev)
    tb = None
    if tiling is not None:
        tb = torch.frombuffer(bytearray(tiling), dtype=torch.uint8).to(dev)
    rc = lib().svd_DC(M, N, _ptr(a), _ptr(U), _ptr(Vt), _ptr(d), _ptr(e2), _ptr(qt), _ptr(wt), _ptr(idx), _ptr(ws),
                      _ptr(tb) if tb is not None else None, _stream())
    _check(rc, "svd_DC")
    if check:
        rc, info = sync_status(ws)
        _check(rc, f"svd_DC (device, info={info})")
    return d, U, Vt


class Workspace:
    """Device buffers of the one-shot path for one (M, N), reusable."""

    def __init__(self, M: int, N: int, device="cuda"):
        torch = _torch()
        self.M, self.N = M, N
        self.nbytes = int(lib().paco_svd_workspace_size(M, N))
        if self.nbytes == 0:
            raise PacoError(PACO_ERR_UNSUPPORTED if N >= 1 and M >= N else PACO_ERR_INVALID_ARG, "paco_svd_workspace_size")
        self.ws = torch.empty(self.nbytes, dtype=torch.uint8, device=device)
        self.A = torch.empty(M, N, device=device)
        self.U = torch.empty(M, M, device=device)
        self.Vt = torch.empty(N, N, device=device)
        self.sigma = torch.empty(N, device=device)

    def run(self, A=None, stream=None):
        """SVD of A (copied into the workspace's A) or of the resident A."""
        if A is not None:
            self.A.copy_(A)
        rc = lib().paco_svd(self.M, self.N, _ptr(self.A), _ptr(self.U), _ptr(self.Vt), _ptr(self.sigma),
                            _ptr(self.ws), self.nbytes, _stream(stream))
        _check(rc, "paco_svd")
        return self.sigma, self.U, self.Vt


def svd_thin(A, check=True):
    """SVD with the thin U: returns (sigma, U M x N, Vt N x N) for a float32
    CUDA matrix A (M >= N), A = U diag(sigma) Vt."""
    torch = _torch()
    A = _check_matrix(A)
    M, N = A.shape
    nbytes = int(lib().paco_svd_workspace_size(M, N))
    if nbytes == 0:
        raise PacoError(PACO_ERR_UNSUPPORTED if N >= 1 and M >= N else PACO_ERR_INVALID_ARG, "paco_svd_thin")
    ws = torch.empty(nbytes, dtype=torch.uint8, device=A.device)
    Aw = A.clone()
    U = torch.empty(M, N, device=A.device)
    Vt = torch.empty(N, N, device=A.device)
    s = torch.empty(N, device=A.device)
    _check(lib().paco_svd_thin(M, N, _ptr(Aw), _ptr(U), _ptr(Vt), _ptr(s), _ptr(ws), nbytes, _stream()),
           "paco_svd_thin")
    if check:
        rc, info = sync_status(ws)
        _check(rc, f"paco_svd_thin (device, info={info})")
    return s, U, Vt


def svd(A, check=True):
    """Full SVD of a float32 CUDA matrix (M >= N): returns (sigma, U, Vt),
    sigma descending, U M x M, Vt N x N."""
    A = _check_matrix(A)
    M, N = A.shape
    w = Workspace(M, N, device=A.device)
    s, U, Vt = w.run(A)
    if check:
        rc, info = sync_status(w.ws)
        _check(rc, f"paco_svd (device, info={info})")
    return s.clone(), U.clone(), Vt.clone()


TUNE_CANDIDATES = ["persistent, 16 rows/CTA, tcgen05", "persistent, 8 rows/CTA, tcgen05",
                   "persistent, 32 rows/CTA, tcgen05", "persistent, 16 rows/CTA, SIMT products",
                   "row/column passes, 16 rows/CTA, tcgen05", "persistent, 16 rows/CTA, tcgen05, no cluster tail"]


def autotune(M: int, N: int, stream=None) -> dict:
    """Times the single-matrix configurations for (M, N) and keeps the fastest
    for later calls of that shape (svd_tiling.cpp's fixed tiling, measured)."""
    out = (ctypes.c_double * 4)()
    _check(lib().paco_autotune(M, N, _stream(stream), out), "paco_autotune")
    k = int(out[0])
    return {"choice": k, "name": TUNE_CANDIDATES[k] if k < len(TUNE_CANDIDATES) else str(k),
            "ms": out[1], "default_ms": out[2], "candidates": int(out[3]), "config": tune_get(M, N),
            "fields": {f: tune_param(M, N, f) for f in TUNE_FIELDS}}


TUNE_FIELDS = ["persistent", "rows_per_cta", "tc", "no_tail", "wy", "qb", "mk", "qr", "ts"]


def tune_param(M: int, N: int, name: str, value: int = -1) -> int:
    """One field of the tuning entry of (M, N) (TUNE_FIELDS); value -1 queries."""
    r = int(lib().paco_tune_param(M, N, TUNE_FIELDS.index(name), int(value)))
    if r < 0 and value != -1:
        raise PacoError(PACO_ERR_INVALID_ARG, f"paco_tune_param {name}={value}")
    return r


def autotune_multi(count: int, M: int, N: int, stream=None) -> dict:
    """Times lockstep groups of 2, 4 and 8 matrices of the multi-matrix form
    on `count` synthetic M x N matrices and keeps the fastest for the shape."""
    out = (ctypes.c_double * 4)()
    _check(lib().paco_autotune_multi(count, M, N, _stream(stream), out), "paco_autotune_multi")
    return {"group": int(out[0]), "ms": out[1], "ms_group2": out[2], "candidates": int(out[3])}


def tune_get(M: int, N: int):
    cfg = (ctypes.c_int * 4)()
    _check(lib().paco_tune_get(M, N, cfg), "paco_tune_get")
    return list(cfg)


def tune_qr(M: int, N: int, mode: int = -1) -> int:
    """QR-first choice for (M, N): 0 off, 1 on, 2 automatic (M >= 1.6 N);
    -1 queries the mode, -2 whether calls of this shape take the QR-first
    path now.  Applies to M > N with N >= 1024."""
    r = int(lib().paco_tune_qr(M, N, int(mode)))
    if r < 0:
        raise PacoError(PACO_ERR_INVALID_ARG, "paco_tune_qr")
    return r


def tune_set(M: int, N: int, cfg) -> None:
    c = (ctypes.c_int * 4)(*[int(x) for x in cfg])
    _check(lib().paco_tune_set(M, N, c), "paco_tune_set")


PACO_BATCH_MAX_M = 2048


def _int_array(vals):
    return (ctypes.c_int * len(vals))(*[int(v) for v in vals])


def batched_workspace_size(shapes) -> int:
    """Workspace bytes of paco_svd_batched for a list of (M, N); 0 if invalid."""
    Ms, Ns = _int_array([m for m, _ in shapes]), _int_array([n for _, n in shapes])
    return int(lib().paco_batched_workspace_size(len(shapes), Ms, Ns))


class Batch:
    """Device buffers of the batched form for a fixed list of shapes
    (M <= 2048, N <= M); reusable across calls.  A, U, Vt and sigma of all
    matrices live in four flat buffers (A_flat, U_flat, Vt_flat, sigma_flat),
    so a whole batch moves between host and device in one copy each; the
    per-matrix tensors in A, U, Vt, sigma are views into them."""

    def __init__(self, shapes, device="cuda"):
        torch = _torch()
        self.shapes = [(int(m), int(n)) for m, n in shapes]
        self.count = len(self.shapes)
        self.nbytes = batched_workspace_size(self.shapes)
        if self.nbytes == 0:
            bad = any(n >= 1 and m >= n and m > PACO_BATCH_MAX_M for m, n in self.shapes)
            raise PacoError(PACO_ERR_UNSUPPORTED if bad else PACO_ERR_INVALID_ARG, "paco_batched_workspace_size")
        self.ws = torch.empty(self.nbytes, dtype=torch.uint8, device=device)

        def flat(sizes):
            buf = torch.empty(max(1, sum(sizes)), device=device)
            views, off = [], 0
            for n in sizes:
                views.append(buf.narrow(0, off, n))
                off += n
            return buf, views

        self.A_flat, a = flat([m * n for m, n in self.shapes])
        self.U_flat, u = flat([m * m for m, _ in self.shapes])
        self.Vt_flat, v = flat([n * n for _, n in self.shapes])
        self.sigma_flat, self.sigma = flat([n for _, n in self.shapes])
        self.A = [t.view(m, n) for t, (m, n) in zip(a, self.shapes)]
        self.U = [t.view(m, m) for t, (m, _) in zip(u, self.shapes)]
        self.Vt = [t.view(n, n) for t, (_, n) in zip(v, self.shapes)]
        self.status = torch.zeros(self.count, dtype=torch.int32, device=device)
        vpa = ctypes.c_void_p * self.count
        self._Ms = _int_array([m for m, _ in self.shapes])
        self._Ns = _int_array([n for _, n in self.shapes])
        self._pA = vpa(*[t.data_ptr() for t in self.A])
        self._pU = vpa(*[t.data_ptr() for t in self.U])
        self._pV = vpa(*[t.data_ptr() for t in self.Vt])
        self._ps = vpa(*[t.data_ptr() for t in self.sigma])

    def load(self, As):
        for dst, src in zip(self.A, As):
            dst.copy_(src if hasattr(src, "data_ptr") else _torch().from_numpy(src), non_blocking=True)

    def run(self, stream=None):
        """Enqueues the batched SVD of the resident A on `stream`."""
        rc = lib().paco_svd_batched(self.count, self._Ms, self._Ns, self._pA, self._pU, self._pV, self._ps,
                                    _ptr(self.status), _ptr(self.ws), self.nbytes, _stream(stream))
        _check(rc, "paco_svd_batched")

    def statuses(self):
        return self.status.cpu().tolist()


def svd_batched(As, check=True):
    """SVD of a list of float32 CUDA (or numpy) matrices, M <= 2048, N <= M, in
    one batched launch.  Returns lists (sigma, U, Vt) and the per-matrix status."""
    torch = _torch()
    As = [a if hasattr(a, "data_ptr") else torch.from_numpy(np.ascontiguousarray(a, np.float32)) for a in As]
    b = Batch([tuple(a.shape) for a in As])
    b.load(As)
    b.run()
    torch.cuda.synchronize()
    st = b.statuses()
    if check:
        for k, c in enumerate(st):
            _check(c, f"paco_svd_batched matrix {k}")
    return [s.clone() for s in b.sigma], [u.clone() for u in b.U], [v.clone() for v in b.Vt], st


def multi_group(k: int) -> int:
    """Matrices per lockstep group of the multi-matrix form (1..8, 0 =
    automatic); returns the previous setting."""
    return int(lib().paco_multi_group(int(k)))


class Multi:
    """Device buffers of the multi-matrix form (paco_svd_multi) for `count`
    matrices of one shape (M >= N), reusable across calls: A (count x M x N,
    read only), U (count x M x M), Vt (count x N x N), sigma (count x N) and
    the per-matrix status.  The lockstep group size is fixed when the
    workspace is sized (multi_group)."""

    def __init__(self, count: int, M: int, N: int, device="cuda"):
        torch = _torch()
        self.count, self.M, self.N = int(count), int(M), int(N)
        self.nbytes = int(lib().paco_svd_multi_workspace_size(self.count, self.M, self.N))
        if self.nbytes == 0:
            raise PacoError(PACO_ERR_UNSUPPORTED if N >= 1 and M >= N else PACO_ERR_INVALID_ARG,
                            "paco_svd_multi_workspace_size")
        self.ws = torch.empty(self.nbytes, dtype=torch.uint8, device=device)
        self.A = torch.empty(self.count, M, N, device=device)
        self.U = torch.empty(self.count, M, M, device=device)
        self.Vt = torch.empty(self.count, N, N, device=device)
        self.sigma = torch.empty(self.count, N, device=device)
        self.status = torch.zeros(self.count, dtype=torch.int32, device=device)
        vpa = ctypes.c_void_p * self.count
        self._pA = vpa(*[self.A[b].data_ptr() for b in range(self.count)])
        self._pU = vpa(*[self.U[b].data_ptr() for b in range(self.count)])
        self._pV = vpa(*[self.Vt[b].data_ptr() for b in range(self.count)])
        self._ps = vpa(*[self.sigma[b].data_ptr() for b in range(self.count)])

    def run(self, stream=None):
        """Enqueues the SVDs of the resident A on `stream`."""
        rc = lib().paco_svd_multi(self.count, self.M, self.N, self._pA, self._pU, self._pV, self._ps,
                                  _ptr(self.status), _ptr(self.ws), self.nbytes, _stream(stream))
        _check(rc, "paco_svd_multi")

    def statuses(self):
        return self.status.cpu().tolist()


def svd_multi(As, check=True):
    """SVDs of a list of float32 matrices of one shape through the
    multi-matrix form.  Returns lists (sigma, U, Vt) and the statuses."""
    torch = _torch()
    As = [a if hasattr(a, "data_ptr") else torch.from_numpy(np.ascontiguousarray(a, np.float32)) for a in As]
    M, N = As[0].shape
    m = Multi(len(As), M, N)
    for b, a in enumerate(As):
        m.A[b].copy_(a)
    m.run()
    torch.cuda.synchronize()
    st = m.statuses()
    if check:
        for k, c in enumerate(st):
            _check(c, f"paco_svd_multi matrix {k}")
    return [x.clone() for x in m.sigma], [x.clone() for x in m.U], [x.clone() for x in m.Vt], st


class HostContext:
    """The svd_main path: host float32 buffers in, host buffers out."""

    def __init__(self, M: int, N: int):
        self.M, self.N = M, N
        h = ctypes.c_void_p()
        _check(lib().paco_ctx_create(M, N, ctypes.byref(h)), "paco_ctx_create")
        self._h = h

    def svd(self, A, U=None, Vt=None, sigma=None):
        """A: host float32 (numpy array or pinned torch tensor).  Outputs are
        written into the given host buffers (allocated when None)."""
        M, N = self.M, self.N

        def hp(x):
            return ctypes.c_void_p(x.data_ptr()) if hasattr(x, "data_ptr") else x.ctypes.data_as(ctypes.c_void_p)

        if U is None: U = np.empty((M, M), np.float32)
        if Vt is None: Vt = np.empty((N, N), np.float32)
        if sigma is None: sigma = np.empty(N, np.float32)
        if isinstance(A, np.ndarray):
            A = np.ascontiguousarray(A, dtype=np.float32)
        _check(lib().paco_ctx_svd_host(self._h, hp(A), hp(U), hp(Vt), hp(sigma)), "paco_ctx_svd_host")
        return sigma, U, Vt

    def close(self):
        if self._h:
            lib().paco_ctx_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
