"""GPU parity of the two-stage reduction (dense -> band -> bidiagonal by bulge
chasing), selected per shape by the tuning entry's band width:

* stages 1 and 2 alone (test hook paco_debug_ts): the band matrix has the
  singular values of A, and so has the bidiagonal (d, e) the chase leaves;
* the whole SVD (paco_svd, paco_svd_thin) on square, ragged and tall shapes
  with bands of 32 and 64 columns.
Tolerances (FP32, against FP64 LAPACK dgesdd): sigma <= 1e-5 sigma_1,
residual and orthogonality <= 1e-5 N."""
import ctypes

import numpy as np
import pytest

import oracle as O
import pacosvd as P

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def check(A, s, U, Vt, thin=False):
    A = np.asarray(A, np.float64)
    N = A.shape[1]
    s, U, Vt = (x.cpu().numpy().astype(np.float64) for x in (s, U, Vt))
    assert O.sigma_err(s, O.lapack_dgesdd_sigma(A)) <= 1e-5
    assert O.residual(A, U[:, :N], s, Vt) <= 1e-5 * N
    assert O.orth_err(U) <= 1e-5 * N and O.orth_err(Vt.T) <= 1e-5 * N


def ts_stages(A, b):
    L = P.lib()
    vp, i = ctypes.c_void_p, ctypes.c_int
    L.paco_debug_ts.argtypes = [i, i, i, vp, vp, vp, vp, vp, ctypes.c_size_t, vp]
    L.paco_debug_ts.restype = i
    M, N = A.shape
    Ad = torch.from_numpy(A).cuda()
    band = torch.zeros(N * 3 * b, device="cuda")
    d = torch.zeros(N, device="cuda")
    e = torch.zeros(N, device="cuda")
    nb = int(L.paco_svd_workspace_size(M, N))
    ws = torch.empty(nb, dtype=torch.uint8, device="cuda")
    rc = L.paco_debug_ts(M, N, b, Ad.data_ptr(), band.data_ptr(), d.data_ptr(), e.data_ptr(), ws.data_ptr(), nb,
                         None)
    assert rc == P.PACO_OK, rc
    band = band.cpu().numpy().reshape(N, 3 * b).astype(np.float64)
    B = np.zeros((N, N))
    for o in range(b, 2 * b + 1):
        k = o - b
        B[np.arange(N - k), np.arange(k, N)] = band[:N - k, o]
    return B, d.cpu().numpy().astype(np.float64), e.cpu().numpy()[:N - 1].astype(np.float64)


@pytest.mark.parametrize("M,N,b", [(1024, 1024, 32), (1100, 1030, 32), (1300, 1100, 64)])
def test_band_and_bidiagonal_keep_the_singular_values(M, N, b):
    A = np.random.default_rng(M + b).standard_normal((M, N)).astype(np.float32)
    B, d, e = ts_stages(A, b)
    ref = O.lapack_dgesdd_sigma(A.astype(np.float64))
    # the band holds no entries outside its b superdiagonals by construction;
    # its singular values are A's
    assert O.sigma_err(np.linalg.svd(B, compute_uv=False), ref) <= 1e-5
    Bd = np.diag(d) + np.diag(e, 1)
    assert O.sigma_err(np.linalg.svd(Bd, compute_uv=False), ref) <= 1e-5


@pytest.mark.parametrize("M,N,b", [(1024, 1024, 32), (1024, 1024, 64), (1100, 1030, 32), (2048, 1024, 64),
                                   (1536, 1536, 32), (4096, 4096, 32)])
def test_two_stage_svd_matches_lapack(M, N, b):
    A = np.random.default_rng(M * 3 + N + b).standard_normal((M, N)).astype(np.float32)
    try:
        assert P.tune_param(M, N, "ts", b) == b
        s, U, Vt = P.svd(torch.from_numpy(A).cuda())
    finally:
        P.tune_param(M, N, "ts", 0)
    check(A, s, U, Vt)


def test_two_stage_thin_u_and_graded_spectrum():
    M, N, b = 1800, 1200, 32
    rng = np.random.default_rng(7)
    Q1, _ = np.linalg.qr(rng.standard_normal((M, N)))
    Q2, _ = np.linalg.qr(rng.standard_normal((N, N)))
    A = ((Q1 * np.logspace(0, -6, N)) @ Q2.T).astype(np.float32)
    try:
        P.tune_param(M, N, "ts", b)
        s, U, Vt = P.svd_thin(torch.from_numpy(A).cuda())
    finally:
        P.tune_param(M, N, "ts", 0)
    assert tuple(U.shape) == (M, N)
    check(A, s, U, Vt)
