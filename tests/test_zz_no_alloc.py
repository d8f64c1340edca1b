"""GPU test of paco_svd_noalloc, the entry point for callers that cannot call
cudaMalloc (a framework allocator owns the device memory, or the host must
not grow its memory after start-up).  Its scratch is a device array inside
the library, so the test checks that two calls in a row, sharing that array,
each give the same SVD as the allocating entry point paco_svd, and singular
values within 1e-5 * sigma_1 of FP64 LAPACK dgesdd, within the tolerances of
the other GPU tests, and that a stream under capture is rejected (the call
ends by synchronizing its stream).  The file name sorts last so that a run
that stops at the first failure has already run every other test."""
import ctypes

import numpy as np
import pytest

import oracle as O
import pacosvd as P

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

SIGMA_TOL = 1e-5


def tol_n(N):
    return 1e-5 * max(N, 1)


def noalloc_fn():
    f = P.lib().paco_svd_noalloc
    f.argtypes = [ctypes.c_int, ctypes.c_int] + [ctypes.c_void_p] * 5
    f.restype = ctypes.c_int
    return f


def svd_noalloc(A_np):
    M, N = A_np.shape
    A = torch.from_numpy(np.ascontiguousarray(A_np)).cuda()
    U = torch.empty(M, M, device="cuda")
    Vt = torch.empty(N, N, device="cuda")
    s = torch.empty(N, device="cuda")
    stream = torch.cuda.current_stream()
    rc = noalloc_fn()(M, N, A.data_ptr(), U.data_ptr(), Vt.data_ptr(), s.data_ptr(), stream.cuda_stream)
    return rc, s, U, Vt


@pytest.mark.parametrize("shapes", [((200, 120), (300, 64)), ((1024, 512), (33, 32))])
def test_noalloc_matches_allocating_entry_point_twice(shapes):
    rng = np.random.default_rng(2024)
    for (M, N) in shapes:  # two calls in a row share the device scratch
        A = rng.standard_normal((M, N)).astype(np.float32)
        rc, s, U, Vt = svd_noalloc(A)
        assert rc == P.PACO_OK
        s_ref, U_ref, Vt_ref = P.svd(torch.from_numpy(A).cuda())
        s, U, Vt = (x.cpu().numpy().astype(np.float64) for x in (s, U, Vt))
        s_ref, U_ref, Vt_ref = (x.cpu().numpy().astype(np.float64) for x in (s_ref, U_ref, Vt_ref))
        assert O.sigma_err(s, s_ref) <= SIGMA_TOL
        assert O.sigma_err(s, O.lapack_dgesdd_sigma(A)) <= SIGMA_TOL
        assert np.max(np.abs(U[:, :N] - U_ref[:, :N])) <= tol_n(N)
        assert np.max(np.abs(Vt - Vt_ref)) <= tol_n(N)
        assert O.residual(A, U, s, Vt) <= tol_n(N)
        assert O.orth_err(U) <= tol_n(N) and O.orth_err(Vt.T) <= tol_n(N)


def test_noalloc_rejects_shapes_beyond_its_scratch():
    f = noalloc_fn()
    assert f(2048, 64, None, None, None, None, None) == P.PACO_ERR_UNSUPPORTED
    assert f(1024, 600, None, None, None, None, None) == P.PACO_ERR_UNSUPPORTED
    assert f(8, 16, None, None, None, None, None) == P.PACO_ERR_INVALID_ARG


def test_noalloc_rejects_a_capturing_stream():
    f = noalloc_fn()
    A = torch.randn(64, 32, device="cuda")
    U = torch.empty(64, 64, device="cuda")
    Vt = torch.empty(32, 32, device="cuda")
    s = torch.empty(32, device="cuda")
    x = torch.zeros(4, device="cuda")
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        rc = f(64, 32, A.data_ptr(), U.data_ptr(), Vt.data_ptr(), s.data_ptr(),
               torch.cuda.current_stream().cuda_stream)
        x += 1
    assert rc == P.PACO_ERR_INVALID_ARG
    g.replay()  # the capture was left intact
    torch.cuda.synchronize()
    assert x[0].item() == 1.0
