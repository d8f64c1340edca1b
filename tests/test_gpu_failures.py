"""GPU tests of the failure paths, in forms that fault, trap or hang no GPU:

* a bounded device-side wait runs out (an mbarrier nothing arrives at, in a
  kernel holding tensor memory; a grid barrier whose target is never
  reached): the library reports PACO_ERR_TIMEOUT, the kernel frees its
  tensor memory and returns, and the context stays usable (an SVD on the
  tensor-core path runs and meets the LAPACK tolerances afterwards);
* the secular-equation solver is held to one iteration: the library reports
  PACO_ERR_NONCONVERGENCE (the reference accepts a root at its iteration
  limit silently, svd.cpp:1184-1191), single-matrix and batched, and the
  default limit restores correct results;
* the serving loop cancels a request whose batch is on the GPU and one that
  is still queued: neither returns a result, and every other request of the
  trace, the cancelled one's batch mates included, is the same as when it
  runs alone.
Tolerances (FP32 outputs, Frobenius): sigma <= 1e-5 sigma_1 against FP64
LAPACK dgesdd, residual and orthogonality <= 1e-5 N."""
import ctypes
import time

import numpy as np
import pytest

import oracle as O
import pacosvd as P
import serve as S

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def hooks():
    L = P.lib()
    L.paco_debug_timeout_ws_bytes.restype = ctypes.c_size_t
    L.paco_debug_wait_timeout.argtypes = [ctypes.c_int, ctypes.c_longlong, ctypes.c_int, ctypes.c_void_p,
                                          ctypes.c_void_p]
    L.paco_debug_wait_timeout.restype = ctypes.c_int
    L.paco_debug_secular_maxit.argtypes = [ctypes.c_int]
    L.paco_debug_secular_maxit.restype = None
    return L


def check(A, s, U, Vt):
    A = np.asarray(A, np.float64)
    N = A.shape[1]
    s, U, Vt = (x.cpu().numpy().astype(np.float64) if hasattr(x, "cpu") else np.asarray(x, np.float64)
                for x in (s, U, Vt))
    assert O.sigma_err(s, O.lapack_dgesdd_sigma(A)) <= 1e-5
    assert O.residual(A, U, s, Vt) <= 1e-5 * N
    assert O.orth_err(U) <= 1e-5 * N and O.orth_err(Vt.T) <= 1e-5 * N


def svd_after():
    # 1100 x 1100: the large products go to the tcgen05 GEMM, the panels to the
    # persistent kernel's grid barrier
    rng = np.random.default_rng(41)
    A = rng.standard_normal((1100, 1100)).astype(np.float32)
    s, U, Vt = P.svd(torch.from_numpy(A).cuda())
    check(A, s, U, Vt)


@pytest.mark.parametrize("which,ctas", [(0, 1), (1, 8), (1, 148)])
def test_bounded_wait_gives_up_with_timeout_status(which, ctas):
    L = hooks()
    ctas = min(ctas, torch.cuda.get_device_properties(0).multi_processor_count)
    ws = torch.zeros(L.paco_debug_timeout_ws_bytes(), dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream()
    t = time.perf_counter()
    rc = L.paco_debug_wait_timeout(which, 200000, ctas, ws.data_ptr(), stream.cuda_stream)
    assert rc == P.PACO_ERR_TIMEOUT
    assert time.perf_counter() - t < 30.0
    # the status block records where the wait gave up and was then cleared
    assert L.paco_debug_wait_timeout(which, 200000, ctas, ws.data_ptr(), stream.cuda_stream) == P.PACO_ERR_TIMEOUT
    svd_after()


def test_secular_iteration_limit_reports_nonconvergence():
    L = hooks()
    rng = np.random.default_rng(8)
    A = rng.standard_normal((300, 200)).astype(np.float32)
    B = [rng.standard_normal((m, n)).astype(np.float32) for m, n in ((120, 90), (64, 64), (200, 33))]
    try:
        L.paco_debug_secular_maxit(1)
        with pytest.raises(P.PacoError) as ei:
            P.svd(torch.from_numpy(A).cuda())
        assert ei.value.code == P.PACO_ERR_NONCONVERGENCE
        _, _, _, st = P.svd_batched(B, check=False)
        assert all(c == P.PACO_ERR_NONCONVERGENCE for c in st)
    finally:
        L.paco_debug_secular_maxit(0)
    s, U, Vt = P.svd(torch.from_numpy(A).cuda())
    check(A, s, U, Vt)
    ss, Us, Vs, st = P.svd_batched(B)
    assert st == [0, 0, 0]
    for a, s1, u1, v1 in zip(B, ss, Us, Vs):
        check(a, s1, u1, v1)


def test_serving_cancels_in_flight_and_queued_requests():
    gen = torch.Generator(device="cuda")
    gen.manual_seed(12)
    shapes = [(300, 200), (256, 128), (180, 180), (90, 60), (400, 100), (128, 100), (64, 40), (350, 300)]
    reqs = [S.Request(k, S.make_input(m, n, k % 3 == 0, gen), keep=True) for k, (m, n) in enumerate(shapes)]
    inputs = {r.rid: r.A.cpu().numpy() for r in reqs}
    srv = S.SvdServer(cap_bytes=8 << 30, max_batch=3, max_inflight=(1, 1), small_max=256)
    t0 = time.perf_counter()
    now = lambda: time.perf_counter() - t0
    for r in reqs:
        srv.submit(r)
    srv.step(now)  # admits all, launches one batch per class
    flying = [r for bs in srv.busy for b in bs if b is not None for r in b.reqs]
    queued = [r for q in srv.pending for r in q]
    assert flying and queued
    victim_f, victim_q = flying[0], queued[-1]
    assert srv.cancel(victim_f.rid, now()) and srv.cancel(victim_q.rid, now())
    assert victim_q.status == S.CANCELLED  # left at once
    while len(srv.completed) + len(srv.cancelled) < len(reqs):
        srv.step(now)
    assert sorted(r.rid for r in srv.cancelled) == sorted([victim_f.rid, victim_q.rid])
    assert victim_f.status == S.CANCELLED and victim_f.U is None and victim_q.U is None
    assert srv.inflight == 0 and not srv.live
    assert srv.status_errors() == []
    assert len(srv.completed) == len(reqs) - 2
    for r in srv.completed:
        check(inputs[r.rid], r.sigma, r.U, r.Vt)
        alone = S.Request(r.rid, torch.from_numpy(inputs[r.rid]).cuda(), keep=True)
        one = S.SvdServer(cap_bytes=8 << 30)
        S.run_trace(one, [alone], np.zeros(1))
        assert torch.equal(alone.sigma, r.sigma) and torch.equal(alone.U, r.U) and torch.equal(alone.Vt, r.Vt)
