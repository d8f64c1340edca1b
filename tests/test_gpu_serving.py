"""GPU tests of the serving loop (paco-svd_b200/serve.py): a Poisson trace of
mixed sizes runs through continuous batching; every result meets the
single-matrix tolerances against LAPACK, and each result is bit for bit the
same when its request runs alone.  Tolerances (FP32 outputs, Frobenius):
sigma <= 1e-5 sigma_1, residual and orthogonality <= 1e-5 N."""
import numpy as np
import pytest

import oracle as O
import pacosvd as P
import serve as S

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def trace(count_rate=2000.0, seconds=0.12, seed=5, mmax=600):
    arr = S.poisson_arrivals(count_rate, seconds, seed)
    M, N, graded = S.serving_shapes(len(arr), seed + 1)
    M = np.minimum(M, mmax)
    N = np.minimum(N, M)
    gen = torch.Generator(device="cuda")
    gen.manual_seed(seed)
    reqs = [S.Request(k, S.make_input(int(m), int(n), bool(g), gen), keep=True)
            for k, (m, n, g) in enumerate(zip(M, N, graded))]
    torch.cuda.synchronize()
    return reqs, arr


def check(A, s, U, Vt):
    A = A.astype(np.float64)
    M, N = A.shape
    s, U, Vt = (x.cpu().numpy().astype(np.float64) for x in (s, U, Vt))
    assert O.sigma_err(s, O.lapack_dgesdd_sigma(A)) <= 1e-5
    tol = 1e-5 * max(N, 1)
    assert O.residual(A, U, s, Vt) <= tol
    assert O.orth_err(U) <= tol and O.orth_err(Vt.T) <= tol


def test_serving_trace_matches_lapack_and_is_the_same_alone():
    reqs, arr = trace()
    inputs = {r.rid: r.A.cpu().numpy() for r in reqs}
    srv = S.SvdServer(cap_bytes=8 << 30, max_batch=64, max_inflight=4)
    S.run_trace(srv, reqs, arr)
    assert len(srv.completed) == len(reqs) and srv.batches > 1
    assert srv.status_errors() == []
    for r in srv.completed:
        assert r.done >= r.arrival
        check(inputs[r.rid], r.sigma, r.U, r.Vt)
    # alone: a fresh server, one request at a time
    for r in sorted(srv.completed, key=lambda x: -x.M)[:6]:
        alone = S.Request(r.rid, torch.from_numpy(inputs[r.rid]).cuda(), keep=True)
        one = S.SvdServer(cap_bytes=8 << 30)
        S.run_trace(one, [alone], np.zeros(1))
        assert torch.equal(alone.sigma, r.sigma) and torch.equal(alone.U, r.U) and torch.equal(alone.Vt, r.Vt)


def test_serving_admission_under_a_tight_cap():
    reqs, arr = trace(seconds=0.03, seed=9, mmax=300)
    inputs = {r.rid: r.A.cpu().numpy() for r in reqs}
    cap = max(r.nbytes for r in reqs) + (64 << 20)   # about one request at a time
    srv = S.SvdServer(cap_bytes=cap, max_batch=64, max_inflight=4)
    S.run_trace(srv, reqs, arr)
    assert len(srv.completed) == len(reqs)
    for r in srv.completed:
        check(inputs[r.rid], r.sigma, r.U, r.Vt)
