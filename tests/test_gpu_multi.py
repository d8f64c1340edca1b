"""GPU tests of the multi-matrix form (paco_svd_multi): several large SVDs of
one shape share the GPU, stage 1 of each group of k in lockstep.  Every
result meets the single-matrix tolerances against FP64 LAPACK dgesdd
(Frobenius: sigma <= 1e-5 sigma_1, residual and orthogonality <= 1e-5 N);
a matrix's result depends only on its own data and the group size (bitwise
the same with other group mates); paco_svd_batched routes a list of one
shape with M > PACO_BATCH_MAX_M here, and A stays unchanged."""
import numpy as np
import pytest

import oracle as O
import pacosvd as P

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def check(A, s, U, Vt):
    A = np.asarray(A, np.float64)
    N = A.shape[1]
    s, U, Vt = (x.cpu().numpy().astype(np.float64) for x in (s, U, Vt))
    assert O.sigma_err(s, O.lapack_dgesdd_sigma(A)) <= 1e-5
    assert np.all(np.diff(s) <= 0)
    assert O.residual(A, U, s, Vt) <= 1e-5 * N
    assert O.orth_err(U) <= 1e-5 * N and O.orth_err(Vt.T) <= 1e-5 * N


def graded(rng, m, n):
    Q1, _ = np.linalg.qr(rng.standard_normal((m, n)))
    Q2, _ = np.linalg.qr(rng.standard_normal((n, n)))
    return ((Q1 * 10.0 ** (-6 * np.arange(n) / (n - 1))[None, :]) @ Q2.T).astype(np.float32)


@pytest.mark.parametrize("group", [1, 2, 4])
def test_multi_matches_lapack(group):
    rng = np.random.default_rng(100 + group)
    M, N = 1300, 900
    As = [rng.standard_normal((M, N)).astype(np.float32) if k % 2 == 0 else graded(rng, M, N) for k in range(5)]
    prev = P.multi_group(group)
    try:
        s, U, Vt, st = P.svd_multi(As)
    finally:
        P.multi_group(prev)
    assert st == [0] * 5
    for k in range(5):
        check(As[k], s[k], U[k], Vt[k])


def test_multi_result_is_independent_of_group_mates():
    rng = np.random.default_rng(7)
    M, N = 1100, 1000
    mates1 = [rng.standard_normal((M, N)).astype(np.float32) for _ in range(3)]
    mates2 = [rng.standard_normal((M, N)).astype(np.float32) for _ in range(3)]
    x = rng.standard_normal((M, N)).astype(np.float32)
    prev = P.multi_group(4)
    try:
        r1 = P.svd_multi(mates1 + [x])
        r2 = P.svd_multi([x] + mates2)
    finally:
        P.multi_group(prev)
    for a, b in zip((r1[0][3], r1[1][3], r1[2][3]), (r2[0][0], r2[1][0], r2[2][0])):
        assert torch.equal(a, b)
    check(x, r1[0][3], r1[1][3], r1[2][3])


def test_batched_routes_large_equal_shapes_to_multi():
    rng = np.random.default_rng(3)
    M, N = 2100, 700
    As = [rng.standard_normal((M, N)).astype(np.float32) for _ in range(3)]
    b = P.Batch([(M, N)] * 3)
    b.load(As)
    b.run()
    torch.cuda.synchronize()
    assert b.statuses() == [0, 0, 0]
    for k in range(3):
        assert np.array_equal(b.A[k].cpu().numpy(), As[k])  # A is read only
        check(As[k], b.sigma[k], b.U[k], b.Vt[k])


def test_batched_rejects_mixed_large_shapes():
    assert P.batched_workspace_size([(2100, 700), (2100, 600)]) == 0
    with pytest.raises(P.PacoError) as ei:
        P.Batch([(2100, 700), (300, 200)])
    assert ei.value.code == P.PACO_ERR_UNSUPPORTED


def test_multi_with_qr_first_matches_lapack():
    # tall shape: every matrix takes the QR-first path (QR per matrix on its
    # own stream, stage 1 of the R factors in lockstep)
    rng = np.random.default_rng(11)
    M, N = 2300, 1100
    As = [rng.standard_normal((M, N)).astype(np.float32) if k != 1 else graded(rng, M, N) for k in range(3)]
    prev = P.multi_group(2)
    try:
        s, U, Vt, st = P.svd_multi(As)
    finally:
        P.multi_group(prev)
    assert st == [0, 0, 0]
    for k in range(3):
        check(As[k], s[k], U[k], Vt[k])
