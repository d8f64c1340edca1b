"""GPU tests of the tiling autotuner: it picks one of its candidates, the
chosen configuration is used by later calls of that shape, and every
candidate gives a correct SVD (same tolerances as the parity tests)."""
import numpy as np
import pytest

import oracle as O
import pacosvd as P

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def check(A, s, U, Vt):
    A = A.astype(np.float64)
    N = A.shape[1]
    s, U, Vt = (x.cpu().numpy().astype(np.float64) for x in (s, U, Vt))
    assert O.sigma_err(s, O.lapack_dgesdd_sigma(A)) <= 1e-5
    assert O.residual(A, U, s, Vt) <= 1e-5 * N
    assert O.orth_err(U) <= 1e-5 * N and O.orth_err(Vt.T) <= 1e-5 * N


def test_autotune_picks_a_candidate_and_keeps_it():
    r = P.autotune(1100, 1030)
    assert 0 <= r["choice"] < r["candidates"] and r["ms"] > 0 and r["ms"] <= r["default_ms"] * 1.0001
    assert r["config"] == P.tune_get(1100, 1030)


@pytest.mark.parametrize("cfg", [[1, 16, 1, 0], [1, 8, 1, 0], [1, 32, 1, 0], [1, 16, 0, 0], [0, 16, 1, 0],
                                 [1, 16, 1, 1]])
def test_every_candidate_is_correct(cfg):
    M, N = 1100, 1030
    P.tune_set(M, N, cfg)
    A = np.random.default_rng(42).standard_normal((M, N)).astype(np.float32)
    s, U, Vt = P.svd(torch.from_numpy(A).cuda())
    check(A, s, U, Vt)


@pytest.mark.parametrize("wy,qb", [(64, 0), (0, 32), (64, 32)])
def test_tile_shape_variants_are_correct(wy, qb):
    # 64-reflector WY blocks and 32-column QR blocks on a tall shape (QR-first)
    M, N = 2400, 1100
    A = np.random.default_rng(43).standard_normal((M, N)).astype(np.float32)
    try:
        P.tune_param(M, N, "wy", wy)
        P.tune_param(M, N, "qb", qb)
        assert P.tune_qr(M, N, -2) == 1
        s, U, Vt = P.svd(torch.from_numpy(A).cuda())
        check(A, s, U, Vt)
    finally:
        P.tune_param(M, N, "wy", 0)
        P.tune_param(M, N, "qb", 0)


def test_autotune_tall_shape_and_multi_group():
    M, N = 2400, 1100
    r = P.autotune(M, N)
    assert r["ms"] <= r["default_ms"] * 1.0001 and r["candidates"] >= 8
    assert r["fields"]["wy"] in (0, 64) and r["fields"]["qb"] in (0, 32) and r["fields"]["ts"] in (0, 32, 64)
    m = P.autotune_multi(4, M, N)
    assert m["group"] in (2, 4) and m["candidates"] == 3 and P.tune_param(M, N, "mk") == m["group"]
    A = [np.random.default_rng(50 + k).standard_normal((M, N)).astype(np.float32) for k in range(3)]
    s, U, Vt, st = P.svd_multi(A)
    assert st == [0, 0, 0]
    for a, s1, u1, v1 in zip(A, s, U, Vt):
        check(a, s1, u1, v1)
    for f in ("wy", "qb", "mk", "ts"):
        P.tune_param(M, N, f, 0)
    P.tune_qr(M, N, 2)
    P.tune_set(M, N, [1, 16, 1, 0])
