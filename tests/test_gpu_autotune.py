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
