"""CPU tests: the oracle (FP64 restatement of the reference path) pinned
against the LAPACK goldens in tests/golden/ and against the reference's own
verification criteria (scripts/verify_svd.py, scripts/verify_result.py)."""
import numpy as np
import pytest

import oracle as O
from conftest import load_secular_golden, load_svd_golden

GOLD = load_svd_golden()
SEC = load_secular_golden()

# The deflation tolerance is the reference's FP32 one (8 * FLT_EPSILON * max,
# svd.cpp:637-638), so sigma may move by up to ~1e-6 * sigma_1 where values
# deflate; generic matrices agree with dgesdd to ~1e-12.
SIGMA_TOL = 2e-6


@pytest.mark.parametrize("N", list(range(1, 40)) + [64, 100, 4096])
def test_leaf_partition_follows_reference_tiling(N):
    leaves = O.leaf_partition(N)
    # contiguous cover of [0, N)
    assert leaves[0][0] == 0 and leaves[-1][1] == N
    for (s0, e0), (s1, e1) in zip(leaves, leaves[1:]):
        assert e0 == s1
    if N <= 2:
        assert leaves == [(0, N)]
        return
    assert len(leaves) == N // 3 + 1  # svd_tiling.cpp:71
    widths = [e - s for s, e in leaves]
    rem = N % 3
    if rem == 0:
        assert widths == [3] * (N // 3 - 1) + [2, 1]
    elif rem == 1:
        assert widths == [3] * (N // 3) + [1]
    else:
        assert widths == [3] * (N // 3) + [2]


@pytest.mark.parametrize("name", sorted(GOLD))
def test_oracle_sigma_matches_dgesdd(name):
    c = GOLD[name]
    s, U, Vt = O.svd(c["A"])
    assert O.sigma_err(s, c["sigma_d"]) <= SIGMA_TOL
    assert np.all(np.diff(s) <= 0), "sigma must be descending"


@pytest.mark.parametrize("name", sorted(GOLD))
def test_oracle_vectors_reconstruct_and_are_orthogonal(name):
    c = GOLD[name]
    A = c["A"].astype(np.float64)
    M, N = A.shape
    s, U, Vt = O.svd(c["A"])
    assert O.residual(A, U, s, Vt) <= 1e-5
    assert O.orth_err(U) <= 1e-12 * M
    assert O.orth_err(Vt.T) <= 1e-12 * N


@pytest.mark.parametrize("name", sorted(GOLD))
def test_oracle_bidiag_matches_dgebrd_up_to_sign(name):
    # B is unique up to the signs of its rows/columns; the reference's reflector
    # (mu = +sqrt) and LAPACK's (beta = -sign(alpha)|x|) differ only by sign.
    # B's forward error grows with clustering (clustered64 agrees to ~2e-9,
    # generic inputs to ~1e-14); 1e-8 * |A|_F is far below FP32 resolution.
    c = GOLD[name]
    b = O.bidiag(c["A"])
    scale = max(1.0, float(np.linalg.norm(c["A"].astype(np.float64))))
    assert np.max(np.abs(np.abs(b["d"]) - c["absd"])) <= 1e-8 * scale
    if c["A"].shape[1] > 1:
        assert np.max(np.abs(np.abs(b["e"]) - c["abse"])) <= 1e-8 * scale


@pytest.mark.parametrize("name", ["cfg1", "u33x31", "ref32x32", "u5x4", "u1x1", "rank2_20x13"])
def test_oracle_stage1_properties(name):
    """verify_result.py:58-123,194-198: orthogonal U, Vt; upper bidiagonal B;
    U B Vt = A."""
    A = GOLD[name]["A"].astype(np.float64)
    M, N = A.shape
    b = O.bidiag(A)
    B = np.zeros((M, N))
    B[np.arange(N), np.arange(N)] = b["d"]
    if N > 1:
        B[np.arange(N - 1), np.arange(1, N)] = b["e"]
    assert np.linalg.norm(b["U"] @ B @ b["Vt"] - A) <= 1e-12 * max(1.0, np.linalg.norm(A))
    assert O.orth_err(b["U"]) <= 1e-12 * M
    assert O.orth_err(b["Vt"]) <= 1e-12 * N
    # reflector convention of upper_bidiagonalization.cpp:193-207: d_i = +mu
    # unless the reflected part is exactly zero
    assert np.all(b["d"][b["tauq"] != 0] >= 0)


def test_oracle_passes_reference_verifier_on_cfg1():
    """The checks of scripts/verify_svd.py:35-65,102-104 with its tolerances."""
    A = GOLD["cfg1"]["A"]
    s, U, Vt = O.svd(A)
    U = U.astype(np.float32); Vt = Vt.astype(np.float32); s = s.astype(np.float32)
    M, N = A.shape
    assert np.allclose(U @ U.T, np.eye(M), rtol=1e-3, atol=1e-5)
    assert np.allclose(Vt @ Vt.T, np.eye(N), rtol=1e-3, atol=1e-5)
    assert np.allclose(s, GOLD["cfg1"]["sigma_s"], rtol=1e-3, atol=1e-5)
    S = np.zeros((M, N), np.float32); np.fill_diagonal(S, s)
    assert np.max(np.abs(U @ S @ Vt - A)) <= 1e-3


@pytest.mark.parametrize("name", sorted(SEC))
def test_oracle_secular_roots_match_dlasd4(name):
    p = SEC[name]
    d, z, roots = p["d"], p["z"], p["roots"]
    for i in range(len(d)):
        s, diff, it = O.secular_root(d, z, i)
        assert it >= 0, "root did not converge"
        assert abs(s - roots[i]) <= 1e-13 * max(roots[i], 1e-300)
        # the stored differences are d_j^2 - sigma_i^2 with their relative accuracy
        np.testing.assert_allclose(diff, (d - s) * (d + s), rtol=1e-9, atol=1e-15)


def test_oracle_secular_roots_interlace():
    rng = np.random.default_rng(3)
    d = np.sort(rng.uniform(0, 1, 64)); d[0] = 0
    z = rng.standard_normal(64) * 0.2
    roots = [O.secular_root(d, z, i)[0] for i in range(64)]
    assert all(d[i] < roots[i] < (d[i + 1] if i < 63 else np.inf) for i in range(64))


def test_oracle_rejects_wide_matrix():
    with pytest.raises(ValueError):
        O.svd(np.zeros((3, 5), np.float32))
