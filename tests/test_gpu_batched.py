"""GPU tests of the batched form (paco_svd_batched): every matrix of a mixed
batch against LAPACK with the tolerances of the single-matrix path, the
same result alone and inside a mix, reproducibility, per-matrix status of a
non-finite input, and the shape limits.

Tolerances (FP32 outputs, Frobenius norms):
  sigma:          max_i |s_i - s_ref_i| / s_ref_1   <= 1e-5
  residual:       ||A - U[:, :N] S Vt|| / ||A||     <= 1e-5 * N
  orthogonality:  ||U^T U - I||, ||V^T V - I||      <= 1e-5 * N"""
import numpy as np
import pytest

import oracle as O
import pacosvd as P

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def check(A, s, U, Vt):
    A = A.astype(np.float64)
    M, N = A.shape
    s, U, Vt = (x.cpu().numpy().astype(np.float64) for x in (s, U, Vt))
    s_ref = O.lapack_dgesdd_sigma(A)
    assert np.all(np.isfinite(s)) and np.all(np.isfinite(U)) and np.all(np.isfinite(Vt))
    assert O.sigma_err(s, s_ref) <= 1e-5, (M, N, O.sigma_err(s, s_ref))
    assert np.all(np.diff(s) <= 0)
    tol = 1e-5 * max(N, 1)
    assert O.residual(A, U, s, Vt) <= tol, (M, N, O.residual(A, U, s, Vt))
    assert O.orth_err(U) <= tol, (M, N, O.orth_err(U))
    assert O.orth_err(Vt.T) <= tol, (M, N, O.orth_err(Vt.T))


EDGE = [(1, 1), (2, 1), (2, 2), (3, 3), (5, 2), (7, 7), (31, 31), (32, 32), (33, 33), (64, 32), (65, 64),
        (100, 3), (128, 128), (200, 199), (511, 17), (512, 512), (512, 16), (300, 257)]


def mixed_batch(seed, count):
    rng = np.random.default_rng(seed)
    mats = []
    for k in range(count):
        M = int(rng.integers(32, 513))
        N = int(rng.integers(16, M + 1))
        mats.append(rng.standard_normal((M, N)).astype(np.float32))
    return mats


def test_batched_edge_shapes_match_lapack():
    rng = np.random.default_rng(3)
    mats = [rng.uniform(-1, 1, (m, n)).astype(np.float32) for m, n in EDGE]
    s, U, Vt, st = P.svd_batched(mats)
    assert st == [0] * len(mats)
    for k, A in enumerate(mats):
        check(A, s[k], U[k], Vt[k])


def test_batched_random_mix_matches_lapack():
    mats = mixed_batch(11, 120)
    s, U, Vt, st = P.svd_batched(mats)
    assert st == [0] * len(mats)
    for k, A in enumerate(mats):
        check(A, s[k], U[k], Vt[k])


def test_batched_special_spectra():
    rng = np.random.default_rng(5)
    mats = [np.zeros((12, 9), np.float32), -np.eye(8, dtype=np.float32), np.ones((16, 16), np.float32),
            np.diag(np.arange(1, 12, dtype=np.float32))]
    # graded: Q1 diag(10^(-6 i/(N-1))) Q2^T
    N = 96
    Q1, _ = np.linalg.qr(rng.standard_normal((128, N)))
    Q2, _ = np.linalg.qr(rng.standard_normal((N, N)))
    mats.append((Q1 * 10.0 ** (-6 * np.arange(N) / (N - 1))) @ Q2.T)
    # rank 2
    mats.append((rng.standard_normal((40, 2)) @ rng.standard_normal((2, 30))))
    mats = [m.astype(np.float32) for m in mats]
    s, U, Vt, st = P.svd_batched(mats)
    assert st == [0] * len(mats)
    for k, A in enumerate(mats):
        check(A, s[k], U[k], Vt[k])


def test_batched_result_is_the_same_alone_and_in_a_mix():
    mats = mixed_batch(21, 40)
    s_mix, U_mix, V_mix, _ = P.svd_batched(mats)
    for k in (0, 7, 39):
        s1, U1, V1, _ = P.svd_batched([mats[k]])
        assert torch.equal(s1[0], s_mix[k]) and torch.equal(U1[0], U_mix[k]) and torch.equal(V1[0], V_mix[k])


def test_batched_is_deterministic():
    mats = mixed_batch(8, 30)
    a = P.svd_batched(mats)
    b = P.svd_batched(mats)
    for k in range(len(mats)):
        assert torch.equal(a[0][k], b[0][k]) and torch.equal(a[1][k], b[1][k]) and torch.equal(a[2][k], b[2][k])


def test_batched_flags_a_nonfinite_matrix_only():
    mats = mixed_batch(4, 6)
    mats[2] = mats[2].copy()
    mats[2][3, 1] = np.nan
    s, U, Vt, st = P.svd_batched(mats, check=False)
    assert st[2] == P.PACO_ERR_NONFINITE
    assert [c for k, c in enumerate(st) if k != 2] == [0] * 5
    for k in (0, 1, 3, 4, 5):
        check(mats[k], s[k], U[k], Vt[k])


def test_batched_wide_rows_match_lapack():
    # rows wider than 512 columns take the segmented sweeps
    rng = np.random.default_rng(17)
    shapes = [(600, 513), (700, 650), (1100, 600), (2048, 64), (530, 530), (64, 60)]
    mats = [rng.standard_normal(s).astype(np.float32) for s in shapes]
    s, U, Vt, st = P.svd_batched(mats)
    assert st == [0] * len(mats)
    for k, A in enumerate(mats):
        check(A, s[k], U[k], Vt[k])


def test_batched_matches_single_matrix_path_within_tolerance():
    mats = mixed_batch(13, 5)
    s, U, Vt, _ = P.svd_batched(mats)
    for k, A in enumerate(mats):
        s1, _, _ = P.svd(torch.from_numpy(A).cuda())
        ref = s1.cpu().numpy().astype(np.float64)
        assert O.sigma_err(s[k].cpu().numpy().astype(np.float64), ref) <= 2e-5
