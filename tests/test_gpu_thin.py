"""GPU tests of the thin-U form (paco_svd_thin: U is M x N, where the
reference always forms the M x M U, main.cpp:33,173), on the one-stage path
and on the QR-first path, against FP64 LAPACK dgesdd with the single-matrix
tolerances (Frobenius): sigma <= 1e-5 sigma_1, ||A - U S Vt|| / ||A|| and
||U^T U - I||, ||V^T V - I|| <= 1e-5 N.  Its U matches the first N columns of
paco_svd's U, and sigma and Vt match paco_svd's, within 1e-5 N entry-wise."""
import numpy as np
import pytest

import oracle as O
import pacosvd as P

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("shape,qr", [((1, 1), 2), ((7, 3), 2), ((300, 200), 2), ((1300, 1200), 2),
                                      ((2600, 1100), 2), ((2600, 1100), 0)])
def test_thin_u_matches_full_and_lapack(shape, qr):
    M, N = shape
    rng = np.random.default_rng(M * 7 + N)
    A = rng.standard_normal((M, N)).astype(np.float32)
    prev = P.tune_qr(M, N) if M > N and N >= 1024 else None
    try:
        if prev is not None:
            P.tune_qr(M, N, qr)
        s, U, Vt = P.svd_thin(torch.from_numpy(A).cuda())
        sf, Uf, Vtf = P.svd(torch.from_numpy(A).cuda())
    finally:
        if prev is not None:
            P.tune_qr(M, N, prev)
    assert U.shape == (M, N)
    s, U, Vt = (x.cpu().numpy().astype(np.float64) for x in (s, U, Vt))
    sf, Uf, Vtf = (x.cpu().numpy().astype(np.float64) for x in (sf, Uf, Vtf))
    tol = 1e-5 * max(N, 1)
    assert O.sigma_err(s, O.lapack_dgesdd_sigma(A)) <= 1e-5
    A64 = A.astype(np.float64)
    assert np.linalg.norm(A64 - (U * s[None, :]) @ Vt) / np.linalg.norm(A64) <= tol
    assert np.linalg.norm(U.T @ U - np.eye(N)) <= tol
    assert O.orth_err(Vt.T) <= tol
    assert np.max(np.abs(s - sf)) <= 1e-5 * sf[0]
    assert np.max(np.abs(U - Uf[:, :N])) <= tol
    assert np.max(np.abs(Vt - Vtf)) <= tol
