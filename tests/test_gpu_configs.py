"""GPU parity at the benchmark configurations' full sizes, through the C ABI
(paco_svd), on the same seeded matrices bench.py runs (workloads.make_matrix):

  cfg2a  4096 x 4096, entries iid N(0,1)
  cfg2b  4096 x 4096, graded spectrum sigma_i = 10^(-6 i/(N-1))
  cfg3   8192 x 4096, 512 clusters of 8 singular values, relative spacing
         1e-7 inside a cluster (the deflation stress case)

Each result is checked against FP64 LAPACK dgesdd of the FP32 input (the
oracle of the reference's scripts/verify_svd.py:55-65,89, in double
precision), with the tolerances (Frobenius norms):
  sigma:          max_i |s_i - s_ref_i| / s_ref_1      <= 1e-5
  residual:       ||A - U[:, :N] S Vt||_F / ||A||_F    <= 1e-5 * N
  orthogonality:  ||U^T U - I||_F, ||V^T V - I||_F     <= 1e-5 * N
For the graded and clustered generators the singular values are also checked
against the exact spectrum the generator built (same 1e-5 bound).
Residual and orthogonality are computed in FP64 on the device."""
import numpy as np
import pytest
import scipy.linalg

import pacosvd as P
from workloads import WORKLOADS, make_matrix

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

SIGMA_TOL = 1e-5


def device_errors(A, s, U, Vt):
    """(residual, orth_U, orth_V) in FP64 on the device."""
    M, N = A.shape
    Ad, Ud, Vd, sd = A.double(), U.double(), Vt.double(), s.double()
    res = (torch.linalg.norm(Ad - (Ud[:, :N] * sd[None, :]) @ Vd) / torch.linalg.norm(Ad)).item()
    ou = torch.linalg.norm(Ud.T @ Ud - torch.eye(M, dtype=torch.float64, device=A.device)).item()
    ov = torch.linalg.norm(Vd @ Vd.T - torch.eye(N, dtype=torch.float64, device=A.device)).item()
    return res, ou, ov


@pytest.mark.parametrize("name", ["cfg2a", "cfg2b", "cfg3"])
def test_config_matches_dgesdd(name):
    wl = WORKLOADS[name]
    A_np, sig_exact = make_matrix(wl, seed=1234, with_sigma=True)
    M, N = A_np.shape
    A = torch.from_numpy(A_np).cuda()
    s, U, Vt = P.svd(A)
    assert torch.isfinite(s).all() and torch.isfinite(U).all() and torch.isfinite(Vt).all()
    res, ou, ov = device_errors(A, s, U, Vt)
    del U, Vt
    torch.cuda.empty_cache()
    s = s.cpu().numpy().astype(np.float64)
    ref = scipy.linalg.svd(A_np.astype(np.float64), compute_uv=False, lapack_driver="gesdd")
    err = float(np.max(np.abs(s - ref)) / ref[0])
    print(f"{name}: sigma_err(dgesdd)={err:.3e} residual={res:.3e} orth_U={ou:.3e} orth_V={ov:.3e}"
          + (f" sigma_err(exact)={np.max(np.abs(s - sig_exact)) / sig_exact[0]:.3e}" if sig_exact is not None
             else ""))
    assert np.all(np.diff(s) <= 0), "sigma must be descending"
    assert err <= SIGMA_TOL
    assert res <= 1e-5 * N
    assert ou <= 1e-5 * N and ov <= 1e-5 * N
    if sig_exact is not None:
        assert np.max(np.abs(s - sig_exact)) / sig_exact[0] <= SIGMA_TOL
