"""GPU parity tests: the CUDA library (through its C ABI) against the oracle
and the LAPACK goldens.

Tolerances (FP32 outputs, Frobenius norms):
  sigma:          max_i |s_i - s_ref_i| / s_ref_1            <= 1e-5
  residual:       ||A - U[:, :N] S Vt||_F / ||A||_F          <= 1e-5 * N
  orthogonality:  ||U^T U - I||_F, ||V^T V - I||_F           <= 1e-5 * N
Stage 1 alone: d, e against the oracle's FP64 values (same reflector
convention, so the signs agree) within 5e-5 * max(|d|, |e|) (the largest
deviation measured on these shapes is 2.7e-5 of it: single entries of the
bidiagonal are less well conditioned than the singular values); every reflector is
exactly orthogonal, tau * (1 + |v[1:]|^2) = 2 within 1e-4, for the vectors
the GPU left in A; tau itself is compared with the oracle only loosely
(1e-2): late reflectors come from small trailing matrices whose FP32
rounding has grown with the step count, so their tau is ill-conditioned."""
import numpy as np
import pytest

import oracle as O
import pacosvd as P
from conftest import load_svd_golden

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

GOLD = load_svd_golden()
SIGMA_TOL = 1e-5


def tol_n(N):
    return 1e-5 * max(N, 1)


def run_svd(A_np):
    A = torch.from_numpy(np.ascontiguousarray(A_np, dtype=np.float32)).cuda()
    s, U, Vt = P.svd(A)
    return (s.cpu().numpy().astype(np.float64), U.cpu().numpy().astype(np.float64),
            Vt.cpu().numpy().astype(np.float64))


def check_svd(A, s, U, Vt, s_ref):
    M, N = A.shape
    assert np.all(np.isfinite(s)) and np.all(np.isfinite(U)) and np.all(np.isfinite(Vt))
    assert O.sigma_err(s, s_ref) <= SIGMA_TOL
    assert np.all(np.diff(s) <= 0), "sigma must be descending"
    assert O.residual(A, U, s, Vt) <= tol_n(N)
    assert O.orth_err(U) <= tol_n(N)
    assert O.orth_err(Vt.T) <= tol_n(N)


@pytest.mark.parametrize("name", sorted(GOLD))
def test_svd_matches_lapack_golden_and_oracle(name):
    c = GOLD[name]
    A = c["A"]
    s, U, Vt = run_svd(A)
    check_svd(A, s, U, Vt, c["sigma_d"])
    so, _, _ = O.svd(A)
    assert O.sigma_err(s, so) <= SIGMA_TOL


SHAPES = [(1, 1), (5, 1), (2, 2), (3, 3), (4, 4), (7, 5), (32, 32), (33, 32), (64, 32), (65, 33), (96, 95),
          (100, 64), (129, 65), (200, 150), (300, 40), (257, 256)]


@pytest.mark.parametrize("shape", SHAPES)
def test_bidiag_matches_oracle(shape):
    M, N = shape
    rng = np.random.default_rng(M * 1000 + N)
    A = rng.standard_normal((M, N)).astype(np.float32)
    g = P.bidiag(torch.from_numpy(A).cuda())
    o = O.bidiag(A)
    nrm = np.linalg.norm(A.astype(np.float64))
    d = g["d"].cpu().numpy(); e = g["e"].cpu().numpy()
    scale = max(np.max(np.abs(o["d"])), np.max(np.abs(o["e"])) if N > 1 else 0.0)
    assert np.max(np.abs(d - o["d"])) <= 5e-5 * scale
    tq = g["tauq"].cpu().numpy().astype(np.float64)
    tp = g["taup"].cpu().numpy().astype(np.float64)
    Ah = g["A"].cpu().numpy().astype(np.float64)
    if N > 1:
        assert np.max(np.abs(e - o["e"])) <= 5e-5 * scale
        assert np.max(np.abs(tp - o["taup"])) <= 1e-2
    assert np.max(np.abs(tq - o["tauq"])) <= 1e-2
    for i in range(N):  # column reflectors: v = [1, A[i+1:, i]]
        if tq[i] != 0:
            assert abs(tq[i] * (1 + np.sum(Ah[i + 1:, i] ** 2)) - 2) <= 1e-4
    for i in range(N - 1):  # row reflectors: u = [1, A[i, i+2:]]
        if tp[i] != 0:
            assert abs(tp[i] * (1 + np.sum(Ah[i, i + 2:] ** 2)) - 2) <= 1e-4
    # U B Vt = A and orthogonality (verify_result.py:58-123,194-198)
    U = g["U"].cpu().numpy().astype(np.float64); Vt = g["Vt"].cpu().numpy().astype(np.float64)
    B = np.zeros((M, N)); B[np.arange(N), np.arange(N)] = d
    if N > 1:
        B[np.arange(N - 1), np.arange(1, N)] = e
    assert np.linalg.norm(U @ B @ Vt - A) <= tol_n(N) * nrm
    assert O.orth_err(U) <= tol_n(N)
    assert O.orth_err(Vt.T) <= tol_n(N)
    # d on the diagonal of the returned A (upper_bidiagonalization.cpp:193-207)
    np.testing.assert_allclose(np.diag(Ah), d, rtol=0, atol=0)


@pytest.mark.parametrize("shape", [(64, 32), (130, 97), (256, 256), (512, 300)])
def test_svd_random_matches_lapack(shape):
    M, N = shape
    rng = np.random.default_rng(7 + M)
    A = rng.standard_normal((M, N)).astype(np.float32)
    s, U, Vt = run_svd(A)
    check_svd(A, s, U, Vt, O.lapack_dgesdd_sigma(A))


def test_svd_1024_graded_spectrum():
    n = 1024
    rng = np.random.default_rng(11)
    Q1, _ = np.linalg.qr(rng.standard_normal((n, n)))
    Q2, _ = np.linalg.qr(rng.standard_normal((n, n)))
    sig = 10.0 ** (-6 * np.arange(n) / (n - 1))
    A = (Q1 * sig[None, :]) @ Q2.T
    A = A.astype(np.float32)
    s, U, Vt = run_svd(A)
    check_svd(A, s, U, Vt, O.lapack_dgesdd_sigma(A))


def test_svd_streamed_panels_match_lapack_and_repeat_bitwise():
    # 3200 x 3000: the first panels' rows do not fit in shared memory and are
    # streamed (with the next step's first batches prefetched); a stale row
    # would show in the residual, a race in the repeat
    rng = np.random.default_rng(29)
    A_np = rng.standard_normal((3200, 3000)).astype(np.float32)
    A = torch.from_numpy(A_np).cuda()
    r1 = P.svd(A)
    r2 = P.svd(A)
    for x, y in zip(r1, r2):
        assert torch.equal(x, y)
    s, U, Vt = (x.cpu().numpy().astype(np.float64) for x in r1)
    check_svd(A_np, s, U, Vt, O.lapack_dgesdd_sigma(A_np))


@pytest.mark.parametrize("shape", [(65, 33), (300, 200), (900, 777), (1300, 800)])
def test_cluster_tail_and_panel_kernel_both_match_lapack(shape):
    # the last columns of stage 1 run on one thread-block cluster when their
    # block fits in its shared memory (all of these shapes, from column 0 or
    # later), or on the grid-wide panel kernel (tuning entry no_tail = 1)
    M, N = shape
    rng = np.random.default_rng(M + 3 * N)
    A = rng.standard_normal((M, N)).astype(np.float32)
    ref = O.lapack_dgesdd_sigma(A)
    try:
        for no_tail in (0, 1):
            P.tune_set(M, N, [1, 16, 1, no_tail])
            s, U, Vt = run_svd(A)
            check_svd(A, s, U, Vt, ref)
    finally:
        P.tune_set(M, N, [1, 16, 1, 0])


def test_results_are_bitwise_deterministic():
    rng = np.random.default_rng(5)
    A = torch.from_numpy(rng.standard_normal((300, 200)).astype(np.float32)).cuda()
    r1 = P.svd(A)
    r2 = P.svd(A)
    for x, y in zip(r1, r2):
        assert torch.equal(x, y)


def test_dropin_two_kernel_flow_with_tiling_blob():
    """main.cpp:56-165: caller-allocated buffers, upper_bidiagonalization then
    svd_DC with the GenerateTiling blob on the device."""
    A = GOLD["cfg1"]["A"]
    M, N = A.shape
    b = P.bidiag(torch.from_numpy(A).cuda())
    s, U, Vt = P.svd_dc(M, b["d"], b["e"], b["U"], b["Vt"], tiling=P.generate_tiling(N))
    check_svd(A, s.cpu().numpy().astype(np.float64), U.cpu().numpy().astype(np.float64),
              Vt.cpu().numpy().astype(np.float64), GOLD["cfg1"]["sigma_d"])


def test_tiling_blob_for_another_n_is_reported():
    A = GOLD["cfg1"]["A"]
    M, N = A.shape
    b = P.bidiag(torch.from_numpy(A).cuda())
    with pytest.raises(P.PacoError) as ei:
        P.svd_dc(M, b["d"], b["e"], b["U"], b["Vt"], tiling=P.generate_tiling(N + 1))
    assert ei.value.code == P.PACO_ERR_BAD_TILING


def test_nonfinite_input_is_reported():
    A = np.ones((16, 8), np.float32)
    A[3, 2] = np.nan
    with pytest.raises(P.PacoError) as ei:
        P.svd(torch.from_numpy(A).cuda())
    assert ei.value.code == P.PACO_ERR_NONFINITE


def test_host_context_matches_device_path():
    A = GOLD["u48x17"]["A"]
    ctx = P.HostContext(*A.shape)
    s, U, Vt = ctx.svd(A)
    ctx.close()
    check_svd(A, s.astype(np.float64), U.astype(np.float64), Vt.astype(np.float64), GOLD["u48x17"]["sigma_d"])


def test_svd_main_cli_writes_reference_files(tmp_path):
    """The svd_main file contract (main.cpp:20-24,64,171-174) end to end."""
    import os
    import subprocess
    A = GOLD["cfg1"]["A"]
    M, N = A.shape
    (tmp_path / "args.txt").write_text(f"{M} {N}")
    (tmp_path / "input").mkdir()
    A.tofile(tmp_path / "input" / "A_gm.bin")
    work = tmp_path / "build"
    work.mkdir()
    exe = os.path.join(os.path.dirname(P.LIB_PATH), "svd_main")
    r = subprocess.run([exe], cwd=work, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    s = np.fromfile(tmp_path / "output" / "sigma.bin", np.float32).astype(np.float64)
    U = np.fromfile(tmp_path / "output" / "U.bin", np.float32).reshape(M, M).astype(np.float64)
    Vt = np.fromfile(tmp_path / "output" / "Vt.bin", np.float32).reshape(N, N).astype(np.float64)
    check_svd(A, s, U, Vt, GOLD["cfg1"]["sigma_d"])
    # and the reference's own checker on those files (scripts/verify_svd.py:35-65,102-104):
    # orthogonality and sigma with rtol 1e-3 / atol 1e-5, reconstruction max-abs <= 1e-3
    assert np.allclose(U @ U.T, np.eye(M), rtol=1e-3, atol=1e-5)
    assert np.allclose(Vt @ Vt.T, np.eye(N), rtol=1e-3, atol=1e-5)
    assert np.allclose(s, GOLD["cfg1"]["sigma_s"], rtol=1e-3, atol=1e-5)
    S = np.zeros((M, N))
    S[np.arange(N), np.arange(N)] = s
    assert np.max(np.abs(U @ S @ Vt - A)) <= 1e-3


def test_svd_main_stage1_writes_checker_files(tmp_path):
    """svd_main --stage1 writes U.bin, B.bin, Vt.bin (the stage-1 hook of
    main.cpp:139-151); they pass the reference's stage-1 checker criteria
    (scripts/verify_result.py:7-9,58-123,194-198), and B equals the LAPACK
    golden B that golden_files.py writes (sgebrd, scripts/bidiag_gen.f90:122)
    up to the signs of its entries, within 1e-5 of its largest entry."""
    import os
    import subprocess
    import golden_files as G
    M, N = 96, 64
    (tmp_path / "args.txt").write_text(f"{M} {N}")
    G.write_goldens(str(tmp_path), generate=True, seed=5)
    work = tmp_path / "build"
    work.mkdir()
    exe = os.path.join(os.path.dirname(P.LIB_PATH), "svd_main")
    r = subprocess.run([exe, "--stage1"], cwd=work, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr

    def rd(name, shape):
        return np.fromfile(tmp_path / name, np.float32).reshape(shape).astype(np.float64)

    A = rd("input/A_gm.bin", (M, N))
    U, B, Vt = rd("output/U.bin", (M, M)), rd("output/B.bin", (M, N)), rd("output/Vt.bin", (N, N))
    assert np.allclose(U @ U.T, np.eye(M), rtol=1e-3, atol=1e-5)
    assert np.allclose(Vt @ Vt.T, np.eye(N), rtol=1e-3, atol=1e-5)
    band = np.zeros((M, N), bool)
    band[np.arange(N), np.arange(N)] = True
    band[np.arange(N - 1), np.arange(1, N)] = True
    assert np.max(np.abs(B[~band])) == 0.0
    assert np.max(np.abs(U @ B @ Vt - A)) <= 1e-3
    Bg = rd("output/B_golden.bin", (M, N))
    assert np.max(np.abs(np.abs(B) - np.abs(Bg))) <= 1e-5 * np.max(np.abs(Bg))
