"""The golden-file CLI (paco-svd_b200/golden_files.py), on the CPU: the files
it writes have the reference's layout (scripts/gen_data.py:160-182) and pass
the reference's stage-1 checker criteria (scripts/verify_result.py:7-9,
58-123,194-198): U U^T = I and Vt Vt^T = I within rtol 1e-3 / atol 1e-5, B
upper bidiagonal (nothing above 1e-5 off the two bands) and
max |U B Vt - A| <= 1e-3."""
import os
import subprocess
import sys

import numpy as np
import pytest

import golden_files as G


def read(path, shape):
    a = np.fromfile(path, np.float32)
    assert a.size == int(np.prod(shape)), path
    return a.reshape(shape).astype(np.float64)


def stage1_checker_passes(A, U, B, Vt):
    M, N = A.shape
    assert np.allclose(U @ U.T, np.eye(M), rtol=1e-3, atol=1e-5)
    assert np.allclose(Vt @ Vt.T, np.eye(N), rtol=1e-3, atol=1e-5)
    off = B.copy()
    off[np.arange(N), np.arange(N)] = 0
    if N > 1:
        off[np.arange(N - 1), np.arange(1, N)] = 0
    assert np.max(np.abs(off)) <= 1e-5
    assert np.max(np.abs(U @ B @ Vt - A)) <= 1e-3


@pytest.mark.parametrize("shape", [(64, 32), (97, 97), (150, 61)])
def test_golden_cli_writes_reference_layout(tmp_path, shape):
    M, N = shape
    (tmp_path / "args.txt").write_text(f"{M} {N}\n")
    here = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "paco-svd_b200")
    r = subprocess.run([sys.executable, os.path.join(here, "golden_files.py"), "--root", str(tmp_path),
                        "--generate", "--seed", "3"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    A = read(tmp_path / "input" / "A_gm.bin", (M, N))
    assert A.min() >= -10 and A.max() < 10
    U = read(tmp_path / "output" / "U_golden.bin", (M, M))
    B = read(tmp_path / "output" / "B_golden.bin", (M, N))
    Vt = read(tmp_path / "output" / "Vt_golden.bin", (N, N))
    s = read(tmp_path / "output" / "sigma_golden.bin", (N,))
    stage1_checker_passes(A, U, B, Vt)
    ref = np.linalg.svd(A, compute_uv=False)
    assert np.max(np.abs(s - ref)) <= 1e-6 * ref[0]
    # the bidiagonal has the same singular values
    assert np.max(np.abs(np.linalg.svd(B, compute_uv=False) - ref)) <= 1e-5 * ref[0]


def test_golden_cli_reads_an_existing_input(tmp_path):
    M, N = 40, 40
    (tmp_path / "args.txt").write_text(f"{M} {N}")
    (tmp_path / "input").mkdir()
    A = np.random.default_rng(0).standard_normal((M, N)).astype(np.float32)
    A.tofile(tmp_path / "input" / "A_gm.bin")
    G.write_goldens(str(tmp_path))
    U = read(tmp_path / "output" / "U_golden.bin", (M, M))
    B = read(tmp_path / "output" / "B_golden.bin", (M, N))
    Vt = read(tmp_path / "output" / "Vt_golden.bin", (N, N))
    stage1_checker_passes(A.astype(np.float64), U, B, Vt)


def test_golden_cli_rejects_m_below_n(tmp_path):
    (tmp_path / "args.txt").write_text("8 16")
    with pytest.raises(SystemExit):
        G.write_goldens(str(tmp_path), generate=True)
