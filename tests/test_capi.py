"""CPU tests of the C ABI library: it loads, exports every entry point that
include/paco_svd.h declares, and its host-side logic (tiling blob, buffer
sizes, argument validation, the svd_main CLI's argument handling) behaves as
the reference's host code does.  No kernel runs here."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

import oracle as O
import pacosvd as P

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "paco_svd.h")
PKG = os.path.join(ROOT, "paco-svd_b200")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"^[A-Za-z_][\w\s\*]*?\b(\w+)\s*\(", src, flags=re.M)
    return sorted(set(n for n in names if n not in ("if", "defined")))


def test_header_declares_the_reference_entry_points():
    names = declared_functions()
    for ref in ("upper_bidiagonalization", "svd_DC", "getTilingSize", "GenerateTiling"):
        assert ref in names


@pytest.mark.parametrize("name", declared_functions())
def test_library_exports_declared_symbol(name):
    L = ctypes.CDLL(P.LIB_PATH)
    assert hasattr(L, name), f"{name} declared in paco_svd.h but not exported"


@pytest.mark.parametrize("N", [1, 2, 3, 4, 5, 6, 7, 8, 9, 31, 32, 33, 100, 4096])
def test_tiling_blob_holds_the_reference_leaf_partition(N):
    blob = P.generate_tiling(N)
    assert len(blob) == P.tiling_size(N)
    hdr = np.frombuffer(blob[:32], np.uint32)
    assert hdr[0] == 0x4F434150 and hdr[1] == N and hdr[3] == 32
    leaves = np.frombuffer(blob[32:], np.uint32).reshape(-1, 2)
    assert hdr[2] == len(leaves)
    assert [tuple(map(int, x)) for x in leaves] == O.leaf_partition(N)


def test_buffer_sizes_follow_main_cpp():
    M, N = 64, 32
    b = P.buffer_sizes(M, N)
    # main.cpp:33-43
    assert b["U"] == M * M * 4 and b["A"] == M * N * 4 and b["Vt"] == N * N * 4
    assert b["d"] == N * 4 and b["e"] == (N - 1) * 4 and b["tauq"] == N * 4 and b["taup"] == (N - 1) * 4
    assert b["qt"] == 2 * N * N * 4 and b["wt"] == 2 * N * N * 4 and b["idx"] == 16 * N * 4
    assert b["workspace"] > 0 and b["tiling"] == P.tiling_size(N)


def test_workspace_size_rejects_bad_shapes():
    assert P.workspace_size(4, 8) == 0          # M < N
    assert P.workspace_size(10, 0) == 0         # N = 0
    assert P.workspace_size(10000, P.PACO_MAX_N + 1) == 0
    assert P.workspace_size(64, 32) > 0


def test_entry_points_validate_before_touching_the_device():
    L = P.lib()
    nul = None
    # M < N (main.cpp:25-29 rejects it)
    assert L.upper_bidiagonalization(4, 8, *([nul] * 9)) == P.PACO_ERR_INVALID_ARG
    assert L.svd_DC(4, 8, *([nul] * 11)) == P.PACO_ERR_INVALID_ARG
    # N beyond the stage-1 limit
    assert L.upper_bidiagonalization(9000, 9000, *([nul] * 9)) == P.PACO_ERR_UNSUPPORTED
    # valid shape, missing buffers
    assert L.upper_bidiagonalization(64, 32, *([nul] * 9)) == P.PACO_ERR_INVALID_ARG
    assert L.svd_DC(64, 32, *([nul] * 11)) == P.PACO_ERR_INVALID_ARG
    assert L.paco_svd(64, 32, *([nul] * 4), nul, 0, nul) == P.PACO_ERR_INVALID_ARG
    h = ctypes.c_void_p()
    assert L.paco_ctx_create(3, 5, ctypes.byref(h)) == P.PACO_ERR_INVALID_ARG


def test_version_string():
    assert b"sm_100a" in P.lib().paco_version()


def test_svd_main_rejects_wide_matrix(tmp_path):
    exe = os.path.join(PKG, "svd_main")
    (tmp_path / "args.txt").write_text("3 5")
    r = subprocess.run([exe, "--args", str(tmp_path / "args.txt"), "--input", str(tmp_path / "A.bin"),
                        "--output", str(tmp_path / "out")], capture_output=True, text=True, timeout=60)
    assert r.returncode == 1
    assert "M must be greater than N" in r.stderr


def test_svd_main_reports_short_input(tmp_path):
    exe = os.path.join(PKG, "svd_main")
    (tmp_path / "args.txt").write_text("8 4")
    np.zeros(5, np.float32).tofile(tmp_path / "A.bin")
    r = subprocess.run([exe, "--args", str(tmp_path / "args.txt"), "--input", str(tmp_path / "A.bin"),
                        "--output", str(tmp_path / "out")], capture_output=True, text=True, timeout=60)
    assert r.returncode == 1 and "expected" in r.stderr


def test_noalloc_scratch_covers_its_largest_shape():
    # paco_svd_noalloc serves M <= 1024, N <= 512 from a 16 MiB device array
    assert P.lib().paco_svd_workspace_size(1024, 512) <= 16 << 20


def test_workspace_covers_the_two_stage_buffers():
    # from N = 1024 on, paco_svd_workspace_size also reserves the two-stage
    # path's band (N x 3b) and its two chasing-reflector stores
    # (N x ceil((N-1)/b) x b floats each), sized for the widest band b = 64
    L = P.lib()
    for M, N in ((1023, 1023), (1024, 1024), (4096, 4096), (8192, 4096)):
        ws = L.paco_svd_workspace_size(M, N)
        if N < 1024:
            continue
        jmax = (N - 2 + 64) // 64
        extra = 4 * (N * 3 * 64 + 2 * N * jmax * 64)
        assert ws >= extra
    a, b = L.paco_svd_workspace_size(1023, 1023), L.paco_svd_workspace_size(1024, 1024)
    assert b - a >= 4 * 2 * 1024 * 16 * 64  # the step at N = 1024


def test_batched_workspace_rejects_bad_shapes():
    assert P.batched_workspace_size([(4, 8)]) == 0               # M < N
    assert P.batched_workspace_size([(10, 0)]) == 0              # N = 0
    # beyond the one-CTA-per-matrix limit only lists of one shape (the multi-matrix form)
    assert P.batched_workspace_size([(2049, 10), (2049, 11)]) == 0
    assert P.batched_workspace_size([(2049, 10), (100, 10)]) == 0
    assert P.batched_workspace_size([(2049, 10)] * 3) == P.lib().paco_svd_multi_workspace_size(3, 2049, 10) > 0
    assert P.batched_workspace_size([]) == 0


def test_batched_entry_validates_before_touching_the_device():
    import ctypes as C
    L = P.lib()
    Ms, Ns = (C.c_int * 2)(3000, 100), (C.c_int * 2)(10, 10)
    nul = (C.c_void_p * 2)(None, None)
    # a large matrix among other shapes has no kernel
    assert L.paco_svd_batched(2, Ms, Ns, nul, nul, nul, nul, None, None, 0, None) == P.PACO_ERR_UNSUPPORTED
    # one large shape goes to the multi-matrix form, which checks its pointers
    assert L.paco_svd_batched(1, Ms, Ns, nul, nul, nul, nul, None, None, 0, None) == P.PACO_ERR_INVALID_ARG
    assert L.paco_svd_multi(1, 3000, 10, nul, nul, nul, nul, None, None, 0, None) == P.PACO_ERR_INVALID_ARG
    Ms[0] = 3
    assert L.paco_svd_batched(1, Ms, Ns, nul, nul, nul, nul, None, None, 0, None) == P.PACO_ERR_INVALID_ARG


def test_serving_trace_generators():
    import serve as S
    arr = S.poisson_arrivals(2000.0, 1.0, 3)
    assert 1800 < len(arr) < 2200 and np.all(np.diff(arr) > 0) and arr[-1] < 1.0
    M, N, g = S.serving_shapes(20000, 4)
    assert M.min() >= 16 and M.max() <= 2048 and np.all(N <= M) and np.all(N >= np.maximum(1, M // 4))
    assert 0.08 < np.mean(M > 256) < 0.12 and 0.18 < g.mean() < 0.22
    assert S.footprint(64, 32) > 4 * (64 * 32 + 64 * 64)


def test_tune_table_defaults_and_round_trip():
    assert P.tune_get(300, 200) == [1, 16, 1, 0]
    P.tune_set(301, 201, [1, 32, 0, 0])
    assert P.tune_get(301, 201) == [1, 32, 0, 0]
    P.tune_set(301, 201, [1, 16, 1, 1])                # last columns kept on the panel kernel
    assert P.tune_get(301, 201) == [1, 16, 1, 1]
    assert P.tune_get(300, 200) == [1, 16, 1, 0]     # other shapes keep the defaults
    for bad in ([2, 16, 1, 0], [1, 2, 1, 0], [1, 16, 3, 0], [1, 1000, 1, 0], [1, 16, 1, 2]):
        with pytest.raises(P.PacoError):
            P.tune_set(301, 201, bad)
    with pytest.raises(P.PacoError):
        P.tune_set(4, 8, [1, 16, 1, 0])               # M < N


def test_tuning_fields_validate_and_round_trip():
    M, N = 3001, 1500
    assert P.tune_param(M, N, "wy") == 0 and P.tune_param(M, N, "qb") == 0
    assert P.tune_param(M, N, "wy", 64) == 64 and P.tune_param(M, N, "wy") == 64
    assert P.tune_param(M, N, "qb", 32) == 32 and P.tune_param(M, N, "mk", 8) == 8
    assert P.tune_param(M, N, "ts") == 0 and P.tune_param(M, N, "ts", 64) == 64
    for name, bad in (("wy", 96), ("qb", 48), ("mk", 9), ("rows_per_cta", 2), ("tc", 2), ("ts", 48)):
        with pytest.raises(P.PacoError):
            P.tune_param(M, N, name, bad)
    # paco_tune_set rewrites the first four fields and keeps the tile shapes
    P.tune_set(M, N, [1, 8, 1, 0])
    assert P.tune_get(M, N) == [1, 8, 1, 0] and P.tune_param(M, N, "wy") == 64
    assert P.lib().paco_tune_param(M, N, 9, 0) == -1 and P.lib().paco_tune_param(0, 0, 0, -1) == -1
    for f, v in (("wy", 0), ("qb", 0), ("mk", 0), ("ts", 0)):
        P.tune_param(M, N, f, v)
    P.tune_set(M, N, [1, 16, 1, 0])
