"""One SVD for a profiler: `python paco-svd_b200/profile_svd.py M N [--warm W] [--qr 0|1|2]`.

Runs W warm-up SVDs of an M x N N(0,1) matrix (seed 0) through the one-shot
workspace path, then exactly one more, with CUDA-graph capture off so that a
profiler sees every kernel launch on its own (`ncu -s <skip> -c <count>`
counts them).  Prints the status and the number of library launches of the
last SVD.  --qr sets the QR-first mode for the shape (0 off, 1 on, 2 automatic),
--ts the two-stage band width (32 or 64; 0 off).

`python paco-svd_b200/profile_svd.py batched COUNT [--warm W]` runs the batched
form instead: W warm-up calls and one more on COUNT N(0,1) matrices with the
shapes of the 10,000-matrix batched workload (M uniform on [32, 512], N on
[16, M], seed 0), three kernel launches per call."""
import argparse
import ctypes
import os
import sys

os.environ.setdefault("PACO_GRAPHS", "0")
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))

import torch  # noqa: E402

import pacosvd as P  # noqa: E402


def batched(count, warm):
    import numpy as np
    from workloads import WORKLOADS, batched_shapes
    wl = dict(WORKLOADS["cfg4"], count=count)
    shapes = batched_shapes(wl, 0)
    rng = np.random.default_rng(0)
    b = P.Batch(shapes)
    b.load([rng.standard_normal(s, dtype=np.float32) for s in shapes])
    L = P.lib()
    L.paco_launch_count.restype = ctypes.c_ulonglong
    for _ in range(warm):
        b.run()
    torch.cuda.synchronize()
    c0 = L.paco_launch_count()
    b.run()
    torch.cuda.synchronize()
    bad = sum(1 for x in b.statuses() if x != P.PACO_OK)
    print("matrices", count, "with a non-zero status", bad, "launches of the last call", L.paco_launch_count() - c0)
    sys.exit(0 if bad == 0 else 1)


def main():
    if len(sys.argv) > 1 and sys.argv[1] == "batched":
        ap = argparse.ArgumentParser()
        ap.add_argument("what")
        ap.add_argument("count", type=int)
        ap.add_argument("--warm", type=int, default=1)
        a = ap.parse_args()
        batched(a.count, a.warm)
        return
    ap = argparse.ArgumentParser()
    ap.add_argument("M", type=int)
    ap.add_argument("N", type=int)
    ap.add_argument("--warm", type=int, default=1)
    ap.add_argument("--qr", type=int, default=None)
    ap.add_argument("--ts", type=int, default=None)
    a = ap.parse_args()
    if a.qr is not None:
        P.tune_qr(a.M, a.N, a.qr)
    if a.ts is not None:
        P.tune_param(a.M, a.N, "ts", a.ts)
    torch.manual_seed(0)
    A = torch.randn(a.M, a.N, device="cuda")
    W = P.Workspace(a.M, a.N)
    L = P.lib()
    L.paco_launch_count.restype = ctypes.c_ulonglong
    for _ in range(a.warm):
        W.run(A)
    torch.cuda.synchronize()
    c0 = L.paco_launch_count()
    W.run(A)
    torch.cuda.synchronize()
    code, _ = P.sync_status(W.ws)
    print("status", code, "launches of the last SVD", L.paco_launch_count() - c0)
    sys.exit(0 if code == P.PACO_OK else 1)


if __name__ == "__main__":
    main()
