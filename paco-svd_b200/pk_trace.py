#!/usr/bin/env python
"""Phase trace of one panel of the persistent stage-1 panel kernel.

    python pk_trace.py M N P0

runs stage 1 (upper_bidiagonalization) three times on an M x N N(0,1)
matrix with PACO_PK_TRACE=P0 set, then reads the phase stamps that CTA 0 and
the last CTA of the panel starting at column P0 wrote into the stage-1
workspace (%globaltimer, about 0.26 us resolution) and prints, per column step,
the time of each phase: the row reflector from the partial records
(rowref), the row pass, the partial records' writes, grid barrier A with the
column reflector, the column pass and grid barrier B; then their means over
steps 1..30 and the step period.  A debugging and tuning aid: the kernel runs
at full speed, only the two CTAs' thread 0 write a few stamps per step.
"""
import ctypes
import os
import sys

import numpy as np


def main(M, N, p0):
    os.environ["PACO_PK_TRACE"] = str(p0)
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    import torch
    import pacosvd as P
    lib = P.lib()
    lib.paco_debug_trace_offset.restype = ctypes.c_size_t
    lib.paco_debug_trace_offset.argtypes = [ctypes.c_int, ctypes.c_int]
    off = lib.paco_debug_trace_offset(M, N)
    torch.manual_seed(0)
    A = torch.randn(M, N, device="cuda")
    for _ in range(3):
        g = P.bidiag(A)
        torch.cuda.synchronize()
    tr = g["workspace"][off: off + 33 * 16 * 2 * 8].view(torch.int64).cpu().numpy().reshape(33, 16, 2)
    names = ["rowref", "rowpass", "partials", "barA+colref", "colpass", "barB"]
    print(f"M={M} N={N} p0={p0}: per-step phase durations (us), CTA0 / last CTA")
    rows = []
    for s in range(33):
        d = np.diff(tr[s, :7, 0].astype(np.float64)) / 1e3
        dl = np.diff(tr[s, :7, 1].astype(np.float64)) / 1e3
        rows.append(np.concatenate([d, dl]))
        print(f"step {s:2d}: " + " ".join(f"{n}={x:6.2f}/{y:6.2f}" for n, x, y in zip(names, d, dl)) +
              f"  waited={tr[s, 7, 0] / 1e3:.2f}us batches={tr[s, 8, 0]}")
    r = np.array(rows)[1:31]
    ok = np.all(np.abs(r) < 1e4, axis=1)
    print("mean CTA0   : " + " ".join(f"{n}={x:6.2f}" for n, x in zip(names, r[ok, :6].mean(axis=0))))
    print("mean lastCTA: " + " ".join(f"{n}={x:6.2f}" for n, x in zip(names, r[ok, 6:].mean(axis=0))))
    starts = tr[:32, 0, 0].astype(np.float64)
    print("period us:", np.round(np.diff(starts) / 1e3, 2).tolist())


if __name__ == "__main__":
    if len(sys.argv) != 4:
        raise SystemExit(__doc__)
    main(int(sys.argv[1]), int(sys.argv[2]), int(sys.argv[3]))
