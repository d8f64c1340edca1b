#!/usr/bin/env python
"""Benchmark of the B200 SVD (libpacosvd.so).  The default workload is the
precision-form configuration: one 8192 x 4096 FP32 matrix whose spectrum is
512 clusters of 8 singular values (centres log-uniform in [1e-4, 1],
relative spacing 1e-7 inside a cluster), A = Q1 diag(sigma) Q2^T with
Haar-random Q1, Q2 from a seed; synthetic data.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--workload cfg3|cfg2a|cfg2b|cfg1|cfg4|cfg5]

A step is one full SVD (stage 1 bidiagonalization + U/Vt formation, stage 2
divide and conquer + final products) of a matrix already resident in HBM.
Metric: SVDs/s (whole job).  One process per GPU; the SVD does not shard, so
N > 1 runs independent replicas (weak scaling) and takes the max time over
ranks.  Between timed steps a 512 MiB buffer is written to flush L2.
Accuracy of the last step is reported against FP64 LAPACK dgesdd of the FP32
input (computed on the host, outside the timed region).

`--impl reference` times the reference's CPU path: the reference itself is
Ascend C for a Huawei NPU and cannot be built here, so its CPU path is the
LAPACK golden its own checker compares with (scripts/verify_svd.py:89,
numpy.linalg.svd = sgesdd in FP32 with the full U, on every host thread),
run on the full workload matrix at every step.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "paco-svd_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from workloads import WORKLOADS, batched_shapes, make_matrix  # noqa: E402

CPU_SAMPLE_N = 768  # oracle sample size (about 5 s of single-thread work)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1])); smax = float(p[2])
            except ValueError:
                continue
            for nm, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))), "measured"
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


def traffic_ratio(resident=False):
    """DRAM bytes per streamed byte of the persistent panel kernel, from the
    committed ncu summaries: profiles/bd_panel_pk_8192x4096.txt (a trailing
    matrix larger than L2, line 'dram_per_alg_byte: X') or, when the matrix
    fits L2, profiles/bd_panel_pk_4096_l2resident.txt ('dram_per_streamed_byte: X')."""
    name, key = (("bd_panel_pk_4096_l2resident.txt", "dram_per_streamed_byte:") if resident
                 else ("bd_panel_pk_8192x4096.txt", "dram_per_alg_byte:"))
    try:
        for ln in open(os.path.join(ROOT, "profiles", name)):
            if ln.startswith(key):
                return float(ln.split(":")[1])
    except Exception:
        pass
    return None


def max_over_ranks(total_ms, dist, device="cuda"):
    """Slowest rank's timed-region length (replicas run concurrently)."""
    if dist is None:
        return float(total_ms)
    import torch
    t = torch.tensor([float(total_ms)], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_value(world, steps, total_ms):
    """SVDs/s of the whole job: every rank ran `steps` SVDs in at most total_ms."""
    return world * steps / (total_ms / 1000.0)


def batched_accuracy(As, Us, Vts, sigmas):
    """Worst sigma error (against FP64 LAPACK dgesdd of the FP32 input),
    residual ||A - U S Vt||_F / ||A||_F and orthogonality ||Q^T Q - I||_F over
    a sample of batched results (numpy arrays, FP64 on the host)."""
    import scipy.linalg
    worst = {"sigma_err": 0.0, "residual": 0.0, "orth_U": 0.0, "orth_V": 0.0, "max_N": 0}
    for A, U, Vt, s in zip(As, Us, Vts, sigmas):
        A, U, Vt, s = (np.asarray(x, np.float64) for x in (A, U, Vt, s))
        n = A.shape[1]
        ref = scipy.linalg.svd(A, compute_uv=False, lapack_driver="gesdd")
        r = {"sigma_err": float(np.max(np.abs(s - ref)) / max(ref[0], np.finfo(float).tiny)),
             "residual": float(np.linalg.norm(A - (U[:, :n] * s[None, :]) @ Vt) / max(np.linalg.norm(A), 1e-300)),
             "orth_U": float(np.linalg.norm(U.T @ U - np.eye(U.shape[1]))),
             "orth_V": float(np.linalg.norm(Vt @ Vt.T - np.eye(n)))}
        for k, v in r.items():
            worst[k] = max(worst[k], v)
        worst["max_N"] = max(worst["max_N"], n)
    worst["matrices"] = len(As)
    worst["tolerance"] = {"sigma_err": 1e-5, "residual_and_orth": "1e-5 * N of each matrix"}
    return worst


def cpu_baseline_batched(wl, nsample=30):
    """Oracle port (FP64 C restatement, 1 thread) on `nsample` matrices drawn
    from the batch's size distribution: SVDs/s of that sample."""
    import oracle
    rng = np.random.default_rng(77)
    shapes = batched_shapes(dict(wl, count=nsample), 99)
    t = time.perf_counter()
    for M, N in shapes:
        oracle.svd(rng.standard_normal((M, N)).astype(np.float32))
    t = time.perf_counter() - t
    return {"value": nsample / t, "unit": "SVDs/s", "cores": 1, "kind": "port",
            "sample": f"oracle.svd on {nsample} N(0,1) matrices drawn from the batch's size distribution "
                      f"({t:.1f} s)"}


def cpu_oracle(wl, steps=1):
    """Oracle port (FP64 C restatement of the reference algorithm, 1 thread)
    on a CPU_SAMPLE_N-column sample with the workload's aspect ratio, scaled
    to the workload's SVDs/s by the M*N^2 work ratio.  A side figure only:
    the measured CPU baseline is lapack_svd_timed on the full matrix."""
    import oracle
    n = min(CPU_SAMPLE_N, wl["N"])
    A = make_matrix(dict(M=n * wl["M"] // wl["N"], N=n, gen=wl["gen"]), seed=99)
    times = []
    for _ in range(max(1, steps)):
        t = time.perf_counter()
        oracle.svd(A)
        times.append(time.perf_counter() - t)
    t = statistics.median(times)
    scale = (wl["M"] * wl["N"] ** 2) / (A.shape[0] * A.shape[1] ** 2)
    return {"value": 1.0 / (t * scale), "unit": "SVDs/s", "cores": 1, "kind": "port",
            "sample": f"oracle.svd on a {A.shape[0]}x{A.shape[1]} {wl['gen']} matrix, median of {len(times)} "
                      f"({t:.2f} s), scaled by the M*N^2 work ratio {scale:.1f} (extrapolated; not the baseline)"}


def host_threads():
    """Threads numpy's OpenBLAS runs LAPACK on (all host cores unless limited)."""
    threads = os.cpu_count() or 1
    try:
        import threadpoolctl
        threads = max([i.get("num_threads", 0) for i in threadpoolctl.threadpool_info()
                       if i.get("internal_api") == "openblas"] or [threads])
    except Exception:
        pass
    return int(threads)


def lapack_svd_timed(A, steps, budget_s):
    """Times numpy.linalg.svd(A, full_matrices=True) -- LAPACK sgesdd in FP32
    with the full M x M U, as the C ABI returns it, on every host thread --
    on the whole matrix: `steps` calls, or as many as fit in budget_s (at
    least one).  Returns the seconds of each call."""
    times = []
    t_all = time.perf_counter()
    for _ in range(max(1, steps)):
        t = time.perf_counter()
        np.linalg.svd(A, full_matrices=True)
        times.append(time.perf_counter() - t)
        if time.perf_counter() - t_all + times[-1] > budget_s:
            break
    return times


def cpu_baseline(wl, A):
    """The reference's CPU path (the LAPACK golden, sgesdd) on the workload's
    own full matrix, one call, every host thread."""
    times = lapack_svd_timed(A, 1, 0.0)
    t = times[0]
    return {"value": 1.0 / t, "unit": "SVDs/s", "cores": host_threads(), "kind": "lapack sgesdd",
            "sample": f"numpy.linalg.svd (OpenBLAS sgesdd, FP32, full U) on the workload's own "
                      f"{A.shape[0]}x{A.shape[1]} matrix, 1 call ({t:.2f} s)"}


def dgesdd_sigma(A):
    """Singular values of the FP32 matrix A by FP64 LAPACK dgesdd (the
    oracle of scripts/verify_svd.py:89, in double precision)."""
    import scipy.linalg
    return scipy.linalg.svd(np.asarray(A, np.float64), compute_uv=False, lapack_driver="gesdd")


def single_config(name, wl):
    """`config` of a single-matrix workload, the same in both arms."""
    return {"workload": f"{name}: {wl['M']}x{wl['N']} FP32 {wl['gen']}, one full SVD per step (sigma, U {wl['M']}x"
                        f"{wl['M']}, Vt {wl['N']}x{wl['N']})",
            "M": wl["M"], "N": wl["N"], "l2": "a 512 MiB buffer is written between timed GPU steps (L2 flush)"}


def multi_config(name, wl):
    """`config` of the multi-matrix workload, the same in both arms."""
    return {"workload": f"{name}: {wl['count']} FP32 {wl['M']}x{wl['N']} matrices with clustered spectra "
                        f"(512 clusters of 8, spacing 1e-7), full SVD of each per step",
            "count": wl["count"], "M": wl["M"], "N": wl["N"],
            "l2": "a 512 MiB buffer is written between timed GPU steps (L2 flush)"}


def batched_config(name, wl):
    """`config` of the batched workload, the same in both arms."""
    return {"workload": f"{name}: {wl['count']} FP32 N(0,1) matrices, M uniform on [{wl['Mlo']}, {wl['Mhi']}], "
                        f"N uniform on [{wl['Nlo']}, M], the whole batch per step",
            "count": wl["count"], "l2": "a 512 MiB buffer is written between timed GPU steps (L2 flush)"}


REF_BUDGET_S = 150.0  # timed CPU work of one reference-arm run


def run_reference(args, wl, rank):
    """The reference arm: its CPU path (LAPACK sgesdd, FP32, full U, every
    host thread) on the same workload, timed on the host.  Under torchrun
    only rank 0 runs; the other ranks exit without work."""
    if rank != 0:
        return
    batched = wl.get("kind") == "batched"
    if wl.get("kind") == "serving":
        print(json.dumps({"impl": "reference", "unavailable": "the reference has no serving mode; its CPU "
                          "algorithm is timed per matrix by the batched and single-matrix workloads"}))
        return
    threads = host_threads()
    multi = wl.get("kind") == "multi"
    if batched:
        # the batch's own shapes in order, N(0,1) entries, as many matrices as fit in the budget
        shapes = batched_shapes(wl, 4321)
        rng = np.random.default_rng(1234)
        np.linalg.svd(rng.standard_normal((64, 32)).astype(np.float32))  # thread pool start-up
        done, t0 = 0, time.perf_counter()
        for M, N in shapes[: wl["count"]]:
            np.linalg.svd(rng.standard_normal((M, N), dtype=np.float32), full_matrices=True)
            done += 1
            if time.perf_counter() - t0 > min(REF_BUDGET_S, 60.0):
                break
        t = time.perf_counter() - t0
        value = done / t
        sample = (f"numpy.linalg.svd (OpenBLAS sgesdd, FP32, full U) on the first {done} of the batch's "
                  f"{wl['count']} shapes (N(0,1), {t:.1f} s)")
        steps_done = 1
        ms = 1000.0 * wl["count"] / value
        config = batched_config(args.workload, wl)
        value_unit = value
    else:
        A = make_matrix(dict(M=wl["M"], N=wl["N"], gen=wl["gen"]), seed=1234)
        warm = lapack_svd_timed(A, 1, 0.0) if args.warmup > 0 else []
        times = lapack_svd_timed(A, args.steps, REF_BUDGET_S)
        steps_done = len(times)
        ms = 1000.0 * statistics.mean(times)
        value_unit = 1000.0 / ms
        sample = (f"the full {wl['M']}x{wl['N']} workload matrix at every step: numpy.linalg.svd (OpenBLAS "
                  f"sgesdd, FP32, full U), {len(warm)} warm-up call, {steps_done} timed calls "
                  f"(of {args.steps} requested; the run stops after {REF_BUDGET_S:.0f} s of timed work)")
        config = multi_config(args.workload, wl) if multi else single_config(args.workload, wl)
        if multi:
            sample += f"; one matrix per timed call (the workload has {wl['count']} per step)"
    cb = {"value": value_unit, "unit": "SVDs/s", "cores": threads, "kind": "lapack sgesdd", "sample": sample}
    line = {"metric": "SVDs/sec", "value": value_unit, "unit": "SVDs/s", "impl": "reference",
            "n_gpus": args.gpus, "steps": steps_done, "steps_requested": args.steps,
            "warmup": 0 if batched else len(warm), "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": config, "parallelism": "host CPU", "cpu_baseline": cb,
            "e2e": {"value": value_unit, "unit": "SVDs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="cfg3", choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer end-to-end measurement")
    ap.add_argument("--serve-seconds", type=float, default=None, help="length of the serving trace")
    ap.add_argument("--no-autotune", action="store_true", help="keep the default configuration (no paco_autotune)")
    ap.add_argument("--multi-group", type=int, default=0, help="matrices per lockstep group of the multi form")
    args = ap.parse_args()
    wl = WORKLOADS[args.workload]

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, wl, rank)
        return

    import torch
    import pacosvd as P

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    if wl.get("kind") == "batched":
        run_batched(args, wl, rank, world, local, dist)
        return
    if wl.get("kind") == "serving":
        run_serving(args, wl, rank, world, local, dist)
        return
    if wl.get("kind") == "multi":
        run_multi(args, wl, rank, world, local, dist)
        return
    M, N = wl["M"], wl["N"]
    # the tiling autotuner picks this shape's configuration before the clock starts
    tune = None if args.no_autotune else P.autotune(M, N)
    A_host, sig_exact = make_matrix(wl, seed=1234 + rank, with_sigma=True)
    A0 = torch.from_numpy(A_host).cuda()
    W = P.Workspace(M, N)
    flush = torch.empty(512 << 20, dtype=torch.uint8, device="cuda")
    # a non-default stream lets the library record the SVD as a CUDA graph
    stream = torch.cuda.Stream()
    lib = P.lib()
    lib.paco_launch_count.restype = ctypes.c_ulonglong
    lib.paco_profile_read.argtypes = [ctypes.POINTER(ctypes.c_double)]
    prof = (ctypes.c_double * 4)()

    def step():
        W.A.copy_(A0)
        W.run(stream=stream)

    # row-pass timing events are part of the recorded graph: enable first
    lib.paco_profile_enable(1)
    with torch.cuda.stream(stream):
        for _ in range(max(3, args.warmup)):
            step()
    stream.synchronize()
    rc, info = P.sync_status(W.ws, stream)
    if rc:
        raise SystemExit(f"device status {rc} ({info}) during warm-up")
    lib.paco_profile_enable(1)  # reset the totals, keep the recorded graph

    clocks = ClockSampler(local)
    clocks.start()
    launches0 = lib.paco_launch_count()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with torch.cuda.stream(stream):
        for k in range(args.steps):
            flush.fill_(k & 0xff)  # L2 flush, outside the timed window
            ev[k][0].record(stream)
            step()
            ev[k][1].record(stream)
            stream.synchronize()
            lib.paco_profile_read(prof)  # accumulates this step's row-pass events
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    launches = lib.paco_launch_count() - launches0
    lib.paco_profile_enable(0)
    clk = clocks.stop()
    step_ms = [a.elapsed_time(b) for a, b in ev]
    total_ms = max_over_ranks(sum(step_ms), dist)
    rc, info = P.sync_status(W.ws, stream)
    if rc:
        raise SystemExit(f"device status {rc} ({info}) in the timed region")

    # accuracy of the last step (Frobenius norms): sigma against FP64 LAPACK
    # dgesdd of the FP32 input (host) and, for the graded and clustered
    # generators, against the exact spectrum they built; the reconstruction
    # residual and the orthogonality of U and V in FP64 on the device
    s = W.sigma.float().cpu().numpy().astype(np.float64)
    acc = None
    if rank == 0:
        Ad = A0.double()
        Ud, Vd, sd = W.U.double(), W.Vt.double(), W.sigma.double()
        nA = torch.linalg.norm(Ad).item()
        res = torch.linalg.norm(Ad - (Ud[:, :N] * sd[None, :]) @ Vd).item() / nA
        eye_m = torch.eye(M, dtype=torch.float64, device="cuda")
        eye_n = torch.eye(N, dtype=torch.float64, device="cuda")
        acc = {"residual": res, "orth_U": torch.linalg.norm(Ud.T @ Ud - eye_m).item(),
               "orth_V": torch.linalg.norm(Vd @ Vd.T - eye_n).item(), "tolerance": 1e-5 * N}
        del Ad, Ud, Vd, eye_m, eye_n
        torch.cuda.empty_cache()
        ref = dgesdd_sigma(A_host)
        acc["sigma_err"] = float(np.max(np.abs(s - ref)) / ref[0])
        acc["sigma_tolerance"] = 1e-5
        acc["sigma_reference"] = "FP64 LAPACK dgesdd of the FP32 input (scipy, host)"
        if sig_exact is not None:
            acc["sigma_err_exact"] = float(np.max(np.abs(s - sig_exact)) / sig_exact[0])

    # end to end through the host-buffer C ABI (H2D of A, D2H of U, Vt, sigma)
    e2e_t = None
    if not args.no_e2e:
        ctx = P.HostContext(M, N)
        pin = lambda shape: torch.empty(shape, dtype=torch.float32).pin_memory()
        Ah, Uh, Vh, sh = pin((M, N)), pin((M, M)), pin((N, N)), pin((N,))
        Ah.copy_(torch.from_numpy(A_host))
        e2e_ms = []
        ctx.svd(Ah, Uh, Vh, sh)
        for _ in range(max(1, min(args.steps, 3))):
            t = time.perf_counter()
            ctx.svd(Ah, Uh, Vh, sh)
            e2e_ms.append((time.perf_counter() - t) * 1000)
        ctx.close()
        e2e_t = statistics.median(e2e_ms)

    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return
    peaks, peak_kind = measured_peaks()
    rp_ms, rp_launches, rp_bytes = prof[0], prof[1], prof[2]
    kname = ("bd_panel_pk (persistent stage-1 panel kernel: all column steps of a 32-column panel) "
             "and bd_tail_k (the last columns on one thread-block cluster, one launch per SVD)"
             if prof[3] == 1 else "bd_row_pass (stage-1 fused GEMV row pass)")
    # algorithmic bytes of the GEMV phase: two FP32 reads of the trailing matrix
    # per column step, 8 * sum_i (M-i)(N-i) bytes per SVD; the fused panel
    # kernel physically streams the live block once per step (rp_bytes)
    # with the QR-first path the column steps run on the N x N factor R
    qr_first = P.tune_qr(M, N, -2) == 1
    Mg = N if qr_first else M
    classic = 8.0 * sum((Mg - i) * (N - i) for i in range(N))
    n_launch = max(rp_launches, 1)
    alg_per_launch = classic * args.steps / n_launch
    avg_s = rp_ms / 1e3 / n_launch
    achieved = (alg_per_launch / 1e9) / avg_s if rp_ms > 0 else None
    # the trailing matrix of the column steps fits L2 (126 MB) or streams from DRAM
    ratio = traffic_ratio(resident=4.0 * Mg * N <= 96 * 2**20)
    roof = {"kernel": kname, "bound": "hbm",
            "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
            "frac": (achieved / peaks["hbm_gbs"]) if achieved else None,
            "traffic": (ratio * rp_bytes / n_launch) if (ratio and rp_launches) else None,
            "alg_bytes_per_launch": alg_per_launch,
            "alg_bytes_definition": ("8*sum_i (N-i)^2 per SVD: two FP32 reads of the trailing matrix per step of the "
                                     "bidiagonalization of R (QR-first)") if qr_first else
                                    "8*sum_i (M-i)(N-i) per SVD (two FP32 reads of the trailing matrix per step)",
            "streamed_bytes_per_launch": rp_bytes / n_launch,
            "avg_launch_us": 1e6 * avg_s,
            "launches": int(rp_launches), "peak_source": f"{peak_kind} hbm_gbs (MEASURED_PEAKS.json)"}
    value = whole_job_value(world, args.steps, total_ms)
    line = {"metric": "SVDs/sec", "value": value, "unit": "SVDs/s", "n_gpus": world, "steps": args.steps,
            "warmup": max(3, args.warmup), "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": single_config(args.workload, wl),
            "parallelism": f"replicas x{world}" if world > 1 else "1 GPU",
            "sigma_max": float(s[0]), "sigma_min": float(s[-1]), "accuracy": acc,
            "autotune": ({"choice": tune["name"], "ms": tune["ms"], "default_ms": tune["default_ms"]}
                         if tune else None),
            "roofline": roof, "clocks": clk,
            "e2e": ({"value": 1000.0 / e2e_t * world, "unit": "SVDs/s",
                     "h2d_bytes_per_step": 4 * M * N, "d2h_bytes_per_step": 4 * (M * M + N * N + N)}
                    if e2e_t else None),
            "gpu_launches": int(launches)}
    if not args.no_cpu_baseline and world == 1:
        line["cpu_baseline"] = cpu_baseline(wl, A_host)
        line["cpu_oracle"] = cpu_oracle(wl)
    print(json.dumps(line))
    if dist:
        dist.destroy_process_group()


def run_multi(args, wl, rank, world, local, dist):
    """cfg3x8: one step = one paco_svd_multi call over `count` matrices of the
    precision-form shape.  Beside it, the same matrices one at a time through
    paco_svd: the plain FP32 form (SIMT FP32 products, tuning entry tc = 0)
    and the precision form (3xTF32 tcgen05 products, the default)."""
    import torch
    import pacosvd as P
    from workloads import make_clustered_device

    M, N, count = wl["M"], wl["N"], wl["count"]
    lib = P.lib()
    lib.paco_launch_count.restype = ctypes.c_ulonglong
    lib.paco_profile_read.argtypes = [ctypes.POINTER(ctypes.c_double)]
    # the tiling autotuner: the single-matrix configuration of the shape, then
    # the lockstep group size (before the workspace is sized)
    tune = tune_m = None
    if not args.no_autotune:
        tune = P.autotune(M, N)
        if not args.multi_group:
            tune_m = P.autotune_multi(count, M, N)
    if args.multi_group:
        P.multi_group(args.multi_group)
    group = args.multi_group or P.tune_param(M, N, "mk") or 4
    m = P.Multi(count, M, N)
    sig_exact = []
    for b in range(count):
        A, sg = make_clustered_device(M, N, 5000 + 100 * rank + b)
        m.A[b].copy_(A)
        sig_exact.append(sg)
        del A
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    flush = torch.empty(512 << 20, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.Stream()
    prof = (ctypes.c_double * 4)()
    lib.paco_profile_enable(1)
    with torch.cuda.stream(stream):
        for _ in range(max(3, args.warmup)):
            m.run(stream)
    stream.synchronize()
    bad = [c for c in m.statuses() if c]
    if bad:
        raise SystemExit(f"statuses {bad} during warm-up")
    lib.paco_profile_enable(1)
    clocks = ClockSampler(local)
    clocks.start()
    launches0 = lib.paco_launch_count()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with torch.cuda.stream(stream):
        for k in range(args.steps):
            flush.fill_(k & 0xff)
            ev[k][0].record(stream)
            m.run(stream)
            ev[k][1].record(stream)
            stream.synchronize()
            lib.paco_profile_read(prof)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    launches = lib.paco_launch_count() - launches0
    lib.paco_profile_enable(0)
    clk = clocks.stop()
    step_ms = [a.elapsed_time(b) for a, b in ev]
    total_ms = max_over_ranks(sum(step_ms), dist)
    if any(m.statuses()):
        raise SystemExit(f"statuses {m.statuses()} in the timed region")

    # accuracy of two matrices of the last call against dgesdd and the exact spectrum
    acc = None
    if rank == 0:
        worst = {"sigma_err": 0.0, "sigma_err_exact": 0.0, "residual": 0.0, "orth_U": 0.0, "orth_V": 0.0}
        for b in (0, count - 1):
            Ad, Ud, Vd = m.A[b].double(), m.U[b].double(), m.Vt[b].double()
            sd = m.sigma[b].double()
            r = {"residual": (torch.linalg.norm(Ad - (Ud[:, :N] * sd[None, :]) @ Vd) / torch.linalg.norm(Ad)).item(),
                 "orth_U": torch.linalg.norm(Ud.T @ Ud - torch.eye(M, dtype=torch.float64, device="cuda")).item(),
                 "orth_V": torch.linalg.norm(Vd @ Vd.T - torch.eye(N, dtype=torch.float64, device="cuda")).item()}
            del Ud, Vd
            s = m.sigma[b].cpu().numpy().astype(np.float64)
            ref = dgesdd_sigma(m.A[b].cpu().numpy())
            r["sigma_err"] = float(np.max(np.abs(s - ref)) / ref[0])
            r["sigma_err_exact"] = float(np.max(np.abs(s - sig_exact[b])) / sig_exact[b][0])
            for key, v in r.items():
                worst[key] = max(worst[key], v)
            del Ad
            torch.cuda.empty_cache()
        acc = dict(worst, matrices=2, tolerance=1e-5 * N, sigma_tolerance=1e-5,
                   sigma_reference="FP64 LAPACK dgesdd of the FP32 input (scipy, host)")

    # the same matrices one at a time through paco_svd: plain FP32 form (SIMT
    # products) and the precision form (tcgen05 3xTF32 products)
    singles = {}
    if rank == 0:
        W = P.Workspace(M, N)
        tuned_cfg, tuned_qr = P.tune_get(M, N), P.tune_qr(M, N)
        for name, cfg in (("plain_fp32_single", [1, 16, 0, 0]), ("precision_single", None)):
            # plain: the reference's method (one-stage bidiagonalization, no QR
            # first) with SIMT FP32 products; precision: the tuned configuration
            # the multi-matrix form runs with
            if cfg is not None:
                P.tune_set(M, N, cfg)
                P.tune_qr(M, N, 0)
            else:
                P.tune_set(M, N, tuned_cfg)
                P.tune_qr(M, N, tuned_qr)
            qr_in_use = P.tune_qr(M, N, -2) == 1
            times = []
            with torch.cuda.stream(stream):
                for k in range(3 + 3):
                    W.A.copy_(m.A[k % count])
                    flush.fill_(k & 0xff)
                    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    e0.record(stream)
                    W.run(stream=stream)
                    e1.record(stream)
                    stream.synchronize()
                    if k >= 3:
                        times.append(e0.elapsed_time(e1))
            rc, info = P.sync_status(W.ws, stream)
            if rc:
                raise SystemExit(f"single-matrix status {rc} ({info})")
            singles[name] = {"value": 1000.0 / statistics.mean(times), "unit": "SVDs/s",
                             "ms_per_svd": statistics.mean(times),
                             "form": ("one paco_svd call per matrix, the one-stage method with SIMT FP32 "
                                      "products (tuning entry tc = 0, QR-first off)"
                                      if cfg is not None else
                                      "one paco_svd call per matrix, the tuned configuration ("
                                      + ("QR-first, " if qr_in_use else "one-stage, ")
                                      + "3xTF32 tcgen05 products)")}
        P.tune_set(M, N, tuned_cfg)
        P.tune_qr(M, N, tuned_qr)
        del W

    e2e = None
    if not args.no_e2e:
        pin = lambda t: torch.empty(t.shape, dtype=t.dtype).pin_memory()
        Ah, Uh, Vh, sh = pin(m.A), pin(m.U), pin(m.Vt), pin(m.sigma)
        Ah.copy_(m.A.cpu())
        times = []
        for k in range(max(1, min(args.steps, 3))):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            with torch.cuda.stream(stream):
                e0.record(stream)
                m.A.copy_(Ah, non_blocking=True)
                m.run(stream)
                Uh.copy_(m.U, non_blocking=True)
                Vh.copy_(m.Vt, non_blocking=True)
                sh.copy_(m.sigma, non_blocking=True)
                e1.record(stream)
            stream.synchronize()
            times.append(e0.elapsed_time(e1))
        e2e = {"value": world * count / (statistics.median(times) / 1000.0), "unit": "SVDs/s",
               "h2d_bytes_per_step": 4 * m.A.numel(),
               "d2h_bytes_per_step": 4 * (m.U.numel() + m.Vt.numel() + m.sigma.numel())}

    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return
    peaks, peak_kind = measured_peaks()
    rp_ms, rp_launches = prof[0], prof[1]
    qr_first = P.tune_qr(M, N, -2) == 1
    Mg = N if qr_first else M  # with QR first the column steps run on R (N x N)
    classic = 8.0 * sum((Mg - i) * (N - i) for i in range(N))
    n_launch = max(rp_launches, 1)
    alg_per_launch = classic * count * args.steps / n_launch
    avg_s = rp_ms / 1e3 / n_launch
    achieved = (alg_per_launch / 1e9) / avg_s if rp_ms > 0 else None
    value = whole_job_value(world, args.steps * count, total_ms)
    lat = sorted(step_ms)
    plain = singles.get("plain_fp32_single")
    prec = singles.get("precision_single")
    line = {"metric": "SVDs/sec", "value": value, "unit": "SVDs/s", "n_gpus": world, "steps": args.steps,
            "warmup": max(3, args.warmup), "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": multi_config(args.workload, wl),
            "parallelism": f"replicas x{world}" if world > 1 else "1 GPU",
            "form": f"paco_svd_multi, lockstep groups of {group}, 3xTF32 tcgen05 products",
            "autotune": ({"single": {"choice": tune["name"], "ms": tune["ms"], "fields": tune["fields"]},
                          "multi": tune_m} if tune else None),
            "latency": {"p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
                        "definition": "a result is delivered when its call returns: the call's duration"},
            "accuracy": acc, "clocks": clk,
            "roofline": {"kernel": "bd_panel_pk (persistent stage-1 panel kernel, k matrices per launch) and "
                                   "bd_tail_k", "bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"],
                         "unit": "GB/s", "frac": (achieved / peaks["hbm_gbs"]) if achieved else None,
                         "traffic": None, "alg_bytes_per_launch": alg_per_launch,
                         "alg_bytes_definition": ("8*sum_i (N-i)^2 per matrix (bidiagonalization of R after the "
                                                  "QR), summed over the matrices") if qr_first else
                                                 "8*sum_i (M-i)(N-i) per matrix, summed over the matrices",
                         "avg_launch_us": 1e6 * avg_s, "launches": int(rp_launches),
                         "peak_source": f"{peak_kind} hbm_gbs (MEASURED_PEAKS.json)"},
            "e2e": e2e, "gpu_launches": int(launches), "singles": singles,
            "multi_over_plain_fp32_single": (value / world / plain["value"]) if plain else None,
            "multi_over_precision_single": (value / world / prec["value"]) if prec else None}
    if not args.no_cpu_baseline and world == 1:
        line["cpu_baseline"] = cpu_baseline(wl, m.A[0].cpu().numpy())
    print(json.dumps(line))
    if dist:
        dist.destroy_process_group()


def run_batched(args, wl, rank, world, local, dist):
    """cfg4: one step = one paco_svd_batched call over the whole batch."""
    import torch
    import pacosvd as P

    lib = P.lib()
    lib.paco_launch_count.restype = ctypes.c_ulonglong
    lib.paco_debug_batched_timing.argtypes = [ctypes.c_int]
    lib.paco_debug_batched_times.argtypes = [ctypes.POINTER(ctypes.c_float)]
    shapes = batched_shapes(wl, 4321 + rank)
    count = len(shapes)
    b = P.Batch(shapes)
    gen = torch.Generator(device="cuda")
    gen.manual_seed(1234 + rank)
    b.A_flat.normal_(generator=gen)  # A is read only: every step sees the same inputs
    flush = torch.empty(512 << 20, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.Stream()
    for _ in range(max(3, args.warmup)):
        b.run(stream)
    stream.synchronize()
    bad = sum(1 for c in b.statuses() if c)
    if bad:
        raise SystemExit(f"{bad} matrices reported a non-zero status during warm-up")
    lib.paco_debug_batched_timing(1)
    kt = (ctypes.c_float * 3)()
    ksum = [0.0, 0.0, 0.0]
    clocks = ClockSampler(local)
    clocks.start()
    launches0 = lib.paco_launch_count()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with torch.cuda.stream(stream):
        for k in range(args.steps):
            flush.fill_(k & 0xff)  # L2 flush, outside the timed window
            ev[k][0].record(stream)
            b.run(stream)
            ev[k][1].record(stream)
            stream.synchronize()
            lib.paco_debug_batched_times(kt)
            for j in range(3):
                ksum[j] += kt[j]
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    launches = lib.paco_launch_count() - launches0
    lib.paco_debug_batched_timing(0)
    clk = clocks.stop()
    total_ms = max_over_ranks(sum(a.elapsed_time(c) for a, c in ev), dist)
    # accuracy of the last timed call on 40 matrices spread over the batch (outside the timing)
    acc = None
    if rank == 0:
        pick = list(range(0, count, max(1, count // 40)))[:40]
        acc = batched_accuracy([b.A[k].cpu().numpy() for k in pick], [b.U[k].cpu().numpy() for k in pick],
                               [b.Vt[k].cpu().numpy() for k in pick], [b.sigma[k].cpu().numpy() for k in pick])

    # end to end: host (pinned) inputs in, host outputs back, every step
    e2e = None
    if not args.no_e2e:
        pin = lambda t: torch.empty(t.shape, dtype=t.dtype).pin_memory()
        Ah, Uh, Vh, sh = pin(b.A_flat), pin(b.U_flat), pin(b.Vt_flat), pin(b.sigma_flat)
        Ah.copy_(b.A_flat.cpu())
        times = []
        for k in range(max(1, min(args.steps, 3))):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            with torch.cuda.stream(stream):
                e0.record(stream)
                b.A_flat.copy_(Ah, non_blocking=True)
                b.run(stream)
                Uh.copy_(b.U_flat, non_blocking=True)
                Vh.copy_(b.Vt_flat, non_blocking=True)
                sh.copy_(b.sigma_flat, non_blocking=True)
                e1.record(stream)
            stream.synchronize()
            times.append(e0.elapsed_time(e1))
        e2e = {"value": world * count / (statistics.median(times) / 1000.0), "unit": "SVDs/s",
               "h2d_bytes_per_step": 4 * b.A_flat.numel(),
               "d2h_bytes_per_step": 4 * (b.U_flat.numel() + b.Vt_flat.numel() + b.sigma_flat.numel())}

    # the plain single-matrix path (paco_svd, direct launches) over a sample of the shapes
    plain = None
    if rank == 0:
        sample = shapes[:: max(1, count // 60)][:60]
        ws = [P.Workspace(m, n) for m, n in sample]
        for w, (m, n) in zip(ws, sample):
            w.A.normal_(generator=gen)
        torch.cuda.synchronize()
        t = time.perf_counter()
        for w in ws:
            w.run()
        torch.cuda.synchronize()
        t = time.perf_counter() - t
        plain = {"value": len(sample) / t, "unit": "SVDs/s",
                 "sample": f"{len(sample)} matrices of the batch, one paco_svd call each, direct launches"}

    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return
    peaks, peak_kind = measured_peaks()
    steps = args.steps
    # GEMV-phase algorithmic bytes: 8 * sum_i (M-i)(N-i) per matrix
    alg = sum(8.0 * sum((m - i) * (n - i) for i in range(n)) for m, n in shapes)
    k1 = ksum[0] / steps
    achieved = alg / 1e9 / (k1 / 1e3)
    value = world * steps * count / (total_ms / 1000.0)
    line = {"metric": "SVDs/sec", "value": value, "unit": "SVDs/s", "n_gpus": world, "steps": steps,
            "warmup": max(3, args.warmup), "ms_per_step": total_ms / steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": batched_config(args.workload, wl),
            "parallelism": f"replicas x{world}" if world > 1 else "1 GPU",
            "roofline": {"kernel": "bt_bidiag_k (batched bidiagonalization, one CTA per matrix)", "bound": "hbm",
                         "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                         "frac": achieved / peaks["hbm_gbs"], "traffic": None,
                         "alg_bytes_per_launch": alg,
                         "alg_bytes_definition": "sum over matrices of 8*sum_i (M-i)(N-i)",
                         "kernel_ms": {"bt_bidiag_k": k1, "bt_bdc_k": ksum[1] / steps, "bt_apply_k": ksum[2] / steps},
                         "peak_source": f"{peak_kind} hbm_gbs (MEASURED_PEAKS.json)"},
            "clocks": clk, "e2e": e2e, "gpu_launches": int(launches), "accuracy": acc,
            "plain_single_matrix": plain,
            "batched_over_plain": (value / world / plain["value"]) if plain else None}
    if not args.no_cpu_baseline and world == 1:
        line["cpu_baseline"] = cpu_baseline_batched(wl)
    print(json.dumps(line))
    if dist:
        dist.destroy_process_group()


def run_serving(args, wl, rank, world, local, dist):
    """cfg5: a Poisson trace through the continuous-batching loop of serve.py.
    Inputs are generated on the device before the clock starts (a request's A
    is resident when it arrives); latency = completion - arrival."""
    import torch
    import pacosvd as P
    import serve as S

    seconds = args.serve_seconds or wl["seconds"]
    arr = S.poisson_arrivals(wl["rate"], seconds, 2024 + rank)
    M, N, graded = S.serving_shapes(len(arr), 2025 + rank)
    gen = torch.Generator(device="cuda")
    gen.manual_seed(7 + rank)
    t = time.perf_counter()
    reqs = [S.Request(k, S.make_input(int(m), int(n), bool(g), gen)) for k, (m, n, g) in enumerate(zip(M, N, graded))]
    torch.cuda.synchronize()
    setup_s = time.perf_counter() - t
    # warm the loop (library plans, allocator pools) on a short slice of the same mix
    warm = [S.Request(-1 - k, r.A.clone()) for k, r in enumerate(reqs[:200])]
    S.run_trace(S.SvdServer(cap_bytes=wl["cap_gb"] << 30), warm, np.zeros(len(warm)))
    srv = S.SvdServer(cap_bytes=wl["cap_gb"] << 30)
    lib = P.lib()
    lib.paco_launch_count.restype = ctypes.c_ulonglong
    launches0 = lib.paco_launch_count()
    clocks = ClockSampler(local)
    clocks.start()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    wall = S.run_trace(srv, reqs, arr)
    torch.cuda.synchronize()
    clk = clocks.stop()
    launches = lib.paco_launch_count() - launches0
    done = srv.completed
    span = max(r.done for r in done) - min(r.arrival for r in done)
    span = max_over_ranks(span * 1000.0, dist) / 1000.0
    stats = S.latency_stats(done)
    errors = len(srv.status_errors())
    small = [r for r in done if r.M <= srv.small_max]
    large = [r for r in done if r.M > srv.small_max]

    # the plain single-matrix path (one paco_svd call per request, direct launches) on a sample
    plain = None
    if rank == 0:
        rng = np.random.default_rng(3)
        idx = rng.choice(len(M), size=min(200, len(M)), replace=False)
        ws = [P.Workspace(int(M[k]), int(N[k])) for k in idx]
        for w in ws:
            w.A.normal_(generator=gen)
        torch.cuda.synchronize()
        t = time.perf_counter()
        for w in ws:
            w.run()
        torch.cuda.synchronize()
        plain = {"value": len(ws) / (time.perf_counter() - t), "unit": "SVDs/s",
                 "sample": f"{len(ws)} requests of the same mix, one paco_svd call each, direct launches"}
    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return
    value = world * len(done) / span
    line = {"metric": "SVDs/sec", "value": value, "unit": "SVDs/s", "n_gpus": world, "steps": 1, "warmup": 1,
            "ms_per_step": span * 1000.0, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"cfg5: Poisson requests at {wl['rate']:.0f}/s for {seconds:.0f} s, 90% M "
                                   f"log-uniform on [16, 256], 10% on [256, 2048], N uniform on [M/4, M], 20% "
                                   f"graded spectra, {wl['cap_gb']} GB working-set cap; continuous batching",
                       "requests": len(done), "parallelism": f"replicas x{world}" if world > 1 else "1 GPU"},
            "latency": dict(stats, small=S.latency_stats(small) if small else None,
                            large=S.latency_stats(large) if large else None),
            "offered_rate": wl["rate"], "wall_s": wall, "batches": srv.batches, "status_errors": errors,
            "peak_working_set_gb": srv.peak_inflight / 1e9, "input_setup_s": setup_s,
            "clocks": clk, "e2e": None, "gpu_launches": int(launches),
            "plain_single_matrix": plain, "served_over_plain": (value / world / plain["value"]) if plain else None}
    print(json.dumps(line))
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
