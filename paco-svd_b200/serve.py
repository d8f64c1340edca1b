"""Serving form of the B200 SVD: a continuous-batching request loop.

Requests (one FP32 matrix each, M <= 2048, N <= M) arrive while others are
on the GPU.  The loop
  * admits an arrived request once its device footprint fits under the
    working-set cap (A, U, Vt, sigma and its per-matrix area of the batched
    workspace),
  * groups admitted requests into batches, small (M <= `small_max`) and large
    separately, and enqueues each batch with one paco_svd_batched call on a
    stream of its own as soon as a stream is free, so batches that arrive
    while others run overlap with them on the device,
  * polls each batch's completion event, stamps its requests done and
    releases their memory,
  * cancels a request on demand: one not yet launched leaves at once (its
    memory is released), one whose batch is on the GPU is dropped when the
    batch completes; the other matrices of that batch are not affected.
Every result depends only on its own matrix (one CTA per matrix), so it is
bit for bit the same alone and in any mix.

The reference has no serving mode (it runs one matrix per process,
main.cpp:15-203); this module drives the same batched kernels as
`pacosvd.svd_batched`.
"""
from __future__ import annotations

import collections
import ctypes
import time

import numpy as np

import pacosvd as P


CANCELLED = -1  # Request.status of a cancelled request


class Request:
    __slots__ = ("rid", "M", "N", "A", "arrival", "admitted", "done", "U", "Vt", "sigma", "status", "keep",
                 "nbytes", "cancel")

    def __init__(self, rid, A, arrival=0.0, keep=False):
        self.rid = rid
        self.A = A
        self.M, self.N = int(A.shape[0]), int(A.shape[1])
        self.arrival = arrival
        self.admitted = self.done = None
        self.U = self.Vt = self.sigma = None
        self.status = None
        self.keep = keep
        self.nbytes = footprint(self.M, self.N)
        self.cancel = False


def footprint(M: int, N: int) -> int:
    """Device bytes one request holds while admitted: A, U, Vt, sigma and its
    per-matrix area of the batched workspace (Householder copy, Q^T, W^T)."""
    return 4 * (M * N + M * M + N * N + N) + 4 * (M * ((N + 3) // 4 * 4) + 2 * N * N + 8 * N) + 4096


class _Batch:
    __slots__ = ("reqs", "ws", "U", "Vt", "s", "status", "event", "nbytes")


class SvdServer:
    def __init__(self, cap_bytes=64 << 30, max_batch=(2048, 16), max_inflight=(4, 16), small_max=256,
                 device="cuda"):
        import torch
        self.torch = torch
        self.cap = int(cap_bytes)
        # per class: large requests go out in small batches (a batch finishes
        # with its slowest matrix) on more streams
        self.max_batch = (max_batch, max_batch) if isinstance(max_batch, int) else tuple(max_batch)
        self.small_max = small_max
        self.device = device
        # a pool of streams per class, so small batches never wait for a free
        # stream behind long-running large ones; the small class's streams
        # have the higher priority, so its CTAs take the SMs that large
        # matrices free first
        if isinstance(max_inflight, int):
            max_inflight = (max_inflight, max_inflight)
        # (a lower number is a higher priority; torch maps it into the device's range)
        self.streams = [[torch.cuda.Stream(priority=(-8 if cls == 0 else 0)) for _ in range(n)]
                        for cls, n in enumerate(max_inflight)]
        self.busy = [[None] * n for n in max_inflight]
        self.waiting = collections.deque()      # arrived, not yet admitted
        self.pending = [collections.deque(), collections.deque()]  # admitted, by class (small, large)
        self.inflight = 0                       # bytes held by admitted requests and batch scratch
        self.peak_inflight = 0
        self.completed = []
        self.cancelled = []
        self.live = {}                          # rid -> request, from submit until done or cancelled
        self.batches = 0
        self.lib = P.lib()

    # -------------------------------------------------------------- intake
    def submit(self, req: Request):
        if not (1 <= req.N <= req.M <= P.PACO_BATCH_MAX_M):
            raise P.PacoError(P.PACO_ERR_UNSUPPORTED, f"request {req.rid}: {req.M}x{req.N}")
        self.waiting.append(req)
        self.live[req.rid] = req

    def cancel(self, rid, now=0.0) -> bool:
        """Cancels request `rid`.  Not yet on the GPU: it leaves now and its
        memory is released.  On the GPU: its batch runs on and the result is
        dropped when the batch completes.  Returns False for an unknown or
        finished request."""
        r = self.live.get(rid)
        if r is None:
            return False
        r.cancel = True
        for q in (self.waiting, self.pending[0], self.pending[1]):
            if r in q:
                q.remove(r)
                if r.admitted is not None:
                    self.inflight -= r.nbytes
                self._drop(r, now)
                return True
        return True  # in flight: _finish drops it

    def _drop(self, r, t):
        r.status = CANCELLED
        r.done = t
        r.A = None
        self.live.pop(r.rid, None)
        self.cancelled.append(r)

    def _admit(self, now):
        while self.waiting and self.inflight + self.waiting[0].nbytes <= self.cap:
            r = self.waiting.popleft()
            r.admitted = now
            self.inflight += r.nbytes
            self.pending[0 if r.M <= self.small_max else 1].append(r)

    # -------------------------------------------------------------- launch
    def _launch(self):
        torch = self.torch
        for cls in (0, 1):
            q = self.pending[cls]
            busy = self.busy[cls]
            while q:
                try:
                    k = busy.index(None)
                except ValueError:
                    break
                reqs = [q.popleft() for _ in range(min(len(q), self.max_batch[cls]))]
                b = _Batch()
                b.reqs = reqs
                n = len(reqs)
                Ms = (ctypes.c_int * n)(*[r.M for r in reqs])
                Ns = (ctypes.c_int * n)(*[r.N for r in reqs])
                nbytes = int(self.lib.paco_batched_workspace_size(n, Ms, Ns))
                stream = self.streams[cls][k]
                with torch.cuda.stream(stream):
                    b.ws = torch.empty(nbytes, dtype=torch.uint8, device=self.device)
                    b.U = torch.empty(sum(r.M * r.M for r in reqs), device=self.device)
                    b.Vt = torch.empty(sum(r.N * r.N for r in reqs), device=self.device)
                    b.s = torch.empty(sum(r.N for r in reqs), device=self.device)
                    b.status = torch.empty(n, dtype=torch.int32, device=self.device)
                vp = ctypes.c_void_p * n
                pU, pV, ps = [], [], []
                ou = ov = os_ = 0
                for r in reqs:
                    pU.append(b.U.data_ptr() + 4 * ou); ou += r.M * r.M
                    pV.append(b.Vt.data_ptr() + 4 * ov); ov += r.N * r.N
                    ps.append(b.s.data_ptr() + 4 * os_); os_ += r.N
                pA = vp(*[r.A.data_ptr() for r in reqs])
                rc = self.lib.paco_svd_batched(n, Ms, Ns, pA, vp(*pU), vp(*pV), vp(*ps),
                                               ctypes.c_void_p(b.status.data_ptr()), ctypes.c_void_p(b.ws.data_ptr()),
                                               nbytes, ctypes.c_void_p(stream.cuda_stream))
                if rc != P.PACO_OK:
                    raise P.PacoError(rc, "paco_svd_batched")
                b.event = torch.cuda.Event()
                b.event.record(stream)
                b.nbytes = nbytes
                self.inflight += nbytes
                self.peak_inflight = max(self.peak_inflight, self.inflight)
                busy[k] = b
                self.batches += 1

    # -------------------------------------------------------------- completion
    def _poll(self, now_fn):
        for busy in self.busy:
            for k, b in enumerate(busy):
                if b is not None and b.event.query():
                    self._finish(b, now_fn())
                    busy[k] = None

    def _finish(self, b, t):
        """Stamps the batch's requests done at t and releases their memory."""
        st = b.status.cpu().tolist()
        ou = ov = os_ = 0
        for j, r in enumerate(b.reqs):
            if r.cancel:
                self.inflight -= r.nbytes
                self._drop(r, t)
                ou += r.M * r.M
                ov += r.N * r.N
                os_ += r.N
                continue
            r.done = t
            if r.keep:
                r.U = b.U[ou:ou + r.M * r.M].view(r.M, r.M).clone()
                r.Vt = b.Vt[ov:ov + r.N * r.N].view(r.N, r.N).clone()
                r.sigma = b.s[os_:os_ + r.N].clone()
            r.status = st[j]
            ou += r.M * r.M
            ov += r.N * r.N
            os_ += r.N
            self.inflight -= r.nbytes
            r.A = None
            self.live.pop(r.rid, None)
            self.completed.append(r)
        # the copies above run on the current stream: keep the batch's buffers
        # out of the allocator's reach until they have, or the next batch on
        # this batch's stream could reuse and overwrite them first
        cur = self.torch.cuda.current_stream()
        for t in (b.U, b.Vt, b.s, b.status):
            t.record_stream(cur)
        self.inflight -= b.nbytes

    def step(self, now_fn):
        self._admit(now_fn())
        self._launch()
        self._poll(now_fn)

    def idle(self):
        return not self.waiting and not any(self.pending) and all(b is None for bs in self.busy for b in bs)

    def status_errors(self):
        return [r.rid for r in self.completed if r.status not in (None, 0)]


# ------------------------------------------------------------------ traces

def serving_shapes(count, seed):
    """Request sizes of the serving benchmark: 90% M log-uniform on [16, 256],
    10% on [256, 2048], N uniform on [M/4, M]; 20% graded spectra."""
    rng = np.random.default_rng(seed)
    big = rng.random(count) < 0.10
    lo = np.where(big, np.log(256.0), np.log(16.0))
    hi = np.where(big, np.log(2048.0), np.log(256.0))
    M = np.exp(lo + (hi - lo) * rng.random(count)).round().astype(int)
    M = np.clip(M, 1, 2048)
    N = np.array([int(rng.integers(max(1, m // 4), m + 1)) for m in M])
    graded = rng.random(count) < 0.20
    return M, N, graded


def poisson_arrivals(rate, seconds, seed):
    rng = np.random.default_rng(seed)
    t, out = 0.0, []
    while True:
        t += rng.exponential(1.0 / rate)
        if t >= seconds:
            return np.array(out)
        out.append(t)


def make_input(M, N, graded, gen, device="cuda"):
    """N(0,1) entries, or A = Q1 diag(10^(-6 i/(N-1))) Q2^T with Haar-random
    orthonormal Q1 (M x N), Q2 (N x N) (QR of a Gaussian, sign-fixed)."""
    import torch
    if not graded:
        return torch.randn(M, N, device=device, generator=gen)

    def haar(m, n):
        Q, R = torch.linalg.qr(torch.randn(m, n, device=device, generator=gen, dtype=torch.float64))
        return Q * torch.sign(torch.diagonal(R))[None, :]

    sig = 10.0 ** (-6.0 * torch.arange(N, device=device, dtype=torch.float64) / max(N - 1, 1))
    return ((haar(M, N) * sig[None, :]) @ haar(N, N).T).float()


def run_trace(server, reqs, arrivals, poll_sleep=0.0):
    """Feeds requests at their arrival times (seconds from start) and runs the
    loop until every request is done.  Returns the wall time of the run."""
    t0 = time.perf_counter()
    now = lambda: time.perf_counter() - t0
    i, n = 0, len(reqs)
    while len(server.completed) + len(server.cancelled) < n:
        t = now()
        while i < n and arrivals[i] <= t:
            reqs[i].arrival = arrivals[i]
            server.submit(reqs[i])
            i += 1
        server.step(now)
        if poll_sleep and server.idle() and i < n:
            time.sleep(min(poll_sleep, max(0.0, arrivals[i] - now())))
    return now()


def latency_stats(reqs):
    lat = np.array([r.done - r.arrival for r in reqs])
    return {"p50_ms": float(np.percentile(lat, 50) * 1e3), "p99_ms": float(np.percentile(lat, 99) * 1e3),
            "mean_ms": float(lat.mean() * 1e3), "max_ms": float(lat.max() * 1e3)}
