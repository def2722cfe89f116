"""Continuous-batching solve server on one GPU (built on mgp.Batch).

Requests (grid dims, boundary kinds, a right-hand side given by sine modes, tolerance)
arrive over time.  The server loop:

* admits arrived requests while the device has memory for them (free HBM from
  cudaMemGetInfo plus what the batch's memory pool holds from retired requests, minus a
  reserve; per-problem bytes from mgp_batch_problem_bytes) and the batch has a free slot; an
  admitted request's hierarchy stays resident until it finishes, and its right-hand side is
  generated on the device;
* runs one batched refinement step (mgp_batch_step) for every resident request -- each
  level operation of every request is one persistent kernel over a (request, tile) work
  list, so requests of different sizes share launches;
* retires requests whose FP64 relative residual ||r||inf/||f||inf is below their
  tolerance: the solution comes back to the host (into a reused page-locked buffer) and the
  slot and memory free up.

Requests that arrive while others are on the GPU join at the next step boundary (continuous
batching, not a queue in front of a one-at-a-time solver).  Latency = finish - arrival.
"""
from __future__ import annotations

import collections
import hashlib
import time
from dataclasses import dataclass, field

import numpy as np

from . import F32, F64, FULLWEIGHTING, GAUSSSEIDEL, Batch, host_array

KINDS = ("dirichlet", "neumann", "mixed")


@dataclass
class Request:
    rid: int
    arrival: float                  # seconds after the start of the stream
    dims: tuple
    levels: int
    h: float
    bc: tuple                       # requested kinds, N S E W T B (0 Dirichlet, 1 Neumann)
    kind: str
    amp: np.ndarray
    kx: np.ndarray
    ky: np.ndarray
    kz: np.ndarray
    tol: float = 1e-8
    admitted: float = float("nan")
    finished: float = float("nan")
    iterations: int = 0
    rel_res: float = float("nan")
    digest: str = ""
    solution: np.ndarray | None = field(default=None, repr=False)

    @property
    def lengths(self):
        return tuple((n - 1) * self.h for n in self.dims)

    @property
    def dof(self):
        return self.dims[0] * self.dims[1] * self.dims[2]


def make_request(rid: int, arrival: float, seed: int, kmin=5, kmax=9, tol=1e-8, rng=None, kmax_z=None) -> Request:
    """Box sides 2^k+1 (k uniform in [kmin, kmax] independently per axis, z at most kmax_z),
    levels down to a
    5-point coarsest side, boundary kind uniform over Dirichlet / Neumann (the reference's
    default {N,N,N,N,D,D}) / mixed (random per face pair: north with south, east, west, top
    with bottom, so that the red-black colouring is a true checkerboard), zero boundary
    data, and a right-hand side of 8
    sine modes with wavenumbers uniform in 1..8 and N(0,1) amplitudes from the request's seed."""
    rng = rng or np.random.default_rng((seed, rid, 1))
    k = rng.integers(kmin, kmax + 1, size=3)
    if kmax_z is not None:
        k[2] = rng.integers(kmin, min(kmax, kmax_z) + 1)
    dims = tuple(int(2 ** kk + 1) for kk in k)
    levels = int(k.min()) - 1
    kind = KINDS[int(rng.integers(0, 3))]
    if kind == "dirichlet":
        bc = (0,) * 6
    elif kind == "neumann":
        bc = (1, 1, 1, 1, 0, 0)
    else:
        ns, ew = rng.integers(0, 2, size=4), int(rng.integers(0, 2))
        # north/south alike and top/bottom alike keep the padded y and z extents odd: the
        # reference's red-black colouring is then a true checkerboard (its degenerate
        # layouts, swept column by column, are left out of the served mix)
        bc = (int(ns[0]), int(ns[0]), int(ns[2]), int(ns[3]), ew, ew)
    mr = np.random.default_rng((seed, rid, 2))
    return Request(rid, arrival, dims, levels, 1.0 / (max(dims) - 1), bc, kind, mr.standard_normal(8),
                   mr.integers(1, 9, size=8).astype(np.float64), mr.integers(1, 9, size=8).astype(np.float64),
                   mr.integers(1, 9, size=8).astype(np.float64), tol)


def make_stream(n: int, rate: float, seed: int = 0, **kw) -> list:
    """Open-loop Poisson arrivals at `rate` requests/s."""
    rng = np.random.default_rng((seed, 0))
    t = 0.0
    out = []
    for rid in range(n):
        t += rng.exponential(1.0 / rate)
        out.append(make_request(rid, t, seed, **kw))
    return out


class Server:
    def __init__(self, inner=F32, max_batch=64, reserve_bytes=4 << 30, device=0, max_steps=200,
                 keep_solutions=False, nsmooth=2, digest=False, pool_bytes=None):
        """pool_bytes: device memory the batch's pool takes up front (default: what
        cudaMemGetInfo reports free, less reserve_bytes and 1 GiB), so that admitting and
        retiring requests never grows or shrinks it; 0 lets the pool grow on demand."""
        self.batch = Batch(FULLWEIGHTING, GAUSSSEIDEL, inner, "Fcycle", nsmooth, max_problems=max_batch,
                           device=device)
        if pool_bytes is None:
            free, _ = self.batch.mem_info()
            pool_bytes = max(0, free - reserve_bytes - (1 << 30))
        if pool_bytes:
            self.batch.reserve(pool_bytes)
        self.max_batch = max_batch
        self.reserve = reserve_bytes
        self.device = device
        self.max_steps = max_steps
        self.keep = keep_solutions
        self.digest = digest
        self.steps = 0
        self.batch_sizes = []
        self._landing = None  # page-locked download buffer, grown to the largest solution
        self._free = None     # device bytes left for admissions (the server's own count)
        self._asked = False   # the device was asked in the current tick
        self._need = {}       # bytes each resident request took

    def close(self):
        self.batch.close()

    def _admit(self, req: Request, now: float) -> bool:
        need = self.batch.problem_bytes(req.dims, req.levels, req.h, req.bc)
        # The server keeps its own count of free device memory: admissions take from it and
        # retirements give back; the device is asked again (cudaMemGetInfo takes milliseconds)
        # only when the count says no, at most once per tick.
        if self._free is None or (self._free - need < self.reserve and not self._asked):
            self._free, _ = self.batch.mem_info()
            self._asked = True
        if self._free - need < self.reserve:
            return False
        self._free -= need
        self._need[req.rid] = need
        pid = self.batch.add(req.dims, req.levels, req.h, req.bc)
        s = self.batch.problem(pid)
        s.fill_sine_modes(req.amp, req.kx, req.ky, req.kz, req.lengths)
        req.admitted = now
        self._active[pid] = req
        return True

    def _retire(self, pid: int, req: Request, now: float):
        st = self.batch.status(pid)
        req.iterations, req.rel_res = int(st.iterations), st.rel_res
        s = self.batch.problem(pid)
        lv = s.level[0]
        if self._landing is None or self._landing.size < lv.size:
            self._landing = host_array((lv.size,), s.np_dtype, pinned=True)
        u = self._landing[:lv.size].reshape(lv.pad)
        # the download writes the shape points; the halo of the reused buffer is zeroed so
        # the result is what a fresh zeroed array would hold
        ix, iy, iz = lv.interior
        u[:ix.start] = 0
        u[ix.stop:] = 0
        u[:, :iy.start] = 0
        u[:, iy.stop:] = 0
        u[:, :, :iz.start] = 0
        u[:, :, iz.stop:] = 0
        s.download("u", 0, out=u)
        if self.digest:
            req.digest = hashlib.sha256(u.tobytes()).hexdigest()[:16]
        if self.keep:
            req.solution = u.copy()
        self.batch.remove(pid)
        if self._free is not None:
            self._free += self._need.pop(req.rid, 0)
        req.finished = now

    def run(self, requests, time_scale: float = 1.0, clock=time.perf_counter) -> dict:
        """Serve `requests` (sorted by arrival); arrival times are multiplied by time_scale."""
        pending = collections.deque(sorted(requests, key=lambda r: r.arrival))
        waiting = collections.deque()
        self._active = {}
        self.steps = 0
        self.batch_sizes = []
        t0 = clock()
        while pending or waiting or self._active:
            now = clock() - t0
            while pending and pending[0].arrival * time_scale <= now:
                waiting.append(pending.popleft())
            self._asked = False
            while waiting and len(self._active) < self.max_batch and self._admit(waiting[0], now):
                waiting.popleft()
            if not self._active:
                if waiting:
                    raise RuntimeError(f"request {waiting[0].rid} {waiting[0].dims} does not fit on the device")
                if pending:
                    time.sleep(max(0.0, min(0.01, pending[0].arrival * time_scale - now)))
                continue
            self.batch.step()
            self.steps += 1
            self.batch_sizes.append(len(self._active))
            now = clock() - t0
            for pid, req in list(self._active.items()):
                st = self.batch.status(pid)
                if st.rel_res < req.tol or st.iterations >= self.max_steps:
                    self._retire(pid, req, clock() - t0)
                    del self._active[pid]
        return summarize(requests, time_scale, self.steps, self.batch_sizes)


def summarize(requests, time_scale, steps, batch_sizes) -> dict:
    lat = np.array([(r.finished - r.arrival * time_scale) for r in requests])
    span = max(r.finished for r in requests) - min(r.arrival * time_scale for r in requests)
    dof = sum(r.dof for r in requests)
    return {
        "requests": len(requests),
        "p50_ms": float(np.percentile(lat, 50) * 1e3),
        "p99_ms": float(np.percentile(lat, 99) * 1e3),
        "mean_ms": float(lat.mean() * 1e3),
        "solves_per_s": len(requests) / span,
        "dof_per_s": dof / span,
        "span_s": span,
        "converged": int(sum(r.rel_res < r.tol for r in requests)),
        "mean_iterations": float(np.mean([r.iterations for r in requests])),
        "steps": steps,
        "mean_batch": float(np.mean(batch_sizes)) if batch_sizes else 0.0,
        "max_batch_seen": int(max(batch_sizes)) if batch_sizes else 0,
    }
