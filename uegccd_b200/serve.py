"""Serving loop: continuous batching of independent UEG solves on one GPU.

Requests (N, rs, basis ratio M/(N/2), twist, method) arrive over time.

* Set-up off the dispatcher: each arriving request goes to a pool of host threads that
  builds its basis and eigenvalues (heg) and its device footprint (uegccd_footprint, the
  amplitudes, index tables and DIIS history it will hold).  A request larger than the
  whole HBM budget is refused at once (UEGCCD_ERR_ALLOC) and never touches the GPU.
* Admission: the dispatcher admits every set-up request whose footprint fits the free
  part of the budget, groups them by method and starts each group as a cohort: one batch
  on its own CUDA stream, driven by its own host thread.  With a batching window
  (batch_window seconds, default 0) it first lets requests gather: it admits once the
  oldest waiting request has waited that long, or when no other request is on its way.
  At most max_cohorts cohorts run at a time (default 4): under light load every request
  starts at once, under heavy load arrivals gather while the cohorts run and start
  together in larger cohorts.  Cohorts that run at the same time overlap on the device
  (the ctypes calls release the GIL).
* Iteration-level retirement: a cohort runs the incremental solve of the library
  (uegccd_batch_start / uegccd_batch_advance): after every round of four iterations, each
  solve that stopped -- converged, or at MaxIter -- is retired at once, with its final
  residual, and its result goes back to its request then, not when the cohort's slowest
  solve ends.  A retired solve's kernels return at once; the cohort's device memory goes
  back to the budget (and the library's chunk cache, which the next cohort reuses) when its
  last solve retires, which admits the next requests.
* MP2 requests need no iteration: their cohort runs the MP2 kernel alone (uegccd_batch_mp2).

The result of a solve does not depend on its cohort: each solve's arithmetic, including its
reductions, touches only its own data, in a fixed order (tests/test_gpu_serve.py).
"""
from __future__ import annotations

import dataclasses
import threading
import time
from collections import deque
from concurrent.futures import ThreadPoolExecutor

import numpy as np

from . import _capi, heg
from .solver import Batch

METHODS = ("MP2", "dRPA", "CCD")


@dataclasses.dataclass
class Request:
    rid: int
    nelectron: int
    rs: float
    ratio: int
    twist: tuple
    method: str
    t_arrival: float = 0.0
    # filled by the server
    system: tuple | None = None
    nbytes: int = 0
    t_ready: float = 0.0      # set-up done
    t_admit: float = 0.0
    t_done: float = 0.0
    e2: float = float("nan")
    ecorr: float = float("nan")
    ecorr_sosex: float = float("nan")
    niter: int = 0
    status: int = 0

    @property
    def latency(self) -> float:
        return self.t_done - self.t_arrival


_SHELLS = None


def _pool_for(nocc: int, nbasis: int) -> int:
    """Smallest |n|^2 cutoff whose lattice holds 1.5x the basis (room for the twist sort)."""
    global _SHELLS
    if _SHELLS is None:
        r = 16
        g = np.arange(-r, r + 1)
        n2 = (g[:, None, None] ** 2 + g[None, :, None] ** 2 + g[None, None, :] ** 2).ravel()
        _SHELLS = np.cumsum(np.bincount(n2, minlength=r * r + 1))[: r * r + 1]
    need = int(1.5 * nbasis) + 8
    k = int(np.searchsorted(_SHELLS, need))
    if k >= len(_SHELLS):
        raise ValueError("basis too large for the serving set-up")
    return max(k, 1)


def build_system(req: Request):
    """Host set-up of one request: the req.ratio * N/2 lowest |n + k_s|^2 plane waves."""
    nocc = req.nelectron // 2
    nbasis = req.ratio * nocc
    fcut = float(req.ratio) ** (2.0 / 3.0)
    inp = heg.default_input(nelectron=req.nelectron, maxkpoint=_pool_for(nocc, nbasis), rsmin=req.rs,
                            rsmax=req.rs, fcut=fcut, ntwist=req.twist)
    return heg.Heg(inp).system()


def poisson_stream(n: int, rate: float, seed: int = 7, nelectrons=(14, 54, 66, 114), ratios=(4, 8, 12, 16, 20),
                   weights=(0.2, 0.2, 0.6)):
    """Seeded request stream: Poisson arrivals, N uniform over `nelectrons`, rs log-uniform
    in [0.5, 5], basis ratio uniform over `ratios`, twist U[-0.5,0.5)^3, method MP2/dRPA/CCD."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for k in range(n):
        t += rng.exponential(1.0 / rate)
        out.append(Request(
            rid=k,
            nelectron=int(rng.choice(nelectrons)),
            rs=float(np.exp(rng.uniform(np.log(0.5), np.log(5.0)))),
            ratio=int(rng.choice(ratios)),
            twist=tuple(float(x) for x in rng.random(3) - 0.5),
            method=str(rng.choice(METHODS, p=list(weights))),
            t_arrival=t,
        ))
    return out


class Server:
    """Continuous-batching request loop over the uegccd batch API (see the module text)."""

    def __init__(self, hbm_budget: int = 40 << 30, max_batch: int = 64, ndiis: int = 6, tol: float = 1e-8,
                 max_iter: int = 200, setup_threads: int = 8, rounds: int = 1, device: int = 0,
                 batch_window: float = 0.0, max_cohorts: int = 4):
        self.budget = hbm_budget
        self.max_batch = max_batch
        self.opts = dict(scheme=1, ndiis=ndiis, denom_factor=1.0, tol=tol, max_iter=max_iter)
        self.ndiis = ndiis
        self.setup_threads = setup_threads
        self.rounds = rounds
        self.device = device
        self.batch_window = batch_window
        self.max_cohorts = max_cohorts
        self.lock = threading.Lock()
        self.in_use = 0
        self.batches_started = 0
        self.max_concurrent = 0
        self._live = 0

    def _retire(self, r: Request, t0: float, e2: float, res: dict | None, status: int):
        r.e2 = float(e2)
        if res is None:              # MP2
            r.ecorr = float(e2)
        else:
            r.ecorr = res["ecorr"]
            r.ecorr_sosex = res["ecorr_sosex"]
            r.niter = res["niter"]
        r.status = status
        r.t_done = time.perf_counter() - t0

    def _run_cohort(self, reqs, t0):
        method = reqs[0].method
        try:
            b = Batch([r.system for r in reqs], device=self.device)
            try:
                if method == "MP2":
                    e2 = b.mp2()
                    for r, e in zip(reqs, e2):
                        self._retire(r, t0, e, None, 0)
                else:
                    e2 = b.start(drpa=(method == "dRPA"), **self.opts)
                    active = len(reqs)
                    while active > 0:
                        active, done = b.advance(self.rounds)
                        for s, res in done:
                            self._retire(reqs[s], t0, e2[s], res, res["status"])
            finally:
                b.close()
        except _capi.UegccdError as exc:
            t_done = time.perf_counter() - t0
            for r in reqs:
                if r.t_done == 0.0:
                    r.status = exc.code
                    r.t_done = t_done
        finally:
            with self.lock:
                self.in_use -= sum(r.nbytes for r in reqs)
                self._live -= 1

    @staticmethod
    def _set_up(r: Request, ndiis: int):
        r.system = build_system(r)
        r.nbytes = _capi.footprint(r.system, ndiis)[0]
        return r

    def run(self, requests, realtime: bool = True, poll: float = 0.0005):
        """Serve `requests` (sorted by t_arrival).  realtime=False: every request arrives at t=0."""
        pending = deque(sorted(requests, key=lambda r: r.t_arrival))
        setting_up = []   # futures of the set-up pool
        waiting = []      # set up, not yet admitted
        threads = []
        t0 = time.perf_counter()
        with ThreadPoolExecutor(max_workers=self.setup_threads) as pool:
            while pending or setting_up or waiting or any(t.is_alive() for t in threads):
                now = time.perf_counter() - t0
                while pending and (not realtime or pending[0].t_arrival <= now):
                    r = pending.popleft()
                    if not realtime:
                        r.t_arrival = now
                    setting_up.append(pool.submit(self._set_up, r, self.ndiis))
                still = []
                for f in setting_up:
                    if not f.done():
                        still.append(f)
                        continue
                    r = f.result()
                    r.t_ready = time.perf_counter() - t0
                    if r.nbytes > self.budget:   # can never be admitted
                        r.status = _capi.UEGCCD_ERR_ALLOC
                        r.t_done = time.perf_counter() - t0
                    else:
                        waiting.append(r)
                setting_up = still
                started = False
                now = time.perf_counter() - t0
                hold = (self.batch_window > 0 and waiting and (pending or setting_up)
                        and now - min(r.t_ready for r in waiting) < self.batch_window)
                for method in METHODS if not hold else ():
                    group = []
                    with self.lock:
                        free = self.budget - self.in_use
                        if self._live >= self.max_cohorts:
                            free = -1   # wait for a running cohort to finish
                        for r in [w for w in waiting if w.method == method]:
                            if len(group) >= self.max_batch:
                                break
                            if r.nbytes <= free:
                                group.append(r)
                                free -= r.nbytes
                        if group:
                            self.in_use += sum(r.nbytes for r in group)
                            self._live += 1
                            self.max_concurrent = max(self.max_concurrent, self._live)
                    if group:
                        t_admit = time.perf_counter() - t0
                        for r in group:
                            r.t_admit = t_admit
                            waiting.remove(r)
                        th = threading.Thread(target=self._run_cohort, args=(group, t0), daemon=True)
                        th.start()
                        threads.append(th)
                        self.batches_started += 1
                        started = True
                if not started:
                    time.sleep(poll)
                threads = [t for t in threads if t.is_alive()] if len(threads) > 256 else threads
        for th in threads:
            th.join()
        return time.perf_counter() - t0


def summarize(reqs, wall: float) -> dict:
    lat = np.array([r.latency for r in reqs])
    done = [r for r in reqs if r.status >= 0]
    return {
        "requests": len(reqs), "completed": len(done), "wall_s": wall,
        "solves_per_s": len(done) / wall if wall > 0 else float("nan"),
        "p50_ms": float(np.percentile(lat, 50) * 1e3), "p99_ms": float(np.percentile(lat, 99) * 1e3),
        "by_method": {m: sum(1 for r in reqs if r.method == m) for m in METHODS},
    }
