#!/usr/bin/env python
"""Benchmark: batched twist-averaged CCD solves per second on the B200.

Workload ("ccd-twist-batch", the batched twist-average configuration):
  N=54 electrons (27 occupied), rs=1.0, per twist k_s ~ U[-0.5,0.5)^3 (units of 2*pi/L,
  numpy default_rng seed 2024): occupy the 27 lowest |n+k_s|^2, basis = the 485
  lowest from the |n|^2 <= 30 pool (fcut 6.857 -> NAO 485); HF eigenvalues; MP2 start;
  FP64 CCD with Pulay DIIS over 6 vectors to max|dT| < 1e-9 (the FP64 GPU configuration).
  One step = MP2 + CCD of every twist.  The reference's own iteration (1/2-damped
  Jacobi, inert DIIS, max|dT| < 1e-8) is run once per bench as a check (not timed).
  Inputs are synthetic: the reference publishes no dataset, only this recipe.

Metric: CCD solves/s (whole job; N GPUs each solve their own twist batch, weak scaling).
  value  device-timed (CUDA events on the library's stream), inputs resident;
  e2e    the same through the C ABI with host buffers: batch create (plan + uploads),
         solve, amplitudes copied back to a page-locked host buffer, every step; the next
         step's create and the previous step's download overlap the current solve.
--impl reference times the oracle (C restatement of the reference Fortran) on the
host cores: one process per core, each running CCD iterations of its own twist.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_ELECTRONS = 54
RS = 1.0
MAXK = 30          # candidate pool |n|^2 <= 30 (739 plane waves)
FCUT = 6.857       # round(fcut^1.5 * 27) = 485 orbitals
SEED = 2024
# Mean CCD iteration count of this workload in the reference's iteration (replay mode
# reproduces the reference's iterations exactly); measured by the GPU arm, which
# checks it every run.  Used to turn the oracle's time per iteration into a time per solve.
REF_ITERS_PER_SOLVE = 33.16  # measured: replay mode on this workload, 100 twists (min 30, max 35)
SOLVE_OPTS = dict(scheme=1, ndiis=6, denom_factor=1.0, tol=1e-9)
E2E_CREATORS = 2   # host threads creating the next batches of the e2e pipeline
# Nominal FP64 peak of a B200 (datasheet); the bench measures it each run with the register-only
# probe of bench_peak.cu (37.0 TFLOP/s measured on B200) and uses this only if the probe fails.
FP64_PEAK_TFLOPS = 37.0


def _nvtx():
    """torch's NVTX markers (a no-op stand-in where torch has no CUDA)."""
    try:
        import torch

        if torch.cuda.is_available():
            return torch.cuda.nvtx
    except Exception:
        pass

    class _Off:
        @staticmethod
        def range_push(_name):
            pass

        @staticmethod
        def range_pop():
            pass

    return _Off


def probe_fp64_peak():
    """FP64 tensor-core TFLOP/s of this GPU from bench_peak.so's register-only probe (None on failure)."""
    import ctypes as C

    path = os.path.join(ROOT, "bench_peak.so")
    if not os.path.exists(path):
        return None
    lib = C.CDLL(path)
    lib.bench_fp64_peak.argtypes = [C.POINTER(C.c_double), C.c_char_p, C.c_int]
    v = C.c_double()
    msg = C.create_string_buffer(256)
    return v.value if lib.bench_fp64_peak(C.byref(v), msg, 256) == 0 else None


def pinned_buffer(n: int):
    """n doubles of page-locked host memory (cudaHostAlloc) as a numpy array; held until exit."""
    import ctypes as C

    import numpy as np

    rt = C.CDLL("libcudart.so.12")
    p = C.c_void_p()
    rc = rt.cudaHostAlloc(C.byref(p), C.c_size_t(8 * n), C.c_uint(0))
    if rc != 0 or not p.value:
        raise RuntimeError(f"cudaHostAlloc of {8 * n} bytes failed ({rc})")
    return np.ctypeslib.as_array((C.c_double * n).from_address(p.value))


def _measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d.get("hbm_gbs", 6650.0)), float(d.get("bf16_tflops", 1590.0))
    except Exception:
        return 6650.0, 1590.0  # fallback figures: an earlier measurement on B200


HBM_PEAK, BF16_PEAK = _measured_peaks()
# DRAM bytes of one launch per solve: dram__bytes_read.sum + dram__bytes_write.sum of every class
# launch of one residual, from one ncu capture of the 100-twist batch itself (a one-pass
# metric set), divided by the 100 solves of a launch.
TRAFFIC_PER_SOLVE = {"k_ladder": 193.4e6 / 100, "k_ladder_hh": 101.5e6 / 100, "k_mosaic_blk": 116.7e6 / 100,
                     "k_rings": 310.0e6 / 100, "k_ring_stage": 496.8e6 / 100, "k_update": 968.7e6 / 100}


def twists(n: int, seed: int = SEED, rank: int = 0):
    import numpy as np

    rng = np.random.default_rng(seed + 7919 * rank)
    return rng.random((n, 3)) - 0.5


def reduce_max(values):
    """Max over ranks of each value (gloo/NCCL all-reduce); identity on one process."""
    try:
        import torch.distributed as dist

        if not (dist.is_available() and dist.is_initialized()):
            return list(values)
        import torch

        t = torch.tensor(list(values), dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return [float(x) for x in t]
    except ImportError:
        return list(values)


def build_systems(tw):
    from uegccd_b200 import heg

    inp = heg.default_input(nelectron=N_ELECTRONS, maxkpoint=MAXK, rsmin=RS, rsmax=RS, fcut=FCUT)
    h = heg.Heg(inp)
    out = []
    for t in tw:
        h.change_twist(t)
        out.append(h.system())
    return out


# ------------------------------------------------------------------- clocks
class ClockSampler:
    """SM clock and clock-event reasons while the timed region runs: in-process NVML reads every
    10 ms (reads only; no setting of the GPU is touched), else nvidia-smi.  NVML is opened before
    the region starts, and the last sample is taken when it ends, so even a short region has
    samples."""

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.samples = []
        self._stop = threading.Event()
        self._t = None
        self._nvml = None

    def _nvml_sample(self):
        N, h, mx, bits = self._nvml
        sm = N.nvmlDeviceGetClockInfo(h, N.NVML_CLOCK_SM)
        pw = N.nvmlDeviceGetPowerUsage(h) / 1000.0
        r = N.nvmlDeviceGetCurrentClocksEventReasons(h)
        self.samples.append([str(sm), str(mx), f"{pw:.1f}"] + ["Active" if r & b else "Not Active" for b in bits])

    def _run_nvml(self):
        while not self._stop.is_set():
            try:
                self._nvml_sample()
            except Exception:
                return
            self._stop.wait(0.01)

    def _run_smi(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        while not self._stop.is_set():
            try:
                r = subprocess.run(["nvidia-smi", "-i", str(self.idx), f"--query-gpu={q}",
                                    "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                f = [x.strip() for x in r.stdout.strip().split(",")]
                if len(f) >= 7:
                    self.samples.append(f)
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        try:
            import pynvml as N

            N.nvmlInit()
            h = N.nvmlDeviceGetHandleByIndex(self.idx)
            mx = N.nvmlDeviceGetMaxClockInfo(h, N.NVML_CLOCK_SM)
            bits = [N.nvmlClocksEventReasonHwSlowdown, N.nvmlClocksEventReasonHwThermalSlowdown,
                    N.nvmlClocksEventReasonSwThermalSlowdown, N.nvmlClocksEventReasonSwPowerCap]
            self._nvml = (N, h, mx, bits)
        except Exception:
            self._nvml = None
        self._t = threading.Thread(target=self._run_nvml if self._nvml else self._run_smi, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        if self._nvml:
            try:
                self._nvml_sample()   # the region's end
            except Exception:
                pass
        self._stop.set()
        self._t.join(timeout=10)
        if self._nvml:
            try:
                self._nvml[0].nvmlShutdown()
            except Exception:
                pass

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for s in self.samples for k in range(4) if s[3 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


# ------------------------------------------------------------------- GPU arm
def plan_stats(sysl):
    """Per-solve sizes of the momentum-block plan: O, V, A, sum o v^2, sum o^2 v, and the
    ring flops over the {Q, -Q} particle-hole group pairs."""
    from collections import defaultdict

    import numpy as np

    nocc, L, mad, eig, nv = sysl
    O = nocc
    M = len(nv)
    idx = {tuple(v): p for p, v in enumerate(nv)}
    blocks = defaultdict(lambda: [0, None, 0])   # rows, columns, rows with i <= j
    for i in range(O):
        for j in range(O):
            K = tuple(nv[i] + nv[j])
            blocks[K][0] += 1
            blocks[K][2] += i <= j
            if blocks[K][1] is None:
                blocks[K][1] = sum(1 for a in range(O, M) if idx.get(tuple(np.array(K) - nv[a]), -1) >= O)
    ov = [(o, v) for o, v, _ in blocks.values() if v > 0]
    # the FP64 ladders form the rows i <= j (the mirrors (j,i) follow by the pair symmetry)
    ocv = [(oc, o, v) for o, v, oc in blocks.values() if v > 0]
    groups = defaultdict(int)
    for i in range(O):
        for x in range(O, M):
            groups[tuple(nv[x] - nv[i])] += 1
    ring = 0
    for Q, n1 in groups.items():
        mq = tuple(-q for q in Q)
        if Q < mq and mq in groups:
            n2 = groups[mq]
            a, b = min(n1, n2), max(n1, n2)
            ring += 10 * a * a * b + 4 * a * b * b
    return {"O": O, "V": M - O, "A": sum(o * v for o, v in ov), "A_half": sum(oc * v for oc, o, v in ocv),
            "ov2": sum(o * v * v for o, v in ov),
            "ov2_half": sum(oc * v * v for oc, o, v in ocv), "o2v_half": sum(oc * o * v for oc, o, v in ocv),
            "ring_flop": ring}


def kernel_units(st):
    """Algorithmic work of one launch per solve: ('flop', F) or ('byte', B)."""
    A = st["A"]
    ndiis = SOLVE_OPTS["ndiis"]
    return {
        # rows i <= j: pp ladder sum_c v(a-c) t(p,c) and hole-hole apply sum_q H(p,q) t(q,a)
        "k_ladder": ("flop", 2 * (st["ov2_half"] + st["o2v_half"])),
        "k_ladder_hh": ("flop", 2 * st["o2v_half"]),
        # pp ladder on the tensor cores (FP16 operands)
        "k_ladder_tc": ("tflop16", 2 * st["ov2"]),
        # per {Q, -Q} group pair, n1 <= n2 rows: X W and Y W of the smaller group, 4 n1^2 n2,
        # and the ring and crossed-ring products of one direction (the other is its mirror),
        # 6 n1^2 n2 + 4 n1 n2^2
        "k_rings": ("flop", st["ring_flop"]),
        # reads the rows i <= j of t once (s is formed in registers; the partial sums are small)
        "k_mosaic_blk": ("byte", 8 * st["A_half"]),
        # the particle-hole copy: every amplitude read once through a 4-byte index and written
        # once (the pairs' X1 and Y1 hold A entries between them)
        "k_ring_stage": ("byte", (8 + 4 + 8) * A),
        # every amplitude: the mirror index (4 B); the amplitudes i <= j: t, the ladder G and the
        # two ring G, the Pulay push (t' FP64 and e FP32 to the history) and the other ndiis - 1
        # error vectors (FP32)
        "k_update": ("byte", 4 * A + (4 * 8 + 8 + 4 + (ndiis - 1) * 4) * st["A_half"]),
    }


def ladder_flops(batch_systems):
    """Algorithmic FLOPs of one particle-particle ladder pass: 2 * sum_K o_K v_K^2."""
    from collections import defaultdict

    import numpy as np

    tot = 0
    for (nocc, L, mad, eig, nv) in batch_systems:
        O = nocc
        idx = {tuple(v): p for p, v in enumerate(nv)}
        blocks = defaultdict(lambda: [0, None])
        for i in range(O):
            for j in range(O):
                K = tuple(nv[i] + nv[j])
                blocks[K][0] += 1
                if blocks[K][1] is None:
                    cnt = 0
                    for a in range(O, len(nv)):
                        b = idx.get(tuple(np.array(K) - nv[a]), -1)
                        if b >= O:
                            cnt += 1
                    blocks[K][1] = cnt
        tot += sum(2 * o * v * v for o, v in blocks.values())
    return tot


def job_rates(args, world: int, device_ms: float, e2e_ms_per_step: float):
    """Whole-job rates from this rank's times: every rank solves its own args.twists per
    step, and the job takes as long as its slowest rank (max over ranks).  Returns
    (solves/s on the device, the max device ms, e2e solves/s)."""
    e_max, e2e_max = reduce_max([device_ms, e2e_ms_per_step])
    value = args.twists * world * args.steps / (e_max / 1e3)
    e2e_value = args.twists * world / (e2e_max / 1e3)
    return value, e_max, e2e_value


def run_gpu(args, rank, world):
    import numpy as np

    from uegccd_b200 import Batch
    from uegccd_b200.solver import SystemSet

    opts = dict(SOLVE_OPTS)
    if args.precision == "mixed":
        opts["precision"] = 1
    tw = twists(args.twists, rank=rank)
    systems = build_systems(tw)
    device = int(os.environ.get("LOCAL_RANK", 0))   # one GPU per rank; batches live on it
    batch = Batch(systems, device=device)
    # the reference's own iteration once (untimed): iteration count and energies
    rc_r, e2_r, res_r = batch.solve()
    # warm-up (untimed)
    for _ in range(args.warmup):
        rc, e2, res = batch.solve(**opts)
    dist = None
    if world > 1:
        import torch.distributed as dist
    if dist:
        dist.barrier()
    # timed steps: graph replays only, no per-kernel events; an NVTX range marks them for
    # a profiler's launch list (ncu --nvtx --nvtx-include "timed_steps/")
    step_ms = []
    nvtx = _nvtx()
    with ClockSampler(int(os.environ.get("LOCAL_RANK", 0))) as clk:
        nvtx.range_push("timed_steps")
        for _ in range(args.steps):
            rc, e2, res = batch.solve(**opts)
            step_ms.append(res[0]["gpu_ms"])
        nvtx.range_pop()
    # per-kernel times from separate steps with one event-bracketed iteration per poll round
    batch.set_profiling(True)
    for _ in range(max(1, min(args.steps, 3))):
        batch.solve(**opts)
    stats = batch.kernel_stats()
    batch.set_profiling(False)
    ring_threads = batch.launch_shapes()  # the tuner's picks, from the first CCD solve
    fp64_peak = probe_fp64_peak()           # the FP64 tensor-core roofline denominator, measured
    niters = [r["niter"] for r in res]
    fails = sum(r["fail"] for r in res)
    total_ms = float(sum(step_ms))
    # e2e: through the C ABI with host buffers, every step: batch create (plan, uploads),
    # solve, and every twist's T2 read back into page-locked host memory.  The stages run
    # at once, as a serving host runs them: the next step's batch is created on a host
    # thread (E2E_CREATORS), this step solves, and the previous step's amplitudes are
    # downloaded on another thread (the C calls release the GIL; each batch has its own
    # stream).  The timed run starts before its first create and ends after its last
    # download: the pipeline's fill and drain (one create and one download that overlap
    # nothing) are inside it, spread over at least 32 steps.
    out_bufs = [pinned_buffer(batch.amplitude_count()) for _ in range(2)]
    xfer = [0, 0]
    stage_ms = {"create": [], "solve": [], "download": []}   # host wall time of each stage

    sset = SystemSet(systems)   # the systems' C structs, as the host set-up hands them over

    def create():
        t = time.perf_counter()
        b2 = Batch(sset, device=device)   # a creator thread starts on device 0: name the rank's
        stage_ms["create"].append((time.perf_counter() - t) * 1e3)
        return b2

    def finish(b2, buf):
        t = time.perf_counter()
        b2.all_amplitudes(out=buf)
        xfer[0], xfer[1] = b2.transfer_bytes()
        b2.close()
        stage_ms["download"].append((time.perf_counter() - t) * 1e3)

    def e2e_run(nsteps):
        from concurrent.futures import ThreadPoolExecutor

        for v in stage_ms.values():
            v.clear()
        t0 = time.perf_counter()
        with ThreadPoolExecutor(max_workers=E2E_CREATORS) as creator, ThreadPoolExecutor(max_workers=1) as reader:
            futs = [creator.submit(create)]   # the first create runs alone: nothing to overlap
            submitted = 1
            done = None
            for k in range(nsteps):
                b2 = futs.pop(0).result()
                while submitted < nsteps and len(futs) < E2E_CREATORS:
                    futs.append(creator.submit(create))
                    submitted += 1
                ts = time.perf_counter()
                b2.solve(**opts)
                stage_ms["solve"].append((time.perf_counter() - ts) * 1e3)
                if done is not None:
                    done.result()
                done = reader.submit(finish, b2, out_bufs[k % 2])
            done.result()
        return (time.perf_counter() - t0) * 1e3 / nsteps

    # warm-up: fills the device-memory cache for the pipeline's four live batches and the
    # pinned buffers; then three timed runs, the median reported
    if args.no_e2e:
        e2e_runs = []
        e2e_ms = [float("nan")]
    else:
        e2e_run(max(6, args.warmup))
        e2e_runs = [e2e_run(max(32, 4 * args.steps)) for _ in range(3)]
        e2e_ms = [float(np.median(e2e_runs))]
    h2d, d2h = xfer
    # the other precision on the same batch (timed the same way): mixed beside FP64
    other = None
    if not args.no_other_precision:
        oopts = dict(SOLVE_OPTS)
        if args.precision != "mixed":
            oopts["precision"] = 1
        for _ in range(args.warmup):
            batch.solve(**oopts)
        oms = []
        for _ in range(args.steps):
            rco, e2o, reso = batch.solve(**oopts)
            oms.append(reso[0]["gpu_ms"])
        dE = max(abs(a["ecorr"] - c["ecorr"]) for a, c in zip(res, reso))
        other = {"precision": "mixed" if args.precision != "mixed" else "fp64",
                 "ms": float(sum(oms)), "niter_mean": float(np.mean([r["niter"] for r in reso])),
                 "fails": int(sum(r["fail"] for r in reso)), "max_dE": float(dE)}
    value, e_max, e2e_value = job_rates(args, world, total_ms, float(np.mean(e2e_ms)))
    if other is not None:
        other["ms"] = reduce_max([other["ms"]])[0]
    out = {
        "value": value, "ms_per_step": e_max / args.steps, "e2e_value": e2e_value, "h2d": h2d, "d2h": d2h,
        "niter_mean": float(np.mean(niters)), "niter_min": int(min(niters)), "niter_max": int(max(niters)),
        "fails": int(fails), "rc": rc, "stats": stats, "clocks": clk.summary(), "ring_threads": ring_threads,
        "fp64_peak": fp64_peak,
        "e2e_stage_ms": {k: round(float(np.median(v)), 2) for k, v in stage_ms.items() if v},
        "e2e_runs_ms": [round(x, 2) for x in e2e_runs],
        "ecorr_first": res[0]["ecorr"], "e2_first": float(e2[0]), "launches_per_step": res[0]["kernel_launches"],
        "systems": systems,
        "replay_niter_mean": float(np.mean([r["niter"] for r in res_r])),
        "replay_vs_diis_max_dE": float(max(abs(a["ecorr"] - b["ecorr"]) for a, b in zip(res_r, res))),
        "other": other,
    }
    return out


# ------------------------------------------------------------------- oracle arm
def _oracle_iter_worker(q):
    """Runs `iters` CCD iterations of one twist in the oracle, pinned to one host core (the
    reference is serial); returns seconds per iteration."""
    tw, iters, core = q
    if core is not None and hasattr(os, "sched_setaffinity"):
        os.sched_setaffinity(0, {core})
    sys.path.insert(0, ROOT)
    import numpy as np  # noqa: F401

    from oracle.oracle import Oracle, parse_input_text

    vals = parse_input_text("")
    vals.update({"# Electrons": str(N_ELECTRONS), "Momentum Cutoff": str(MAXK), "rSMin": str(RS),
                 "rSMax": str(RS), "fcut": str(FCUT), "NTwist": " ".join(str(x) for x in tw)})
    o = Oracle(vals)
    e2, ta, tb, tc, _ = o.mp2()
    t0 = time.perf_counter()
    o.ccd(ta, tb, tc, max_iter=iters + 1)  # iters updates + the final residual
    dt = time.perf_counter() - t0
    return dt / (iters + 1)


def oracle_rate(ncores: int, iters: int, iters_per_solve: float, rank: int = 0):
    """Solves/s of the oracle on ncores processes (one twist each), from a bounded sample."""
    import multiprocessing as mp

    tw = twists(max(ncores, 1), rank=rank)
    cores = sorted(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else []
    pin = [cores[k] if k < len(cores) else None for k in range(ncores)]   # one worker per core
    ctx = mp.get_context("spawn")
    t0 = time.perf_counter()
    with ctx.Pool(ncores) as pool:
        per_iter = pool.map(_oracle_iter_worker, [(tuple(t), iters, pin[k]) for k, t in enumerate(tw[:ncores])])
    wall = time.perf_counter() - t0
    sec_per_solve = statistics.mean(per_iter) * iters_per_solve
    return ncores / sec_per_solve, per_iter, wall


def _rank_entry(target, env, argv):
    os.environ.update(env)
    target(argv)


def launch_ranks(n: int, target, argv) -> int:
    """Without torchrun: one process per GPU of this node, ranks 0..n-1 (RANK, LOCAL_RANK,
    WORLD_SIZE and a 127.0.0.1 rendezvous in each one's environment), each running
    target(argv).  Returns 0 when every rank exited 0, else the first non-zero exit code."""
    import multiprocessing as mp
    import socket

    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    ctx = mp.get_context("spawn")
    procs = []
    for r in range(n):
        env = {"RANK": str(r), "LOCAL_RANK": str(r), "WORLD_SIZE": str(n), "LOCAL_WORLD_SIZE": str(n),
               "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)}
        p = ctx.Process(target=_rank_entry, args=(target, env, list(argv)))
        p.start()
        procs.append(p)
    rc = 0
    for p in procs:
        p.join()
        if rc == 0 and p.exitcode:
            rc = p.exitcode if p.exitcode > 0 else 1
    return rc


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--twists", type=int, default=100)
    ap.add_argument("--cpu-iters", type=int, default=1)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-other-precision", action="store_true",
                    help="skip the second timing of the batch in the other precision")
    ap.add_argument("--iters-per-solve", type=float, default=None)
    ap.add_argument("--serve-requests", type=int, default=150,
                    help="requests of the serving stream reported under 'serve' (0: skip)")
    ap.add_argument("--serve-rate", type=float, default=150.0, help="Poisson arrival rate, requests/s")
    ap.add_argument("--serve-requests-saturated", type=int, default=600,
                    help="requests of the saturating serving stream (reported under serve.saturated)")
    ap.add_argument("--serve-rate-saturated", type=float, default=4000.0,
                    help="its arrival rate, requests/s: well above what the GPU serves")
    ap.add_argument("--no-e2e", action="store_true",
                    help="skip the end-to-end pipeline (for profiling the timed device solve alone)")
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="fp64",
                    help="mixed: particle-particle ladder on the tensor cores (FP16/FP32, defect correction)")
    args = ap.parse_args(argv)
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ and args.impl == "ours":
        # not under torchrun: start one rank per GPU here
        sys.exit(launch_ranks(args.gpus, main, sys.argv[1:] if argv is None else argv))
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    metric = "CCD solves/s (N=54 rs=1 twist batch, FP64)"
    config = {"workload": "ccd-twist-batch", "n_electrons": N_ELECTRONS, "rs": RS, "nao": 485,
              "twists_per_gpu": args.twists, "twist_seed": SEED, "maxkpoint_pool": MAXK, "fcut": FCUT,
              "iteration": "Pulay DIIS 6 vectors, undamped Jacobi step, max|dT| < 1e-9",
              "l2": "inputs larger than L2 (each step reads >1 GB of amplitudes and tables)",
              "parallelism": f"independent solves, {world} GPU(s)"}
    ips = args.iters_per_solve or REF_ITERS_PER_SOLVE
    if args.impl == "reference":
        if rank != 0:
            return
        ncores = os.cpu_count() or 1
        vals = []
        for _ in range(args.warmup + args.steps):
            r, per_iter, wall = oracle_rate(ncores, args.cpu_iters, ips)
            vals.append(r)
        v = statistics.mean(vals[args.warmup:]) if args.steps > 0 else vals[-1]
        line = {"impl": "reference", "metric": metric, "value": v, "unit": "solves/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": config,
                "cpu_baseline": {"value": v, "unit": "solves/s", "cores": ncores, "kind": "port",
                                 "sample": f"{args.cpu_iters} CCD iteration(s) of one twist per core (one "
                                           f"process pinned to each), x {ips} iterations per solve"},
                "e2e": {"value": v, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return

    if world > 1:
        import torch
        import torch.distributed as dist

        if torch.cuda.is_available():
            torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
        from datetime import timedelta

        # host-side timing reduction only (the solves exchange nothing): gloo, short timeout
        dist.init_process_group("gloo", timeout=timedelta(seconds=300))
    g = run_gpu(args, rank, world)
    if rank != 0:
        if world > 1:
            import torch.distributed as dist

            dist.barrier()
            dist.destroy_process_group()
        return
    stats = g["stats"]
    per_solve = [plan_stats(x) for x in g["systems"][: min(8, len(g["systems"]))]]
    nsys = len(g["systems"])
    kern = {}
    for k, (ms, launches) in stats.items():
        kinds = [kernel_units(ps).get(k) for ps in per_solve]
        if kinds[0] is None:
            continue
        kind = kinds[0][0]
        units = sum(u[1] for u in kinds) / len(kinds) * nsys  # one launch covers every solve
        avg_s = ms / 1e3 / max(launches, 1)
        if kind == "tflop16":
            ach = units / avg_s / 1e12
            kern[k] = {"bound": "tensor", "achieved": ach, "peak": BF16_PEAK, "unit": "TFLOP/s",
                       "frac": ach / BF16_PEAK, "avg_ms": avg_s * 1e3, "launches": launches,
                       "peak_source": "measured (dense 16-bit tensor)"}
        elif kind == "flop":
            ach = units / avg_s / 1e12
            p64 = g.get("fp64_peak") or FP64_PEAK_TFLOPS
            kern[k] = {"bound": "tensor", "achieved": ach, "peak": p64, "unit": "TFLOP/s",
                       "frac": ach / p64, "avg_ms": avg_s * 1e3, "launches": launches,
                       "peak_source": ("measured in this run: register-only mma.sync m8n8k4 f64 probe"
                                       if g.get("fp64_peak") else "nominal FP64")}
        else:
            ach = units / avg_s / 1e9
            kern[k] = {"bound": "hbm", "achieved": ach, "peak": HBM_PEAK, "unit": "GB/s", "frac": ach / HBM_PEAK,
                       "avg_ms": avg_s * 1e3, "launches": launches, "peak_source": "measured"}
    top = max(kern, key=lambda k: kern[k]["avg_ms"] * kern[k]["launches"])
    roof = dict(kern[top])
    roof["kernel"] = top
    tr = TRAFFIC_PER_SOLVE.get(top)
    roof["traffic"] = tr * nsys if tr else None
    flops_pp = sum(ps["ov2_half"] * 2 for ps in per_solve) / len(per_solve) * nsys
    config["launch_shapes"] = g["ring_threads"]   # picked by the launch-shape tuner on the batch
    if args.precision == "mixed":
        config["precision"] = "particle-particle ladder FP16 tensor cores (FP32 accumulate), rest FP64"
    line = {"metric": metric, "value": g["value"], "unit": "solves/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": g["ms_per_step"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64" if args.precision == "fp64" else "f16/f64", "data": "synthetic", "config": config,
            "e2e": {"value": g["e2e_value"], "unit": "solves/s", "h2d_bytes_per_step": g["h2d"],
                    "d2h_bytes_per_step": g["d2h"], "stage_ms_median": g["e2e_stage_ms"],
                    "ms_per_step_runs": g["e2e_runs_ms"],
                    "note": "per step: batch create (plan + uploads), solve, T2 of every twist to page-locked host "
                            f"memory; the create of the next step ({E2E_CREATORS} host thread(s)) and the download of "
                            "the previous one overlap the solve"},
            "gpu_launches": int(g["launches_per_step"]) * args.steps,
            "clocks": g["clocks"], "roofline": roof,
            "kernels": {k: {"ms": v[0], "launches": v[1], **({"roofline": kern[k]} if k in kern else {})}
                        for k, v in stats.items()},
            "ccd_iterations_per_s": g["value"] * g["niter_mean"],   # solve-iterations of all twists per second
            "check": {"niter_mean": g["niter_mean"], "niter_min": g["niter_min"], "niter_max": g["niter_max"],
                      "not_converged": g["fails"], "ecorr_twist0": g["ecorr_first"], "e2_twist0": g["e2_first"],
                      "pp_ladder_gflop_per_iter": flops_pp / 1e9,
                      "replay_niter_mean": g["replay_niter_mean"],
                      "replay_vs_diis_max_dE": g["replay_vs_diis_max_dE"],
                      # how much of a solves/s ratio against the reference's iteration is the
                      # iteration count (Pulay DIIS here, 1/2-damped Jacobi there) and how much
                      # the rate of iterations
                      "iterations_ratio_replay_over_diis": g["replay_niter_mean"] / g["niter_mean"],
                      "solve_iterations_per_s": g["value"] * g["niter_mean"]}}
    if g.get("other"):
        o = g["other"]
        line[o["precision"]] = {
            "value": args.twists * world * args.steps / (o["ms"] / 1e3), "unit": "solves/s",
            "ms_per_step": o["ms"] / args.steps, "niter_mean": o["niter_mean"], "not_converged": o["fails"],
            "max_abs_dE_vs_" + args.precision + "_Ha": o["max_dE"],
            "max_abs_dE_per_electron_uHa": o["max_dE"] / N_ELECTRONS * 1e6,
            "note": "the same batch, solved in this precision after the headline one (tcgen05 FP16 particle-"
                    "particle ladder on t - t_ref, FP64 refresh per poll round, FP64 sweeps at the end)"
                    if o["precision"] == "mixed" else "the same batch in plain FP64"}
    if world == 1 and args.serve_requests > 0:
        from uegccd_b200 import serve

        def serve_point(n, rate):
            reqs = serve.poisson_stream(n, rate=rate, seed=SEED)
            srv = serve.Server(hbm_budget=40 << 30, max_batch=64, tol=1e-8)
            wall = srv.run(reqs, realtime=True)
            sv = serve.summarize(reqs, wall)
            sv.update({"arrival_rate": rate, "batches": srv.batches_started,
                       "max_concurrent_batches": srv.max_concurrent})
            return sv

        # the arrival-bound point, then a saturating stream (arrivals far above the service rate)
        sv = serve_point(args.serve_requests, args.serve_rate)
        sv.update({"stream": "Poisson; N in {14,54,66,114}; rs log-uniform [0.5,5]; M/(N/2) in {4,8,12,16,20}; "
                             "twist U[-0.5,0.5)^3; MP2/dRPA/CCD 0.2/0.2/0.6", "hbm_budget_gib": 40,
                   "retirement": "per solve, after each round of four iterations (incremental batch solve)"})
        sv["saturated"] = serve_point(args.serve_requests_saturated, args.serve_rate_saturated)
        line["serve"] = sv
    if world == 1 and not args.no_cpu_baseline:
        ncores = 1
        r, per_iter, wall = oracle_rate(ncores, args.cpu_iters, g["replay_niter_mean"])
        line["cpu_baseline"] = {"value": r, "unit": "solves/s", "cores": ncores, "kind": "port",
                                "sample": f"{args.cpu_iters} CCD iteration(s) of twist 0 in the oracle (the "
                                          f"reference's iteration) on one pinned core, x "
                                          f"{g['replay_niter_mean']:.2f} mean iterations per solve "
                                          f"({per_iter[0]:.2f} s/iter); host cores: {os.cpu_count()}"}
    print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
