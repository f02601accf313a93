"""Benchmark of the shear_fdtd hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload c1] [--impl ours|reference]

One bench step is one full solve of the workload (force projection, the whole
time loop, outputs) on seeded synthetic inputs with the config's shapes.
Prints ONE JSON line (rank 0).  Multi-GPU runs are launched by torchrun, one
rank per GPU; the solves are independent replicas (weak scaling, no
collective on the data path) and the time is the max over ranks.

value   Gcell-steps/s with inputs resident in HBM (device-timed, CUDA events)
e2e     the same through the public API with numpy inputs and outputs
        (host<->device copies inside the timed region, wall clock)
roofline  the fused step kernel: algorithmic bytes per launch / mean launch
        time, against the measured HBM copy bandwidth
cpu_baseline  the FP32 CPU port of the reference time loop on a bounded
        sample of the same workload, on this host's cores
"""

from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "Gcell-steps/s mixed+batched vs plain FP64 GPU @relL2≤1e-4; HBM %; p99 lat"
UNIT = "Gcell-steps/s"
FALLBACK_HBM_GBS = 6650.0
# algorithmic bytes per cell-step of the fused step kernel (FP32 mixed form):
# read u_c, u_p and write u_n (9 x 4 B) + mu/rho, eta/rho (2 x 4 B); push
# steps read the projected force (3 x 4 B) in addition
BYTES_CELL_STEP = {"mixed": 44.0, "fp64": 88.0}
BYTES_PUSH = {"mixed": 12.0, "fp64": 24.0}


# ---------------------------------------------------------------------------
# helpers
# ---------------------------------------------------------------------------
def rank_info():
    r = int(os.environ.get("RANK", "0"))
    w = int(os.environ.get("WORLD_SIZE", "1"))
    lr = int(os.environ.get("LOCAL_RANK", str(r)))
    return r, w, lr


def reduce_scalar(x: float, op: str, device, world: int) -> float:
    """Max or sum of a per-rank number over all ranks (identity for one rank)."""
    if world == 1:
        return float(x)
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return float(t.item())


def measured_hbm():
    p = ROOT / "MEASURED_PEAKS.json"
    try:
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def ncu_bytes_per_cell_step(kernel: str):
    """DRAM bytes (read + write) per cell-step of a step kernel, from an ncu
    capture summarised in profiles/traffic.txt (lines ``<kernel>
    bytes_per_cell_step <B>``); None when absent."""
    p = ROOT / "profiles" / "traffic.txt"
    if not p.exists():
        return None
    for line in p.read_text().splitlines():
        parts = line.split()
        if len(parts) >= 3 and parts[0] == kernel and parts[1] == "bytes_per_cell_step":
            try:
                return float(parts[2])
            except ValueError:
                return None
    return None


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []
        self.reader = None
        self.first = threading.Event()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line)
            self.first.set()
        self.first.set()

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200", "-i", str(self.gpu)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return self
        self.reader = threading.Thread(target=self._read, daemon=True)
        self.reader.start()
        # nvidia-smi's start-up (driver and NVML initialisation) ends before
        # the timed region begins: wait for its first sample, then drop it
        self.first.wait(timeout=10)
        self.skip = len(self.lines)
        return self

    def __exit__(self, *exc):
        self.out = ""
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            if self.reader is not None:
                self.reader.join(timeout=5)
            self.out = "".join(self.lines[self.skip:])

    def summary(self):
        rows = []
        for line in (self.out or "").splitlines():
            p = [x.strip() for x in line.split(",")]
            if len(p) < 9:
                continue
            try:
                rows.append((float(p[1]), float(p[2]), p[5:9]))
            except ValueError:
                continue
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for _, _, r in rows for i, v in enumerate(r)
                          if v.lower() == "active"})
        return {"sm_mhz": statistics.median(r[0] for r in rows), "sm_max_mhz": rows[0][1],
                "reasons": reasons, "samples": len(rows)}


# ---------------------------------------------------------------------------
# workloads
# ---------------------------------------------------------------------------
def make_workload(name: str, rank: int, grid=None, nsteps=None, shrink=1.0, instances=48):
    from shearwave_b200 import workloads as W

    if name == "c1":
        shape = (grid, grid, grid) if grid else (192, 192, 192)
        return [W.problem_c1(seed=rank, shape=shape, n_steps=nsteps or 2000)]
    if name == "c0":
        return [W.problem_c0()]
    if name == "c3":
        return W.batch_c3(seed=rank, n=instances, shrink=shrink)
    raise SystemExit(f"unknown workload {name}")


def describe(name: str, probs, shrink: float = 1.0) -> dict:
    cs = sum(_cell_steps(p) for p in probs)
    if name == "c1" and (_shape(probs[0]) != (192, 192, 192) or probs[0]["n_steps"] != 2000):
        name = "c1"  # overridden size: grid / n_steps below say which
    desc = {"workload": {"c0": "config-0 64^3 homogeneous, nT=500, snapshots every 10",
                         "c1": "config-1 192^3 heterogeneous (12 inclusions), nT=2000, "
                               "snapshots every 10, dT viscous clamp",
                         "c3": "config-3 batch of 48 seeded solves 64^3..160x160x224, "
                               "nT 500..3000"}[name],
            "instances": len(probs), "cell_steps_per_rank": cs,
            "grid": list(_shape(probs[0])) if len(probs) == 1 else "varied",
            "n_steps": probs[0]["n_steps"] if len(probs) == 1 else "varied",
            "dX_m": probs[0]["dX"], "precision": "mixed (FP32 u and increment, FP64 projection)",
            "full_size": bool(name != "c3" or (len(probs) == 48 and shrink == 1.0)),
            "l2_flush": "none needed: per-solve state is larger than the 126 MB L2",
            "data": "seeded synthetic inputs with the config shapes"}
    return desc


def _shape(p):
    ref = p["bx"] if p["bx"] is not None else (p["by"] if p["by"] is not None else p["bz"])
    return tuple(ref.shape[:3])


def _cell_steps(p):
    nx, ny, nz = _shape(p)
    return nx * ny * nz * p["n_steps"]


def _to_dev(obj, dev):
    import torch

    if isinstance(obj, np.ndarray):
        return torch.from_numpy(obj).to(dev)
    if isinstance(obj, dict):
        return {k: _to_dev(v, dev) for k, v in obj.items()}
    if isinstance(obj, (list, tuple)):
        return type(obj)(_to_dev(v, dev) for v in obj)
    return obj


def _solve(p, precision, device_io, info=None):
    import shearwave_b200 as sw

    opts = dict(p["opts"], precision=precision)
    if info is not None:
        opts["info"] = info
    return sw.shear_fdtd(p["bx"], p["by"], p["bz"], p["rho"], p["mu"], p["dX"], p["dY"], p["dZ"],
                         p["dT"], p["n_steps"], opts, snapshot_stride=p.get("snapshot_stride"),
                         return_device=device_io)


def _solve_all(probs, precision, device_io, infos=None):
    """One bench step: every problem of the workload (batched when > 1)."""
    import shearwave_b200 as sw

    if len(probs) == 1:
        info = {} if infos is not None else None
        out = [_solve(probs[0], precision, device_io, info)]
        if infos is not None:
            infos.append(info)
        return out
    batch = []
    for p in probs:
        q = dict(p, opts=dict(p["opts"]))
        if infos is not None:
            info = {}
            q["opts"]["info"] = info
            infos.append(info)
        batch.append(q)
    return sw.shear_fdtd_batch(batch, precision=precision, return_device=device_io)


def _to_pinned(obj):
    """numpy arrays of a problem as page-locked host tensors (the e2e inputs)."""
    import torch

    if isinstance(obj, np.ndarray):
        return torch.from_numpy(np.ascontiguousarray(obj)).pin_memory()
    if isinstance(obj, dict):
        return {k: _to_pinned(v) for k, v in obj.items()}
    if isinstance(obj, (list, tuple)):
        return type(obj)(_to_pinned(v) for v in obj)
    return obj


def _nbytes(obj) -> int:
    if hasattr(obj, "is_pinned"):  # a host torch tensor
        return obj.numel() * obj.element_size()
    if isinstance(obj, np.ndarray):
        return obj.nbytes
    if isinstance(obj, dict):
        return sum(_nbytes(v) for v in obj.values())
    if isinstance(obj, (list, tuple)):
        return sum(_nbytes(v) for v in obj)
    return 0


# ---------------------------------------------------------------------------
# CPU baseline: the FP32 port of the reference time loop (oracle) on a sample
# ---------------------------------------------------------------------------
def _cpu_sample(p, budget_s: float):
    from oracle import shearwave_oracle as O

    shape = _shape(p)
    rng = np.random.default_rng(0)
    iu = (1e-6 * rng.standard_normal((*shape, 3))).astype(np.float32)
    opts = dict(p["opts"])
    opts.pop("force_terms", None)
    opts["initial_u"] = iu
    zero = np.zeros(shape, np.float32)
    def timed(steps):
        o = dict(opts, env_t=np.zeros(steps, np.float32))
        t0 = time.perf_counter()
        O.shear_fdtd(None, None, zero, p["rho"], p["mu"], p["dX"], p["dY"], p["dZ"], p["dT"],
                     steps, opts=o, dtype=np.float32)
        return time.perf_counter() - t0

    t1 = timed(1)  # one step sizes the sample
    steps = max(2, min(4096, int(budget_s / max(t1, 1e-4))))
    t = timed(steps)
    n = shape[0] * shape[1] * shape[2]
    return n * steps / t / 1e9, steps, shape


def cpu_baseline(probs, budget_s=12.0):
    p = max(probs, key=_cell_steps)
    v, steps, shape = _cpu_sample(p, budget_s)
    return {"value": v, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"FP32 CPU port of the reference time loop (oracle/shearwave_oracle.py), "
                      f"{steps} steps on the {shape[0]}x{shape[1]}x{shape[2]} grid of this "
                      f"workload, projection excluded, numpy single-threaded"}


def _ref_worker(args):
    p, budget = args
    return _cpu_sample(p, budget)


def run_reference(a, rank, world):
    """Reference arm: the CPU port of the reference on the host's cores."""
    if rank != 0:
        return 0
    probs = make_workload(a.workload, 0, a.grid, a.nsteps, a.shrink, a.instances)
    ncpu = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    procs = ncpu if len(probs) > 1 else 1
    budget = 2.0
    import multiprocessing as mp

    ctx = mp.get_context("spawn")
    samples = []
    with ctx.Pool(procs) as pool:
        for i in range(a.warmup + a.steps):
            work = [(probs[(i * procs + j) % len(probs)], budget) for j in range(procs)]
            t0 = time.perf_counter()
            res = pool.map(_ref_worker, work)
            el = time.perf_counter() - t0
            cells = sum(r[1] * r[2][0] * r[2][1] * r[2][2] for r in res)
            if i >= a.warmup:
                samples.append((cells / el / 1e9, el))
    val = statistics.median(s[0] for s in samples)
    line = {
        "metric": METRIC, "value": val, "unit": UNIT, "impl": "reference", "n_gpus": a.gpus,
        "steps": a.steps, "warmup": a.warmup,
        "ms_per_step": 1e3 * statistics.median(s[1] for s in samples),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic", "config": describe(a.workload, probs, a.shrink),
        "cpu_baseline": {"value": val, "unit": UNIT, "cores": procs, "kind": "port",
                         "sample": f"{procs} process(es) x ~{budget:.0f} s of the FP32 CPU port "
                                   "of the reference time loop on this workload's grids"},
        "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# serving: config-4 request stream through the continuous-batching server
# ---------------------------------------------------------------------------
def c4_requests(n_requests: int, seed: int = 0, pool: int = 0):
    """The config-4 request list: n seeded requests, or, with ``pool`` > 0,
    ``pool`` distinct seeded requests drawn in a seeded order for n arrivals
    (a long stream whose inputs would not fit in host memory, or could not be
    generated between arrivals)."""
    from shearwave_b200 import workloads as W

    rng = np.random.default_rng(1234 + seed)
    if pool <= 0 or pool >= n_requests:
        return [W.problem_c4(rng) for _ in range(n_requests)]
    distinct = [W.problem_c4(rng) for _ in range(pool)]
    order = np.random.default_rng(99 + seed).integers(0, pool, size=n_requests)
    return [distinct[int(k)] for k in order]


def serving_run(n_requests: int, rate_hz: float, seed: int = 0, probs=None,
                n_fp64: int = 2, pool: int = 0) -> dict:
    """Poisson arrivals of config-4 requests (log-uniform 64^3..256^3 cubes,
    1 or 4 pushes, nT 500..4000, inclusion media, HBM budget 150 GB)."""
    from shearwave_b200 import workloads as W
    from shearwave_b200.serve import ShearServer, poisson_arrivals, run_stream

    if probs is None:
        probs = c4_requests(n_requests, seed, pool)
    arrivals = poisson_arrivals(rate_hz, n_requests, seed=seed)
    with ShearServer(hbm_budget=150e9, chunk_steps=50) as srv:
        failed = run_stream(srv, probs, arrivals, keep=False)
    st = srv.stats()
    out = {"requests": n_requests, "rate_hz": rate_hz,
           "latency_s": st["latency_s"], "queue_s": st["queue_s"],
           "gcell_steps_per_s": st["gcell_steps_per_s"], "failed": int(failed),
           "wall_s": st["wall_s"],
           "cell_steps": int(sum(W.cell_steps(p) for p in probs)),
           "distinct_requests": len({id(p) for p in probs}),
           "workload": "config-4 requests (log-uniform 64^3..256^3, 1 or 4 pushes, "
                       "nT 500..4000), Poisson arrivals, budget 150 GB, mixed form"}
    if n_fp64 > 0:
        out["fp64_one_at_a_time"] = _fp64_one_at_a_time(probs[:n_fp64])
    return out


def serving_sweep(rates, n_requests: int, n_fp64: int, seed: int = 0, pool: int = 0) -> dict:
    """The config-4 stream at several arrival rates (the same seeded requests
    at every rate), and the first ``n_fp64`` requests solved one at a time in
    plain FP64 (device-resident inputs, CUDA events) as the comparison."""
    import torch

    from shearwave_b200 import workloads as W

    probs = c4_requests(n_requests, seed, pool)
    runs = [serving_run(n_requests, r, seed, probs, n_fp64=0) for r in rates]
    out = {"rates": [{k: r[k] for k in ("rate_hz", "latency_s", "queue_s", "gcell_steps_per_s",
                                        "wall_s", "failed")}
                     for r in runs],
           "requests": n_requests, "distinct_requests": runs[0]["distinct_requests"],
           "workload": runs[0]["workload"]}
    if n_fp64 > 0:
        out["fp64_one_at_a_time"] = _fp64_one_at_a_time(probs[:n_fp64])
    return out


def _fp64_one_at_a_time(sample) -> dict:
    """Plain-FP64 shear_fdtd calls one after another on requests of the
    stream (inputs in HBM, CUDA events): the serving comparison."""
    import torch

    from shearwave_b200 import workloads as W

    dev = torch.device("cuda", torch.cuda.current_device())
    dsample = [_to_dev(p, dev) for p in sample]
    _solve(dsample[0], "fp64", True)  # warm
    torch.cuda.synchronize()
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record()
    for p in dsample:
        _solve(p, "fp64", True)
    e.record()
    torch.cuda.synchronize()
    cs = sum(W.cell_steps(p) for p in sample)
    return {"value": cs / (s.elapsed_time(e) / 1e3) / 1e9, "unit": UNIT,
            "sample": f"{len(sample)} requests of the stream, plain FP64 shear_fdtd calls one "
                      "after another, inputs in HBM"}


# ---------------------------------------------------------------------------
# accuracy and phase-time extras of the bench line
# ---------------------------------------------------------------------------
def _knobs():
    from shearwave_b200 import tune

    return tune.get_knobs()


def _split(infos, batched: bool) -> dict:
    """Device time of the phases of one bench step (CUDA events in the solver):
    setup + force projection, the time loop, the output conversion.  A batch
    runs each phase for all solves together (max over solves); sequential
    solves add up."""
    agg = max if batched else sum
    out = {k: agg(i[f"t_{k}_ms"] for i in infos) for k in ("setup", "steps", "finish")}
    out["projection_method"] = sorted({c.get("method", "cg") for i in infos for c in i["cg"]})
    out["cg_iterations"] = int(sum(c["iters"] for i in infos for c in i["cg"]))
    out["note"] = ("setup = materials, initial state and the force projection; steps = the "
                   "time loop; finish = output conversion")
    return out


def _strain_rel(outs, o64, probs) -> dict:
    """Max over solves of the relative L2 of each strain invariant of the mixed
    result against the plain FP64 result (fused strain post-pass on both)."""
    import shearwave_b200 as sw

    worst = {}
    for (u32, *_), (u64, *_), p in zip(outs, o64, probs):
        _e, i32 = sw.compute_strain_fields(u32, p["dX"], p["dY"], p["dZ"], return_tensor=False,
                                           return_device=True)
        _e, i64 = sw.compute_strain_fields(u64, p["dX"], p["dY"], p["dZ"], return_tensor=False,
                                           return_device=True)
        for k in i64:
            a, b = i32[k].double(), i64[k].double()
            r = float((a - b).norm() / b.norm().clamp_min(1e-300))
            worst[k] = max(worst.get(k, 0.0), r)
    return worst


def _divergence_residual(dprobs) -> dict:
    """Divergence residual max|div_c f_S| / max|div_c f| of each solve's
    projected force: the mixed form's projection (spectral solve) and the
    plain FP64 form's CG at the solve's tolerance, and the relative L2 of the
    mixed projected force against the FP64 one."""
    import torch

    import shearwave_b200 as sw

    rows = []
    for p in dprobs:
        z = torch.zeros_like(p["bz"], dtype=torch.float64)
        bz = p["bz"].double()
        h = (p["dX"], p["dY"], p["dZ"])
        tol, it = p["opts"]["poisson_tol"], p["opts"]["poisson_max_iters"]
        din = sw.divergence_center(z, z, bz, *h).abs().max()
        fs = sw.project_vector_field(z, z, bz, *h, tol, it, method="spectral")
        fc = sw.project_vector_field(z, z, bz, *h, tol, it, method="cg")
        rs = float(sw.divergence_center(*fs, *h).abs().max() / din)
        rc = float(sw.divergence_center(*fc, *h).abs().max() / din)
        num = sum(float((a - b).norm() ** 2) for a, b in zip(fs, fc)) ** 0.5
        den = sum(float(b.norm() ** 2) for b in fc) ** 0.5
        rows.append((rs, rc, num / den))
    return {"mixed_spectral": max(r[0] for r in rows), "fp64_cg": max(r[1] for r in rows),
            "rel_l2_mixed_vs_fp64_force": max(r[2] for r in rows),
            "solves": len(rows),
            "note": "max over the first solves of the workload, each at its own poisson_tol"}


def _kahan_run(dprobs, cs_rank, o64, max_over_ranks, sum_over_ranks) -> dict:
    """One bench step with the compensated displacement sum (kahan=True: one
    step per launch, 12 more bytes per cell-step), device-timed."""
    import torch

    kprobs = [dict(p, opts=dict(p["opts"], kahan=True)) for p in dprobs]
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record()
    outs = _solve_all(kprobs, "mixed", True)
    e.record()
    torch.cuda.synchronize()
    t = max_over_ranks(s.elapsed_time(e) / 1e3)
    ru = max(float((o[0].double() - r[0]).norm() / r[0].norm()) for o, r in zip(outs, o64))
    rv = max(float((o[1].double() - r[1]).norm() / r[1].norm()) for o, r in zip(outs, o64))
    return {"value": sum_over_ranks(cs_rank) / t / 1e9, "unit": UNIT, "rel_l2_u": ru,
            "rel_l2_v": rv, "how": "the same batch with opts kahan=True (one step per "
                                   "launch), one device-timed bench step"}


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--workload", default="c3", choices=["c0", "c1", "c3"])
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--grid", type=int, default=None, help="c1 only: cubic grid override")
    ap.add_argument("--nsteps", type=int, default=None, help="c1 only: nT override")
    ap.add_argument("--shrink", type=float, default=1.0,
                    help="c3 only: scale grids and nT down (small cases for profiling)")
    ap.add_argument("--instances", type=int, default=48, help="c3 only: solves in the batch")
    ap.add_argument("--serve-requests", type=int, default=16,
                    help="requests of the config-4 serving stream run after the timing (0: skip)")
    ap.add_argument("--serve-rate", type=float, default=4.0,
                    help="mean Poisson arrival rate of the serving stream (requests/s)")
    ap.add_argument("--serve-pool", type=int, default=0,
                    help="distinct seeded requests the serving stream draws from (0: every "
                         "request distinct)")
    ap.add_argument("--serve-sweep", default=None,
                    help="comma-separated arrival rates (requests/s): run the serving stream "
                         "at each rate instead of --serve-rate, plus plain-FP64 one-at-a-time "
                         "solves of its first requests")
    ap.add_argument("--steps-per-pass", type=int, default=0, choices=[0, 1, 2],
                    help="mixed form: time steps fused per pass over HBM (0 = library default)")
    ap.add_argument("--no-tune", action="store_true",
                    help="skip the autotuner (library default launch shapes)")
    ap.add_argument("--knobs", default=None,
                    help="launch-shape knobs name=value,... set instead of the autotuner "
                         "(shearwave_b200.tune.KNOBS)")
    ap.add_argument("--tune-steps", type=int, default=128,
                    help="time steps of the shortened workload each autotuner candidate runs")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the compensated-sum run, the pageable e2e run and the "
                         "divergence / strain-invariant accuracy checks")
    a = ap.parse_args(argv)
    rank, world, local = rank_info()
    if a.impl == "reference":
        return run_reference(a, rank, world)

    import torch
    import torch.distributed as dist

    import shearwave_b200._native as native

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(x: float) -> float:
        return reduce_scalar(x, "max", dev, world)

    def sum_over_ranks(x: float) -> float:
        return reduce_scalar(x, "sum", dev, world)

    probs = make_workload(a.workload, rank, a.grid, a.nsteps, a.shrink, a.instances)
    if a.steps_per_pass:
        for p in probs:
            p["opts"] = dict(p["opts"], steps_per_pass=a.steps_per_pass)
    dprobs = [_to_dev(p, dev) for p in probs]
    cs_rank = sum(_cell_steps(p) for p in probs)

    # ---- launch shapes chosen by the autotuner (shearwave_b200/tune.py) ----
    tune_info = None
    default_knobs = _knobs()
    if a.knobs:
        from shearwave_b200 import tune

        tune.set_knobs(**{k: int(v) for k, v in (kv.split("=") for kv in a.knobs.split(","))})
        tune_info = {"knobs": tune.get_knobs(), "set_by": "--knobs"}
    elif not a.no_tune and not a.steps_per_pass:
        from shearwave_b200 import tune

        t0 = time.perf_counter()
        cands = tune.fused_batch_candidates() if len(dprobs) > 1 else None
        res = tune.autotune(dprobs, steps=a.tune_steps, repeats=1, candidates=cands)
        tune_info = {"knobs": res["best"], "candidates": len(res["results"]),
                     "tune_steps": a.tune_steps, "seconds": time.perf_counter() - t0,
                     "scores_gcell_steps_s": [round(r["gcell_steps_per_s"], 2)
                                              for r in res["results"]]}

    # ---- device-resident timing -------------------------------------------
    for _ in range(a.warmup):
        _solve_all(dprobs, "mixed", True)
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    infos = []
    n0, h0 = native.launch_count(), native.host_enqueue_count()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        start.record()
        for _ in range(a.steps):
            infos = []
            outs = _solve_all(dprobs, "mixed", True, infos)
        end.record()
        torch.cuda.synchronize()
    barrier()
    launches = native.launch_count() - n0
    host_enqueues = native.host_enqueue_count() - h0
    t_dev = max_over_ranks(start.elapsed_time(end) / 1e3)
    value = sum_over_ranks(cs_rank) * a.steps / t_dev / 1e9

    # roofline of the step kernel (the dominant kernel).  The step loop
    # launches one kernel per pair of time steps (one per single step at an
    # odd end); a batched run covers all running solves in each launch.
    # achieved = algorithmic bytes of the launches / their device time.
    # the library fuses step pairs by default, batched or alone
    spl = 1 if a.steps_per_pass == 1 else 2
    if len(probs) > 1:
        step_ms = max(i["t_steps_ms"] for i in infos)
        steps_total = max(p["n_steps"] for p in probs)
    else:
        step_ms = infos[0]["t_steps_ms"]
        steps_total = probs[0]["n_steps"]
    launches_step = (steps_total + spl - 1) // spl
    alg_bytes = 0.0
    for p, i in zip(probs, infos):
        nx, ny, nz = _shape(p)
        alg_bytes += nx * ny * nz * (BYTES_CELL_STEP["mixed"] * p["n_steps"]
                                     + BYTES_PUSH["mixed"] * i["n_push_steps"])
    per_launch_ms = step_ms / launches_step
    achieved = alg_bytes / (step_ms / 1e3) / 1e9
    peak, peak_kind = measured_hbm()
    bpcs = ncu_bytes_per_cell_step("step_f32_fused2" if spl == 2 else "step_f32_tma")
    cells_per_launch = sum(math.prod(_shape(p)) * p["n_steps"] for p in probs) / launches_step
    traffic = None if bpcs is None else bpcs * cells_per_launch
    roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "traffic": traffic, "peak_source": peak_kind,
            "frac_of_nominal_8000_gbs": achieved / 8000.0,
            "traffic_note": ("DRAM bytes per launch: ncu's read+write bytes per cell-step "
                             "(profiles/traffic.txt) x the cells a launch updates"),
            "traffic_bytes_per_cell_step": bpcs,
            "kernel": ("step_f32_fused2 (two KV steps per pass, mixed form)" if spl == 2
                       else "step_f32_tma (fused KV step, mixed form)"),
            "steps_per_launch": spl,
            "mean_launch_us": per_launch_ms * 1e3,
            "alg_bytes_per_launch": alg_bytes / launches_step,
            "step_only_gcell_steps_s": cs_rank / (step_ms / 1e3) / 1e9}

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": 1e3 * t_dev / a.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": dict(describe(a.workload, probs, a.shrink), autotune=tune_info,
                       knobs=_knobs()), "roofline": roof,
        "clocks": clk.summary(), "gpu_launches": int(launches),
        "host_enqueues": int(host_enqueues),
        "cg_iters": [c["iters"] for i in infos for c in i["cg"]],
        "time_split_ms": {"mixed": _split(infos, batched=len(probs) > 1)},
    }

    # ---- plain FP64 GPU drop-in on the same workload: one solve at a time ----
    if not a.no_fp64:
        _solve(dprobs[0], "fp64", True)  # warm
        torch.cuda.synchronize()
        barrier()
        s2, e2 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        infos64 = [{} for _ in dprobs]
        from shearwave_b200 import tune

        with tune.knobs(**default_knobs):  # the plain drop-in runs the library defaults
            s2.record()
            o64 = [_solve(p, "fp64", True, i) for p, i in zip(dprobs, infos64)]
            e2.record()
            torch.cuda.synchronize()
        t64 = max_over_ranks(s2.elapsed_time(e2) / 1e3)
        v64 = sum_over_ranks(cs_rank) / t64 / 1e9
        line["time_split_ms"]["fp64"] = _split(infos64, batched=False)
        rl = []
        for (u32, v32, *_), (u64, v64_, *_) in zip(outs, o64):
            du = torch.linalg.vector_norm(u32.double() - u64) / torch.linalg.vector_norm(u64)
            dv = torch.linalg.vector_norm(v32.double() - v64_) / torch.linalg.vector_norm(v64_)
            rl.append((float(du), float(dv)))
        line["vs_plain_fp64"] = {"value": v64, "unit": UNIT, "ratio": value / v64,
                                 "how": "the same problems as sequential plain-FP64 "
                                        "shear_fdtd calls, device-resident, CUDA events",
                                 "rel_l2_u": max(r[0] for r in rl),
                                 "rel_l2_v": max(r[1] for r in rl)}
        if not a.no_extras:
            line["vs_plain_fp64"]["rel_l2_strain_invariants"] = _strain_rel(outs, o64, probs)
            line["divergence_residual"] = _divergence_residual(dprobs[:4])
            line["kahan"] = _kahan_run(dprobs, cs_rank, o64, max_over_ranks, sum_over_ranks)
        del o64

    # ---- end to end through the public API with host arrays ---------------
    # inputs in page-locked host memory, outputs returned as numpy arrays;
    # every timed step copies the inputs in and the results out
    if not a.no_e2e:
        hprobs = [_to_pinned(p) for p in probs]
        h2d = sum(_nbytes({k: p[k] for k in ("bx", "by", "bz", "rho", "mu", "opts")})
                  for p in hprobs)
        e2e_steps = max(1, min(a.steps, 3))
        _solve_all(hprobs, "mixed", False)  # warm-up: allocator and pinned-buffer caches
        torch.cuda.synchronize()
        barrier()
        t0 = time.perf_counter()
        d2h = 0
        for _ in range(e2e_steps):
            outs = _solve_all(hprobs, "mixed", False)
            d2h = sum(o.nbytes for out in outs for o in out)
            del outs
        torch.cuda.synchronize()
        te = max_over_ranks(time.perf_counter() - t0)
        line["e2e"] = {"value": sum_over_ranks(cs_rank) * e2e_steps / te / 1e9, "unit": UNIT,
                       "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                       "steps": e2e_steps,
                       "note": "page-locked host inputs in, numpy outputs back, through "
                               "shear_fdtd_batch (projection included), wall clock after "
                               "one warm-up step"}
        if not a.no_extras:
            # the same with the plain (pageable) numpy arrays a drop-in caller passes
            t0 = time.perf_counter()
            for _ in range(e2e_steps):
                outs = _solve_all(probs, "mixed", False)
                del outs
            torch.cuda.synchronize()
            tp = max_over_ranks(time.perf_counter() - t0)
            line["e2e_pageable"] = {
                "value": sum_over_ranks(cs_rank) * e2e_steps / tp / 1e9, "unit": UNIT,
                "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                "steps": e2e_steps,
                "note": "pageable numpy inputs in (as a drop-in caller passes them), numpy "
                        "outputs back, otherwise as e2e"}

    if rank == 0 and world == 1 and a.serve_requests > 0:
        if a.serve_sweep:
            rates = [float(r) for r in a.serve_sweep.split(",")]
            line["serving_sweep"] = serving_sweep(rates, a.serve_requests, 6, seed=rank,
                                                  pool=a.serve_pool)
        else:
            line["serving"] = serving_run(a.serve_requests, a.serve_rate, seed=rank,
                                          pool=a.serve_pool)

    if rank == 0 and world == 1 and not a.no_cpu:
        line["cpu_baseline"] = cpu_baseline(probs)

    if world > 1:
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
