"""Throughput benchmark of the fused lattice-Boltzmann step (one JSON line on stdout).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME] [--impl b200|reference]

Default workload: D2Q9 BGK, tau = 0.6, 4096 x 4096 fully periodic, fp32 storage (f - w,
shifted arithmetic), pull two-buffer; rho = 1 + 0.01 N(0,1), u = 8 seeded Fourier modes with
max|u| = 0.05. One benchmark step = 1000 lattice time steps of the whole lattice. The state
(2 x 604 MB) is larger than L2, so no flush is needed between steps.

Batched workload ``d2q9-mrt-batch64-f16``: 64 independent D2Q9 MRT lid-driven cavities, edges
log-uniform in [128, 1024] (multiples of 8), tau ~ U[0.51, 1], lid speed ~ U[0.05, 0.1], fp16
storage, advanced together by one launch per lattice step; one benchmark step = 2000 lattice
steps replayed from one CUDA graph (2 x 209 MB of state, larger than L2).

* ``value``    MLUPS with the state resident in HBM, CUDA events on the launching stream,
               max over ranks (replicas: every rank advances its own lattice, no collective
               on the data path).
* ``e2e``      the same through the solver API with host buffers: every step copies the
               stored state host -> device from pinned memory, advances 1000 steps and copies
               the state back.
* ``roofline`` algorithmic bytes (2 q s per node and launch) / average launch time, against
               the measured HBM copy bandwidth.
* ``cpu_baseline``  the float64 NumPy oracle (a port of pylbm's own CPU path) on a bounded
               sample of the same workload, one host core.

``--impl reference`` times that CPU implementation instead, on all host cores (one process
per core, each advancing its own 4096-wide periodic band of the workload).
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

# name -> (lattice, n, collision, tau, variant)
WORKLOADS = {
    "d2q9-bgk-ab-f32": ("D2Q9", 4096, "bgk", 0.6, "fused"),
    "d2q9-trt-ab-f32": ("D2Q9", 4096, "trt", 0.6, "fused"),
    "d2q9-bgk-aa-f32": ("D2Q9", 4096, "bgk", 0.6, "fused-aa"),
    "d2q9-trt-aa-f32": ("D2Q9", 4096, "trt", 0.6, "fused-aa"),
    "d2q9-bgk-ab-f16": ("D2Q9", 4096, "bgk", 0.6, "fused-fp16"),
    "d2q9-bgk-aa-f16": ("D2Q9", 4096, "bgk", 0.6, "fused-aa-fp16"),
    "d2q9-bgk-ab-plain": ("D2Q9", 4096, "bgk", 0.6, "fused-plain"),
    "d3q19-trt-ab-f32": ("D3Q19", 256, "trt", 0.55, "fused"),
    "d3q19-trt-ab-f16": ("D3Q19", 256, "trt", 0.55, "fused-fp16"),
    "d3q19-trt-ab-bf16": ("D3Q19", 256, "trt", 0.55, "fused-bf16"),
    "d3q19-trt-aa-f32": ("D3Q19", 256, "trt", 0.55, "fused-aa"),
    # lid-driven cavities (walls on every axis, lid U = 0.05 on the top of the last axis)
    "d2q9-bgk-cavity-f32": ("D2Q9", 4096, "bgk", 0.6, "fused"),
    "d2q9-mrt-cavity-f32": ("D2Q9", 4096, "mrt", 0.6, "fused"),
    "d2q9-mrt-cavity-f16": ("D2Q9", 4096, "mrt", 0.6, "fused-fp16"),
    "d3q19-bgk-cavity-f32": ("D3Q19", 256, "bgk", 0.6, "fused"),
}


# batches of independent lattices: name -> (count, collision, variant, seed)
BATCHES = {
    "d2q9-mrt-batch64-f16": (64, "mrt", "fused-fp16", 0),
}


# pylbm's published MLUPS for the same lattice, collision, size, storage and pattern on its
# benchmark problem (the 4096^2 lid-driven cavity, README.md:84-115, on an RTX 3070 Laptop
# GPU; its Re = 1000 sets a different relaxation rate, which changes no work per node);
# vs_baseline is null for workloads without such a figure
PUBLISHED_MLUPS = {
    "d2q9-bgk-cavity-f32": 5024.0,  # CUDA C fused, fp32 (README.md:97)
}


def is_cavity(name: str) -> bool:
    return "cavity" in name


def batch_problems(name: str) -> list:
    from pylbm_b200 import workloads as W

    count, coll, _, seed = BATCHES[name]
    return W.cavity_batch_problems(count, seed=seed, collision=coll)


def dominant_kernel(name: str) -> str:
    """The step kernel the workload runs (the only kernel launched in the timed region)."""
    if name in BATCHES:
        return "k_d2q9_batch_ab"
    lat, _, _, _, variant = WORKLOADS[name]
    if "-aa" in variant:
        return ("k_d2q9_aa_odd + k_d2q9_aa_even" if lat == "D2Q9"
                else "k_staged (AA odd) + k_aa_even")
    return "k_d2q9_ab" if lat == "D2Q9" else "rows3d::k_ab"


def default_lbm_steps(name: str) -> int:
    return 2000 if name in BATCHES else 1000
FALLBACK_HBM_GBS = 6650.0


def log(*a) -> None:  # noqa: ANN002
    print(*a, file=sys.stderr, flush=True)


def measured_peak() -> tuple[float, str]:
    p = ROOT / "MEASURED_PEAKS.json"
    try:
        return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def traffic_from_profiles(kernel_tag: str) -> float | None:
    """Per-launch DRAM bytes recorded from an ncu capture in profiles/traffic.json."""
    p = ROOT / "profiles" / "traffic.json"
    try:
        return float(json.loads(p.read_text())[kernel_tag]["bytes_per_launch"])
    except Exception:
        return None


def make_problem(name: str, n: int | None = None):
    from pylbm_b200.problem import Problem

    lat, n0, coll, tau, _ = WORKLOADS[name]
    n = n or n0
    shape = (n, n) if lat == "D2Q9" else (n, n, n)
    if is_cavity(name):
        return Problem(shape, tau=tau, collision=coll, u_lid=0.05)
    return Problem(shape, tau=tau, collision=coll, periodic=(True,) * len(shape))


def initial_state(name: str, seed: int, n: int | None = None) -> np.ndarray:
    from pylbm_b200 import workloads as W

    lat, n0, *_ = WORKLOADS[name]
    n = n or n0
    if is_cavity(name):  # fluid at rest, set in motion by the lid
        return make_problem(name, n).initial_populations()
    if lat == "D2Q9":
        return W.fourier_populations(n, seed)
    return W.taylor_green_3d_populations(n)


# ----------------------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi clock / throttle-reason samples during the timed region (read-only)."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int) -> None:
        self.gpu = gpu
        self.tmp = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.proc = None

    def __enter__(self) -> ClockSampler:
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.tmp, stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc) -> None:  # noqa: ANN002
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self) -> dict:
        self.tmp.flush()
        rows = []
        for line in Path(self.tmp.name).read_text().splitlines():
            parts = [v.strip() for v in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.tmp.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if v == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(rows)}


# ----------------------------------------------------------------------------- CPU legs
def _oracle_band_worker(args: tuple) -> float:
    """Time ``steps`` oracle steps on one periodic 4096-wide band (runs in a spawned process)."""
    name, rows, steps, warmup, seed, barrier = args
    sys.path.insert(0, str(ROOT))
    from oracle import lbm_oracle as O
    from pylbm_b200 import workloads as W
    from pylbm_b200.lattice import D2Q9, D3Q19, equilibrium

    lat, n, coll, tau, _ = WORKLOADS[name]
    if is_cavity(name):  # a cavity of the band's size: walls everywhere, lid on top
        shape = (n, rows) if lat == "D2Q9" else (n, n, rows)
        case = O.Case(shape, tau, coll, (False,) * len(shape), u_lid=0.05)
        lattice = D2Q9 if lat == "D2Q9" else D3Q19
        f = equilibrium(lattice, np.ones(shape[::-1]), np.zeros((len(shape),) + shape[::-1]))
    elif lat == "D2Q9":
        rho, u = W.fourier_state(n, seed)
        f = equilibrium(D2Q9, rho[:rows], u[:, :rows])
        case = O.Case((n, rows), tau, coll, (True, True))
    else:
        rho, u = W.taylor_green_3d(n)
        f = equilibrium(D3Q19, rho[:rows], u[:, :rows])
        case = O.Case((n, n, rows), tau, coll, (True, True, True))
    for _ in range(warmup):
        f = O.step(f, case)
    if barrier is not None:
        barrier.wait()
    t0 = time.perf_counter()
    for _ in range(steps):
        f = O.step(f, case)
    return time.perf_counter() - t0


def _oracle_batch_worker(args: tuple) -> tuple[float, int]:
    """Time ``steps`` oracle steps on lattice ``i`` of a batch (runs in a spawned process);
    returns (seconds, nodes)."""
    name, i, steps, warmup, barrier = args
    sys.path.insert(0, str(ROOT))
    from oracle import lbm_oracle as O

    p = batch_problems(name)[i]
    case = O.Case(tuple(p.shape), p.tau, p.collision, (False, False), u_lid=p.u_lid)
    f = p.initial_populations()
    for _ in range(warmup):
        f = O.step(f, case)
    if barrier is not None:
        barrier.wait()
    t0 = time.perf_counter()
    for _ in range(steps):
        f = O.step(f, case)
    return time.perf_counter() - t0, p.n_nodes


def band_nodes(name: str, rows: int) -> int:
    lat, n, *_ = WORKLOADS[name]
    return n * rows if lat == "D2Q9" else n * n * rows


def cpu_baseline(name: str) -> dict:
    """The oracle on one core, a bounded sample of the workload (about 10 s)."""
    if name in BATCHES:
        dt, nodes = _oracle_batch_worker((name, 0, 3, 1, None))
        return {"value": nodes * 3 / dt / 1e6, "unit": "MLUPS", "cores": 1, "kind": "port",
                "sample": f"float64 NumPy oracle, 3 steps of lattice 0 of the batch "
                          f"({nodes} nodes)"}
    lat = WORKLOADS[name][0]
    rows, steps = (512, 3) if lat == "D2Q9" else (8, 3)
    dt = _oracle_band_worker((name, rows, steps, 1, 0, None))
    mlups = band_nodes(name, rows) * steps / dt / 1e6
    return {"value": mlups, "unit": "MLUPS", "cores": 1, "kind": "port",
            "sample": f"float64 NumPy oracle, {steps} steps of a periodic band of "
                      f"{band_nodes(name, rows)} nodes of the same workload"}


def run_reference(a: argparse.Namespace) -> None:
    """--impl reference: the CPU implementation on all host cores."""
    import multiprocessing as mp

    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    name = a.workload
    cores = min(os.cpu_count() or 1, a.cpu_procs)
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    barrier = mgr.Barrier(cores)
    if name in BATCHES:  # one lattice of the batch per process
        count = BATCHES[name][0]
        with ctx.Pool(cores) as pool:
            res = pool.map(_oracle_batch_worker,
                           [(name, i % count, a.steps, a.warmup, barrier) for i in range(cores)])
        dt = max(r[0] for r in res)
        total = sum(r[1] for r in res) * a.steps
        sample = (f"float64 NumPy oracle, {cores} processes x {a.steps} steps, each on one "
                  f"lattice of the batch")
    else:
        lat = WORKLOADS[name][0]
        rows = 64 if lat == "D2Q9" else 2
        with ctx.Pool(cores) as pool:
            times = pool.map(_oracle_band_worker,
                             [(name, rows, a.steps, a.warmup, 0, barrier)] * cores)
        dt = max(times)
        total = cores * band_nodes(name, rows) * a.steps
        sample = (f"float64 NumPy oracle, {cores} processes x {a.steps} steps of a periodic "
                  f"band of {band_nodes(name, rows)} nodes each")
    mlups = total / dt / 1e6
    out = {"impl": "reference", "metric": "MLUPS", "value": mlups, "unit": "MLUPS",
           "n_gpus": a.gpus, "steps": a.steps, "warmup": a.warmup,
           "ms_per_step": 1e3 * dt / a.steps, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f64", "data": "synthetic",
           "config": config_of(name, a),
           "cpu_baseline": {"value": mlups, "unit": "MLUPS", "cores": cores, "kind": "port",
                            "sample": sample},
           "e2e": {"value": mlups, "unit": "MLUPS", "h2d_bytes_per_step": 0,
                   "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


def config_of(name: str, a: argparse.Namespace) -> dict:
    if name in BATCHES:
        count, coll, variant, seed = BATCHES[name]
        probs = batch_problems(name)
        return {"workload": name, "lattice": "D2Q9", "lattices": count,
                "nodes": int(sum(p.n_nodes for p in probs)), "collision": coll,
                "variant": variant, "edges": "log-uniform [128, 1024], multiples of 8",
                "tau": "U[0.51, 1.0]", "u_lid": "U[0.05, 0.1]", "seed": seed,
                "lbm_steps_per_step": a.lbm_steps, "launch": "CUDA graph, one launch per step",
                "launch_shape": getattr(a, "launch_shape", None),
                "init": "lid-driven cavities, fluid at rest",
                "l2": "state larger than L2 (no flush needed)",
                "parallelism": f"replicas x{a.gpus}"}
    lat, n, coll, tau, variant = WORKLOADS[name]
    n = a.n or n
    shape = [n, n] if lat == "D2Q9" else [n, n, n]
    if is_cavity(name):
        init = "lid-driven cavity, walls on every axis, lid U=0.05, fluid at rest"
    elif lat == "D2Q9":
        init = "rho=1+0.01N(0,1), u=8 seeded Fourier modes, max|u|=0.05"
    else:
        init = "Taylor-Green vortex u0=0.05, rho=1"
    return {"workload": name, "lattice": lat, "shape": shape, "collision": coll, "tau": tau,
            "variant": variant, "periodic": not is_cavity(name),
            "lbm_steps_per_step": a.lbm_steps, "init": init,
            "l2": "state larger than L2 (no flush needed)", "parallelism": f"replicas x{a.gpus}"}


# ----------------------------------------------------------------------------- ranks
def rank_barrier(world: int, device: str) -> None:
    """All ranks meet here, with the device idle on both sides (no-op for one rank)."""
    import torch

    if device == "cuda":
        torch.cuda.synchronize()
    if world > 1:
        import torch.distributed as dist

        dist.barrier()
        if device == "cuda":
            torch.cuda.synchronize()


def ranks_max(v: float, world: int, device: str) -> float:
    """The maximum of v over the ranks (the job's time is its slowest rank's)."""
    if world == 1:
        return v
    import torch
    import torch.distributed as dist

    t = torch.tensor([v], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_mlups(world: int, nodes: int, steps: int, seconds: float) -> float:
    """Whole-job throughput of ``world`` replicas, each advancing ``nodes`` nodes ``steps``
    times, over the max-over-ranks time."""
    return world * nodes * steps / seconds / 1e6


# ----------------------------------------------------------------------------- GPU arm
def run_b200(a: argparse.Namespace) -> None:
    import torch
    import torch.distributed as dist

    from pylbm_b200.backend import VARIANTS

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    name = a.workload
    if name in BATCHES:
        from pylbm_b200.autotune import autotune_batch
        from pylbm_b200.batched import BatchedSolver

        s = BatchedSolver(batch_problems(name), BATCHES[name][2])
        a.launch_shape = autotune_batch(s)["launch"]  # threads per block, blocks per SM (0: one item per warp)
        nodes = s.nodes
    else:
        cls = VARIANTS[WORKLOADS[name][4]]
        p = make_problem(name, a.n)
        s = cls(p)
        s.set_populations(initial_state(name, seed=rank, n=a.n))
        nodes = p.n_nodes
    L = a.lbm_steps

    def barrier() -> None:
        rank_barrier(world, "cuda")

    def max_over_ranks(v: float) -> float:
        return ranks_max(v, world, "cuda")

    # ---------------- device-resident throughput
    for _ in range(a.warmup):
        s.step(L)
    barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        ev0.record()
        for _ in range(a.steps):
            s.step(L)
        ev1.record()
        ev1.synchronize()
    barrier()
    dt = max_over_ranks(ev0.elapsed_time(ev1) / 1e3)
    clocks = clk.summary()
    launches = a.steps * L  # one kernel launch per lattice time step (AB and AA alike)
    value = replica_mlups(world, nodes, L * a.steps, dt)

    # ---------------- end to end through the solver API, host buffers
    e2e = None
    if not a.no_e2e:
        host_in = torch.empty(s.A.numel(), dtype=s.A.dtype, pin_memory=True)
        host_in.copy_(s.A)
        host_out = torch.empty_like(host_in, pin_memory=True)
        for _ in range(1):
            s.A.copy_(host_in, non_blocking=True)
            s.step(L)
            host_out.copy_(s.A, non_blocking=True)
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(a.steps):
            s.A.copy_(host_in, non_blocking=True)
            s.step(L)
            host_out.copy_(s.A, non_blocking=True)
        e1.record()
        e1.synchronize()
        barrier()
        dte = max_over_ranks(e0.elapsed_time(e1) / 1e3)
        nbytes = s.A.numel() * s.A.element_size()
        e2e = {"value": replica_mlups(world, nodes, L * a.steps, dte), "unit": "MLUPS",
               "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": nbytes}

    if rank == 0:
        peak, peak_kind = measured_peak()
        bpn = s.bytes_per_node
        achieved = bpn * nodes / (dt / launches) / 1e9
        tag = f"{name}"
        traffic = traffic_from_profiles(tag)
        out = {
            "metric": "MLUPS", "value": value, "unit": "MLUPS", "n_gpus": world,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": 1e3 * dt / a.steps,
            "higher_is_better": True, "scaling": "weak",
            "vs_baseline": (value / PUBLISHED_MLUPS[name]) if name in PUBLISHED_MLUPS else None,
            "dtype": "f32" if s.storage == "f32" else s.storage, "data": "synthetic",
            "config": config_of(name, a),
            "bytes_per_update": bpn, "effective_GBs": value * 1e6 * bpn / 1e9,
            "roofline": {"bound": "hbm", "kernel": dominant_kernel(name),
                         "achieved": achieved, "peak": peak,
                         "unit": "GB/s", "frac": achieved / peak, "peak_kind": peak_kind,
                         "traffic": traffic, "algorithmic_bytes_per_launch": bpn * nodes},
            "gpu_launches": launches,
            "clocks": clocks,
        }
        if e2e is not None:
            out["e2e"] = e2e
        if world == 1 and not a.no_cpu:
            out["cpu_baseline"] = cpu_baseline(name)
        print(json.dumps(out), flush=True)
    if world > 1:
        dist.destroy_process_group()


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__,
                                 formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="d2q9-bgk-ab-f32",
                    choices=sorted(WORKLOADS) + sorted(BATCHES))
    ap.add_argument("--lbm-steps", type=int, default=None,
                    help="lattice time steps per benchmark step (1000; 2000 for batches)")
    ap.add_argument("--n", type=int, default=None, help="override the lattice edge (profiling)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--cpu-procs", type=int, default=64)
    a = ap.parse_args()
    if a.lbm_steps is None:
        a.lbm_steps = default_lbm_steps(a.workload)
    if a.workload in BATCHES and a.n is not None:
        ap.error("--n does not apply to batches")
    if a.warmup < 3 and a.impl == "b200":
        log("note: fewer than 3 warm-up steps")
    if a.impl == "reference":
        run_reference(a)
    else:
        run_b200(a)


if __name__ == "__main__":
    main()
