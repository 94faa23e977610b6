"""Throughput benchmark of the fused lattice-Boltzmann step (one JSON line on stdout).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME] [--impl b200|reference]
                    [--no-extras] [--no-e2e] [--no-cpu]

Default workload: D2Q9 BGK, tau = 0.6, 4096 x 4096 fully periodic, fp32 storage (f - w,
shifted arithmetic), pull two-buffer; rho = 1 + 0.01 N(0,1), u = 8 seeded Fourier modes with
max|u| = 0.05. One benchmark step = 1000 lattice time steps of the whole lattice. The state
(2 x 604 MB) is larger than L2, so no flush is needed between steps.

* ``value``    MLUPS with the state resident in HBM, CUDA events on the launching stream,
               max over ranks (replicas: every rank advances its own lattice, no collective
               on the data path).
* ``e2e``      the same through the solver API with host buffers: every step copies the
               stored state host -> device from pinned memory, advances 1000 steps and copies
               the state back. ``e2e_canonical``: the same through pylbm's state exchange,
               ``set_populations`` / ``populations`` with the float64 canonical array.
* ``roofline`` algorithmic bytes (2 q s per node and launch) / average launch time, against
               the measured HBM copy bandwidth (and ``frac_spec`` against the 8 TB/s HBM3e
               figure).
* ``cpu_baseline``  pylbm's own float64 NumPy solver (``baseline/_ref``; the oracle port when
               pylbm is not installed) on a bounded sample of the same workload, one host core.
* ``extra``    (one GPU, default workload) every other configuration measured in the same
               process, each with its own warm-up, CUDA-event timing, roofline and clocks:
               the D2Q9 4096^2 TRT / AA / 16-bit variants, D3Q19 256^3 TRT in fp32 / fp16 /
               bf16 (AB and AA), 64 uneven D2Q9 MRT fp16 cavities in one CUDA-graph launch
               per step against 64 separate fp32 solvers, the adjoint of the 1024 x 256 channel
               against its forward step; the ratios the targets are stated on; and parity
               against pylbm's float64 algorithm (``core.step`` on float64 tensors) on the
               256^2 crop of the same seed (1000 steps) and the 64^3 Taylor-Green vortex
               (500 steps), computed outside the timed regions.

``--impl reference`` times pylbm's NumPy solver instead, on all host cores (one process per
core, each advancing its own 4096-wide periodic band of the workload).
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
    "d2q9-bgk-ab-bf16": ("D2Q9", 4096, "bgk", 0.6, "fused-bf16"),
    "d2q9-bgk-aa-f16": ("D2Q9", 4096, "bgk", 0.6, "fused-aa-fp16"),
    "d2q9-bgk-ab-plain": ("D2Q9", 4096, "bgk", 0.6, "fused-plain"),
    "d3q19-trt-ab-f32": ("D3Q19", 256, "trt", 0.55, "fused"),
    "d3q19-trt-ab-f16": ("D3Q19", 256, "trt", 0.55, "fused-fp16"),
    "d3q19-trt-ab-bf16": ("D3Q19", 256, "trt", 0.55, "fused-bf16"),
    "d3q19-trt-aa-f32": ("D3Q19", 256, "trt", 0.55, "fused-aa"),
    "d3q19-trt-aa-f16": ("D3Q19", 256, "trt", 0.55, "fused-aa-fp16"),
    "d3q19-trt-aa-bf16": ("D3Q19", 256, "trt", 0.55, "fused-aa-bf16"),
    # d'Humieres et al. (2002) MRT (no pylbm counterpart)
    "d3q19-mrt-ab-f32": ("D3Q19", 256, "mrt", 0.55, "fused"),
    "d3q19-mrt-ab-f16": ("D3Q19", 256, "mrt", 0.55, "fused-fp16"),
    "d3q19-mrt-aa-f16": ("D3Q19", 256, "mrt", 0.55, "fused-aa-fp16"),
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

# the configurations measured beside the default workload (``extra`` of the JSON line)
EXTRA_SINGLE = ("d2q9-trt-ab-f32", "d2q9-bgk-aa-f32", "d2q9-trt-aa-f32", "d2q9-bgk-ab-f16",
                "d2q9-bgk-ab-bf16", "d2q9-bgk-aa-f16", "d3q19-trt-ab-f32", "d3q19-trt-ab-f16",
                "d3q19-trt-ab-bf16", "d3q19-trt-aa-f32", "d3q19-trt-aa-f16", "d3q19-mrt-ab-f32",
                "d3q19-mrt-ab-f16", "d3q19-mrt-aa-f16")
EXTRA_WARMUP, EXTRA_STEPS = 3, 3
HBM3E_SPEC_GBS = 8000.0  # B200 HBM3e specification (DGX figure)

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
                else "rows3d::k_aa_odd + k_aa_even")
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


def traffic_from_profiles(kernel_tag: str) -> dict | None:
    """Per-launch DRAM bytes of an ncu capture recorded in profiles/traffic.json."""
    p = ROOT / "profiles" / "traffic.json"
    try:
        e = json.loads(p.read_text())[kernel_tag]
        return {"bytes_per_launch": float(e["bytes_per_launch"]), "source": e.get("source")}
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


def initial_state(name: str, seed: int, n: int | None = None):  # noqa: ANN201
    """The workload's float64 canonical initial state, built on the device."""
    import torch

    from pylbm_b200 import workloads as W

    lat, n0, *_ = WORKLOADS[name]
    n = n or n0
    if is_cavity(name):  # fluid at rest, set in motion by the lid
        return torch.as_tensor(make_problem(name, n).initial_populations(), device="cuda")
    if lat == "D2Q9":
        return W.fourier_populations_device(n, seed)
    return W.taylor_green_3d_populations_device(n)


def load_pylbm():  # noqa: ANN201
    """pylbm itself (the offline install ``baseline/_ref`` or ``PYLBM_SRC``), or None."""
    try:
        from baseline import import_pylbm

        return import_pylbm()
    except ImportError:
        return None


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
def _cpu_stepper(shape: tuple, tau: float, coll: str, periodic: tuple, u_lid: float,
                 f: np.ndarray, use_pylbm: bool):  # noqa: ANN202
    """One float64 CPU step function: pylbm's NumpySolver, or the oracle port of it."""
    if use_pylbm:
        load_pylbm()
        from pylbm.backends.numpy_backend import NumpySolver
        from pylbm.problem import Problem as PProblem

        s = NumpySolver(PProblem(shape, tau=tau, collision=coll, periodic=periodic,
                                 u_lid=u_lid))
        s.set_populations(f)
        return lambda: s.step(1)
    from oracle import lbm_oracle as O

    case = O.Case(shape, tau, coll, periodic, u_lid=u_lid)
    box = [f]

    def one() -> None:
        box[0] = O.step(box[0], case)

    return one


def _cpu_band_worker(args: tuple) -> float:
    """Time ``steps`` float64 CPU steps on one band of the workload (runs in a spawned
    process): a periodic 4096-wide band of the periodic cases, a cavity of the band's size
    for the cavity workloads."""
    name, rows, steps, warmup, seed, barrier, use_pylbm = args
    sys.path.insert(0, str(ROOT))
    from pylbm_b200 import workloads as W
    from pylbm_b200.lattice import D2Q9, D3Q19, equilibrium

    lat, n, coll, tau, _ = WORKLOADS[name]
    if is_cavity(name):
        shape = (n, rows) if lat == "D2Q9" else (n, n, rows)
        lattice = D2Q9 if lat == "D2Q9" else D3Q19
        f = equilibrium(lattice, np.ones(shape[::-1]), np.zeros((len(shape),) + shape[::-1]))
        one = _cpu_stepper(shape, tau, coll, (False,) * len(shape), 0.05, f, use_pylbm)
    elif lat == "D2Q9":
        rho, u = W.fourier_state(n, seed)
        f = equilibrium(D2Q9, rho[:rows], u[:, :rows])
        one = _cpu_stepper((n, rows), tau, coll, (True, True), 0.0, f, use_pylbm)
    else:
        rho, u = W.taylor_green_3d(n)
        f = equilibrium(D3Q19, rho[:rows], u[:, :rows])
        one = _cpu_stepper((n, n, rows), tau, coll, (True, True, True), 0.0, f, use_pylbm)
    for _ in range(warmup):
        one()
    if barrier is not None:
        barrier.wait()
    t0 = time.perf_counter()
    for _ in range(steps):
        one()
    return time.perf_counter() - t0


def _cpu_batch_worker(args: tuple) -> tuple[float, int]:
    """Time ``steps`` float64 CPU steps on lattice ``i`` of a batch (runs in a spawned
    process); returns (seconds, nodes)."""
    name, i, steps, warmup, barrier, use_pylbm = args
    sys.path.insert(0, str(ROOT))
    p = batch_problems(name)[i]
    one = _cpu_stepper(tuple(p.shape), p.tau, p.collision, (False, False), p.u_lid,
                       p.initial_populations(), use_pylbm)
    for _ in range(warmup):
        one()
    if barrier is not None:
        barrier.wait()
    t0 = time.perf_counter()
    for _ in range(steps):
        one()
    return time.perf_counter() - t0, p.n_nodes


def band_nodes(name: str, rows: int) -> int:
    lat, n, *_ = WORKLOADS[name]
    return n * rows if lat == "D2Q9" else n * n * rows


def cpu_kind() -> tuple[bool, str, str]:
    """(use pylbm, cpu_baseline kind, what ran)."""
    if load_pylbm() is not None:
        return True, "reference", "pylbm's NumpySolver (float64, backends/numpy_backend.py)"
    return False, "port", "the float64 NumPy oracle (a port of pylbm's NumpySolver)"


def cpu_baseline(name: str) -> dict:
    """The float64 CPU path on one core, a bounded sample of the workload (about 10 s)."""
    use, kind, what = cpu_kind()
    if name in BATCHES:
        dt, nodes = _cpu_batch_worker((name, 0, 3, 1, None, use))
        return {"value": nodes * 3 / dt / 1e6, "unit": "MLUPS", "cores": 1, "kind": kind,
                "sample": f"{what}, 3 steps of lattice 0 of the batch ({nodes} nodes)"}
    lat = WORKLOADS[name][0]
    rows, steps = (512, 3) if lat == "D2Q9" else (8, 3)
    dt = _cpu_band_worker((name, rows, steps, 1, 0, None, use))
    mlups = band_nodes(name, rows) * steps / dt / 1e6
    return {"value": mlups, "unit": "MLUPS", "cores": 1, "kind": kind,
            "sample": f"{what}, {steps} steps of a band of {band_nodes(name, rows)} nodes "
                      f"of the same workload"}


def run_reference(a: argparse.Namespace) -> None:
    """--impl reference: pylbm's CPU implementation on all host cores."""
    import multiprocessing as mp

    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    name = a.workload
    use, kind, what = cpu_kind()
    cores = min(os.cpu_count() or 1, a.cpu_procs)
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    barrier = mgr.Barrier(cores)
    if name in BATCHES:  # one lattice of the batch per process
        count = BATCHES[name][0]
        with ctx.Pool(cores) as pool:
            res = pool.map(_cpu_batch_worker,
                           [(name, i % count, a.steps, a.warmup, barrier, use)
                            for i in range(cores)])
        dt = max(r[0] for r in res)
        total = sum(r[1] for r in res) * a.steps
        sample = f"{what}, {cores} processes x {a.steps} steps, each on one lattice of the batch"
    else:
        lat = WORKLOADS[name][0]
        rows = 64 if lat == "D2Q9" else 2
        with ctx.Pool(cores) as pool:
            times = pool.map(_cpu_band_worker,
                             [(name, rows, a.steps, a.warmup, 0, barrier, use)] * cores)
        dt = max(times)
        total = cores * band_nodes(name, rows) * a.steps
        sample = (f"{what}, {cores} processes x {a.steps} steps of a band of "
                  f"{band_nodes(name, rows)} nodes each")
    mlups = total / dt / 1e6
    out = {"impl": "reference", "metric": "MLUPS", "value": mlups, "unit": "MLUPS",
           "n_gpus": a.gpus, "steps": a.steps, "warmup": a.warmup,
           "ms_per_step": 1e3 * dt / a.steps, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f64", "data": "synthetic",
           "config": config_of(name, a),
           "cpu_baseline": {"value": mlups, "unit": "MLUPS", "cores": cores, "kind": kind,
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


# ----------------------------------------------------------------------------- timing
def timed(fn, warmup: int, steps: int, gpu: int) -> tuple[float, dict]:  # noqa: ANN001
    """Run ``fn`` (one benchmark step, queued on the current stream) ``warmup`` times, then
    time ``steps`` calls with CUDA events, sampling the clocks meanwhile: (seconds, clocks)."""
    import torch

    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(gpu) as clk:
        e0.record()
        for _ in range(steps):
            fn()
        e1.record()
        e1.synchronize()
    return e0.elapsed_time(e1) / 1e3, clk.summary()


def entry(nodes: int, bpn: float, lbm_steps: int, warmup: int, steps: int, dt: float,
          clocks: dict, peak: float, kernel: str) -> dict:
    """One measured configuration: MLUPS, time per benchmark step, roofline, clocks."""
    updates = nodes * lbm_steps * steps
    achieved = bpn * updates / dt / 1e9
    return {"value": updates / dt / 1e6, "unit": "MLUPS", "ms_per_step": 1e3 * dt / steps,
            "lbm_steps_per_step": lbm_steps, "warmup": warmup, "steps": steps,
            "nodes": nodes, "bytes_per_update": bpn,
            "roofline": {"bound": "hbm", "kernel": kernel, "achieved": achieved,
                         "unit": "GB/s", "frac": achieved / peak,
                         "frac_spec": achieved / HBM3E_SPEC_GBS},
            "clocks": clocks}


def free_cuda() -> None:
    import gc

    import torch

    gc.collect()
    torch.cuda.empty_cache()


# ----------------------------------------------------------------------------- extras
def extra_single(name: str, f0, peak: float, gpu: int) -> dict:  # noqa: ANN001
    from pylbm_b200.backend import VARIANTS

    s = VARIANTS[WORKLOADS[name][4]](make_problem(name))
    s.set_populations(f0)
    L = 1000
    dt, clk = timed(lambda: s.step(L), EXTRA_WARMUP, EXTRA_STEPS, gpu)
    out = entry(s.N, s.bytes_per_node, L, EXTRA_WARMUP, EXTRA_STEPS, dt, clk, peak,
                dominant_kernel(name))
    out["variant"] = WORKLOADS[name][4]
    out["roofline"]["traffic"] = traffic_from_profiles(name)
    del s
    free_cuda()
    return out


def extra_batch(name: str, peak: float, gpu: int) -> dict:
    """Config 4: the batch in one CUDA-graph launch per step, and the same lattices as 64
    separate fp32 solvers (pylbm's way: one solver per lattice, stepped one after another)."""
    from pylbm_b200.autotune import autotune_batch
    from pylbm_b200.backend import B200FusedPlain
    from pylbm_b200.batched import BatchedSolver

    probs = batch_problems(name)
    b = BatchedSolver(probs, BATCHES[name][2])
    tune = autotune_batch(b, use_cache=False)
    L = 2000
    dt, clk = timed(lambda: b.step(L), EXTRA_WARMUP, EXTRA_STEPS, gpu)
    out = entry(b.nodes, b.bytes_per_node, L, EXTRA_WARMUP, EXTRA_STEPS, dt, clk, peak,
                "k_d2q9_batch_ab")
    out.update(lattices=len(probs), launch_shape=tune["launch"], variant=BATCHES[name][2])
    out["roofline"]["traffic"] = traffic_from_profiles(name)
    b.close()
    del b
    free_cuda()
    solvers = [B200FusedPlain(p) for p in probs]
    Ls = 256

    def seq() -> None:
        for s in solvers:
            s.step(Ls)

    dts, clks = timed(seq, EXTRA_WARMUP, EXTRA_STEPS, gpu)
    nodes = sum(s.N for s in solvers)
    seq_e = entry(nodes, 72, Ls, EXTRA_WARMUP, EXTRA_STEPS, dts, clks, peak, "k_d2q9_ab")
    seq_e["how"] = ("64 fused-plain fp32 solvers (pylbm's fp32 arithmetic), each advanced "
                    "by its own step() in turn (CUDA graphs of 64 launches below 2^20 nodes)")
    out["sequential_fp32"] = seq_e
    out["speedup_vs_sequential_fp32"] = out["value"] / seq_e["value"]
    del solvers
    free_cuda()
    return out


def extra_adjoint(peak: float, gpu: int) -> dict:
    """Config 5: D2Q9 BGK channel 1024 x 256 with a disc of diameter 40 at (200, 129), tau
    0.56, g_x = 1e-6 plus a seeded N(0, 1e-7) control field; J = mean x drag over steps
    1500..2000 of T = 2000, checkpoints every 45 steps."""
    import torch

    from pylbm_b200 import workloads as W
    from pylbm_b200.adjoint import DragAdjoint
    from pylbm_b200.problem import Problem

    solid, F = W.cylinder_channel(1024, 256, 200.0, 129.0, 40.0, 1e-7, seed=0)
    p = Problem((1024, 256), tau=0.56, periodic=(True, False), force=(1e-6, 0.0), solid=solid)
    adj = DragAdjoint(p, steps=2000, t0=1500, checkpoint=45)
    Fd = torch.as_tensor(F, dtype=torch.float32, device="cuda")
    adj.solver.set_force_field(Fd)
    L = 2000
    dtf, clkf = timed(lambda: adj.forward_step(L), EXTRA_WARMUP, EXTRA_STEPS, gpu)
    dtr, clkr = timed(lambda: adj.reverse_step(L), EXTRA_WARMUP, EXTRA_STEPS, gpu)
    # algorithmic bytes per node: forward 9+9 populations, force field (8 B); recompute
    # (9+9 populations, force field, rho and u written) + reverse (rho, u, force field, 9+9
    # adjoint populations, FP64 gradient read and written)
    fwd = entry(p.n_nodes, 80, L, EXTRA_WARMUP, EXTRA_STEPS, dtf, clkf, peak, "k_generic (AB)")
    rev = entry(p.n_nodes, 216, L, EXTRA_WARMUP, EXTRA_STEPS, dtr, clkr, peak,
                "k_forward_record + k_adjoint_bgk")
    # the whole gradient: checkpointed forward (J) and the reverse sweep
    J = adj.objective(Fd)
    g = adj.gradient()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    J = adj.objective(Fd)
    g = adj.gradient()
    e1.record()
    e1.synchronize()
    gn = float(g.abs().max().item())
    out = {"forward": fwd, "recompute_plus_reverse": rev,
           "ratio_reverse_over_forward": dtr / dtf,
           "gradient": {"ms": e0.elapsed_time(e1), "J": J, "max_abs_dJdF": gn,
                        "finite": bool(np.isfinite(J) and np.isfinite(gn)),
                        "checkpoints": len(adj._checkpoints)}}
    del adj
    free_cuda()
    return out


def _pylbm_f64(pylbm, problem_kw: dict, f0, steps: int):  # noqa: ANN001, ANN202
    """pylbm's own float64 algorithm (core.step over torch float64 tensors on the device)."""
    import torch
    from pylbm.core import Ops, make_geometry, step
    from pylbm.problem import Problem as PProblem

    p = PProblem(**problem_kw)

    def to(a):  # noqa: ANN001, ANN202
        a = np.asarray(a)
        return torch.as_tensor(a, device=f0.device,
                               dtype=None if a.dtype == bool else torch.float64)

    geo, ops = make_geometry(p, to), Ops(torch)
    f = f0.clone()
    with torch.no_grad():
        for _ in range(steps):
            f = step(f, geo, ops)
    return f, p


def extra_parity() -> dict:
    """Distances to pylbm's float64 algorithm: the 256^2 crop of config 2 after 1000 steps
    (max relative per population) and the 64^3 Taylor-Green vortex of config 3 after 500 steps
    (velocity L-inf / U0 and kinetic-energy decay)."""
    import torch

    from pylbm_b200 import workloads as W
    from pylbm_b200.backend import VARIANTS
    from pylbm_b200.problem import Problem

    pylbm = load_pylbm()
    if pylbm is None:
        return {"unavailable": "pylbm is not installed (baseline/_ref)"}
    from pylbm.core import macroscopic

    out: dict = {"reference": "pylbm core.step on float64 tensors"}
    f0 = W.fourier_populations_device(256, 0)
    crop = {}
    for coll in ("bgk", "trt"):
        kw = dict(shape=(256, 256), tau=0.6, collision=coll, periodic=(True, True))
        ref, _ = _pylbm_f64(pylbm, kw, f0, 1000)
        for variant in ("fused", "fused-aa", "fused-fp16"):
            s = VARIANTS[variant](Problem(**kw))
            s.set_populations(f0)
            s.step(1000)
            got = torch.as_tensor(s.populations(), device="cuda")
            crop[f"{coll}/{variant}"] = {
                "max_rel": float(((got - ref).abs() / ref.abs()).max().item()),
                "max_abs": float((got - ref).abs().max().item())}
    out["c2_crop_256_1000"] = crop
    out["f64_crop_max_rel"] = max(v["max_rel"] for k, v in crop.items() if "fp16" not in k)

    n, u0 = 64, 0.05
    kw = dict(shape=(n, n, n), tau=0.55, collision="trt", periodic=(True, True, True))
    g0 = W.taylor_green_3d_populations_device(n, u0)
    ref, pp = _pylbm_f64(pylbm, kw, g0, 500)
    rho_r, u_r = macroscopic(ref, pp)
    u_r = torch.stack(u_r)

    def energy(rho, u):  # noqa: ANN001, ANN202
        return float((0.5 * rho * (u * u).sum(0)).sum().item())

    rho0, u0_field = macroscopic(g0, pp)
    e0 = energy(rho0, torch.stack(u0_field))
    tgv = {"energy_ratio_f64": energy(rho_r, u_r) / e0}
    for variant in ("fused", "fused-fp16", "fused-bf16", "fused-aa-fp16"):
        s = VARIANTS[variant](Problem(**kw))
        s.set_populations(g0)
        s.step(500)
        rho, u = macroscopic(torch.as_tensor(s.populations(), device="cuda"), pp)
        u = torch.stack(u)
        tgv[variant] = {"u_linf_over_U": float((u - u_r).abs().max().item()) / u0,
                        "energy_ratio": energy(rho, u) / e0}
    out["c3_tgv_64_500"] = tgv
    free_cuda()
    return out


def run_extras(headline: dict, peak: float, gpu: int) -> dict:
    """Every other configuration, measured in this process after the headline."""
    ex: dict = {"protocol": f"each entry: {EXTRA_WARMUP} warm-up + {EXTRA_STEPS} timed "
                            "benchmark steps, CUDA events, state larger than L2 (no flush); "
                            "frac against the measured copy bandwidth, frac_spec against "
                            "8 TB/s"}
    wl: dict = {}
    f0 = {}
    for name in EXTRA_SINGLE:
        lat = WORKLOADS[name][0]
        if lat not in f0:
            f0.clear()
            free_cuda()
            f0[lat] = initial_state(name, seed=0)
        t0 = time.perf_counter()
        wl[name] = extra_single(name, f0[lat], peak, gpu)
        log(f"extra {name}: {wl[name]['value']:.0f} MLUPS "
            f"({wl[name]['roofline']['frac']:.3f}) in {time.perf_counter() - t0:.1f} s")
    f0.clear()
    free_cuda()
    bname = "d2q9-mrt-batch64-f16"
    wl[bname] = extra_batch(bname, peak, gpu)
    log(f"extra {bname}: {wl[bname]['value']:.0f} MLUPS ({wl[bname]['roofline']['frac']:.3f})")
    wl["d2q9-bgk-adjoint-channel"] = extra_adjoint(peak, gpu)
    ex["workloads"] = wl

    v = {k: e["value"] for k, e in wl.items() if "value" in e}
    v["d2q9-bgk-ab-f32"] = headline["value"]
    adj = wl["d2q9-bgk-adjoint-channel"]
    ratios = {
        "d2q9_bgk_ab_f16_over_f32": v["d2q9-bgk-ab-f16"] / v["d2q9-bgk-ab-f32"],
        "d2q9_bgk_aa_f16_over_f32": v["d2q9-bgk-aa-f16"] / v["d2q9-bgk-aa-f32"],
        "d3q19_trt_ab_f16_over_f32": v["d3q19-trt-ab-f16"] / v["d3q19-trt-ab-f32"],
        "d3q19_trt_aa_f16_over_f32": v["d3q19-trt-aa-f16"] / v["d3q19-trt-aa-f32"],
        "batch64_over_sequential_fp32": wl[bname]["speedup_vs_sequential_fp32"],
        "adjoint_over_forward": adj["ratio_reverse_over_forward"],
    }
    ex["ratios"] = ratios
    t0 = time.perf_counter()
    ex["parity"] = extra_parity()
    log(f"parity in {time.perf_counter() - t0:.1f} s")

    c2 = [headline["roofline"]["frac"]] + [wl[k]["roofline"]["frac"] for k in
                                           ("d2q9-trt-ab-f32", "d2q9-bgk-aa-f32",
                                            "d2q9-trt-aa-f32")]
    par = ex["parity"]
    targets = {
        "c2_fp32_min_frac_ge_0.90": {"value": min(c2), "met": min(c2) >= 0.90},
        "c3_fp16_ge_1.8x_fp32": {"value": ratios["d3q19_trt_ab_f16_over_f32"],
                                 "met": ratios["d3q19_trt_ab_f16_over_f32"] >= 1.8},
        "d2q9_fp16_ge_1.8x_fp32": {"value": ratios["d2q9_bgk_ab_f16_over_f32"],
                                   "met": ratios["d2q9_bgk_ab_f16_over_f32"] >= 1.8},
        "c4_batch_frac_ge_0.80": {"value": wl[bname]["roofline"]["frac"],
                                  "met": wl[bname]["roofline"]["frac"] >= 0.80},
        "c5_adjoint_le_3x_forward": {"value": ratios["adjoint_over_forward"],
                                     "met": ratios["adjoint_over_forward"] <= 3.0},
    }
    if "f64_crop_max_rel" in par:
        targets["c2_crop_f64_max_rel_le_1e-5"] = {"value": par["f64_crop_max_rel"],
                                                  "met": par["f64_crop_max_rel"] <= 1e-5}
        fp16 = par["c3_tgv_64_500"]["fused-fp16"]["u_linf_over_U"]
        targets["c3_fp16_velocity_le_1e-2_U"] = {"value": fp16, "met": fp16 <= 1e-2}
    ex["targets"] = targets
    return ex


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
    f0 = None
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
        f0 = initial_state(name, seed=rank, n=a.n)
        s.set_populations(f0)
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
    e2e = e2e_canon = None
    if not a.no_e2e:
        host_in = torch.empty(s.A.numel(), dtype=s.A.dtype, pin_memory=True)
        host_in.copy_(s.A)
        host_out = torch.empty_like(host_in, pin_memory=True)

        def e2e_step() -> None:
            s.A.copy_(host_in, non_blocking=True)
            s.step(L)
            host_out.copy_(s.A, non_blocking=True)

        e2e_step()
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(a.steps):
            e2e_step()
        e1.record()
        e1.synchronize()
        barrier()
        dte = max_over_ranks(e0.elapsed_time(e1) / 1e3)
        nbytes = s.A.numel() * s.A.element_size()
        e2e = {"value": replica_mlups(world, nodes, L * a.steps, dte), "unit": "MLUPS",
               "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": nbytes}
        del host_in, host_out
        if f0 is not None:  # pylbm's state exchange: float64 canonical array both ways
            host_f = f0.cpu().numpy()
            ksteps = min(a.steps, 3)

            def canon_step() -> None:
                s.set_populations(host_f)
                s.step(L)
                s.populations()

            canon_step()
            barrier()
            e0.record()
            for _ in range(ksteps):
                canon_step()
            e1.record()
            e1.synchronize()
            barrier()
            dtc = max_over_ranks(e0.elapsed_time(e1) / 1e3)
            e2e_canon = {"value": replica_mlups(world, nodes, L * ksteps, dtc), "unit": "MLUPS",
                         "steps": ksteps, "h2d_bytes_per_step": host_f.nbytes,
                         "d2h_bytes_per_step": host_f.nbytes,
                         "how": "set_populations(float64 numpy) + step(1000) + populations()"}
            del host_f

    out = None
    if rank == 0:
        peak, peak_kind = measured_peak()
        bpn = s.bytes_per_node
        achieved = bpn * nodes / (dt / launches) / 1e9
        traffic = traffic_from_profiles(name)
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
                         "frac_spec": achieved / HBM3E_SPEC_GBS,
                         "traffic": traffic["bytes_per_launch"] if traffic else None,
                         "traffic_source": traffic["source"] if traffic else None,
                         "algorithmic_bytes_per_launch": bpn * nodes},
            "gpu_launches": launches,
            "clocks": clocks,
        }
        if e2e is not None:
            out["e2e"] = e2e
        if e2e_canon is not None:
            out["e2e_canonical"] = e2e_canon
    del s, f0
    free_cuda()
    if rank == 0:
        if world == 1 and not a.no_extras and name == "d2q9-bgk-ab-f32" and a.n is None:
            t0 = time.perf_counter()
            out["extra"] = run_extras(out, out["roofline"]["peak"], local)
            out["extra"]["seconds"] = time.perf_counter() - t0
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
    ap.add_argument("--no-extras", action="store_true",
                    help="only the selected workload (the other configurations are measured "
                         "by default on one GPU with the default workload)")
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
