"""Launch-shape autotuner for batched lattices, with an on-disk cache.

``autotune_batch`` times every candidate launch shape (threads per block x resident blocks
per SM, which sets how the warp-sized row segments of all lattices are spread over the GPU)
with CUDA events on the batch itself, keeps the fastest, and caches the choice under a key of
(GPU name, lattice set): the shapes, collision and storage of every lattice, order included.
The state is saved before and restored after the trials, so tuning does not advance the
simulation. Cache file: ``$PYLBM_B200_CACHE/autotune.json`` (default
``~/.cache/pylbm_b200``).
"""

from __future__ import annotations

import hashlib
import json
import os
from pathlib import Path
from typing import Any, Callable, Iterable

BLOCKS = (64, 128, 256)
PER_SM = (0, 2, 4, 8, 16, 32)  # resident blocks per SM; 0 = one work item per warp


def cache_path() -> Path:
    root = os.environ.get("PYLBM_B200_CACHE", str(Path.home() / ".cache" / "pylbm_b200"))
    return Path(root) / "autotune.json"


def batch_key(gpu: str, problems: Iterable[Any], variant: str) -> str:
    h = hashlib.sha1()
    for p in problems:
        h.update(repr((tuple(p.shape), p.collision, tuple(p.periodic), bool(p.u_lid))).encode())
    return f"{gpu}|{variant}|{h.hexdigest()[:16]}"


def load_cache(path: Path | None = None) -> dict:
    path = path or cache_path()
    try:
        return json.loads(path.read_text())
    except Exception:
        return {}


def save_cache(cache: dict, path: Path | None = None) -> None:
    path = path or cache_path()
    path.parent.mkdir(parents=True, exist_ok=True)
    tmp = path.with_suffix(f".{os.getpid()}.tmp")
    tmp.write_text(json.dumps(cache, indent=1, sort_keys=True))
    tmp.replace(path)


def choose(candidates: Iterable[tuple[int, int]],
           measure: Callable[[tuple[int, int]], float]) -> tuple[tuple[int, int], dict]:
    """Time every candidate with ``measure`` (seconds per step) and return the fastest."""
    times = {}
    for c in candidates:
        times[c] = measure(c)
    best = min(times, key=times.get)
    return best, {f"{b}x{s}": t for (b, s), t in times.items()}


def autotune_batch(batch: Any, steps: int = 20, reps: int = 2, use_cache: bool = True,
                   path: Path | None = None) -> dict:
    """Pick and apply the fastest launch shape for ``batch`` (a BatchedSolver)."""
    import torch

    gpu = torch.cuda.get_device_name(batch.dev)
    key = batch_key(gpu, batch.problems, batch.variant)
    cache = load_cache(path) if use_cache else {}
    if key in cache:
        block, per_sm = cache[key]["launch"]
        batch.set_launch(block, per_sm)
        return {"key": key, "launch": [block, per_sm], "cached": True}
    saved_a, saved_b, saved_steps = batch.A.clone(), batch.B.clone(), batch.steps_done
    steps += steps % 2  # even step counts leave A and B in place

    def measure(c: tuple[int, int]) -> float:
        batch.set_launch(*c)
        batch.step(2, graph=False)
        best = float("inf")
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            batch.step(steps, graph=False)
            e1.record()
            e1.synchronize()
            best = min(best, e0.elapsed_time(e1) / 1e3 / steps)
        return best

    best, times = choose([(b, s) for b in BLOCKS for s in PER_SM], measure)
    batch.A.copy_(saved_a)
    batch.B.copy_(saved_b)
    batch.steps_done = saved_steps
    batch.set_launch(*best)
    entry = {"launch": list(best), "seconds_per_step": times}
    if use_cache:
        cache = load_cache(path)
        cache[key] = entry
        save_cache(cache, path)
    return {"key": key, "launch": list(best), "cached": False, "times": times}
