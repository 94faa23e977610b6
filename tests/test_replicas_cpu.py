"""The multi-GPU form of the benchmark is replicas (one independent lattice per rank, no
collective on the data path): its host logic on CPU with world size 2 over gloo. The ranks
meet at barriers, the job time is the slowest rank's, the value aggregates all ranks; under
torchrun the reference arm prints exactly one line, from rank 0, and every rank exits 0."""

from __future__ import annotations

import json
import os
import socket
import subprocess
import sys
from pathlib import Path

import pytest

torch = pytest.importorskip("torch")
ROOT = Path(__file__).resolve().parent.parent


def _port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out: str) -> None:
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, str(ROOT))
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    bench.rank_barrier(world, "cpu")
    t = bench.ranks_max(1.0 + rank, world, "cpu")  # the slowest rank's time
    v = bench.replica_mlups(world, 1000, 10, t)
    bench.rank_barrier(world, "cpu")
    dist.destroy_process_group()
    Path(out + f".{rank}").write_text(json.dumps({"t": t, "v": v}))


def test_max_over_ranks_and_aggregate_with_gloo(tmp_path):
    import torch.multiprocessing as mp

    world, port = 2, _port()
    out = str(tmp_path / "r")
    mp.start_processes(_rank, args=(world, port, out), nprocs=world, join=True,
                       start_method="spawn")
    res = [json.loads(Path(out + f".{r}").read_text()) for r in range(world)]
    assert all(r["t"] == 2.0 for r in res)
    assert all(r["v"] == pytest.approx(2 * 1000 * 10 / 2.0 / 1e6) for r in res)


def test_reference_arm_under_torchrun_prints_once():
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
           "--master-addr", "127.0.0.1", "--master-port", str(_port()), "bench.py",
           "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "0",
           "--cpu-procs", "1"]
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
