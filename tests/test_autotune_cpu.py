"""Autotuner selection and cache logic (no GPU)."""

from __future__ import annotations

from pylbm_b200 import autotune as A
from pylbm_b200 import workloads as W
from pylbm_b200.problem import Problem


def test_choose_picks_fastest():
    times = {(64, 2): 3.0, (128, 8): 1.0, (256, 4): 2.0}
    best, table = A.choose(times, lambda c: times[c])
    assert best == (128, 8)
    assert table["128x8"] == 1.0


def test_batch_key_depends_on_lattice_set_and_gpu():
    a = [Problem((64, 32), u_lid=0.1, collision="mrt"), Problem((48, 40), u_lid=0.1, collision="mrt")]
    b = list(reversed(a))
    assert A.batch_key("B200", a, "fused-fp16") != A.batch_key("B200", b, "fused-fp16")
    assert A.batch_key("B200", a, "fused-fp16") != A.batch_key("H100", a, "fused-fp16")
    assert A.batch_key("B200", a, "fused-fp16") == A.batch_key("B200", list(a), "fused-fp16")


def test_cache_round_trip(tmp_path):
    path = tmp_path / "sub" / "tune.json"
    assert A.load_cache(path) == {}
    A.save_cache({"k": {"launch": [128, 8]}}, path)
    assert A.load_cache(path)["k"]["launch"] == [128, 8]


def test_cavity_batch_generator():
    cav = W.cavity_batch(64, seed=0)
    assert len(cav) == 64
    for c in cav:
        nx, ny = c["shape"]
        assert 128 <= nx <= 1024 and 128 <= ny <= 1024 and nx % 8 == 0 and ny % 8 == 0
        assert 0.51 <= c["tau"] <= 1.0 and 0.05 <= c["u_lid"] <= 0.1
    assert cav == W.cavity_batch(64, seed=0)
    probs = W.cavity_batch_problems(4, seed=1)
    assert all(p.collision == "mrt" and p.u_lid > 0 for p in probs)
