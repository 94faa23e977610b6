"""Loading of the committed golden fixtures (tests/golden/*.npz) as oracle cases."""

from __future__ import annotations

import json
from pathlib import Path

import numpy as np

from oracle.lbm_oracle import D2Q9, D3Q19, Case

GOLDEN = Path(__file__).resolve().parent / "golden"


def load(name: str) -> dict:
    with np.load(GOLDEN / f"{name}.npz", allow_pickle=False) as z:
        d = {k: z[k] for k in z.files}
    d["params"] = json.loads(str(d["params"]))
    return d


def case_of(d: dict) -> Case:
    p = d["params"]
    return Case(tuple(p["shape"]), p["tau"], p["collision"], tuple(p["periodic"]), p["u_lid"],
                tuple(p["force"]), p["magic"], p["s_e"], p["s_eps"], d.get("solid"),
                inlet=d.get("inlet"), outlet=bool(d.get("outlet", False)))


def rest_state(case: Case) -> np.ndarray:
    lat = D2Q9 if case.dim == 2 else D3Q19
    w = np.array(lat.w).reshape((-1,) + (1,) * case.dim)
    return np.broadcast_to(w, (lat.q,) + case.array_shape).copy()


def initial(d: dict, case: Case) -> np.ndarray:
    return d["f0"] if "f0" in d else rest_state(case)


def names(prefix: str) -> list[str]:
    return sorted(p.stem for p in GOLDEN.glob(f"{prefix}*.npz"))
