"""Build pylbm's own CUDA C kernel as GPU parity comparators -- test infrastructure only.

    python oracle/build_ref.py        (also run by __graft_entry__.build())

For each configuration below this writes a header of #defines (the role of pylbm's
kernel_source(), cupy_backend.py:51-70, generated here from this repository's lattice tables)
into ``oracle/_ref/`` and compiles ``oracle/ref_launch.cu`` -- which #includes pylbm's
``backends/cuda/lbm.cu`` where pylbm is installed (``PYLBM_SRC`` or ``baseline/_ref``),
unmodified and uncopied -- into ``oracle/_ref/lbmref_<name>.so`` for sm_100a. Nothing is built
when pylbm is absent (the GPU box uses the prebuilt files, which travel with the working tree
but are not committed).
"""

from __future__ import annotations

import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "_ref"
sys.path.insert(0, str(HERE.parent))
from baseline import pylbm_path  # noqa: E402
from oracle.lbm_oracle import D2Q9, D3Q19, MRT_M, MRT_NORM  # noqa: E402

# pylbm's kernel source, from PYLBM_SRC or the offline install baseline/_ref
_PYLBM = pylbm_path()
REF_CU = (_PYLBM / "pylbm" / "backends" / "cuda" / "lbm.cu") if _PYLBM else Path("/nonexistent")

# name: (lattice, periodic, lid, force, collision, storage, pattern)
CONFIGS = {
    "cavity_bgk_f32_ab": ("D2Q9", (0, 0), 1, 0, "bgk", "f32", "ab"),
    "cavity_mrt_f32_ab": ("D2Q9", (0, 0), 1, 0, "mrt", "f32", "ab"),
    "cavity_bgk_f16_ab": ("D2Q9", (0, 0), 1, 0, "bgk", "f16", "ab"),
    "periodic_bgk_f32_ab": ("D2Q9", (1, 1), 0, 0, "bgk", "f32", "ab"),
    "periodic_trt_f32_ab": ("D2Q9", (1, 1), 0, 0, "trt", "f32", "ab"),
    "periodic_trt_f32_aaodd": ("D2Q9", (1, 1), 0, 0, "trt", "f32", "aa-odd"),
    "periodic_trt_f32_aaeven": ("D2Q9", (1, 1), 0, 0, "trt", "f32", "aa-even"),
    "periodic_bgk_f16_ab": ("D2Q9", (1, 1), 0, 0, "bgk", "f16", "ab"),
    "periodic_bgk_bf16_ab": ("D2Q9", (1, 1), 0, 0, "bgk", "bf16", "ab"),
    "channel_trt_f32_ab_force": ("D2Q9", (1, 0), 0, 1, "trt", "f32", "ab"),
    "periodic3d_trt_f32_ab": ("D3Q19", (1, 1, 1), 0, 0, "trt", "f32", "ab"),
    "periodic3d_trt_f16_ab": ("D3Q19", (1, 1, 1), 0, 0, "trt", "f16", "ab"),
    "cavity3d_bgk_f32_ab": ("D3Q19", (0, 0, 0), 1, 0, "bgk", "f32", "ab"),
}
BLOCK_X = 128


def _arr(vals, fmt: str = "{}") -> str:
    return "{" + ", ".join(fmt.format(v) for v in vals) + "}"


def header(cfg: tuple) -> str:
    lat_name, per, lid, force, coll, storage, pattern = cfg
    lat = D2Q9 if lat_name == "D2Q9" else D3Q19
    c = [list(ci) + [0] * (3 - lat.d) for ci in lat.c]
    per3 = tuple(per) + (1,) * (3 - lat.d)
    defs = {
        "Q": lat.q, "D": lat.d, "BLOCK_X": BLOCK_X,
        "CX_INIT": _arr([v[0] for v in c]), "CY_INIT": _arr([v[1] for v in c]),
        "CZ_INIT": _arr([v[2] for v in c]), "W_INIT": _arr(lat.w, "{!r}f"),
        "OPP_INIT": _arr(lat.opp), "PER_X": per3[0], "PER_Y": per3[1], "PER_Z": per3[2],
        "LID": lid, "FORCE": force, "COLL": {"bgk": 0, "trt": 1, "mrt": 2}[coll],
        "STORAGE": {"f32": 0, "f16": 1, "bf16": 2}[storage],
        "PATTERN": {"ab": 0, "aa-odd": 1, "aa-even": 2}[pattern],
    }
    if coll == "mrt":
        defs["M_INIT"] = "{" + ", ".join(_arr([float(v) for v in r], "{!r}f") for r in MRT_M) + "}"
        defs["NORM_INIT"] = _arr(MRT_NORM, "{!r}f")
    return "\n".join(f"#define {k} {v}" for k, v in defs.items()) + "\n"


def build(force: bool = False) -> list[Path]:
    if not REF_CU.exists():
        return []
    OUT.mkdir(exist_ok=True)
    nvcc = "/usr/local/cuda/bin/nvcc" if Path("/usr/local/cuda/bin/nvcc").exists() else "nvcc"
    built = []
    procs = []
    for name, cfg in CONFIGS.items():
        hdr = OUT / f"cfg_{name}.h"
        so = OUT / f"lbmref_{name}.so"
        text = header(cfg)
        if not force and so.exists() and hdr.exists() and hdr.read_text() == text and \
                so.stat().st_mtime >= max(REF_CU.stat().st_mtime,
                                          (HERE / "ref_launch.cu").stat().st_mtime):
            built.append(so)
            continue
        hdr.write_text(text)
        cmd = [nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++14",
               "-shared", "-Xcompiler", "-fPIC", "-include", str(hdr),
               f'-DLBM_REF_CU="{REF_CU}"', str(HERE / "ref_launch.cu"), "-o", str(so)]
        procs.append((so, subprocess.Popen(cmd, stdout=subprocess.PIPE,
                                           stderr=subprocess.STDOUT, text=True)))
    for so, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            raise RuntimeError(f"building {so.name} failed:\n{out}")
        built.append(so)
    return built


if __name__ == "__main__":
    for p in build(force="--force" in sys.argv):
        print(p)
