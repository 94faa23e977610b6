"""Install the unmodified pylbm package into ``baseline/_ref`` (git-ignored; it travels to GPU
machines with the working tree, where the reference tree itself is absent).

    python baseline/install_ref.py [--src DIR] [--force]

``--src`` (or ``PYLBM_REF``) is the pylbm project directory; the default is the read-only
reference checkout at /root/reference. pylbm declares hatchling as its build backend and this
image has no hatchling, so the project is copied to a temporary directory, the copy's
``[build-system]`` table is switched to setuptools (the package sources are untouched) and
pip installs it offline with ``--target baseline/_ref``. The installed ``pylbm`` package is
then compared file by file with the project's ``src/pylbm``; any difference is an error.

Users of the installed copy: ``bench.py --impl reference`` (pylbm's NumPy solver), the
drop-in tests through pylbm's registry, CLI and benchmark engine, and ``oracle/build_ref.py``
(pylbm's CUDA C kernel as a comparator).
"""

from __future__ import annotations

import argparse
import filecmp
import os
import shutil
import subprocess
import sys
import tempfile
from pathlib import Path

HERE = Path(__file__).resolve().parent
TARGET = HERE / "_ref"
DEFAULT_SRC = Path("/root/reference")

_SETUPTOOLS_BACKEND = """[build-system]
requires = ["setuptools"]
build-backend = "setuptools.build_meta"

[tool.setuptools.packages.find]
where = ["src"]

[tool.setuptools.package-data]
"*" = ["*.cu", "*.json", "data/*"]
"""


def installed() -> bool:
    return (TARGET / "pylbm" / "__init__.py").exists()


def _rewrite_pyproject(text: str) -> str:
    """pylbm's pyproject.toml with its hatchling tables replaced by setuptools ones."""
    out, skip = [], False
    for line in text.splitlines():
        if line.startswith("["):
            skip = line.strip() in ("[build-system]", "[tool.hatch.build.targets.wheel]")
        if not skip:
            out.append(line)
    return _SETUPTOOLS_BACKEND + "\n" + "\n".join(out) + "\n"


def _same_tree(a: Path, b: Path) -> list[str]:
    """Relative paths that differ between two package trees (bytecode caches ignored)."""
    bad = []
    cmp = filecmp.dircmp(a, b, ignore=["__pycache__"])
    stack = [(cmp, Path("."))]
    while stack:
        c, rel = stack.pop()
        bad += [str(rel / n) for n in c.left_only + c.right_only]
        _, mismatch, errors = filecmp.cmpfiles(c.left, c.right, c.common_files, shallow=False)
        bad += [str(rel / n) for n in mismatch + errors]
        stack += [(sub, rel / name) for name, sub in c.subdirs.items()]
    return bad


def install(src: Path | None = None, force: bool = False) -> Path:
    src = Path(src or os.environ.get("PYLBM_REF") or DEFAULT_SRC)
    if installed() and not force:
        return TARGET
    if not (src / "src" / "pylbm" / "__init__.py").exists():
        raise FileNotFoundError(f"no pylbm project at {src}")
    with tempfile.TemporaryDirectory() as tmp:
        proj = Path(tmp) / "pylbm"
        shutil.copytree(src, proj, ignore=shutil.ignore_patterns("__pycache__", ".git"))
        pp = proj / "pyproject.toml"
        pp.write_text(_rewrite_pyproject(pp.read_text()))
        if TARGET.exists():
            shutil.rmtree(TARGET)
        cmd = [sys.executable, "-m", "pip", "install", "--no-index", "--no-build-isolation",
               "--no-deps", "--find-links", "/opt/wheelhouse", "--target", str(TARGET),
               str(proj)]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"pip install of pylbm failed:\n{r.stdout}\n{r.stderr}")
    bad = _same_tree(src / "src" / "pylbm", TARGET / "pylbm")
    if bad:
        raise RuntimeError(f"installed pylbm differs from its sources: {bad[:10]}")
    return TARGET


if __name__ == "__main__":
    ap = argparse.ArgumentParser(description=__doc__,
                                 formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--src", type=Path, default=None)
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    print(install(a.src, a.force))
