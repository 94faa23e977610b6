"""The #define headers used to build pylbm's own kernel as a comparator equal the header that
pylbm's kernel_source() (cupy_backend.py:51-70) prints for the same problem. Needs pylbm
(``baseline/_ref`` or ``PYLBM_SRC``; skipped without it)."""

from __future__ import annotations

import re

import pytest

from oracle import build_ref

pytestmark = pytest.mark.skipif(not build_ref.REF_CU.exists(), reason="pylbm not installed")


def _defines(text: str) -> dict:
    """The leading block of #define lines (the configuration header, not the kernel body)."""
    head = []
    for line in text.splitlines():
        if not line.startswith("#define "):
            break
        head.append(line)
    return dict(re.findall(r"^#define (\w+) (.*)$", "\n".join(head), re.M))


@pytest.mark.parametrize("name", list(build_ref.CONFIGS))
def test_header_matches_pylbm_kernel_source(name):
    from baseline import import_pylbm

    import_pylbm()
    from pylbm.backends.cupy_backend import kernel_source
    from pylbm.problem import Problem

    lat, per, lid, force, coll, storage, pattern = build_ref.CONFIGS[name]
    d = 2 if lat == "D2Q9" else 3
    p = Problem((8,) * d, collision=coll, periodic=tuple(bool(v) for v in per),
                u_lid=0.1 if lid else 0.0, force=(1e-5,) + (0.0,) * (d - 1) if force else None)
    theirs = _defines(kernel_source(p, storage, pattern, build_ref.BLOCK_X))
    mine = _defines(build_ref.header(build_ref.CONFIGS[name]))
    assert mine == theirs
