"""Where the unmodified pylbm package is found: ``PYLBM_SRC`` (a directory holding the
``pylbm`` package, e.g. a checkout's ``src``) or the offline install ``baseline/_ref`` made by
``baseline/install_ref.py``. Used by the reference arm of ``bench.py``, the drop-in tests and
the oracle's fixture and comparator builders; the product package never imports pylbm from
here.
"""

from __future__ import annotations

import os
import sys
from pathlib import Path

INSTALLED = Path(__file__).resolve().parent / "_ref"


def pylbm_path() -> Path | None:
    """The directory to put on ``sys.path`` for ``import pylbm``, or None when absent."""
    env = os.environ.get("PYLBM_SRC")
    for d in ([Path(env)] if env else []) + [INSTALLED]:
        if (d / "pylbm" / "__init__.py").exists():
            return d
    return None


def import_pylbm():  # noqa: ANN201
    """Import pylbm from :func:`pylbm_path` (no bytecode written next to it); raises
    ImportError when it is not installed."""
    d = pylbm_path()
    if d is None:
        raise ImportError("pylbm not found: set PYLBM_SRC or run baseline/install_ref.py")
    if str(d) not in sys.path:
        sys.path.insert(0, str(d))
    prev = sys.dont_write_bytecode
    sys.dont_write_bytecode = True
    try:
        import pylbm
    finally:
        sys.dont_write_bytecode = prev
    return pylbm
