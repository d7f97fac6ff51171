"""Loads the package in ``cuda-k-svd-denoising_b200/`` as module ``ksvd_b200``.

The directory name is not a Python identifier, so it is imported by path.
"""

from __future__ import annotations

import importlib.util
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent
PKG_DIR = ROOT / "cuda-k-svd-denoising_b200"


def load():
    if "ksvd_b200" in sys.modules:
        return sys.modules["ksvd_b200"]
    spec = importlib.util.spec_from_file_location("ksvd_b200", PKG_DIR / "__init__.py",
                                                  submodule_search_locations=[str(PKG_DIR)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["ksvd_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def load_oracle():
    """The CPU oracle (test infrastructure)."""
    if str(ROOT / "oracle") not in sys.path:
        sys.path.insert(0, str(ROOT / "oracle"))
    import oracle  # noqa: E402
    return oracle
