"""B200 (sm_100a) K-SVD denoiser: Python helpers around libksvd_sm100.so.

The package directory name contains hyphens, so it is loaded by path (see
``load()`` below, used by tests/, bench.py and __graft_entry__.py) under the
module name ``ksvd_b200``.
"""

from . import ksvd, synth  # noqa: F401

__all__ = ["ksvd", "synth"]
