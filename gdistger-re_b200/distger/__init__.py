"""distger: DistGER's walk + SGNS hot path on B200 (sm_100a) behind a C ABI.

The compute lives in libdistger.so (CUDA, built in-tree by `build()`); this
package is the host-side mirror of the reference's interfaces over that ABI.
"""
from ._lib import DistgerError, build, lib  # noqa: F401
from .walk import Graph, Paths, WalkEngine  # noqa: F401

__all__ = ["DistgerError", "build", "lib", "Graph", "Paths", "WalkEngine"]
