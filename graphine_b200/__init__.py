"""graphine_b200: B200-native GRE vertex-centric superstep (PageRank, BFS, SSSP, CC, BC).

The compute lives in libgre_gpu.so (C ABI, include/gre_gpu.h; CUDA sm_100a kernels in csrc/).
This package is its Python mirror; see :mod:`graphine_b200.gre`.
"""
from .gre import *  # noqa: F401,F403
from .gre import Graph, GreError, Stats, lib  # noqa: F401

__all__ = ["Graph", "GreError", "Stats", "lib"]
