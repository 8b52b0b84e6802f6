"""KGraph on NVIDIA B200: NN-descent k-NN graph construction and graph-walk
k-NN search as hand-written sm_100a CUDA kernels behind the reference's API.

``kgraph_b200.KGraph(data, metric)`` is the drop-in for the reference's
Python ``kgraph.KGraph`` (same methods, keyword arguments and defaults);
``import kgraph_b200 as kgraph`` keeps existing scripts working.
``kgraph_b200.capi`` binds the C-ABI directly.

Importing fails if the compiled extension is missing (build it with
``python -m kgraph_b200.build``): there is no CPU fallback.
"""
from ._kgraph import KGraph, arch, git_commit, version  # noqa: F401

__all__ = ["KGraph", "arch", "git_commit", "version"]
