"""Host-side checks that need no GPU: the C-ABI library loads and exports
every entry point include/kgraph_b200.h declares; defaults match kgraph.h;
the Python module rejects what the reference rejects."""
import os
import re

import numpy as np
import pytest

from conftest import ROOT


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "kgraph_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(kg_[a-z_0-9]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    from kgraph_b200 import capi
    L = capi.lib()
    names = declared_symbols()
    assert len(names) >= 15
    for n in names:
        assert hasattr(L, n), n
    assert sorted(capi.SYMBOLS) == names


def test_defaults_match_reference_header():
    from kgraph_b200 import capi
    p = capi.IndexParams()
    capi.lib().kg_index_params_default(p)
    assert (p.iterations, p.L, p.K, p.S, p.R, p.controls, p.seed, p.prune, p.reverse) == (30, 100, 25, 10, 100, 100,
                                                                                          1998, 0, 0)
    assert abs(p.delta - 0.002) < 1e-9 and abs(p.recall - 0.99) < 1e-7
    s = capi.SearchParams()
    capi.lib().kg_search_params_default(s)
    assert (s.K, s.M, s.P, s.S, s.T, s.seed, s.init) == (25, 0, 100, 10, 1, 1998, 0)
    assert s.epsilon == np.float32(1e30)
    assert "sm_100a" in capi.version()


def test_python_module_errors_match_reference():
    import kgraph_b200 as kgraph
    X = np.zeros((10, 4), np.float32)
    with pytest.raises(RuntimeError, match="metric not supported"):
        kgraph.KGraph(X, "cosine")
    with pytest.raises(RuntimeError, match="data type not supported"):
        kgraph.KGraph(X.astype(np.float64), "euclidean")
    assert kgraph.arch["name"] == "sm_100a"


def test_python_module_has_the_extensions():
    import kgraph_b200 as kgraph
    for name in ("train_router", "set_search_precision", "autotune", "search", "build", "load", "save"):
        assert hasattr(kgraph.KGraph, name), name
    assert "router" in kgraph.KGraph.search.__doc__


def test_context_creation_fails_cleanly_without_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from kgraph_b200 import capi
    with pytest.raises(capi.KGError):
        capi.Context(0)


def test_parameter_keywords_must_name_fields():
    """A misspelt build or router keyword raises instead of landing on the
    ctypes struct as a plain attribute the library never reads."""
    from kgraph_b200 import capi
    p = capi._set_fields(capi.IndexParams(), dict(K=12, recall=1.0, delta=0.0))
    assert (p.K, p.recall, p.delta) == (12, 1.0, 0.0)
    with pytest.raises(TypeError, match="recal"):
        capi._set_fields(capi.IndexParams(), dict(recal=1.0))
    with pytest.raises(TypeError, match="rand_seed"):
        capi._set_fields(capi.IndexParams(), dict(rand_seed=1))
    r = capi._set_fields(capi.RouterParams(), dict(clusters=64, epochs=2))
    assert (r.clusters, r.epochs) == (64, 2)
    with pytest.raises(TypeError):
        capi._set_fields(capi.RouterParams(), dict(epoch=2))
