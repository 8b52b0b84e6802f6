"""Index file formats and the command-line tools on the GPU.

* KGraph::save in FORMAT_TEXT and FORMAT_NO_DIST equals, byte for byte, what
  the reference's own saver writes for the same graph (kgraph.cpp:333-373;
  fixtures from tests/golden/make_formats.py); a FORMAT_NO_DIST file the
  reference wrote loads, saves back identically, searches with the
  reference's results, and refuses what needs distances (get_nn with
  distances, reverse), as the reference does.
* The index / search tools (the reference's index.cpp / search.cpp) build an
  index from an LSHKIT file and search it; the reference's own C++ search on
  the index the tool wrote returns the same ids as the tool.
"""
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN, ROOT, load_golden
from oracle import kgoracle as ko

pytestmark = pytest.mark.gpu


def test_index_formats_match_reference_files(tmp_path):
    g = load_golden("u16")
    f = np.load(os.path.join(GOLDEN, "formats_u16.npz"))
    exe = str(tmp_path / "formats_demo")
    lib = os.path.join(ROOT, "kgraph_b200")
    subprocess.check_call(["g++", "-std=c++17", "-O2", "-I" + os.path.join(ROOT, "include"),
                           os.path.join(ROOT, "tests", "cpp", "formats_demo.cpp"), "-o", exe,
                           "-L" + lib, "-lkgraph_b200", "-Wl,-rpath," + lib])
    (tmp_path / "in.idx").write_bytes(g["index_bytes"].tobytes())
    (tmp_path / "ref_nodist.idx").write_bytes(f["nodist_bytes"].tobytes())
    g["X"].astype(np.float32).tofile(tmp_path / "X.f32")
    g["Q"].astype(np.float32).tofile(tmp_path / "Q.f32")
    s0 = g["searches"][0]
    K, P = s0["K"], s0["P"]
    n, d = g["X"].shape
    args = [exe, tmp_path / "in.idx", tmp_path / "out.txt", tmp_path / "out_nodist.idx", tmp_path / "ref_nodist.idx",
            tmp_path / "resaved_nodist.idx", tmp_path / "X.f32", n, d, tmp_path / "Q.f32", len(g["Q"]), K, P,
            tmp_path / "ids.u32"]
    r = subprocess.run([str(a) for a in args], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert (tmp_path / "out.txt").read_bytes() == f["text_bytes"].tobytes()
    assert (tmp_path / "out_nodist.idx").read_bytes() == f["nodist_bytes"].tobytes()
    assert (tmp_path / "resaved_nodist.idx").read_bytes() == f["nodist_bytes"].tobytes()
    ids = np.fromfile(tmp_path / "ids.u32", np.uint32).reshape(len(g["Q"]), K)
    assert (ids == g["s0_ids"]).all()
    assert "refuses_dists=1" in r.stdout and "refuses_reverse=1" in r.stdout


def _lshkit(path, a):
    a = np.ascontiguousarray(a)
    path.write_bytes(np.array([4, a.shape[0], a.shape[1]], np.uint32).tobytes() + a.tobytes())


def _read_lshkit_u32(path):
    raw = path.read_bytes()
    es, r, c = np.frombuffer(raw, np.uint32, 3)
    assert es == 4
    return np.frombuffer(raw, np.uint32, offset=12).reshape(r, c)


def test_cli_index_and_search_match_reference_search(tmp_path):
    binp = os.path.join(ROOT, "kgraph_b200", "bin")
    rng = np.random.default_rng(17)
    X = rng.random((6000, 24), dtype=np.float32)
    Q = rng.random((200, 24), dtype=np.float32)
    _lshkit(tmp_path / "data", X)
    _lshkit(tmp_path / "query", Q)
    r = subprocess.run([os.path.join(binp, "index"), str(tmp_path / "data"), str(tmp_path / "g.idx"), "-K", "10",
                        "-L", "30", "-S", "8", "--reverse", "-1"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    # exact neighbours by the tool's own --linear mode, used as the gold standard
    r = subprocess.run([os.path.join(binp, "search"), str(tmp_path / "data"), str(tmp_path / "g.idx"),
                        str(tmp_path / "query"), str(tmp_path / "gs"), "-K", "10", "--linear"],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    gs = _read_lshkit_u32(tmp_path / "gs")
    ref = ko.RefLib()
    bf_ids, _, _, _ = ref.search_l2sqr(X, str(tmp_path / "g.idx"), Q, K=10, P=6000)   # P >= N: brute force
    assert (gs == bf_ids).all()
    r = subprocess.run([os.path.join(binp, "search"), str(tmp_path / "data"), str(tmp_path / "g.idx"),
                        str(tmp_path / "query"), str(tmp_path / "res"), "-K", "10", "-P", "30",
                        "--eval", str(tmp_path / "gs")], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    m = re.search(r"Time: (\S+) Recall: (\S+) Cost: (\S+)", r.stdout)
    assert m and float(m.group(2)) > 0.9 and 0 < float(m.group(3)) < 1, r.stdout
    res = _read_lshkit_u32(tmp_path / "res")
    ref_ids, _, _, ref_cost = ref.search_l2sqr(X, str(tmp_path / "g.idx"), Q, K=10, P=30)
    assert (res == ref_ids).all()                                     # the reference's walk on the tool's index
    assert abs(float(m.group(3)) - float(ref_cost.mean())) < 1e-5


@pytest.mark.parametrize("level", [1, 2])
def test_cli_resave_and_prune_tools(tmp_path, level):
    """The reference's resave and prune tools (resave.cpp, prune.cpp): resave
    --no-dist writes the reference's no-dist bytes; --prune and the prune tool
    prune exactly as the reference's prune (the pinned oracle restatement);
    the prune tool's default level is the reference's PRUNE_LEVEL_1 &
    PRUNE_LEVEL_2 = 0, a plain re-save."""
    binp = os.path.join(ROOT, "kgraph_b200", "bin")
    g = load_golden("u16")
    f = np.load(os.path.join(GOLDEN, "formats_u16.npz"))
    src = tmp_path / "in.idx"
    src.write_bytes(g["index_bytes"].tobytes())
    r = subprocess.run([os.path.join(binp, "resave"), str(src), str(tmp_path / "nd.idx"), "--no-dist"],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert (tmp_path / "nd.idx").read_bytes() == f["nodist_bytes"].tobytes()
    G = ko.read_index(g["index_bytes"])
    R = ko.Oracle(g["X"], g["metric"]).prune(G, level)
    r = subprocess.run([os.path.join(binp, "resave"), str(src), str(tmp_path / "pr.idx"), "--prune", str(level)],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    P = ko.read_index(str(tmp_path / "pr.idx"))
    assert (P.offsets == R.offsets).all() and (P.ids == R.ids).all() and (P.M == R.M).all()
    assert (P.dists.view(np.uint32) == R.dists.view(np.uint32)).all()
    _lshkit(tmp_path / "data", g["X"].astype(np.float32))
    r = subprocess.run([os.path.join(binp, "prune"), str(tmp_path / "data"), str(src), str(tmp_path / "p2.idx"),
                        "--prune", str(level)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    P2 = ko.read_index(str(tmp_path / "p2.idx"))
    assert (P2.offsets == R.offsets).all() and (P2.ids == R.ids).all() and (P2.M == R.M).all()
    r = subprocess.run([os.path.join(binp, "prune"), str(tmp_path / "data"), str(src), str(tmp_path / "p0.idx")],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    P0 = ko.read_index(str(tmp_path / "p0.idx"))
    assert (P0.offsets == G.offsets).all() and (P0.ids == G.ids).all() and (P0.M == G.M).all()
