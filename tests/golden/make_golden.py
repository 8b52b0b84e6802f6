"""Generates the golden fixtures in tests/golden/ from the REFERENCE itself.

The reference (aaalgo/kgraph) is compiled from its own sources by
oracle/Makefile into oracle/_ref/v4 (its Python module, python-api.cpp, and
the C++ MatrixOracle driver).  This script runs it -- builds on ONE OpenMP
thread so the graph is deterministic -- and stores inputs and outputs:

  <case>.npz: X (data), Q (queries), metric, build params, the reference's
  graph as the raw bytes of its saved index file, and for each
  search configuration the reference's ids / dists (and counts / costs where
  the C++ driver reports them), plus the brute-force K-NN.

Run where the reference's sources and oracle/_ref are present:
    python tests/golden/make_golden.py [case ...]     (no case: all of them)
The fixtures are committed; the tests never run the reference themselves on
the GPU box.
"""
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import kgoracle as ko  # noqa: E402


def mixture(rng, n, d, centres, spread, lo=0.0, hi=128.0, integer=True):
    c = rng.uniform(lo, hi, (centres, d))
    lab = rng.integers(0, centres, n)
    x = c[lab] + rng.normal(0, spread, (n, d))
    if integer:
        x = np.round(np.maximum(x, 0))
    return x.astype(np.float32)


CASES = {
    # uniform data, python euclidean oracle, reverse=-1
    "u16": dict(n=2000, d=16, nq=64, metric="euclidean", kind="uniform", seed=11,
                build=dict(K=10, L=30, S=8, reverse=-1),
                searches=[dict(K=10, P=20), dict(K=10, P=50, S=4), dict(K=5, P=30, T=3), dict(K=10, P=40, M=20)]),
    # integer-valued mixture: many exact distance ties
    "mix32": dict(n=2000, d=32, nq=64, metric="euclidean", kind="mixture", seed=12,
                  build=dict(K=10, L=40, S=10, reverse=-1),
                  searches=[dict(K=10, P=30), dict(K=10, P=100), dict(K=20, P=60, T=2)]),
    # angular, no reverse: per-node M < L, so SearchParams.M matters
    "ang20": dict(n=1500, d=20, nq=64, metric="angular", kind="normal", seed=13,
                  build=dict(K=8, L=24, S=6, reverse=0),
                  searches=[dict(K=8, P=20), dict(K=8, P=20, M=20), dict(K=8, P=40, T=2), dict(K=8, P=16, S=3)]),
    # wide rows (d = 300, not a multiple of 16: 12 tail terms): wider than the
    # tensor-core brute force takes, integer-valued with exact ties
    "mix300": dict(n=1000, d=300, nq=48, metric="euclidean", kind="mixture", seed=15,
                   build=dict(K=10, L=30, S=8, reverse=-1),
                   searches=[dict(K=10, P=30), dict(K=10, P=80, S=5), dict(K=5, P=40, T=2)]),
}
# C++ MatrixOracle<l2sqr> through the reference's C++ API (search cost, epsilon, init)
L2CASE = dict(name="l2sq24", n=1500, d=24, nq=64, seed=14, build=dict(K=10, L=30, S=8, reverse=-1),
              searches=[dict(K=10, P=30), dict(K=10, P=30, epsilon=None), dict(K=10, P=30, init=5),
                        dict(K=10, P=20, T=2)])


def make_data(spec):
    rng = np.random.default_rng(spec["seed"])
    n, d, nq = spec["n"], spec["d"], spec["nq"]
    kind = spec.get("kind", "uniform")
    if kind == "uniform":
        X = rng.random((n + nq, d), dtype=np.float32)
    elif kind == "mixture":
        X = mixture(rng, n + nq, d, 16, 20.0)
    else:
        X = rng.standard_normal((n + nq, d)).astype(np.float32)
    return X[:n].copy(), X[n:].copy()


WORKER = r"""
import sys, json, numpy as np
sys.path.insert(0, %(root)r)
from oracle import kgoracle as ko
kg = ko.load_reference_module('v4')
a = json.load(open(sys.argv[1]))
X = np.load(a['X']); Q = np.load(a['Q'])
g = kg.KGraph(X, a['metric'])
g.build(**a['build'])
g.save(a['index'])
g2 = kg.KGraph(X, a['metric'])
g2.load(a['index'])
out = {}
for i, s in enumerate(a['searches']):
    ids, d = g2.search(Q, withDistance=True, **s)
    out['s%%d_ids' %% i] = ids; out['s%%d_dists' %% i] = d
g3 = kg.KGraph(X, a['metric'])
ids, d = g3.search(Q, K=a['bfK'], withDistance=True)
out['bf_ids'] = ids; out['bf_dists'] = d
np.savez(a['out'], **out)
"""


def run_case(name, spec, tmp):
    X, Q = make_data(spec)
    xp, qp = os.path.join(tmp, name + "_X.npy"), os.path.join(tmp, name + "_Q.npy")
    np.save(xp, X)
    np.save(qp, Q)
    idx = os.path.join(tmp, name + ".idx")
    outp = os.path.join(tmp, name + "_out.npz")
    args = dict(X=xp, Q=qp, metric=spec["metric"], build=spec["build"], index=idx, searches=spec["searches"],
                bfK=10, out=outp)
    ap = os.path.join(tmp, name + ".json")
    json.dump(args, open(ap, "w"))
    wp = os.path.join(tmp, "worker.py")
    open(wp, "w").write(WORKER % dict(root=ROOT))
    env = dict(os.environ, OMP_NUM_THREADS="1")
    r = subprocess.run([sys.executable, wp, ap], env=env, capture_output=True, text=True)
    if r.returncode:
        raise RuntimeError(r.stderr)
    log = [l for l in r.stderr.splitlines() if l.startswith("iteration")]
    res = dict(np.load(outp))
    G = ko.read_index(idx)
    fx = dict(X=X, Q=Q, metric=np.array(spec["metric"]), build=np.array(json.dumps(spec["build"])),
              searches=np.array(json.dumps(spec["searches"])), index_bytes=np.frombuffer(open(idx, "rb").read(), np.uint8),
              build_log=np.array("\n".join(log)), **res)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **fx)
    print(name, "E", len(G.ids), "log", log[-1] if log else "")


def run_l2(spec, tmp):
    X, Q = make_data(spec)
    ref = ko.RefLib("v4")
    ref.set_verbosity(0)
    ref.set_threads(1)
    idx = os.path.join(tmp, spec["name"] + ".idx")
    info = ref.build_l2sqr(X, idx, **spec["build"])
    G = ko.read_index(idx)
    out = {}
    rng = np.random.default_rng(spec["seed"] + 100)
    eps_used = []
    for i, s in enumerate(spec["searches"]):
        s = dict(s)
        init_ids = None
        if s.get("epsilon", 1) is None:
            # an epsilon that cuts some result lists short
            ids0, d0, _, _ = ref.search_l2sqr(X, idx, Q, K=10, P=30)
            s["epsilon"] = float(np.median(d0[:, 5]))
        if s.get("init"):
            init_ids = rng.integers(0, spec["n"], (spec["nq"], s["init"])).astype(np.uint32)
            out["s%d_init" % i] = init_ids
        ids, d, cnt, cost = ref.search_l2sqr(X, idx, Q, init_ids=init_ids, **s)
        out["s%d_ids" % i], out["s%d_dists" % i], out["s%d_counts" % i], out["s%d_costs" % i] = ids, d, cnt, cost
        eps_used.append(s)
    ids, d, cnt, cost = ref.search_l2sqr(X, idx, Q, K=10, P=spec["n"])   # P >= N: brute force
    out["bf_ids"], out["bf_dists"] = ids, d
    fx = dict(X=X, Q=Q, metric=np.array("l2sqr"), build=np.array(json.dumps(spec["build"])),
              searches=np.array(json.dumps(eps_used)), index_bytes=np.frombuffer(open(idx, "rb").read(), np.uint8), build_info=info, **out)
    np.savez_compressed(os.path.join(HERE, spec["name"] + ".npz"), **fx)
    print(spec["name"], "E", len(G.ids), "info", info)


def main(names):
    if not ko.reference_available("v4"):
        raise SystemExit("oracle/_ref/v4 is not built (make -C oracle ref)")
    known = list(CASES) + [L2CASE["name"]]
    for n in names:
        if n not in known:
            raise SystemExit("unknown case %r (cases: %s)" % (n, ", ".join(known)))
    with tempfile.TemporaryDirectory() as tmp:
        for name, spec in CASES.items():
            if not names or name in names:
                run_case(name, spec, tmp)
        if not names or L2CASE["name"] in names:
            run_l2(L2CASE, tmp)


if __name__ == "__main__":
    main(sys.argv[1:])
