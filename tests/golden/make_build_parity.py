"""Generates tests/golden/build_parity_mix128.json from the REFERENCE itself.

Build parity at the benchmark's graph parameters (K=50, L=100, S=12, R=100,
reverse=-1, 30 iterations) on a mid-size version of the benchmark's data:
100,000 x 128 float32 non-negative integers from a 64-centre Gaussian mixture
(centre coordinates uniform in [0, 128), per-dimension std 20, clipped at 0 and
rounded), euclidean, 1,000 queries from the same mixture.

The reference (compiled from its own sources into oracle/_ref by
oracle/Makefile) builds the graph through its Python module (python-api.cpp,
all host threads) three times; the build is nondeterministic under OpenMP, so
all three results are kept.  Per build:

  graph_recall10   mean over a fixed sample of 2,000 nodes of
                   #(first 10 entries of the node's list, by stored distance,
                   whose exact squared L2 distance is <= the node's exact
                   10th-nearest distance, self excluded) / 10;
  search_recall10  recall@10 of the reference's search (K=10, P in P_LIST,
                   its fixed seeds) over the 1,000 queries, ties counted.

Exact distances are computed in FP64, which is exact on integer data, so the
ground truth does not depend on any FP32 summation order.  The GPU test regenerates
the same data from the same seeds and compares its graph's figures with these.

Run in the build container (needs oracle/_ref):
    python tests/golden/make_build_parity.py
"""
import json
import os
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

N, D, CENTRES, NQ, NSAMPLE = 100_000, 128, 64, 1000, 2000
BUILD = dict(K=50, L=100, S=12, iterations=30, reverse=-1)   # the Python build fixes R=100
P_LIST = [50, 100, 300]
OUT = os.path.join(HERE, "build_parity_mix128.json")


def make_data():
    """Dataset (seed 21), queries (seed 23) and the node sample (seed 22)."""
    rng = np.random.default_rng(21)
    c = rng.uniform(0, 128, (CENTRES, D))

    def draw(r, m):
        x = c[r.integers(0, CENTRES, m)] + r.normal(0, 20, (m, D))
        return np.round(np.maximum(x, 0)).astype(np.float32)
    X = draw(rng, N)
    Q = draw(np.random.default_rng(23), NQ)
    sample = np.sort(np.random.default_rng(22).choice(N, NSAMPLE, replace=False)).astype(np.int64)
    return X, Q, sample


def exact_kth(X, rows, K, exclude_self):
    """FP64 squared distance of each row's K-th nearest dataset row (chunked numpy)."""
    Xd = X.astype(np.float64)
    xn = (Xd * Xd).sum(1)
    out = np.zeros(len(rows))
    for a in range(0, len(rows), 250):
        q = rows[a:a + 250].astype(np.float64)
        d = xn[None, :] - 2.0 * (q @ Xd.T) + (q * q).sum(1)[:, None]
        d = np.maximum(np.rint(d), 0)   # integer data: exact squared distances
        k = K + 1 if exclude_self else K
        out[a:a + 250] = np.partition(d, k - 1, axis=1)[:, k - 1]
    return out


def graph_recall(X, offsets, ids, dists, sample, kth, K=10):
    tot = 0
    for r, kd in zip(sample, kth):
        a, b = int(offsets[r]), int(offsets[r + 1])
        first = ids[a:b][np.argsort(dists[a:b], kind="stable")][:K]
        dd = ((X[first].astype(np.float64) - X[r].astype(np.float64)) ** 2).sum(1)
        tot += int((dd <= kd).sum())
    return tot / (len(sample) * K)


def search_recall(X, Q, ids, kth, K=10):
    ids = np.asarray(ids)[:, :K].astype(np.int64)
    dd = ((X[ids].astype(np.float64) - Q[:, None, :].astype(np.float64)) ** 2).sum(2)
    return float((dd <= kth[:, None]).mean())


def main():
    from oracle import kgoracle as ko
    if not ko.reference_available():
        raise SystemExit("oracle/_ref is not built (make -C oracle ref)")
    kg = ko.load_reference_module()
    X, Q, sample = make_data()
    node_kth = exact_kth(X, X[sample], 10, True)
    query_kth = exact_kth(X, Q, 10, False)
    builds = []
    with tempfile.TemporaryDirectory() as tmp:
        for rep in range(3):
            g = kg.KGraph(X, "euclidean")
            t0 = time.perf_counter()
            g.build(**BUILD)
            secs = time.perf_counter() - t0
            p = os.path.join(tmp, "g%d.idx" % rep)
            g.save(p)
            G = ko.read_index(p)
            rec = {"graph_recall10": graph_recall(X, G.offsets, G.ids, G.dists, sample, node_kth),
                   "search_recall10": {str(P): search_recall(X, Q, g.search(Q, K=10, P=P), query_kth)
                                       for P in P_LIST},
                   "edges": int(len(G.ids)), "build_seconds": secs, "threads": os.cpu_count()}
            print(rec)
            builds.append(rec)
    json.dump({"data": {"N": N, "D": D, "centres": CENTRES, "queries": NQ, "node_sample": NSAMPLE,
                        "seeds": {"data": 21, "sample": 22, "queries": 23}},
               "build": BUILD, "P": P_LIST, "reference_builds": builds,
               # the ground truth's exact 10th-nearest squared distances (integers), stored so the test need not
               # recompute them
               "node_kth": [int(v) for v in node_kth], "query_kth": [int(v) for v in query_kth]},
              open(OUT, "w"))


if __name__ == "__main__":
    main()
