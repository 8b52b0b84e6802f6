import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")


def load_golden(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    d = {k: z[k] for k in z.files}
    d["metric"] = str(d["metric"])
    d["build"] = json.loads(str(d["build"]))
    d["searches"] = json.loads(str(d["searches"]))
    return d


GOLDEN_CASES = ["u16", "mix32", "ang20", "l2sq24"]
# rows wider than the tensor-core brute force takes (d = 300)
WIDE_GOLDEN_CASES = ["mix300"]


@pytest.fixture(scope="session")
def gpu_ctx():
    from kgraph_b200 import capi
    c = capi.Context(0)
    yield c
    c.close()
