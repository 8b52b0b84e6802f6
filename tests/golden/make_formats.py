"""Generates tests/golden/formats_u16.npz from the REFERENCE itself.

The reference (compiled from its own sources into oracle/_ref by
oracle/Makefile; oracle/ref_driver.cpp calls only its public C++ API) loads
the u16 fixture's index file -- written by the reference's build, see
make_golden.py -- and saves it again in the formats its saver writes
(kgraph.cpp:333-373):

  text_bytes     KGraph::FORMAT_TEXT
  nodist_bytes   KGraph::FORMAT_NO_DIST

and writes the fixture's dataset as an LSHKIT matrix with its own
Matrix<float>::save_lshkit (kgraph-data.h:207-218):

  lshkit_bytes

Run where oracle/_ref is built:
    python tests/golden/make_formats.py
"""
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)


def main():
    from oracle import kgoracle as ko
    z = np.load(os.path.join(HERE, "u16.npz"))
    ref = ko.RefLib()
    out = {}
    with tempfile.TemporaryDirectory() as tmp:
        src = os.path.join(tmp, "u16.idx")
        open(src, "wb").write(z["index_bytes"].tobytes())
        for name, fmt in (("text_bytes", 128), ("nodist_bytes", 1)):
            p = os.path.join(tmp, name)
            ref.resave(src, p, fmt)
            out[name] = np.frombuffer(open(p, "rb").read(), np.uint8)
        p = os.path.join(tmp, "X.lshkit")
        ref.save_lshkit(z["X"], p)
        out["lshkit_bytes"] = np.frombuffer(open(p, "rb").read(), np.uint8)
    np.savez_compressed(os.path.join(HERE, "formats_u16.npz"), **out)
    print({k: len(v) for k, v in out.items()})


if __name__ == "__main__":
    main()
