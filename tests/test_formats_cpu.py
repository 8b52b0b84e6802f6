"""LSHKIT matrix files (kgraph-data.h:175-218 of the reference) through
kgraph-b200's kgraph-data.h, against files the reference's own
Matrix<float>::save_lshkit wrote (tests/golden/formats_u16.npz, made by
tests/golden/make_formats.py), and the command-line tools' option handling
(no GPU needed for either)."""
import os
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN, ROOT


def _compile(tmp_path, name):
    exe = str(tmp_path / name)
    subprocess.check_call(["g++", "-std=c++17", "-O2", "-I" + os.path.join(ROOT, "include"),
                           os.path.join(ROOT, "tests", "cpp", name + ".cpp"), "-o", exe])
    return exe


def test_lshkit_round_trip_matches_reference_bytes(tmp_path):
    f = np.load(os.path.join(GOLDEN, "formats_u16.npz"))
    X = np.load(os.path.join(GOLDEN, "u16.npz"))["X"]
    ref_bytes = f["lshkit_bytes"].tobytes()
    # the reference's file: header (element size, rows, cols) then the rows
    hdr = np.frombuffer(ref_bytes, np.uint32, 3)
    assert hdr.tolist() == [4, X.shape[0], X.shape[1]]
    assert (np.frombuffer(ref_bytes, np.float32, offset=12).reshape(X.shape) == X).all()
    src = tmp_path / "X.lshkit"
    src.write_bytes(ref_bytes)
    ids = np.arange(7 * 11, dtype=np.uint32).reshape(7, 11)
    usrc = tmp_path / "ids.lshkit"
    usrc.write_bytes(np.array([4, 7, 11], np.uint32).tobytes() + ids.tobytes())
    exe = _compile(tmp_path, "lshkit_rt")
    out = subprocess.run([exe, str(src), str(tmp_path / "X2"), str(usrc), str(tmp_path / "ids2")],
                         capture_output=True, text=True, check=True).stdout
    assert "f=%dx%d" % X.shape in out and "u=7x11" in out and "rejects_wrong_size=1" in out
    assert (tmp_path / "X2").read_bytes() == ref_bytes            # byte-identical to the reference's writer
    assert (tmp_path / "ids2").read_bytes() == usrc.read_bytes()


def test_cli_tools_usage_and_options():
    binp = os.path.join(ROOT, "kgraph_b200", "bin")
    if not os.path.exists(os.path.join(binp, "index")):
        pytest.skip("command-line tools not built (python -m kgraph_b200.build)")
    r = subprocess.run([os.path.join(binp, "index"), "--help"], capture_output=True, text=True)
    assert r.returncode == 0 and r.stdout.startswith("Usage: index [OTHER OPTIONS]... INPUT [OUTPUT]")
    r = subprocess.run([os.path.join(binp, "index")], capture_output=True, text=True)   # no input: usage, as index.cpp
    assert r.returncode == 0 and "Usage: index" in r.stdout
    r = subprocess.run([os.path.join(binp, "search"), "-v"], capture_output=True, text=True)
    assert r.returncode == 0 and r.stdout.startswith("KGraph version ")
    r = subprocess.run([os.path.join(binp, "search"), "a", "b"], capture_output=True, text=True)
    assert r.returncode == 0 and r.stdout.startswith("search <data> <index> <query> [output]")
    r = subprocess.run([os.path.join(binp, "index"), "--bogus", "1", "x"], capture_output=True, text=True)
    assert r.returncode != 0 and "unrecognised option" in r.stderr
    r = subprocess.run([os.path.join(binp, "prune"), "-h"], capture_output=True, text=True)
    assert r.returncode == 0 and r.stdout.startswith("Usage: prune [OTHER OPTIONS]... DATA INPUT [OUTPUT]")
    r = subprocess.run([os.path.join(binp, "resave")], capture_output=True, text=True)
    assert r.returncode == 0 and "--no-dist" in r.stdout
