"""The C++ API (include/kgraph.h, include/kgraph-data.h) compiles and links
the way code written for the reference's headers does; on a GPU the demo
builds, saves, loads and searches."""
import os
import subprocess

import pytest

from conftest import ROOT


def compile_demo(tmp_path):
    exe = str(tmp_path / "api_demo")
    lib = os.path.join(ROOT, "kgraph_b200")
    subprocess.check_call(["g++", "-std=c++17", "-O2", "-I" + os.path.join(ROOT, "include"),
                           os.path.join(ROOT, "tests", "cpp", "api_demo.cpp"), "-o", exe,
                           "-L" + lib, "-lkgraph_b200", "-Wl,-rpath," + lib])
    return exe


def test_cpp_api_compiles_and_links(tmp_path):
    assert os.path.exists(compile_demo(tmp_path))


@pytest.mark.gpu
def test_cpp_api_build_save_load_search(tmp_path):
    exe = compile_demo(tmp_path)
    out = subprocess.run([exe, str(tmp_path / "g.kgraph")], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    kv = dict(t.split("=", 1) for t in out.stdout.split())
    assert kv["c1"] == "5" and kv["c2"] == "5" and kv["c3"] == "5"
    assert kv["same"] == "1"                       # graph search == brute force here, before and after load
    assert kv["first"] == "17,17,17" and float(kv["self_dist"]) == 0.0
    assert kv["rejects_vector_oracle"] == "1"
    assert int(kv["L"]) >= int(kv["M"]) > 0
