"""The C++ host side (include/tlm_b200.hpp) as a reference-style caller would
use it: compiled with g++ against libtlm_b200.so; on a GPU its probe and port
records equal the reference's golden vectors."""
import os
import subprocess

import numpy as np
import pytest

from tests.conftest import ROOT, golden

SRC = os.path.join(ROOT, "tests", "cpp", "tlm_cpp_client.cpp")
EXE = os.path.join(ROOT, "_build", "tlm_cpp_client")


def compile_client():
    os.makedirs(os.path.dirname(EXE), exist_ok=True)
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-I" + os.path.join(ROOT, "include"), SRC,
           "-L" + os.path.join(ROOT, "emsolver_b200"), "-ltlm_b200",
           "-Wl,-rpath," + os.path.join(ROOT, "emsolver_b200"), "-pthread", "-o", EXE]
    out = subprocess.run(cmd, capture_output=True, text=True)
    assert out.returncode == 0, out.stderr
    return EXE


def test_cpp_client_compiles_and_links(built):
    exe = compile_client()
    assert os.path.exists(exe)


@pytest.mark.gpu
def test_cpp_client_matches_reference(built, tmp_path):
    exe = compile_client()
    out = tmp_path / "rec.bin"
    r = subprocess.run([exe, str(out)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    data = np.fromfile(out, np.float32)
    assert data.size == 1500
    g = golden("plain_free_space")
    assert np.array_equal(data[:500], g["probe0_ez"])
    assert np.array_equal(data[500:1000], g["port0_v"])
    assert np.array_equal(data[1000:], g["port0_i"])
