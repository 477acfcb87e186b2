"""The C ABI library on a machine without a GPU: it loads, exports every
symbol include/tlm_b200.h, fdtd_b200.h and emsim_b200.h declare, its host-only math matches the
reference bit for bit, and compute entry points fail loudly (no fallback)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from tests.conftest import ROOT
from emsolver_b200 import _lib
from oracle import Oracle, RefSolver, ref_available

HEADERS = [os.path.join(ROOT, "include", n) for n in ("tlm_b200.h", "fdtd_b200.h", "emsim_b200.h")]


def declared_symbols():
    src = "".join(open(h).read() for h in HEADERS)
    return sorted(set(re.findall(r"TLM_API\s+[\w\s\*]+?\b((?:tlm|fdtd|emsim)_\w+)\s*\(", src)))


def test_header_declares_entry_points():
    names = declared_symbols()
    assert len(names) >= 40
    assert "tlm_setup" in names and "tlm_step" in names and "tlm_get_probe" in names


@pytest.mark.parametrize("variant", ["", "checked"])
def test_library_exports_every_declared_symbol(built, variant):
    path = _lib.library_path(variant)
    lib = C.CDLL(path)
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, missing
    # the Python binding covers the whole header
    assert set(declared_symbols()) == set(_lib.SIGNATURES)


def test_version_and_defaults(built):
    L = _lib.load()
    assert b"sm_100a" in L.tlm_version()
    c = _lib.ConfigC()
    L.tlm_config_default(C.byref(c))
    # TlmConfig defaults (TlmSolver.h:113-123)
    assert c.f0 == np.float32(1e9) and c.waveform == 0 and c.total_steps == 2000
    assert c.settle_steps == 600 and c.boundary_rho == 0.0 and c.storage == _lib.STORE_F32


def test_waveform_value_bitwise(built):
    L = _lib.load()
    out = C.c_float()
    for wf in (0, 1, 2):
        O = Oracle(False)
        O.setup(4, 4, 4, np.zeros(64, np.uint8), [], dl=2.5e-3, f0=1.3e9, waveform=wf)
        for n in (0, 3, 59, 60, 61, 499, 7999):
            assert L.tlm_waveform_value(wf, 1.3e9, 2.5e-3, n, C.byref(out)) == 0
            assert np.float32(out.value) == np.float32(O.waveform(n)), (wf, n)
            if ref_available():
                R = RefSolver()
                R.setup(4, 4, 4, np.zeros(64, np.uint8), [], dl=2.5e-3, f0=1.3e9, waveform=wf)
                assert np.float32(out.value) == np.float32(R.waveform(n))
    assert L.tlm_waveform_value(9, 1e9, 1e-3, 0, C.byref(out)) == _lib.TLM_EINVAL


def test_null_arguments_are_rejected(built):
    L = _lib.load()
    assert L.tlm_create(None, 0) == _lib.TLM_EINVAL
    assert L.tlm_setup(None, None, None, 0, None, 0, None) == _lib.TLM_EINVAL
    assert L.tlm_step(None, 1) == _lib.TLM_EINVAL
    assert L.tlm_destroy(None) == _lib.TLM_OK
    assert L.tlm_current_step(None) == -1
    assert b"null" in L.tlm_last_error(None)


def test_no_device_fails_loudly(built):
    """Without a CUDA device every compute entry point refuses: there is no
    CPU path to fall back to."""
    L = _lib.load()
    h = C.c_void_p()
    st = L.tlm_create(C.byref(h), 0)
    if st == _lib.TLM_OK:
        L.tlm_destroy(h)
        pytest.skip("a GPU is present")
    assert st == _lib.TLM_ENODEV
    assert L.tlm_last_error(None)
    e = C.c_float()
    assert L.tlm_scatter_unitarity_error(0, C.byref(e)) == _lib.TLM_ENODEV


def test_request_footprint_without_device(built):
    """Admission arithmetic is host-only: FP32 pulses take twice the bytes of
    BF16, and a dielectric adds the stub planes."""
    from emsolver_b200 import workloads
    from emsolver_b200.server import footprint
    w = workloads.dipole(32, 32, 48, 21, steps=500)
    f32, bf16 = footprint(w, storage=0), footprint(w, storage=1)
    P = 32 * 32 * 48
    assert f32 - bf16 == 2 * 12 * P * 2
    w2 = workloads.dipole(32, 32, 48, 21, slab=(2, 6, 3.0), steps=500)
    assert footprint(w2, storage=0) - f32 == 3 * P * 4


# ctypes mirror -> C type of the headers
STRUCTS = {
    "Grid": "tlm_grid", "MatPropsC": "tlm_matprops", "ConfigC": "tlm_config",
    "BatchTuningC": "tlm_batch_tuning", "RequestC": "tlm_request", "ServerStatsC": "tlm_server_stats_t",
    "EmsimFaceC": "emsim_face", "EmsimToolbarC": "emsim_toolbar", "EmsimObjectC": "emsim_object",
    "EmsimPatternC": "emsim_pattern", "EmsimResultC": "emsim_result", "EmsimCurveC": "emsim_curve",
    "EmsimFrameC": "emsim_frame", "EmsimCaptureC": "emsim_capture",
}


def test_ctypes_structs_match_the_headers(tmp_path):
    """Every structure the Python binding passes across the C ABI has the
    size and field offsets the headers give it (compiled here with g++)."""
    import shutil
    import subprocess
    if not shutil.which("g++"):
        pytest.skip("no g++")
    lines = ["#include <cstddef>", "#include <cstdio>", '#include "tlm_b200.h"', '#include "emsim_b200.h"',
             "int main() {"]
    for py, c in STRUCTS.items():
        lines.append(f'std::printf("{py} size %zu\\n", sizeof({c}));')
        for name, _ in getattr(_lib, py)._fields_:
            lines.append(f'std::printf("{py} {name} %zu\\n", offsetof({c}, {name}));')
    lines.append("return 0; }")
    src = tmp_path / "layout.cpp"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["g++", "-std=c++17", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)],
                   check=True, capture_output=True)
    got = {}
    for line in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.splitlines():
        py, name, value = line.split()
        got[(py, name)] = int(value)
    for py in STRUCTS:
        cls = getattr(_lib, py)
        assert got[(py, "size")] == C.sizeof(cls), py
        for name, _ in cls._fields_:
            assert got[(py, name)] == getattr(cls, name).offset, (py, name)
