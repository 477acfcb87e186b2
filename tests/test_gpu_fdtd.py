"""The Yee FDTD solver on a B200 against the reference's own FdtdSolver.

Bar: with the same inputs, every E and H value, port V/I, probe E record,
|Js|, Js DFT, Huygens phasor, cut plane and frame is bitwise the reference's
(golden vectors it produced, and live runs of the reference compiled
headless on fresh random grids); the energy history (an FP64 sum in another
order) within 1e-6 relative; the far field within 1e-3 of the reference's
maximum."""
import numpy as np
import pytest

from tests.conftest import golden
from emsolver_b200 import workloads
from emsolver_b200._lib import TLM_EINVAL, TlmError
from emsolver_b200.fdtd import FIELDS, build_fdtd
from oracle import RefFdtd, drive, ref_available
from tests.golden.cases import fdtd_cases

pytestmark = pytest.mark.gpu

CASES = fdtd_cases()


def gpu_record(s, w):
    out = s.fields()
    for p in range(len(w.ports)):
        out[f"port{p}_v"], out[f"port{p}_i"] = s.port(p)
    for q in range(len(w.probes_cell)):
        out[f"probe{q}_ex"], out[f"probe{q}_ey"], out[f"probe{q}_ez"] = s.probe(q)
    st, ev = s.getEnergyHistory(f64=True)
    out["energy_steps"], out["energy"] = st, ev
    f, h = s.faces(), s.huygensFaces()
    mag, re, im, ns = s.getJsDft(raw=True)
    acc, hs = s.huygensDft()
    out.update({"face_cells": f["cells"], "face_axis": f["axis"], "face_sign": f["sign"],
                "face_center": f["center"], "js_instant": s.getJsInstant(), "js_re": re, "js_im": im,
                "js_mag": mag, "js_samples": ns, "huy_cells": h["cells"], "huy_axis": h["axis"],
                "huy_sign": h["out_sign"], "huy_pos": h["pos"], "huy_acc": acc, "huy_samples": hs})
    plane = s.getFieldPlane()
    if plane is not None:
        out["plane"], out["plane_axis"], out["plane_index"] = plane
    frames = [s.getFrame(i) for i in range(s.frameCount())]
    if frames:
        out["frame_steps"] = np.array([fr["step"] for fr in frames])
        out["frame_js"] = np.stack([fr["js"] for fr in frames])
        last = [fr for fr in frames if fr["plane"] is not None]
        if last:
            out["frame_last_plane"], out["frame_last_plane_step"] = last[-1]["plane"], last[-1]["step"]
    return out


def assert_matches(got, ref):
    for k, v in got.items():
        if k not in ref:
            continue
        r = np.asarray(ref[k])
        if k == "energy":
            scale = max(np.abs(r).max(), 1e-30)
            assert np.abs(np.asarray(v, np.float64) - r).max() <= 1e-6 * scale, k
        else:
            assert np.array_equal(np.asarray(v).astype(r.dtype), r), k


@pytest.mark.parametrize("w", CASES, ids=[w.name for w in CASES])
def test_fdtd_bitwise_vs_reference_golden(built, w):
    g = golden(w.name)
    s = build_fdtd(w)
    s.step(w.steps)
    assert_matches(gpu_record(s, w), g)
    if g["far_U"].size:
        ff = s.computeFarField(19, 37)
        U, Ur = ff["U"].astype(np.float64), g["far_U"].astype(np.float64)
        assert np.abs(U - Ur).max() <= 1e-3 * Ur.max()
        assert abs(ff["directivity"] - float(g["far_directivity"])) <= 1e-3 * float(g["far_directivity"])


@pytest.mark.skipif(not ref_available(), reason="reference library not shipped")
@pytest.mark.parametrize("seed", [41, 42, 43])
def test_fdtd_live_reference_random(built, seed):
    rng = np.random.default_rng(seed)
    nx, ny, nz = (int(v) for v in rng.integers(9, 20, 3))
    w = workloads.random_dipole(rng, nx, ny, nz, int(rng.integers(20, 60)), name="live")
    w.probes_cell = [tuple(int(rng.integers(0, d)) for d in (nx, ny, nz))]
    w.meta.update(settle_steps=int(rng.integers(0, 15)), record_every=int(rng.integers(0, 6)),
                  field_plane=(int(rng.integers(0, 3)), int(rng.integers(0, 8))), surface_monitors=True,
                  huy_offset=2)
    R = RefFdtd()
    drive.setup(R, w)
    drive.advance(R, w, w.steps)
    ref = R.fields()
    for p in range(len(w.ports)):
        ref[f"port{p}_v"], ref[f"port{p}_i"] = R.port(p)
    ref["probe0_ex"], ref["probe0_ey"], ref["probe0_ez"] = R.probe(0)
    ref["js_instant"] = R.js_instant()
    ref["huy_acc"] = R.huygens_dft()[0]
    s = build_fdtd(w)
    s.step(w.steps)
    assert_matches(gpu_record(s, w), ref)


def test_fdtd_in_steps_equals_one_run(built):
    w = CASES[0]
    a = build_fdtd(w)
    a.run()
    b = build_fdtd(w)
    for n in (7, 1, 30, w.steps - 38):
        b.step(n)
    for name in FIELDS:
        assert np.array_equal(a.field(name), b.field(name)), name


def test_fdtd_rejects_bad_input(built):
    w = CASES[0]
    s = build_fdtd(w)
    with pytest.raises(TlmError) as e:
        s.addPort([0], 2, 1.0)    # corner cell: the current loop would leave the grid
    assert e.value.status == TLM_EINVAL
