"""Surface monitors on a B200: PEC-surface currents (|Js| and its DFT),
Huygens-box phasors, the |E| cut plane, playback frames and the far field.

Bar: FP32 storage bitwise the reference (golden vectors it produced) for the
face lists, |Js|, the raw and finalised Js DFT, the Huygens phasors, the cut
plane and the frames; the far field, whose sums the device runs in FP64
(the reference sums in FP32), within 1e-3 of the reference's U maximum and
directivity. FP64 storage bitwise the FP64 oracle."""
import numpy as np
import pytest

from tests.conftest import golden
from emsolver_b200 import Batch, workloads
from emsolver_b200._lib import TLM_EINVAL, TLM_ESTATE, TlmError
from emsolver_b200.runner import build_solver, records
from emsolver_b200.solver import Storage
from oracle import Oracle, drive
from tests.golden.cases import surface_cases

pytestmark = pytest.mark.gpu

CASES = surface_cases()
FAR_TOL = 1e-3


def gpu_record(s):
    f, h = s.faces(), s.huygensFaces()
    mag, re, im, ns = s.getJsDft(raw=True)
    acc, hs = s.huygensDft()
    plane = s.getFieldPlane()
    frames = [s.getFrame(i) for i in range(s.frameCount())]
    out = {"face_cells": f["cells"], "face_axis": f["axis"], "face_sign": f["sign"], "face_center": f["center"],
           "js_instant": s.getJsInstant(), "js_re": re, "js_im": im, "js_mag": mag, "js_samples": ns,
           "huy_cells": h["cells"], "huy_axis": h["axis"], "huy_sign": h["out_sign"], "huy_pos": h["pos"],
           "huy_acc": acc, "huy_samples": hs, "plane": plane[0], "plane_axis": plane[1],
           "plane_index": plane[2], "frame_steps": np.array([fr["step"] for fr in frames]),
           "frame_js": np.stack([fr["js"] for fr in frames])}
    last = [fr for fr in frames if fr["plane"] is not None]
    if last:
        out["frame_last_plane"] = last[-1]["plane"]
        out["frame_last_plane_step"] = last[-1]["step"]
    return out


@pytest.mark.parametrize("w", CASES, ids=[w.name for w in CASES])
def test_surface_monitors_bitwise_vs_reference(built, w):
    g = golden(w.name)
    s = build_solver(w)
    s.step(w.steps)
    got = gpu_record(s)
    for k, v in got.items():
        assert np.array_equal(np.asarray(v).astype(np.asarray(g[k]).dtype), g[k]), k
    ff = s.computeFarField(19, 37)
    U, Ur = ff["U"].astype(np.float64), g["far_U"].astype(np.float64)
    assert np.abs(U - Ur).max() <= FAR_TOL * Ur.max()
    assert abs(ff["directivity"] - float(g["far_directivity"])) <= FAR_TOL * float(g["far_directivity"])
    ti, pj = np.unravel_index(np.argmax(Ur), Ur.shape)
    assert U[ti, pj] >= (1 - FAR_TOL) * U.max()


def test_fp64_storage_matches_fp64_oracle(built):
    w = CASES[0]
    s = build_solver(w, storage=Storage.F64)
    s.step(w.steps)
    O = Oracle(True)
    drive.setup(O, w)
    drive.advance(O, w, w.steps)
    # the device keeps FP64 accumulators; the C ABI hands them out as float
    re_o, im_o, mag_o, ns_o = O.js_dft()
    mag, re, im, ns = s.getJsDft(raw=True)
    assert ns == ns_o
    assert np.array_equal(re, re_o.astype(np.float32)) and np.array_equal(im, im_o.astype(np.float32))
    assert np.array_equal(s.getJsInstant(), O.js_instant().astype(np.float32))
    acc_o, hs_o = O.huygens_dft()
    acc, hs = s.huygensDft()
    assert hs == hs_o and np.array_equal(acc, acc_o.astype(np.float32))
    assert np.array_equal(s.getFieldPlane()[0], O.field_plane()[0].astype(np.float32))
    ff, fo = s.computeFarField(19, 37), O.far_field(19, 37)
    assert np.abs(ff["U"] - fo["U"]).max() <= 1e-5 * fo["U"].max()


@pytest.mark.parametrize("storage", [Storage.BF16, Storage.F16, Storage.BFP16])
def test_16bit_storage_surface_monitors_bounded(built, storage):
    """Same monitors in the 16-bit modes: finite, and the |Js| DFT magnitude
    within 5 % of the FP32 result on the strongest faces."""
    w = CASES[0]
    ref = build_solver(w)
    ref.step(w.steps)
    s = build_solver(w, storage=storage)
    s.step(w.steps)
    a, b = s.getJsDft(), ref.getJsDft()
    strong = b > 0.5 * b.max()
    assert np.all(np.isfinite(a))
    assert np.abs(a[strong] - b[strong]).max() <= 0.05 * b.max()


def test_monitors_do_not_change_the_solve(built):
    w = CASES[0]
    plain = workloads.dipole(24, 26, 30, 13, slab=(2, 6, 3.0), steps=w.steps, nfreq=4)
    a = build_solver(plain)
    a.step(w.steps)
    b = build_solver(w)
    b.step(w.steps)
    assert np.array_equal(a.pulses(), b.pulses())
    ra, rb = records(a, plain), records(b, w)
    for k in ra:
        assert np.array_equal(ra[k], rb[k]), k


def test_monitors_after_set_pulses(built):
    """The first step after tlm_set_pulses reads incident pulses directly."""
    w = CASES[1]
    rng = np.random.default_rng(4)
    v0 = rng.standard_normal(w.ncells * 12).astype(np.float32)
    v0.reshape(-1, 12)[np.asarray(w.mat) == 1] = 0.0
    s = build_solver(w)
    s.setPulses(v0)
    O = Oracle(False)
    drive.setup(O, w)
    O.set_pulses(v0)
    s.step(40)
    drive.advance(O, w, 40)
    assert np.array_equal(s.getJsInstant(), O.js_instant())
    assert np.array_equal(s.huygensDft()[0], O.huygens_dft()[0])
    assert np.array_equal(s.getFieldPlane()[0], O.field_plane()[0])


def test_batch_and_far_field_refusals(built):
    w = CASES[0]
    s = build_solver(w)
    with Batch() as b:
        with pytest.raises(TlmError) as e:
            b.attach(s)
        assert e.value.status == TLM_EINVAL
    plain = workloads.dipole(24, 26, 30, 13, steps=20, nfreq=4)
    p = build_solver(plain)
    p.step(5)
    with pytest.raises(TlmError) as e:
        p.computeFarField()
    assert e.value.status == TLM_ESTATE
    assert p.faces()["cells"].size == 0 and p.getFieldPlane() is None
