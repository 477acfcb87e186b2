"""Saving a finished B200 run as an .emsim project (emsim_from_tlm /
emsim_from_fdtd) and opening it with the reference's own LoadProject.

Bar: the reference loads the file and saves it back to the same bytes; what
the file holds is exactly what the solver's getters return (faces, |Js| DFT,
cut plane, frames, far-field pattern), with the domain box and pattern
placement the reference's main window computes from the grid."""
import numpy as np
import pytest

from emsolver_b200.emsim import Project, load_project
from emsolver_b200.fdtd import build_fdtd
from emsolver_b200.runner import build_solver
from oracle import RefEmsim, ref_available
from tests.golden.cases import fdtd_cases, surface_cases

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not ref_available(), reason="reference library not built")]


def check_capture(s, w, tmp_path):
    p = Project()
    p.capture(s, js_dft=True, n_theta=19, n_phi=37, playback=True)
    path, back = tmp_path / "run.emsim", tmp_path / "back.emsim"
    p.save(path)
    assert RefEmsim.resave(path, back) == ""
    assert back.read_bytes() == path.read_bytes()

    q = load_project(path)
    r, pb = q.result, q.playback
    f = s.faces()
    assert np.array_equal(r["faces"]["cells"], f["cells"]) and np.array_equal(r["faces"]["axis"], f["axis"])
    assert np.array_equal(r["faces"]["sign"], f["sign"]) and np.array_equal(r["faces"]["center"], f["center"])
    assert np.array_equal(r["face_vals"], s.getJsDft())
    plane, axis, index = s.getFieldPlane()
    assert r["has_plane"] and (r["plane_axis"], r["plane_index"]) == (axis, index)
    assert np.array_equal(r["plane_vals"], plane.ravel())
    ff = s.computeFarField(19, 37)
    assert r["has_pattern"] and np.array_equal(r["pattern"]["U"], ff["U"].ravel())
    assert r["pattern"]["directivity"] == np.float32(ff["directivity"])
    dl = np.float32(w.dl)
    ext = [np.float32(n) * dl for n in (w.nx, w.ny, w.nz)]
    o = [np.float32(v) for v in w.origin]
    assert r["domain_lo"] == tuple(np.float32(v) for v in o)
    assert r["domain_hi"] == tuple(np.float32(a + b) for a, b in zip(o, ext))
    assert r["pat_center"] == tuple(np.float32(a + b * np.float32(0.5)) for a, b in zip(o, ext))
    assert r["pat_scale"] == np.float32(np.float32(0.45) * np.float32(min(w.nx, w.ny, w.nz))) * dl
    assert pb["valid"] and pb["grid"]["nx"] == w.nx and len(pb["frames"]) == s.frameCount() > 0
    for i, fr in enumerate(pb["frames"]):
        g = s.getFrame(i)
        assert fr["step"] == g["step"] and np.array_equal(fr["js"], g["js"])
        if g["plane"] is None:
            assert fr["plane"].size == 0 and fr["plane_axis"] == -1
        else:
            assert np.array_equal(fr["plane"], g["plane"].ravel()) and fr["plane_axis"] == g["axis"]


def test_tlm_run_saved_as_emsim(built, tmp_path):
    w = surface_cases()[0]
    s = build_solver(w)
    s.step(w.steps)
    check_capture(s, w, tmp_path)


def test_fdtd_run_saved_as_emsim(built, tmp_path):
    w = fdtd_cases()[0]
    s = build_fdtd(w)
    s.step(w.steps)
    check_capture(s, w, tmp_path)
