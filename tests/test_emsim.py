"""The .emsim project file against the reference's own SaveProject and
LoadProject (ProjectIO.cpp, compiled headless into oracle/_ref).

Bar: byte-identical files both ways (a file the reference writes loads here
and saves back to the same bytes; a file written here loads in the reference
and the reference saves it back to the same bytes), and the same accept /
reject decision with the same message on every truncation and on corrupt
counts."""
import struct

import numpy as np
import pytest

from emsolver_b200._lib import TLM_ESTATE
from emsolver_b200.emsim import EmsimError, Project, load_project
from oracle import RefEmsim, ref_available

pytestmark = pytest.mark.skipif(not ref_available(), reason="reference library not built")


def ours_load_error(path):
    try:
        load_project(path).close()
        return ""
    except EmsimError as e:
        return str(e)


def full_project():
    p = Project()
    p.add_setting("Frequency (GHz)", "1.5")
    p.add_setting("Cell size (mm)", "2")
    p.set_toolbar(solver=1, excitation=2, waveform=1, currents=2, db_range=3, gpu=1, show_model=0, plane_on=1)
    p.add_object(4, "dipole", position=(0.1, 0.2, 0.3), rot_deg=(0, 90, 0), design_freq_hz=1.5e9,
                 params=[("length", 0.1), ("gap", 0.002)])
    p.add_object(0, "part.stl", dielectric=True, epsr=3.5, sigma=0.01,
                 stl_verts=np.arange(9, dtype=np.float32) * 0.5, stl_idx=[0, 1, 2])
    faces = {"cells": [5, 17, 230], "center": [[0, 0, 1], [1, 0.5, 2], [3, 2, 1]], "axis": [0, 1, 2],
             "sign": [1, -1, 1]}
    p.set_result(faces=faces, face_vals=[0.5, 1.5, 2.5], face_dl=2e-3, tri_v=np.ones((3, 3)), tri_idx=[0, 1, 2],
                 tri_mag=[0.7], wire_pts=np.zeros((2, 3)), wire_mag=[0.1], has_plane=True,
                 plane_grid={"nx": 4, "ny": 5, "nz": 6, "origin": (0, 0, 0), "dl": 2e-3}, plane_axis=1,
                 plane_index=2, plane_n1=4, plane_n2=6, plane_vals=np.linspace(0, 1, 24), has_pattern=True,
                 pattern={"n_theta": 2, "n_phi": 3, "U": np.arange(6), "u_max": 5.0, "directivity": 1.7,
                          "peak_theta_deg": 90.0, "peak_phi_deg": 0.0},
                 pat_center=(0.004, 0.005, 0.006), pat_scale=0.0018, domain_lo=(0, 0, 0),
                 domain_hi=(0.008, 0.01, 0.012), domain_visible=True, probe_markers=[[1, 2, 3]])
    p.add_page("Input impedance", "f (GHz)", "Z (ohm)",
               [{"name": "Re Z", "x": [1.0, 1.5], "y": [50.0, 60.0], "color": 255},
                {"name": "Im Z", "x": [1.0, 1.5], "y": [-5.0, 3.0]}])
    p.set_playback({"nx": 4, "ny": 5, "nz": 6, "origin": (0, 0, 0), "dl": 2e-3}, 3.85e-12, faces)
    p.add_frame(7, [1, 2, 3])
    p.add_frame(14, [4, 5, 6], plane=np.arange(24), plane_axis=1, plane_index=2, plane_n1=4, plane_n2=6)
    return p


@pytest.mark.parametrize("seed", [0, 1, 2, 3, 7])
@pytest.mark.parametrize("playback", [False, True])
def test_reference_file_loads_and_saves_back_bytewise(tmp_path, seed, playback):
    ref = tmp_path / "ref.emsim"
    ours = tmp_path / "ours.emsim"
    RefEmsim.write_sample(ref, seed, playback)
    p = load_project(ref)
    p.save(ours)
    assert ours.read_bytes() == ref.read_bytes()
    s = RefEmsim.summary(ref)
    r, pb = p.result, p.playback
    assert (len(p.settings), len(p.objects), len(r["faces"]["cells"]), r["face_vals"].size,
            r["plane_vals"].size, r["pattern"]["U"].size, len(p.pages), len(p.pages[0]["curves"])) == \
        (s["settings"], s["objects"], s["faces"], s["face_vals"], s["plane_vals"], s["pattern_u"], s["pages"],
         s["page0_curves"])
    assert (int(pb["valid"]), len(pb["faces"]["cells"]), len(pb["frames"])) == \
        (s["playback_valid"], s["playback_faces"], s["frames"])
    if pb["frames"]:
        assert pb["frames"][0]["js"].size == s["frame0_js"]
    assert p.file_version == 2


def test_our_file_is_what_the_reference_writes(tmp_path):
    ours, back = tmp_path / "ours.emsim", tmp_path / "back.emsim"
    full_project().save(ours)
    assert RefEmsim.resave(ours, back) == ""
    assert back.read_bytes() == ours.read_bytes()
    s = RefEmsim.summary(ours)
    assert (s["settings"], s["objects"], s["faces"], s["plane_vals"], s["pattern_u"], s["pages"],
            s["page0_curves"], s["playback_valid"], s["frames"], s["frame0_js"]) == (2, 2, 3, 24, 6, 1, 2, 1, 2, 3)


def test_values_round_trip(tmp_path):
    path = tmp_path / "p.emsim"
    full_project().save(path)
    p = load_project(path)
    assert p.settings == [("Frequency (GHz)", "1.5"), ("Cell size (mm)", "2")]
    assert p.toolbar == {"solver": 1, "excitation": 2, "waveform": 1, "currents": 2, "db_range": 3, "gpu": 1,
                         "show_model": 0, "db_scale": 1, "plane_on": 1, "mesh_on": 0}
    o = p.objects
    assert o[0]["params"] == [("length", 0.1), ("gap", 0.002)] and o[0]["design_freq_hz"] == 1.5e9
    assert o[1]["is_stl"] and o[1]["dielectric"] and np.array_equal(o[1]["stl_idx"], [0, 1, 2])
    assert np.array_equal(o[1]["stl_verts"], np.arange(9, dtype=np.float32) * 0.5)
    r = p.result
    assert np.array_equal(r["faces"]["cells"], [5, 17, 230]) and np.array_equal(r["faces"]["sign"], [1, -1, 1])
    assert np.array_equal(r["plane_vals"], np.linspace(0, 1, 24).astype(np.float32))
    assert r["pattern"]["directivity"] == np.float32(1.7) and r["plane_grid"]["nz"] == 6
    assert r["domain_visible"] and r["probe_markers"].tolist() == [[1, 2, 3]]
    pg = p.pages[0]
    assert pg["title"] == "Input impedance" and pg["curves"][0]["color"] == 255
    assert pg["curves"][1]["y"].tolist() == [-5.0, 3.0]
    fr = p.playback["frames"]
    assert [f["step"] for f in fr] == [7, 14] and fr[0]["plane"].size == 0 and fr[0]["plane_axis"] == -1
    assert np.array_equal(fr[1]["plane"], np.arange(24, dtype=np.float32))


def test_defaults_match_the_reference(tmp_path):
    """An empty project saves as the reference saves a default ProjectData."""
    path, back = tmp_path / "e.emsim", tmp_path / "b.emsim"
    Project().save(path)
    assert RefEmsim.resave(path, back) == ""
    assert back.read_bytes() == path.read_bytes()
    r = load_project(path).result
    assert r["plane_axis"] == -1 and r["pat_scale"] == 1.0 and r["domain_lo"][0] == np.float32(1e30)


def test_every_truncation_is_handled_like_the_reference(tmp_path):
    src = tmp_path / "full.emsim"
    full_project().save(src)
    data = src.read_bytes()
    cut = tmp_path / "cut.emsim"
    for n in range(len(data)):
        cut.write_bytes(data[:n])
        assert ours_load_error(cut) == RefEmsim.resave(cut, tmp_path / "x.emsim"), n


def patched(data, offset, value):
    return data[:offset] + struct.pack("<I", value) + data[offset + 4:]


def test_corrupt_counts_and_versions_match_the_reference(tmp_path):
    empty = tmp_path / "e.emsim"
    Project().save(empty)
    e = empty.read_bytes()
    p = Project()
    p.add_setting("", "x")
    p.save(tmp_path / "s.emsim")
    s = (tmp_path / "s.emsim").read_bytes()
    p = Project()
    p.add_object(0, "")
    p.save(tmp_path / "o.emsim")
    o = (tmp_path / "o.emsim").read_bytes()
    p = Project()
    p.add_page("", "", "")
    p.save(tmp_path / "g.emsim")
    g = (tmp_path / "g.emsim").read_bytes()
    p = Project()
    p.set_playback({"nx": 2, "ny": 2, "nz": 2, "origin": (0, 0, 0), "dl": 1e-3}, 1e-12, None)
    p.save(tmp_path / "b.emsim")
    b = (tmp_path / "b.emsim").read_bytes()
    cases = {
        "bad magic": (b"EMSIN" + e[5:], "not an EMSIM project file"),
        "version 0": (patched(e, 8, 0), "unsupported project version"),
        "version 3": (patched(e, 8, 3), "unsupported project version"),
        "version 1": (patched(e, 8, 1)[:-1], ""),
        "1001 settings": (patched(e, 12, 1001), "corrupt settings"),
        "long string": (patched(s, 16, 200000000), "file truncated or corrupt"),
        "100001 objects": (patched(e, 41, 100001), "corrupt object list"),
        "100001 params": (patched(o, 103, 100001), "file truncated or corrupt"),
        "huge face count": (patched(e, 45, 0x40000000), "file truncated or corrupt"),
        "1001 pages": (patched(e, len(e) - 5, 1001), "corrupt plot data"),
        "1001 curves": (patched(g, len(g) - 5, 1001), "corrupt curve data"),
        "10^7+1 frames": (patched(b, len(b) - 4, 10000001), "corrupt playback data"),
        "missing frames": (patched(b, len(b) - 4, 1000), "file truncated or corrupt"),
        "trailing bytes": (e + b"\0\0\0", ""),
    }
    f = tmp_path / "c.emsim"
    for name, (data, msg) in cases.items():
        f.write_bytes(data)
        assert RefEmsim.resave(f, tmp_path / "x.emsim") == msg, name
        assert ours_load_error(f) == msg, name
    f.write_bytes(patched(e, 8, 1)[:-1])
    assert load_project(f).file_version == 1


def test_missing_file_and_misuse(tmp_path):
    assert ours_load_error(tmp_path / "none.emsim") == "cannot open file"
    p = Project()
    with pytest.raises(EmsimError) as e:
        p.add_frame(1, [1.0])
    assert e.value.status == TLM_ESTATE
    with pytest.raises(EmsimError):
        p.save(tmp_path / "no_such_dir" / "x.emsim")
