"""Generate the golden vectors under tests/golden/ from the REFERENCE ITSELF.

The reference's own CPU TLM step (TlmSolver.cpp + Geometry.cpp of
smilima/EMSolver) is compiled headless by oracle/Makefile into
oracle/_ref/libtlmref.so; this script drives it through oracle/ref_harness.cpp
on seeded synthetic workloads and stores its outputs:

  plain_free_space.npz   64^3, 500 steps: probe E series, port V/I, energy
  heterogeneous.npz      192^3, 16 lossy dielectric boxes, 2000 steps:
                         8 probe series, port V/I, energy, yhat/ghat tables,
                         sha256 of the material map
  small_<name>.npz       small grids (PEC, dielectrics, rho != 0, plane wave,
                         odd x extents): full final pulse and stub state plus
                         all records
  fdtd_<name>.npz        the reference's Yee FDTD solver: final E and H
                         fields, port, probe and energy records and every
                         surface monitor (a dipole and a plane-wave case)
  surface_<name>.npz     dipoles with the surface monitors on: PEC faces,
                         |Js| and its DFT (raw and finalised), Huygens faces
                         and phasors, the |E| cut plane, playback frames and
                         the far field (19 x 37 directions)

Run:  python tests/golden/make_golden.py [--skip-large]
(needs the reference sources to build oracle/_ref; takes ~3 minutes)
"""
from __future__ import annotations

import hashlib
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from emsolver_b200 import workloads  # noqa: E402
from oracle import RefFdtd, RefSolver, build_oracle  # noqa: E402
from oracle import drive  # noqa: E402
from tests.golden.cases import fdtd_cases, small_cases, surface_cases  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def run_ref(w, steps=None, solver=RefSolver):
    S = solver()
    drive.setup(S, w)
    if "plane_wave" in w.meta:
        S.add_plane_wave(*w.meta["plane_wave"])
    drive.advance(S, w, w.steps if steps is None else steps)
    return S


def surface_record(S, far=True):
    """Every surface-monitor output of a solver (reference or oracle)."""
    sf, hf = S.surface_faces(), S.huygens_faces()
    re, im, mag, ns = S.js_dft()
    acc, hs = S.huygens_dft()
    plane = S.field_plane()
    frames = S.frames()
    ff = S.far_field(19, 37) if far else {"U": np.zeros((0, 0), np.float32), "u_max": 0.0, "directivity": 0.0,
                                          "peak_theta_deg": 0.0, "peak_phi_deg": 0.0}
    out = {"face_cells": sf["cells"], "face_axis": sf["axis"], "face_sign": sf["sign"],
           "face_center": sf["center"], "js_instant": S.js_instant(), "js_re": re, "js_im": im,
           "js_mag": mag, "js_samples": ns, "huy_cells": hf["cells"], "huy_axis": hf["axis"],
           "huy_sign": hf["out_sign"], "huy_pos": hf["pos"], "huy_acc": acc, "huy_samples": hs,
           "plane": plane[0], "plane_axis": plane[1], "plane_index": plane[2],
           "frame_steps": np.array([f["step"] for f in frames]),
           "frame_js": np.stack([f["js"] for f in frames]),
           "far_U": ff["U"], "far_u_max": ff["u_max"], "far_directivity": ff["directivity"],
           "far_peak": np.array([ff["peak_theta_deg"], ff["peak_phi_deg"]])}
    last = [f for f in frames if f["plane"] is not None]
    if last:
        out["frame_last_plane"] = last[-1]["plane"]
        out["frame_last_plane_step"] = last[-1]["step"]
    return out


def fdtd_record(S, w):
    """Fields, records and surface monitors of an FDTD solver run on `w`."""
    out = {k: v for k, v in S.fields().items()}
    for p in range(len(w.ports)):
        out[f"port{p}_v"], out[f"port{p}_i"] = S.port(p)
    for q in range(len(w.probes_cell)):
        out[f"probe{q}_ex"], out[f"probe{q}_ey"], out[f"probe{q}_ez"] = S.probe(q)
    st, ev = S.energy_history()
    out["energy_steps"], out["energy"] = st, ev
    out.update(surface_record(S, far=S.huygens_faces()["cells"].size > 0))
    return out


def main():
    build_oracle()
    skip_large = "--skip-large" in sys.argv
    for w in small_cases():
        S = run_ref(w)
        rec = drive.records(S, w)
        y, g = S.tables()
        np.savez_compressed(os.path.join(OUT, w.name + ".npz"), pulses=S.pulses(), stubs=S.stubs(),
                            yhat=y, ghat=g, threads=S.threads, **rec)
        print("wrote", w.name, flush=True)
    for w in surface_cases():
        S = run_ref(w)
        np.savez_compressed(os.path.join(OUT, w.name + ".npz"), **surface_record(S))
        print("wrote", w.name, flush=True)
    for w in fdtd_cases():
        np.savez_compressed(os.path.join(OUT, w.name + ".npz"), **fdtd_record(run_ref(w, solver=RefFdtd), w))
        print("wrote", w.name, flush=True)
    if skip_large:
        return
    w = workloads.plain_free_space()
    t = time.time()
    S = run_ref(w)
    dt = time.time() - t
    rec = drive.records(S, w)
    np.savez_compressed(os.path.join(OUT, "plain_free_space.npz"), seconds=dt, threads=S.threads,
                        **rec)
    print(f"wrote plain_free_space ({dt:.1f}s, {S.threads} threads)", flush=True)
    w = workloads.heterogeneous()
    t = time.time()
    S = run_ref(w)
    dt = time.time() - t
    rec = drive.records(S, w)
    y, g = S.tables()
    np.savez_compressed(os.path.join(OUT, "heterogeneous.npz"), seconds=dt, threads=S.threads,
                        yhat=y, ghat=g, mat_sha256=hashlib.sha256(w.mat.tobytes()).hexdigest(),
                        **rec)
    print(f"wrote heterogeneous ({dt:.1f}s, {S.threads} threads)", flush=True)


if __name__ == "__main__":
    main()
