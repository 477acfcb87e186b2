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
from oracle import RefSolver, build_oracle  # noqa: E402
from oracle import drive  # noqa: E402
from tests.golden.cases import small_cases  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def run_ref(w, steps=None):
    S = RefSolver()
    drive.setup(S, w)
    if "plane_wave" in w.meta:
        S.add_plane_wave(*w.meta["plane_wave"])
    drive.advance(S, w, w.steps if steps is None else steps)
    return S


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
