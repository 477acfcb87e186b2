"""The oracle pinned against the reference (CPU only).

Bar: the float oracle is BITWISE the reference's own CPU step -- against the
golden vectors the reference produced (tests/golden/make_golden.py) and, when
the reference library is built here, against live runs on fresh random cases.
The FP64 oracle must agree with the float one to float rounding.
"""
import hashlib

import numpy as np
import pytest

from tests.conftest import golden
from emsolver_b200 import workloads
from oracle import Oracle, RefSolver, drive, ref_available
from tests.golden.cases import small_cases, surface_cases

CASES = small_cases()


def _run_oracle(w, fp64=False, steps=None):
    S = Oracle(fp64=fp64)
    drive.setup(S, w)
    if "plane_wave" in w.meta:
        S.add_plane_wave(*w.meta["plane_wave"])
    drive.advance(S, w, w.steps if steps is None else steps)
    return S


def _same(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return a.shape == b.shape and np.array_equal(a, b)


@pytest.mark.parametrize("w", CASES, ids=[w.name for w in CASES])
def test_small_cases_bitwise_vs_reference_golden(built, w):
    g = golden(w.name)
    S = _run_oracle(w)
    assert _same(S.pulses(), g["pulses"])
    assert _same(S.stubs(), g["stubs"])
    y, gh = S.tables()
    assert _same(y, g["yhat"]) and _same(gh, g["ghat"])
    rec = drive.records(S, w)
    for k, v in rec.items():
        if k == "energy":
            # the reference reports the FP64 sum as float
            assert _same(v.astype(np.float32), g[k].astype(np.float32)), k
        else:
            assert _same(v, g[k]), k


def test_plain_free_space_golden(built):
    w = workloads.plain_free_space()
    g = golden("plain_free_space")
    S = _run_oracle(w)
    rec = drive.records(S, w)
    ez = g["probe0_ez"]
    assert ez.shape == (500,) and np.abs(ez).max() > 0
    for k in ("probe0_ex", "probe0_ey", "probe0_ez", "port0_v", "port0_i"):
        assert _same(rec[k], g[k]), k
    assert _same(rec["energy"].astype(np.float32), g["energy"].astype(np.float32))


def test_heterogeneous_tables_and_prefix(built):
    """192^3 heterogeneous grid: the material map and stub tables match the
    reference bit for bit, and the first 12 steps of every record match (the
    full 2000-step run is compared on the GPU)."""
    w = workloads.heterogeneous()
    g = golden("heterogeneous")
    assert hashlib.sha256(w.mat.tobytes()).hexdigest() == str(g["mat_sha256"])
    S = Oracle(False)
    drive.setup(S, w)
    y, gh = S.tables()
    assert _same(y, g["yhat"]) and _same(gh, g["ghat"])
    drive.advance(S, w, 12)
    rec = drive.records(S, w)
    for k, v in rec.items():
        if k.startswith("energy"):
            continue
        assert _same(v, g[k][:12]), k


@pytest.mark.skipif(not ref_available(), reason="reference library not built here")
@pytest.mark.parametrize("seed", [11, 12, 13])
def test_live_reference_random_cases(built, seed):
    rng = np.random.default_rng(seed)
    nx, ny, nz = (int(v) for v in rng.integers(4, 14, 3))
    mat = np.zeros((nz, ny, nx), np.uint8)
    table = []
    for b in range(int(rng.integers(0, 4))):
        lo = [int(rng.integers(0, d)) for d in (nz, ny, nx)]
        hi = [int(rng.integers(l, d)) + 1 for l, d in zip(lo, (nz, ny, nx))]
        mat[lo[0]:hi[0], lo[1]:hi[1], lo[2]:hi[2]] = 2 + b
        table.append((float(rng.uniform(0.5, 12)), float(rng.uniform(-0.01, 0.1))))
    mat[rng.random((nz, ny, nx)) < 0.1] = 1
    mat = mat.reshape(-1)
    w = workloads.Workload("rand", nx, ny, nz, mat, table, f0=2e10, waveform=int(rng.integers(0, 3)),
                           steps=60, rho=float(rng.choice([-1.0, 0.0, 0.25, 1.0])))
    kk, jj, ii = np.unravel_index(np.arange(mat.size), (nz, ny, nx))
    inner = (ii > 0) & (ii < nx - 1) & (jj > 0) & (jj < ny - 1) & (kk > 0) & (kk < nz - 1)
    air = np.flatnonzero((mat == 0) & inner)
    if air.size:
        w.ports.append(([int(c) for c in rng.choice(air, 2)], int(rng.integers(0, 3)), 1.5))
    w.probes_cell.append((0, 0, 0))
    w.probes_cell.append((nx - 1, ny // 2, nz - 1))
    R = RefSolver()
    drive.run(R, w)
    O = _run_oracle(w)
    assert _same(R.pulses(), O.pulses())
    assert _same(R.stubs(), O.stubs())
    rr, ro = drive.records(R, w), drive.records(O, w)
    for k in rr:
        if k == "energy":
            assert _same(rr[k].astype(np.float32), ro[k].astype(np.float32))
        else:
            assert _same(rr[k], ro[k]), k


def test_unitarity_kats():
    """TlmSolver.cpp:116-169 thresholds (SelfTest.cpp:215-219)."""
    assert Oracle.scatter_unitarity(False) < 1e-5
    assert Oracle.stub_unitarity(3.0, False) < 1e-4
    assert Oracle.scatter_unitarity(True) < 1e-13
    assert Oracle.stub_unitarity(3.0, True) < 1e-12
    if ref_available():
        assert np.float32(Oracle.scatter_unitarity(False)) == np.float32(RefSolver.scatter_unitarity())
        assert np.float32(Oracle.stub_unitarity(3.0, False)) == np.float32(RefSolver.stub_unitarity(3.0))


@pytest.mark.skipif(not ref_available(), reason="reference library not built here")
def test_waveforms_match_reference(built):
    for wf in (0, 1, 2):
        R, O = RefSolver(), Oracle(False)
        for S in (R, O):
            S.setup(4, 4, 4, np.zeros(64, np.uint8), [], dl=2.5e-3, f0=1.3e9, waveform=wf)
        for n in (0, 1, 7, 100, 523, 4000):
            assert np.float32(R.waveform(n)) == np.float32(O.waveform(n)), (wf, n)


def test_fp64_oracle_tracks_fp32(built):
    w = CASES[3]
    a = _run_oracle(w, fp64=False)
    b = _run_oracle(w, fp64=True)
    pa, pb = a.pulses().astype(np.float64), b.pulses()
    assert np.abs(pa - pb).max() <= 1e-4 * np.abs(pb).max()
    ra, rb = drive.records(a, w), drive.records(b, w)
    ez_a, ez_b = ra["probe0_ez"].astype(np.float64), rb["probe0_ez"]
    assert np.abs(ez_a - ez_b).max() <= 1e-4 * max(np.abs(ez_b).max(), 1e-30)


def test_port_loop_outside_grid_is_refused(built):
    """The reference reads out of bounds here (TlmSolver.cpp:695-698); the
    oracle refuses the port, as the product does."""
    S = Oracle(False)
    S.setup(5, 5, 5, np.zeros(125, np.uint8), [])
    assert S.add_port(np.array([0], np.uint64), 2, 1.0) == -1
    assert S.add_port(np.array([62], np.uint64), 2, 1.0) == 0


SURFACE_KEYS_EXACT = ("face_cells", "face_axis", "face_sign", "face_center", "js_instant", "js_re", "js_im",
                      "js_mag", "js_samples", "huy_cells", "huy_axis", "huy_sign", "huy_pos", "huy_acc",
                      "huy_samples", "plane", "plane_axis", "plane_index", "frame_steps", "frame_js", "far_U",
                      "far_u_max", "far_directivity", "far_peak", "frame_last_plane", "frame_last_plane_step")


@pytest.mark.parametrize("w", surface_cases(), ids=[w.name for w in surface_cases()])
def test_surface_monitors_bitwise_vs_reference_golden(built, w):
    """PEC-surface |Js| and its DFT, Huygens phasors, the cut plane, frames and
    the far field of the float oracle equal the reference's, bit for bit."""
    from tests.golden.make_golden import surface_record
    g = golden(w.name)
    O = Oracle(False)
    drive.setup(O, w)
    drive.advance(O, w, w.steps)
    got = surface_record(O)
    for k in SURFACE_KEYS_EXACT:
        if k in g:
            assert np.array_equal(np.asarray(got[k]).astype(np.asarray(g[k]).dtype), g[k]), k


@pytest.mark.skipif(not ref_available(), reason="reference library not built here")
@pytest.mark.parametrize("seed", [21, 22])
def test_surface_monitors_live_reference(built, seed):
    from tests.golden.make_golden import surface_record
    rng = np.random.default_rng(seed)
    nx, ny, nz = (int(v) for v in rng.integers(14, 26, 3))
    w = workloads.random_dipole(rng, nx, ny, nz, 60, name="live")
    w.meta.update(settle_steps=int(rng.integers(0, 30)), huy_offset=2, record_every=int(rng.integers(3, 9)),
                  field_plane=(int(rng.integers(0, 3)), int(rng.integers(0, 12))), surface_monitors=True)
    recs = []
    for S in (RefSolver(), Oracle(False)):
        drive.setup(S, w)
        drive.advance(S, w, w.steps)
        recs.append(surface_record(S))
    for k in SURFACE_KEYS_EXACT:
        if k in recs[0]:
            assert np.array_equal(np.asarray(recs[1][k]).astype(np.asarray(recs[0][k]).dtype), recs[0][k]), k
