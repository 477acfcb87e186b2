"""FP16/BF16 pulse storage with a near-field box (tlm_config.near_field) on a
B200.

Cells of the box keep the FP32 residual of their stored pulses, so that
decode(stored) + residual is exactly the FP32 pulse, and step as FP32
storage would; the rest of the grid is stored in 16 bits. Checks: a box that
covers the whole grid steps bitwise as FP32 storage (every read is then
exact); the S11 of dipole instances of the batched workload stays within
1e-3 (relative) of the FP64 storage mode, which is
itself bitwise the FP64 oracle; a state written by tlm_set_pulses reads back
exactly inside the box and rounded to 16 bits outside; batch members with a
box give bitwise the results they give alone.
"""
import numpy as np
import pytest

from emsolver_b200 import Batch, workloads
from emsolver_b200._lib import TLM_EINVAL, TlmError
from emsolver_b200.runner import build_solver, records
from emsolver_b200.solver import Storage, s11_from_dft
from tests.golden.cases import small_cases

pytestmark = pytest.mark.gpu

S11_TOL = 1e-3        # relative S11 error against the FP64 storage mode
NEAR = 6              # box radius in cells


def s11_of(w, **kw):
    s = build_solver(w, **kw)
    s.step(w.steps)
    v, i = s.portDft(0)
    s.close()
    return s11_from_dft(v, i)[1]


@pytest.mark.parametrize("storage", [Storage.F16, Storage.BF16])
def test_box_over_the_whole_grid_steps_as_fp32(built, storage):
    """Every cell in the box: pulses and records bitwise those of FP32
    storage (energy to the usual 1e-6: the reduction follows the tiles)."""
    w = small_cases()[3]
    ref = build_solver(w, storage=Storage.F32)
    ref.step(w.steps)
    s = build_solver(w, storage=storage, near_field=10 ** 6)
    s.step(w.steps)
    assert np.array_equal(s.pulses(f64=True), ref.pulses(f64=True))
    assert np.array_equal(s.stubs(), ref.stubs())
    ra, rb = records(s, w, f64=True), records(ref, w, f64=True)
    for k in ra:
        if k == "energy":
            assert np.allclose(ra[k], rb[k], rtol=1e-6, atol=0), k
        else:
            assert np.array_equal(ra[k], rb[k]), k


def test_fp16_near_field_s11_within_bar_on_dipoles(built):
    """Dipoles of the batched workload (edges U{24..96}, 1000 steps): FP16
    storage with a box of radius 6 keeps S11 within 1e-3 of the FP64 mode
    at every DFT frequency, where plain FP16 storage does not."""
    worst, worst_plain = 0.0, 0.0
    for w in workloads.batched_instances(count=6, steps=1000)[:6:2]:
        ref = s11_of(w, storage=Storage.F64)
        nf = s11_of(w, storage=Storage.F16, near_field=NEAR)
        plain = s11_of(w, storage=Storage.F16)
        worst = max(worst, float(np.max(np.abs(nf - ref) / np.abs(ref))))
        worst_plain = max(worst_plain, float(np.max(np.abs(plain - ref) / np.abs(ref))))
    assert worst <= S11_TOL, (worst, worst_plain)
    assert worst < worst_plain


def test_near_field_state_round_trip(built):
    """tlm_set_pulses then tlm_get_pulses: box cells exactly the written
    FP32 values, other cells an FP16 value within half an FP16 step of the
    written one (scale 1), PEC cells 0."""
    w = workloads.dipole(24, 20, 30, 11, steps=10)
    s = build_solver(w, storage=Storage.F16, near_field=2, pulse_scale=1.0)
    nx, ny, nz = w.nx, w.ny, w.nz
    rng = np.random.default_rng(7)
    x = (rng.standard_normal((nz, ny, nx, 12)) * 0.3).astype(np.float32)
    s.setPulses(x.reshape(-1))
    got = s.pulses().reshape(nz, ny, nx, 12)
    mat = np.asarray(w.mat).reshape(nz, ny, nx)
    pec = mat == 1
    k, j, i = np.nonzero(pec)
    (cells, _, _), = w.ports
    c = cells[0]
    pts = np.array(list(zip(k, j, i)) + [(c // (nx * ny), c // nx % ny, c % nx)])
    lo = np.maximum(pts.min(0) - 2, 0)
    hi = np.minimum(pts.max(0) + 2, [nz - 1, ny - 1, nx - 1])
    box = np.zeros((nz, ny, nx), bool)
    box[lo[0]:hi[0] + 1, lo[1]:hi[1] + 1, lo[2]:hi[2] + 1] = True
    live = ~pec
    inside = box & live
    outside = ~box & live
    assert np.array_equal(got[inside], x[inside])
    assert np.all(got[pec] == 0.0)
    g, v = got[outside].astype(np.float64), x[outside].astype(np.float64)
    assert np.array_equal(g, g.astype(np.float16).astype(np.float64))   # FP16 values
    step = np.exp2(np.floor(np.log2(np.maximum(np.abs(v), 2.0 ** -14))) - 10)
    assert np.all(np.abs(g - v) <= step / 2)


def test_near_field_batch_members_equal_alone(built):
    rng = np.random.default_rng(31)
    ws = []
    for b in range(3):
        nx, ny, nz = (int(v) for v in rng.integers(20, 40, 3))
        w = workloads.random_dipole(rng, nx, ny, nz, int(rng.integers(120, 200)), name=f"nf{b}")
        w.dft_freqs = w.dft_freqs[:8]
        ws.append(w)
    refs = []
    for w in ws:
        s = build_solver(w, storage=Storage.F16, near_field=NEAR)
        s.step(w.steps)
        refs.append((s.pulses(f64=True), records(s, w, f64=True)))
        s.close()
    solvers = [build_solver(w, storage=Storage.F16, near_field=NEAR) for w in ws]
    with Batch() as b:
        for s in solvers:
            b.attach(s)
        b.run()
    for s, w, (p, r) in zip(solvers, ws, refs):
        assert np.array_equal(s.pulses(f64=True), p), w.name
        got = records(s, w, f64=True)
        for k in got:
            assert np.array_equal(got[k], r[k]), (w.name, k)


def test_near_field_needs_16_bit_storage(built):
    w = workloads.dipole(24, 20, 30, 11, steps=10)
    for storage in (Storage.F32, Storage.F64, Storage.BFP16):
        with pytest.raises(TlmError) as err:
            build_solver(w, storage=storage, near_field=3)
        assert err.value.status == TLM_EINVAL
