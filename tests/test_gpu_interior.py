"""The interior-tile body of the step kernel on a B200.

Tiles away from the y/z faces, PEC and sources take a second step body (all
pulse loads first, packed FP32x2 scatter of node pairs); in FP32 those off
the outer y/z faces are staged in shared memory by bulk copies first. On
grids that hold such tiles: FP32 storage is bitwise the reference's CPU step
(oracle), and for every storage mode and tile shape the interior body gives
bitwise the state and records of the general body (tlm_config.general_tiles
= 1), staged or not (tlm_config.no_staging = 1)."""
import numpy as np
import pytest

from emsolver_b200 import _lib
from emsolver_b200.runner import build_solver, records
from emsolver_b200.solver import Storage
from oracle import Oracle, drive
from emsolver_b200 import workloads
from tests.golden.cases import interior_tiles, mid_cases, staged_tiles, stub_tile_counts

pytestmark = pytest.mark.gpu

MID = mid_cases()


def test_mid_cases_hold_interior_tiles():
    for w in MID:
        assert interior_tiles(w) > 0 and interior_tiles(w, V=2) > 0 and interior_tiles(w, V=8) > 0
        assert staged_tiles(w) > 0


def pair_variant(storage):
    """The tile shape with 2 nodes per thread and the select scatter (the one
    staged tiles run in)."""
    L = _lib.load()
    for v in range(L.tlm_kernel_variants(int(storage))):
        V, minb = _lib.C.c_int(0), _lib.C.c_int(0)
        L.tlm_kernel_variant_info(int(storage), v, _lib.C.byref(V), _lib.C.byref(minb))
        if V.value == 2 and minb.value == 4:
            return v
    raise AssertionError("no 2-node shape")


@pytest.mark.parametrize("storage,rounding", [(Storage.F32, 0), (Storage.F16, 0), (Storage.BF16, 0),
                                              (Storage.F16, 1)])
@pytest.mark.parametrize("case", ["heterogeneous", "mid", "air_odd"])
def test_staged_tiles_equal_direct_loads(built, case, storage, rounding):
    """Staged interior tiles (FP32: 2 nodes per thread; FP16/BF16: 4) against
    the same tiles loading directly: pulses, stubs and every record (energy
    included) bitwise, with round-to-nearest and stochastic 16-bit stores."""
    if case == "heterogeneous":
        w = workloads.heterogeneous(n=96, steps=48)
    elif case == "mid":
        w = MID[0]
    else:
        w = slab_dipole()
    assert staged_tiles(w) > 0
    out = []
    v = pair_variant(storage) if storage == Storage.F32 else 0   # the staged shapes
    for no_staging in (True, False):
        s = build_solver(w, storage=storage, kernel_variant=v, no_staging=no_staging, rounding=rounding,
                         pulse_scale=2.0 ** -10 if storage != Storage.F32 else 0.0)
        s.step(w.steps)
        out.append((s.pulses(), s.stubs() if w.table else None, records(s, w, f64=True)))
        s.close()
    (pa, sa, ra), (pb, sb, rb) = out
    assert np.array_equal(pa, pb)
    if sa is not None:
        assert np.array_equal(sa, sb)
    for k in ra:
        assert np.array_equal(ra[k], rb[k]), k


def slab_dipole():
    """A dipole beside a thin dielectric slab (9 of 61 nodes of every row):
    staged tiles whose few stub-loaded nodes load their stubs directly."""
    return workloads.dipole(61, 70, 33, 20, slab=(3, 12, 4.0), steps=40, name="odd")


def test_cases_hold_sparse_and_dense_stub_tiles():
    sparse, dense = stub_tile_counts(slab_dipole())
    assert sparse > 0
    sparse, dense = stub_tile_counts(workloads.heterogeneous(n=96, steps=48))
    assert sparse > 0 and dense > 0


def test_sparse_stub_tiles_bitwise_vs_oracle(built):
    """Staged tiles with stubs loaded directly (kTileStubSparse) and staged
    (the dense ones), FP32: pulses, stubs and records bitwise the oracle."""
    for w in (slab_dipole(), workloads.heterogeneous(n=64, steps=30)):
        assert stub_tile_counts(w)[0] > 0
        s = build_solver(w, kernel_variant=pair_variant(Storage.F32))
        s.step(w.steps)
        O = Oracle(False)
        drive.setup(O, w)
        drive.advance(O, w, w.steps)
        assert np.array_equal(s.pulses(), O.pulses()), w.name
        assert np.array_equal(s.stubs(), O.stubs()), w.name
        ra, ro = records(s, w), drive.records(O, w)
        for k in ra:
            if not k.startswith("energy"):
                assert np.array_equal(ra[k], ro[k]), (w.name, k)
        s.close()


@pytest.mark.parametrize("w", MID, ids=[w.name for w in MID])
def test_interior_tiles_bitwise_vs_oracle(built, w):
    s = build_solver(w)
    s.step(w.steps)
    O = Oracle(False)
    drive.setup(O, w)
    drive.advance(O, w, w.steps)
    assert np.array_equal(s.pulses(), O.pulses())
    if w.table:
        assert np.array_equal(s.stubs(), O.stubs())
    ra, ro = records(s, w), drive.records(O, w)
    for k in ra:
        if k.startswith("energy"):
            continue
        assert np.array_equal(ra[k], ro[k]), k


@pytest.mark.parametrize("storage", [Storage.F32, Storage.BF16, Storage.F16, Storage.BFP16, Storage.F64])
@pytest.mark.parametrize("rounding", [0, 1])
def test_interior_body_equals_general_body(built, storage, rounding):
    if storage in (Storage.F32, Storage.F64) and rounding:
        pytest.skip("rounding applies to 16-bit storage")
    L = _lib.load()
    w = MID[0]
    for v in range(L.tlm_kernel_variants(int(storage))):
        out = []
        for general in (True, False):
            s = build_solver(w, storage=storage, kernel_variant=v, rounding=rounding, general_tiles=general)
            s.step(w.steps)
            out.append((s.pulses(f64=True), s.stubs(), records(s, w, f64=True)))
            s.close()
        (pa, sa, ra), (pb, sb, rb) = out
        assert np.array_equal(pa, pb), (storage, v)
        assert np.array_equal(sa, sb), (storage, v)
        for k in ra:
            assert np.array_equal(ra[k], rb[k]), (storage, v, k)


def test_stage_wait_running_out_fails_the_step(built):
    """A stage wait that runs out (tlm_config.stage_wait_us < 0: give up at
    the first poll that finds the stage not ready) sets the kernel's fault
    flag instead of hanging: the step returns TLM_ECUDA with the wait's
    message, and the device stays usable -- a fresh handle then steps the
    same grid bitwise like a handle that loads its pulses directly."""
    w = workloads.heterogeneous(n=96, steps=24)
    v = pair_variant(Storage.F32)
    assert staged_tiles(w) > 0
    s = build_solver(w, kernel_variant=v, stage_wait_us=-1)
    with pytest.raises(_lib.TlmError) as err:
        s.step(1)
    assert err.value.status == _lib.TLM_ECUDA
    assert "never arrived" in str(err.value)
    s.close()
    out = []
    for no_staging in (False, True):
        r = build_solver(w, kernel_variant=v, no_staging=no_staging)
        r.step(w.steps)
        out.append((r.pulses(), r.stubs(), records(r, w, f64=True)))
        r.close()
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1])
    for k in out[0][2]:
        assert np.array_equal(out[0][2][k], out[1][2][k]), k
