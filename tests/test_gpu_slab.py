"""A grid split into z-slabs, every slab a B200 solver with ghost planes,
the halo messages traded between steps: either after whole steps
(tlm_halo_pack / tlm_halo_unpack) or overlapped with the step, which then
runs in two launches (tlm_slab_step_begin: the planes next to a ghost plane
and their outgoing halo; tlm_slab_step_end: the received halo and the other
planes).

One GPU here holds every slab: the slabs step one after the other and the
messages are copied between their buffers with the device idle in between
(no kernel waits on another). Bar: the pulses of every slab's own planes and
every port and probe record bitwise those of the undivided grid; the summed
energy history within 1e-12 relative (FP64 sums in another order)."""
import numpy as np
import pytest
import torch

from emsolver_b200 import Batch, workloads
from emsolver_b200._lib import TLM_EINVAL, TLM_ESTATE, TlmError
from emsolver_b200.runner import build_solver, records
from emsolver_b200.slab import DeviceSlab, monitor_intervals, slab_workload, split_planes
from emsolver_b200.solver import Storage

pytestmark = pytest.mark.gpu


def run_split(w, parts, steps, overlapped=False, **kw):
    ranges = split_planes(w.nz, parts, monitor_intervals(w))
    slabs, bufs = [], []
    for k0, k1 in ranges:
        v, glo, ghi, lo = slab_workload(w, k0, k1)
        s = DeviceSlab(v, glo, ghi, 0, **kw)
        slabs.append((s, v, glo, ghi, lo, k0, k1))
        bufs.append({key: (s.buffer() if (glo if key.endswith("lo") else ghi) else None)
                     for key in ("send_lo", "recv_lo", "send_hi", "recv_hi")})

    def trade():
        torch.cuda.synchronize()
        for r in range(len(slabs) - 1):
            bufs[r + 1]["recv_lo"].copy_(bufs[r]["send_hi"])
            bufs[r]["recv_hi"].copy_(bufs[r + 1]["send_lo"])
        torch.cuda.synchronize()

    for _ in range(steps):
        if overlapped:
            for (s, *_), b in zip(slabs, bufs):
                s.begin(b["send_lo"], b["send_hi"])
            trade()
            for (s, *_), b in zip(slabs, bufs):
                s.end(b["recv_lo"], b["recv_hi"])
            continue
        for s, *_ in slabs:
            s.step1()
        for (s, *_), b in zip(slabs, bufs):
            s.pack(b["send_lo"], b["send_hi"])
        trade()
        for (s, *_), b in zip(slabs, bufs):
            s.unpack(b["recv_lo"], b["recv_hi"])
    for s, *_ in slabs:
        if overlapped:
            s.flush()
        s.finish()
    return slabs


def check_split(w, parts, steps, f64=False, overlapped=False, **kw):
    whole = build_solver(w, **kw)
    whole.step(steps)
    ref = records(whole, w, f64=True)
    ref_p = whole.pulses(f64=f64).reshape(w.nz, w.ny * w.nx, 12)
    slabs = run_split(w, parts, steps, overlapped, **kw)
    energy = np.zeros_like(ref["energy"])
    for s, v, glo, ghi, lo, k0, k1 in slabs:
        p = s.solver.pulses(f64=f64).reshape(v.nz, v.ny * v.nx, 12)
        assert np.array_equal(p[glo:v.nz - ghi], ref_p[k0:k1]), (k0, k1)
        rec = s.records()
        for lp, gp in enumerate(v.port_ids):
            assert np.array_equal(rec[f"port{lp}_v"], ref[f"port{gp}_v"])
            assert np.array_equal(rec[f"port{lp}_i"], ref[f"port{gp}_i"])
        for lq, gq in enumerate(v.probe_ids):
            for c in ("ex", "ey", "ez"):
                assert np.array_equal(rec[f"probe{lq}_{c}"], ref[f"probe{gq}_{c}"])
        assert np.array_equal(rec["energy_steps"], ref["energy_steps"])
        energy += rec["energy"]
        s.close()
    assert np.abs(energy - ref["energy"]).max() <= 1e-12 * np.abs(ref["energy"]).max()
    whole.close()


def dipole_workload(seed, nx=26, ny=24, nz=41, steps=120):
    rng = np.random.default_rng(seed)
    w = workloads.random_dipole(rng, nx, ny, nz, steps, name="split")
    w.rho = 0.3
    w.probes_cell = [tuple(int(rng.integers(0, d)) for d in (nx, ny, nz)) for _ in range(6)] + [(3, 4, 0),
                                                                                                (5, 6, nz - 1)]
    return w


@pytest.mark.parametrize("overlapped", [False, True])
@pytest.mark.parametrize("parts", [2, 3, 5])
def test_split_f32_bitwise(built, parts, overlapped):
    check_split(dipole_workload(parts), parts, 120, overlapped=overlapped)


def test_split_overlapped_staged_tiles_and_partial_window(built):
    """A slab grid large enough that its interior planes hold staged tiles,
    stepped a number of steps that leaves a partial launch window."""
    w = dipole_workload(8, 70, 64, 36, 150)
    check_split(w, 3, 150, overlapped=True)


@pytest.mark.parametrize("overlapped", [False, True])
@pytest.mark.parametrize("storage,kw", [(Storage.F64, {}), (Storage.BFP16, {}),
                                        (Storage.F16, {"pulse_scale": 2.0 ** -10})])
def test_split_storage_modes_bitwise(built, storage, kw, overlapped):
    w = dipole_workload(11, 18, 17, 29, 80)
    w.storage = int(storage)
    check_split(w, 3, 80, f64=storage == Storage.F64, overlapped=overlapped, **kw)


@pytest.mark.parametrize("prop", [0, 2])
def test_split_with_plane_wave_through_a_boundary(built, prop):
    w = dipole_workload(5, 20, 18, 30, 90)
    ranges = split_planes(w.nz, 3, monitor_intervals(w))
    w.meta["plane_wave"] = (prop, ranges[1][0] - 1 if prop == 2 else 4, 1, 0.7)
    check_split(w, 3, 90)


def test_slab_misuse_is_refused(built):
    w = dipole_workload(2, 16, 14, 20, 20)
    v, glo, ghi, lo = slab_workload(w, 8, 14)
    s = build_solver(v)
    s.setSlab(glo, ghi)
    s.addProbeCell(2, 2, 0)                        # in the low ghost plane
    with pytest.raises(TlmError) as e:
        s.step(1)
    assert e.value.status == TLM_EINVAL
    s = build_solver(v)
    s.step(1)
    with pytest.raises(TlmError) as e:
        s.setSlab(glo, ghi)
    assert e.value.status == TLM_ESTATE
    s = build_solver(v)
    s.setSlab(glo, ghi)
    with pytest.raises(TlmError) as e:
        s.haloPack(None, None)                     # both sides have neighbours
    assert e.value.status == TLM_EINVAL
    b = Batch()
    with pytest.raises(TlmError):
        b.attach(s)
    v.storage = int(Storage.F16)
    s = build_solver(v)
    with pytest.raises(TlmError) as e:
        s.setSlab(glo, ghi)                        # 16-bit slabs need a shared scale
    assert e.value.status == TLM_EINVAL
