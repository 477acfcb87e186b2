"""Batched execution on a B200: every member of a batch gives bitwise the
results it gives stepped alone -- with uneven grid sizes and step counts,
members joining and leaving mid-run, mixed storage modes, CUDA graphs on and
off, and after the autotuner has re-shaped the kernels."""
import numpy as np
import pytest

from emsolver_b200 import Batch, BatchTuning, workloads
from emsolver_b200._lib import TLM_EBUSY, TLM_ESTATE, TlmError
from emsolver_b200.runner import build_solver, records
from emsolver_b200.solver import Storage

pytestmark = pytest.mark.gpu


def instances(count, seed, lo=16, hi=40, steps=(150, 330)):
    rng = np.random.default_rng(seed)
    out = []
    for b in range(count):
        nx, ny, nz = (int(v) for v in rng.integers(lo, hi + 1, 3))
        w = workloads.random_dipole(rng, nx, ny, nz, int(rng.integers(*steps)), name=f"m{b}")
        w.dft_freqs = w.dft_freqs[:8]
        out.append(w)
    return out


def alone(w, storage=0):
    s = build_solver(w, storage=storage)
    s.step(w.steps)
    return s.pulses(f64=True), records(s, w, f64=True)


def assert_same(s, w, ref, energy_rtol=0.0):
    """Pulses and records bitwise; the FP64 energy sum also bitwise unless the
    tile shape differs from the reference run's (its reduction follows the
    tiles), in which case it agrees to `energy_rtol`."""
    p, r = ref
    assert s.currentStep() == w.steps
    assert np.array_equal(s.pulses(f64=True), p), w.name
    got = records(s, w, f64=True)
    for k in got:
        if k == "energy" and energy_rtol > 0:
            assert np.allclose(got[k], r[k], rtol=energy_rtol, atol=0), (w.name, k)
        else:
            assert np.array_equal(got[k], r[k]), (w.name, k)
    v, i = s.portDft(0)
    return v, i


@pytest.mark.parametrize("graphs,window,overlap", [(True, 64, False), (False, 64, False), (True, 16, False),
                                                    (True, 100, False), (True, 64, True), (False, 64, True)])
def test_batch_members_equal_alone(built, graphs, window, overlap):
    """overlap: the general tiles on a second stream beside the staged ones."""
    ws = instances(7, seed=1)
    refs = [alone(w) for w in ws]
    solvers = [build_solver(w) for w in ws]
    with Batch() as b:
        b.set_tuning(BatchTuning(0, window, 0, graphs, overlap))
        assert b.get_tuning().overlap == overlap
        for s in solvers:
            b.attach(s)
        assert b.size() == 7 and b.active() == 7
        b.run()
        assert b.active() == 0
        for s, w, ref in zip(solvers, ws, refs):
            assert_same(s, w, ref)
            # the port DFT equals the DFT of the same handle stepped alone
            s2 = build_solver(w)
            s2.step(w.steps)
            v1, i1 = s.portDft(0)
            v2, i2 = s2.portDft(0)
            assert np.array_equal(v1, v2) and np.array_equal(i1, i2)


def test_members_join_and_leave_mid_run(built):
    ws = instances(6, seed=2)
    refs = [alone(w) for w in ws]
    solvers = [build_solver(w) for w in ws]
    with Batch() as b:
        for s in solvers[:3]:
            b.attach(s)
        b.step(70)                 # not a multiple of the window
        b.attach(solvers[3])       # joins at its own step 0
        b.step(64)
        b.detach(solvers[0])       # leaves mid-run ...
        solvers[0].step(ws[0].steps - solvers[0].currentStep())   # ... and finishes alone
        b.attach(solvers[4])
        b.attach(solvers[5])
        b.run()
    for s, w, ref in zip(solvers, ws, refs):
        assert_same(s, w, ref)


def test_mixed_storage_batch(built):
    ws = instances(5, seed=3)
    modes = [Storage.F32, Storage.BF16, Storage.F16, Storage.F64, Storage.BFP16]
    refs = [alone(w, m) for w, m in zip(ws, modes)]
    solvers = [build_solver(w, storage=m) for w, m in zip(ws, modes)]
    with Batch() as b:
        for s in solvers:
            b.attach(s)
        b.run()
    for s, w, ref in zip(solvers, ws, refs):
        assert_same(s, w, ref)


def test_autotune_then_run(built):
    ws = instances(5, seed=4)
    refs = [alone(w) for w in ws]
    solvers = [build_solver(w) for w in ws]
    with Batch() as b:
        for s in solvers:
            b.attach(s)
        t = b.autotune(trial_windows=1)
        assert t.ms_per_step > 0 and t.steps_per_launch in (50, 100, 200)
        for s in solvers:
            assert s.currentStep() == 0
        b.run()
    for s, w, ref in zip(solvers, ws, refs):
        assert_same(s, w, ref, energy_rtol=1e-12)


def test_batch_state_rules(built):
    w = instances(1, seed=5)[0]
    s = build_solver(w)
    with Batch() as b:
        b.attach(s)
        with pytest.raises(TlmError) as e:
            b.attach(s)
        assert e.value.status == TLM_ESTATE
        with pytest.raises(TlmError) as e:
            s.step(1)
        assert e.value.status == TLM_ESTATE
        with pytest.raises(TlmError) as e:
            s.close()
        assert e.value.status == TLM_EBUSY
        b.step(10)
        assert s.currentStep() == 10
    s.step(5)          # detached by the batch's destruction: steps alone again
    assert s.currentStep() == 15


def test_pipelined_solve_equals_alone(built):
    """Batch.solve (set-up of the next chunk overlapping the device's window,
    members collected and freed as they finish): every port DFT and record
    bitwise what the instance gives alone."""
    ws = workloads.batched_instances(count=10, steps=150, lo=20, hi=40)
    for k, w in enumerate(ws):
        w.steps = 100 + 13 * k           # members finish in different windows
    alone = []
    for w in ws:
        s = build_solver(w)
        s.step(w.steps)
        alone.append((s.portDft(0), records(s, w, f64=True)))
        s.close()
    with Batch() as b:
        got = b.solve(ws, build_solver, lambda s, w: (s.portDft(0), records(s, w, f64=True)), chunk=3)
    assert len(got) == len(ws)
    for (da, ra), (dg, rg) in zip(alone, got):
        for x, y in zip(da, dg):
            assert np.array_equal(x, y)
        for key in ra:
            assert np.array_equal(ra[key], rg[key]), key
