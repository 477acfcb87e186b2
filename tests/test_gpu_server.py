"""The continuous-batching request server on a B200.

Each served result equals the same solve run alone (bitwise: port DFT and
port records), whatever else is in the mix; admission never exceeds the HBM
budget; requests that arrive while others run join them; cancellation and
bad requests are reported without disturbing the rest."""
import time

import numpy as np
import pytest

from emsolver_b200 import Server, workloads
from emsolver_b200._lib import TLM_ENOMEM, TlmError
from emsolver_b200.runner import build_solver
from emsolver_b200.server import CANCELLED, DONE, FAILED, footprint

pytestmark = pytest.mark.gpu


def requests(count, seed, lo=16, hi=36, steps=(120, 400)):
    rng = np.random.default_rng(seed)
    out = []
    for r in range(count):
        e = int(rng.integers(lo, hi + 1))
        w = workloads.random_dipole(rng, e, e, e, int(rng.integers(*steps)),
                                    storage=int(rng.integers(0, 2)), name=f"r{r}")
        w.dft_freqs = w.dft_freqs[:8]
        out.append(w)
    return out


def solve_alone(w):
    s = build_solver(w)
    s.step(w.steps)
    v, i = s.portDft(0)
    port = s.port(0)
    s.close()
    return v, i, port.vRec, port.iRec


def test_served_results_equal_alone_with_staggered_arrivals(built):
    ws = requests(10, seed=7)
    with Server() as srv:
        ids = []
        for k, w in enumerate(ws):
            ids.append(srv.submit(w))
            if k % 3 == 2:
                time.sleep(0.01)          # later requests arrive while earlier ones run
        for rid in ids:
            assert srv.wait(rid, 120.0) == DONE
        for rid, w in zip(ids, ws):
            v, i, lat = srv.result(rid)
            vr, ir = srv.port_records(rid)
            av, ai, avr, air = solve_alone(w)
            assert np.array_equal(v, av) and np.array_equal(i, ai), w.name
            assert np.array_equal(vr, avr) and np.array_equal(ir, air), w.name
            assert lat > 0
        st = srv.stats()
        assert st["completed"] == 10 and st["failed"] == 0
        assert st["latency_p99_s"] >= st["latency_p50_s"] > 0


def test_admission_respects_budget(built):
    ws = requests(6, seed=8, lo=28, hi=32, steps=(200, 260))
    budget = int(2.5 * max(footprint(w) for w in ws))
    most = budget // min(footprint(w) for w in ws)
    with Server(hbm_budget=budget) as srv:
        ids = [srv.submit(w) for w in ws]
        peak = 0
        while srv.stats()["completed"] < len(ws):
            st = srv.stats()
            peak = max(peak, st["hbm_used_bytes"])
            assert st["hbm_used_bytes"] <= budget
            assert st["running"] <= most
            time.sleep(0.002)
        assert peak > 0
        for rid in ids:
            assert srv.poll(rid) == DONE


def test_cancel_and_bad_request(built):
    ws = requests(4, seed=9, steps=(3000, 3001))
    bad = requests(1, seed=10)[0]
    bad.mat = bad.mat.copy()
    bad.mat[5] = 9                       # dielectric id with no table entry
    with Server() as srv:
        ids = [srv.submit(w) for w in ws]
        bid = srv.submit(bad)
        srv.cancel(ids[1])                # running or queued: ends cancelled
        assert srv.wait(bid, 60.0) == FAILED
        assert srv.wait(ids[1], 60.0) == CANCELLED
        for rid in (ids[0], ids[2], ids[3]):
            assert srv.wait(rid, 120.0) == DONE
        with pytest.raises(TlmError):
            srv.result(bid)


def test_oversized_request_is_refused(built):
    w = requests(1, seed=11)[0]
    with Server(hbm_budget=footprint(w) // 2) as srv:
        with pytest.raises(TlmError) as e:
            srv.submit(w)
        assert e.value.status == TLM_ENOMEM


def test_destroy_cancels_pending(built):
    ws = requests(3, seed=12, steps=(5000, 5001))
    srv = Server(hbm_budget=int(1.2 * footprint(ws[0])))
    for w in ws:
        srv.submit(w)
    srv.close()                           # must not hang with work queued


def test_least_work_first_admission(built):
    """With a running-cells cap that fits one request at a time, a short
    request queued behind a long one is admitted first under the least-work
    order (and finishes first), and after it under the arrival order; both
    results equal the solves run alone."""
    rng = np.random.default_rng(12)
    blocker = workloads.random_dipole(rng, 40, 40, 40, 600, name="blocker")
    long_w = workloads.random_dipole(rng, 40, 40, 40, 600, name="long")
    short_w = workloads.random_dipole(rng, 24, 24, 24, 150, name="short")
    for w in (blocker, long_w, short_w):
        w.dft_freqs = w.dft_freqs[:8]
    for order, short_first in ((Server.LEAST_WORK, True), (Server.ARRIVAL, False)):
        with Server() as srv:
            srv.set_policy(order, 1, 0)           # one request at a time, all in the batch
            ids = [srv.submit(w) for w in (blocker, long_w, short_w)]
            for rid in ids:
                assert srv.wait(rid, 120.0) == DONE
            lat = {w.name: srv.result(rid)[2] for rid, w in zip(ids, (blocker, long_w, short_w))}
            assert (lat["short"] < lat["long"]) == short_first, (order, lat)
            for rid, w in zip(ids, (blocker, long_w, short_w)):
                v, i, _ = srv.result(rid)
                av, ai, _, _ = solve_alone(w)
                assert np.array_equal(v, av) and np.array_equal(i, ai), (order, w.name)


def test_solo_lane_results_equal_alone(built):
    """Requests at or above the solo size run on their own stream beside the
    batch (here: every request of at least 30^3 cells); all results, solo
    and batched, equal the solves run alone."""
    ws = requests(6, seed=21, lo=20, hi=40)
    with Server() as srv:
        srv.set_policy(Server.LEAST_WORK, 0, 30 ** 3)
        ids = [srv.submit(w) for w in ws]
        for rid in ids:
            assert srv.wait(rid, 120.0) == DONE
        for rid, w in zip(ids, ws):
            v, i, _ = srv.result(rid)
            vr, ir = srv.port_records(rid)
            av, ai, avr, air = solve_alone(w)
            assert np.array_equal(v, av) and np.array_equal(i, ai), w.name
            assert np.array_equal(vr, avr) and np.array_equal(ir, air), w.name
