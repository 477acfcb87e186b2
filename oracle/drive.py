"""Feed a synthetic Workload to an oracle solver (TEST INFRASTRUCTURE ONLY).

Works for both ``Oracle`` (the restatement) and ``RefSolver`` (the reference
compiled headless): same setup, ports, probes (at cell centres, through the
world-position addProbe of TlmSolver.cpp:377-391) and source values.
"""
from __future__ import annotations

import numpy as np


def setup(S, w, settle_steps=None):
    """Settle steps, Huygens inset, frame period and cut plane come from
    ``w.meta`` ("settle_steps", "huy_offset", "record_every", "field_plane")
    when present."""
    wf = w.waveform if w.waveform != 3 else 2
    if settle_steps is None:
        settle_steps = w.meta.get("settle_steps", 0)
    S.setup(w.nx, w.ny, w.nz, w.mat, w.table, origin=w.origin, dl=w.dl, f0=w.f0, waveform=wf,
            total_steps=w.steps, settle_steps=settle_steps, rho=w.rho,
            huy_offset=w.meta.get("huy_offset", 0), record_every=w.meta.get("record_every", 0))
    if "field_plane" in w.meta:
        S.set_field_plane(*w.meta["field_plane"])
    port_idx = [S.add_port(np.asarray(cells, np.uint64), pol, amp) for cells, pol, amp in w.ports]
    probe_idx = [S.add_probe(*w.cell_center(i, j, k)) for (i, j, k) in w.probes_cell]
    return port_idx, probe_idx


def advance(S, w, count):
    """Advance `count` steps from the solver's current step."""
    if w.waveform == 3:
        n0 = S.step_index
        sv = np.zeros(count, np.float64)
        avail = max(0, min(count, len(w.sv) - n0))
        sv[:avail] = w.sv[n0:n0 + avail]
        S.steps(count, sv=sv)
    else:
        S.steps(count)


def run(S, w, steps=None):
    setup(S, w)
    advance(S, w, w.steps if steps is None else steps)
    return S


def records(S, w):
    out = {}
    for p in range(len(w.ports)):
        v, i = S.port(p)
        out[f"port{p}_v"] = v
        out[f"port{p}_i"] = i
    for q in range(len(w.probes_cell)):
        ex, ey, ez = S.probe(q)
        out[f"probe{q}_ex"] = ex
        out[f"probe{q}_ey"] = ey
        out[f"probe{q}_ez"] = ez
    st, ev = S.energy_history()
    out["energy_steps"] = st
    out["energy"] = ev
    return out
