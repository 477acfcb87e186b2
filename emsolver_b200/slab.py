"""One TLM grid split along z over the ranks of a process group.

The reference runs one grid in one address space and splits the work into
z-slabs over worker threads (TlmSolver.cpp:174-240, 516-613). For a grid too
large for one GPU's HBM, or to bring several GPUs to one grid, each rank here
owns a contiguous range of z-planes as its own solver: the planes plus one
ghost plane on each side that has a neighbour (the neighbour's boundary plane
with its true material). Every step the ranks trade the z-directed pulses
that cross each shared face (two pulse slots of one plane per face and
direction, nx*ny*8 bytes in FP32) with point-to-point sends over the group
(NCCL between GPUs), overlapped with the step: the planes next to a ghost
plane step first and their halo leaves on a stream of its own while the
other planes step (tlm_slab_step_begin / tlm_slab_step_end), and the next
step waits only for the received halo. Nothing else crosses ranks on the
data path; records are gathered once at the end.

Results are bitwise those of the undivided grid for every pulse, probe and
port record (each node's update reads the same values in the same order);
the energy history is the sum of the slabs' FP64 partial sums.

Monitors (probes, ports with their current loops) must not straddle a slab
boundary: ``split_planes`` moves boundaries off their planes.
"""
from __future__ import annotations

import contextlib
import copy
import os

import numpy as np


def monitor_intervals(w):
    """[kmin, kmax] plane intervals that must lie inside one slab: each probe
    cell, and each port's gap cells with the four neighbours of its middle
    cell that the current loop reads (TlmSolver.cpp:677-703)."""
    plane = w.nx * w.ny
    out = [(k, k) for (_, _, k) in w.probes_cell]
    for cells, pol, _ in w.ports:
        ks = [int(c) // plane for c in cells if w.mat.reshape(-1)[int(c)] == 0]
        if not ks:
            continue
        cells_air = [int(c) for c in cells if w.mat.reshape(-1)[int(c)] == 0]
        mid = cells_air[len(cells_air) // 2]
        km = mid // plane
        lo, hi = min(ks), max(ks)
        if pol != 2:  # the loop around an x or y gap crosses z-neighbours
            lo, hi = min(lo, km - 1), max(hi, km + 1)
        out.append((max(lo, 0), min(hi, w.nz - 1)))
    return out


def split_planes(nz, parts, keep=()):
    """Own-plane ranges [(k0, k1)] of `parts` slabs: near-equal sizes, with
    every boundary moved off the inside of the intervals in `keep`."""
    if parts < 1 or parts > nz:
        raise ValueError(f"cannot split {nz} planes into {parts} slabs")
    bounds = [round(r * nz / parts) for r in range(parts + 1)]
    for r in range(1, parts):
        b = bounds[r]
        for _ in range(len(keep) + 1):
            hit = next(((lo, hi) for lo, hi in keep if lo < b <= hi), None)
            if hit is None:
                break
            cands = [c for c in (hit[0], hit[1] + 1) if bounds[r - 1] < c < bounds[r + 1]]
            if not cands:
                break
            b = min(cands, key=lambda c: abs(c - b))
        if any(lo < b <= hi for lo, hi in keep) or not bounds[r - 1] < b < bounds[r + 1]:
            raise ValueError("no slab boundary avoids the monitors; use fewer slabs")
        bounds[r] = b
    return [(bounds[r], bounds[r + 1]) for r in range(parts)]


def slab_workload(w, k0, k1):
    """The workload of the slab owning planes [k0, k1): those planes plus a
    ghost plane on each side with a neighbour. Returns (workload, ghost_lo,
    ghost_hi, first plane held). Ports and probes are kept when they lie in
    the own planes; a z plane wave is kept when its plane is held."""
    glo, ghi = int(k0 > 0), int(k1 < w.nz)
    lo, hi = k0 - glo, k1 + ghi
    plane = w.nx * w.ny
    v = copy.copy(w)
    v.meta = dict(w.meta)
    v.name = f"{w.name}[{k0}:{k1}]"
    v.nz = hi - lo
    v.mat = np.ascontiguousarray(w.mat.reshape(w.nz, w.ny, w.nx)[lo:hi]).reshape(-1)
    o = [np.float32(c) for c in w.origin]
    o[2] = np.float32(o[2] + np.float32(lo) * np.float32(w.dl))
    v.origin = tuple(float(c) for c in o)
    v.ports, v.port_ids = [], []
    for p, (cells, pol, amp) in enumerate(w.ports):
        ks = [int(c) // plane for c in cells]
        if all(k0 <= k < k1 for k in ks):
            v.ports.append(([int(c) - lo * plane for c in cells], pol, amp))
            v.port_ids.append(p)
    v.probes_cell, v.probe_ids = [], []
    for q, (i, j, k) in enumerate(w.probes_cell):
        if k0 <= k < k1:
            v.probes_cell.append((i, j, k - lo))
            v.probe_ids.append(q)
    if "plane_wave" in w.meta:
        prop, index, pol, amp = w.meta["plane_wave"]
        if prop == 2:
            if lo <= index < hi:
                v.meta["plane_wave"] = (prop, index - lo, pol, amp)
            else:
                del v.meta["plane_wave"]
    return v, glo, ghi, lo


class DeviceSlab:
    """A slab on one GPU: the B200 solver with its ghost planes and the
    device buffers of its halo messages."""

    def __init__(self, w, ghost_lo, ghost_hi, device=0, **solver_kw):
        import torch
        from .runner import build_solver
        self.w = w
        self.solver = build_solver(w, device=device, **solver_kw)
        self.solver.setSlab(ghost_lo, ghost_hi)
        self.nbytes = self.solver.haloBytes()
        self.device = torch.device("cuda", device)
        self.stream = torch.cuda.ExternalStream(self.solver.stream(), device=self.device)

    def buffer(self):
        import torch
        return torch.zeros(self.nbytes, dtype=torch.uint8, device=self.device)

    @staticmethod
    def _addr(t):
        return None if t is None else t.data_ptr()

    def step1(self):
        self.solver.stepAsync(1)

    def begin(self, send_lo, send_hi):
        self.solver.slabStepBegin(self._addr(send_lo), self._addr(send_hi))

    def end(self, recv_lo, recv_hi):
        self.solver.slabStepEnd(self._addr(recv_lo), self._addr(recv_hi))

    def flush(self):
        self.solver.slabFlush()

    def pack(self, send_lo, send_hi):
        self.solver.haloPack(self._addr(send_lo), self._addr(send_hi))

    def unpack(self, recv_lo, recv_hi):
        self.solver.haloUnpack(self._addr(recv_lo), self._addr(recv_hi))

    def exchange_context(self):
        """The stream the halo messages travel on (the slab steps' halo
        stream), so that the exchange overlaps the interior planes."""
        import torch
        if not hasattr(self, "_halo"):
            self._halo = torch.cuda.ExternalStream(self.solver.haloStream(), device=self.device)
        return torch.cuda.stream(self._halo)

    def finish(self):
        self.solver.sync()

    def records(self):
        from .runner import records
        return records(self.solver, self.w, f64=True)

    def close(self):
        self.solver.close()


class SlabSolver:
    """One rank's part of a grid split into z-slabs over a process group.

    Every rank of the group builds a SlabSolver from the same workload;
    ``step(n)`` advances all slabs in lockstep (each step: the slab's step,
    then the halo exchange with its neighbours), ``records()`` returns the
    whole grid's port, probe and energy records on every rank. ``stepper``
    builds the per-rank solver (default: DeviceSlab on this rank's GPU)."""

    def __init__(self, w, group=None, device=None, stepper=None, **solver_kw):
        import torch.distributed as dist
        self._dist = dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.ranges = split_planes(w.nz, self.world, monitor_intervals(w))
        k0, k1 = self.ranges[self.rank]
        self.local, glo, ghi, self.first = slab_workload(w, k0, k1)
        self.global_w = w
        if stepper is None:
            dev = int(os.environ.get("LOCAL_RANK", 0)) if device is None else device
            self.slab = DeviceSlab(self.local, glo, ghi, dev, **solver_kw)
        else:
            self.slab = stepper(self.local, glo, ghi)
        self.below = self._peer(self.rank - 1) if glo else None
        self.above = self._peer(self.rank + 1) if ghi else None
        self.send_lo = self.slab.buffer() if glo else None
        self.recv_lo = self.slab.buffer() if glo else None
        self.send_hi = self.slab.buffer() if ghi else None
        self.recv_hi = self.slab.buffer() if ghi else None

    def _peer(self, r):
        return r if self.group is None else self._dist.get_global_rank(self.group, r)

    def _exchange(self):
        dist = self._dist
        ops = []
        if self.below is not None:
            ops += [dist.P2POp(dist.isend, self.send_lo, self.below, self.group),
                    dist.P2POp(dist.irecv, self.recv_lo, self.below, self.group)]
        if self.above is not None:
            ops += [dist.P2POp(dist.isend, self.send_hi, self.above, self.group),
                    dist.P2POp(dist.irecv, self.recv_hi, self.above, self.group)]
        if ops:
            ctx = getattr(self.slab, "exchange_context", contextlib.nullcontext)()
            with ctx:
                for work in dist.batch_isend_irecv(ops):
                    work.wait()

    def step(self, n=1):
        """n steps in lockstep with the neighbours: per step the slab's
        boundary planes and their outgoing halo (``begin``), the exchange,
        then the received halo and the other planes (``end``), the exchange
        overlapping the other planes' update on the device."""
        for _ in range(n):
            self.slab.begin(self.send_lo, self.send_hi)
            self._exchange()
            self.slab.end(self.recv_lo, self.recv_hi)
        self.slab.flush()
        self.slab.finish()

    def records(self):
        """The undivided grid's records (runner.records naming) on every rank."""
        mine = self.slab.records()
        part = {"ports": {}, "probes": {}, "energy_steps": mine["energy_steps"], "energy": mine["energy"]}
        for lp, gp in enumerate(self.local.port_ids):
            part["ports"][gp] = (mine[f"port{lp}_v"], mine[f"port{lp}_i"])
        for lq, gq in enumerate(self.local.probe_ids):
            part["probes"][gq] = tuple(mine[f"probe{lq}_{c}"] for c in ("ex", "ey", "ez"))
        parts = [None] * self.world
        self._dist.all_gather_object(parts, part, group=self.group)
        out = {}
        for pr in parts:
            for gp, (v, i) in pr["ports"].items():
                out[f"port{gp}_v"], out[f"port{gp}_i"] = v, i
            for gq, (ex, ey, ez) in pr["probes"].items():
                out[f"probe{gq}_ex"], out[f"probe{gq}_ey"], out[f"probe{gq}_ez"] = ex, ey, ez
        out["energy_steps"] = parts[0]["energy_steps"]
        e = np.zeros(len(parts[0]["energy"]), np.float64)
        for pr in parts:
            e = e + np.asarray(pr["energy"], np.float64)
        out["energy"] = e
        return out

    def close(self):
        if hasattr(self.slab, "close"):
            self.slab.close()
