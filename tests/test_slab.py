"""A grid split into z-slabs over a process group, on CPU (gloo ranks).

The host side of emsolver_b200.slab -- the split, the slab workloads, the
per-step halo exchange over torch.distributed, the gathering of records --
runs here with each rank stepping its slab on the oracle (the CPU
restatement, bitwise the reference) instead of a GPU. Bar: every port and
probe record of the split grid bitwise equal to the undivided grid's."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from emsolver_b200 import workloads
from emsolver_b200.slab import monitor_intervals, slab_workload, split_planes
from oracle import Oracle, drive

PEC = 1


class OracleSlab:
    """A slab stepped by the oracle. The oracle keeps incident pulses (after
    connect) in the reference's node-major layout, so its halo is the pulses
    each boundary plane received through its outer z face: the ghost plane's
    copy of what the own boundary plane sent is the message, and the
    neighbour writes it into its own boundary plane, except where either end
    of the link is PEC (there the oracle's connect already used the PEC
    rule)."""

    def __init__(self, w, ghost_lo, ghost_hi):
        self.w, self.glo, self.ghi = w, ghost_lo, ghost_hi
        self.S = Oracle()
        drive.setup(self.S, w)
        self.plane = w.nx * w.ny
        self.mat = np.asarray(w.mat).reshape(w.nz, self.plane)

    def buffer(self):
        return torch.zeros(2 * self.plane, dtype=torch.float64)

    def step1(self):
        drive.advance(self.S, self.w, 1)

    def _state(self):
        return self.S.pulses().astype(np.float64).reshape(self.w.nz, self.plane, 12)

    def pack(self, send_lo, send_hi):
        v = self._state()
        if send_lo is not None:   # ghost plane 0 received (slots 10, 11) what plane 1 sent down
            send_lo.copy_(torch.from_numpy(np.ascontiguousarray(v[0, :, 10:12].T).reshape(-1)))
        if send_hi is not None:   # the top ghost plane received (slots 8, 9) what the last plane sent up
            send_hi.copy_(torch.from_numpy(np.ascontiguousarray(v[-1, :, 8:10].T).reshape(-1)))

    def unpack(self, recv_lo, recv_hi):
        v = self._state()
        nz = self.w.nz
        for recv, own, ghost, slots in ((recv_lo, 1, 0, slice(8, 10)), (recv_hi, nz - 2, nz - 1, slice(10, 12))):
            if recv is None:
                continue
            msg = recv.numpy().reshape(2, self.plane).T
            ok = (self.mat[own] != PEC) & (self.mat[ghost] != PEC)
            v[own, ok, slots] = msg[ok]
        self.S.set_pulses(v.reshape(-1))

    def begin(self, send_lo, send_hi):
        """The first half of an overlapped slab step: the step, then the
        outgoing halo."""
        self.step1()
        self.pack(send_lo, send_hi)

    def end(self, recv_lo, recv_hi):
        self.unpack(recv_lo, recv_hi)

    def flush(self):
        pass

    def finish(self):
        pass

    def records(self):
        out = drive.records(self.S, self.w)
        out["energy"] = np.zeros(len(out["energy"]))   # the oracle's sum includes the ghost planes
        return out


def split_workload(seed=3):
    rng = np.random.default_rng(seed)
    w = workloads.random_dipole(rng, 11, 10, 23, 90, name="split")
    w.rho = 0.5
    w.probes_cell = [(2, 3, 0), (5, 5, 7), (8, 2, 11), (4, 7, 15), (1, 1, 22), (6, 4, 16)]
    return w


def _rank_main(rank, world, port, w, out_path):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch.distributed as dist
    from emsolver_b200.slab import SlabSolver
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        s = SlabSolver(w, stepper=OracleSlab)
        s.step(w.steps)
        rec = s.records()
        if rank == 0:
            np.savez(out_path, ranges=np.array(s.ranges), **rec)
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        return sk.getsockname()[1]


def test_split_planes_balances_and_avoids_monitors():
    assert split_planes(20, 1) == [(0, 20)]
    assert split_planes(20, 4) == [(0, 5), (5, 10), (10, 15), (15, 20)]
    r = split_planes(20, 3, [(6, 8)])
    assert r[0][0] == 0 and r[-1][1] == 20 and all(a[1] == b[0] for a, b in zip(r, r[1:]))
    assert all(not (6 < b <= 8) for _, b in r[:-1])
    with pytest.raises(ValueError):
        split_planes(4, 4, [(0, 3)])
    with pytest.raises(ValueError):
        split_planes(3, 4)


def test_slab_workload_holds_its_planes_and_ghosts():
    w = split_workload()
    ranges = split_planes(w.nz, 3, monitor_intervals(w))
    gm = w.mat.reshape(w.nz, w.ny, w.nx)
    seen_probes, seen_ports = [], []
    for k0, k1 in ranges:
        v, glo, ghi, lo = slab_workload(w, k0, k1)
        assert (glo, ghi) == (int(k0 > 0), int(k1 < w.nz)) and lo == k0 - glo
        assert np.array_equal(v.mat.reshape(v.nz, w.ny, w.nx), gm[lo:k1 + ghi])
        for (i, j, k), q in zip(v.probes_cell, v.probe_ids):
            assert w.probes_cell[q] == (i, j, k + lo) and glo <= k < v.nz - ghi
        seen_probes += v.probe_ids
        seen_ports += v.port_ids
    assert sorted(seen_probes) == list(range(len(w.probes_cell)))
    assert sorted(seen_ports) == list(range(len(w.ports)))


@pytest.mark.parametrize("world", [2, 3])
def test_gloo_slabs_match_the_undivided_grid(tmp_path, world):
    w = split_workload()
    out = tmp_path / "rec.npz"
    mp.start_processes(_rank_main, args=(world, _free_port(), w, str(out)), nprocs=world, join=True,
                       start_method="spawn")
    got = np.load(out)
    assert len(got["ranges"]) == world
    S = Oracle()
    drive.setup(S, w)
    drive.advance(S, w, w.steps)
    ref = drive.records(S, w)
    for k, v in ref.items():
        if k.startswith(("port", "probe")):
            assert np.array_equal(got[k], v), k
