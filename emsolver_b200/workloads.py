"""Seeded synthetic TLM workloads (no dataset is involved anywhere).

Each builder returns a plain ``Workload`` (grid, material map, table, config,
sources, probes) that can be fed to this library's ``TlmSolver``, to the
oracle, or to the reference's own solver compiled headless, so that all three
solve exactly the same problem.

* ``plain_free_space``    64^3 free space, Gaussian pulse on the centre
                          node's Ez links, probe at (48,32,32), 500 steps.
* ``heterogeneous``       192^3 with 16 random lossy dielectric boxes, a
                          z-directed differentiated-Gaussian source on one
                          air node, 8 random probes, 2000 steps.
* ``dipole``              a z-directed PEC wire dipole with a 1-node feed gap
                          (the port), optional dielectric slab; used for the
                          384x384x256 precision run, the batched instances
                          and the served requests.
* ``batched_instances``   256 dipoles with edges U{24..96}, 1000 steps.
* ``request_stream``      Poisson arrivals of dipole solves.
"""
from __future__ import annotations

from dataclasses import dataclass, field
import math

import numpy as np

C0_F32 = np.float32(299792458.0)


@dataclass
class Workload:
    name: str
    nx: int
    ny: int
    nz: int
    mat: np.ndarray                       # uint8, reference cell order
    table: list = field(default_factory=list)   # [(epsr, sigma)]
    dl: float = 1e-3
    origin: tuple = (0.0, 0.0, 0.0)
    f0: float = 1e9
    waveform: int = 2                     # reference WaveformType, 3 = table
    sv: np.ndarray | None = None          # per-step source values (table waveform)
    steps: int = 500
    rho: float = 0.0
    ports: list = field(default_factory=list)    # [(cells, pol, amp)]
    probes_cell: list = field(default_factory=list)  # [(i, j, k)] probe at cell centre
    dft_freqs: np.ndarray | None = None
    storage: int = 0
    meta: dict = field(default_factory=dict)

    @property
    def ncells(self):
        return self.nx * self.ny * self.nz

    def cell(self, i, j, k):
        return (k * self.ny + j) * self.nx + i

    def cell_center(self, i, j, k):
        f = np.float32
        o = [f(v) for v in self.origin]
        dl = f(self.dl)
        return tuple(float(o[a] + (f(c) + f(0.5)) * dl) for a, c in enumerate((i, j, k)))

    def n_diel(self):
        return int(np.count_nonzero(self.mat >= 2))

    def bytes_per_step(self, storage_bytes=4, stub_bytes=4):
        """Algorithmic DRAM bytes of one step: 12 pulses read + 12 written +
        1 material byte per node, + 3 stub pulses read and written per
        dielectric node."""
        return self.ncells * (24 * storage_bytes + 1) + self.n_diel() * 6 * stub_bytes


def gaussian_pulse_f0(dl, width_steps=20):
    """f0 for which the reference's GaussianPulse has tau = width_steps*dt
    (tau = 0.5/f0, dt = dl/(2 c0)) -- in float32 like the reference."""
    return float(C0_F32 / (np.float32(width_steps) * np.float32(dl)))


def differentiated_gaussian(steps, width=20.0, delay=60.0):
    """-2u exp(-u^2), u = (n - delay)/width, scaled to a peak of 1 (float32)."""
    n = np.arange(steps, dtype=np.float64)
    u = (n - delay) / width
    g = -2.0 * u * np.exp(-u * u) / (math.sqrt(2.0) * math.exp(-0.5))
    return g.astype(np.float32)


def plain_free_space(n=64, steps=500, dl=1e-3):
    """Free space, rho = 0, GaussianPulse of width 20 steps and delay 60 on the
    Ez links of the centre node (index n/2), probe Ez at (3n/4, n/2, n/2)."""
    mat = np.zeros(n ** 3, np.uint8)
    w = Workload("plain_free_space", n, n, n, mat, [], dl=dl, f0=gaussian_pulse_f0(dl), waveform=2,
                 steps=steps, rho=0.0)
    c = n // 2
    w.ports.append(([w.cell(c, c, c)], 2, 1.0))
    w.probes_cell.append((3 * n // 4, c, c))
    return w


def heterogeneous(n=192, steps=2000, seed=1, nboxes=16, nprobes=8, dl=1e-3):
    """16 axis-aligned lossy dielectric boxes (corners uniform in the grid,
    eps_r ~ U[1,10], sigma ~ U[0,0.05] S/m, ids 2..17, later boxes win), a
    z-directed differentiated-Gaussian soft source on one interior air node,
    8 probes at uniform random nodes."""
    rng = np.random.default_rng(seed)
    mat = np.zeros((n, n, n), np.uint8)          # [k][j][i]
    table = []
    for b in range(nboxes):
        lo, hi = [], []
        for _ in range(3):
            a, c = rng.integers(0, n, 2)
            lo.append(min(a, c))
            hi.append(max(a, c) + 1)
        mat[lo[2]:hi[2], lo[1]:hi[1], lo[0]:hi[0]] = 2 + b
        table.append((float(np.float32(rng.uniform(1.0, 10.0))),
                      float(np.float32(rng.uniform(0.0, 0.05)))))
    mat = mat.reshape(-1)
    w = Workload("heterogeneous", n, n, n, mat, table, dl=dl, f0=gaussian_pulse_f0(dl),
                 waveform=3, sv=differentiated_gaussian(steps), steps=steps, rho=0.0)
    while True:
        i, j, k = (int(v) for v in rng.integers(1, n - 1, 3))
        if mat[w.cell(i, j, k)] == 0:
            break
    w.ports.append(([w.cell(i, j, k)], 2, 1.0))
    for _ in range(nprobes):
        w.probes_cell.append(tuple(int(v) for v in rng.integers(0, n, 3)))
    w.meta["source_cell"] = (i, j, k)
    return w


def dipole(nx, ny, nz, length, slab=None, steps=8000, dl=1e-3, nfreq=64, storage=0,
           name="dipole"):
    """z-directed PEC wire dipole of `length` nodes (odd: the middle node is
    the air feed gap and carries the port) centred in the grid. `slab` =
    (x0, x1, eps_r) adds a dielectric slab x0 <= i < x1 over all j, k.
    GaussianPulse excitation with f0 = 2 f_res, f_res = c0/(2 L dl); port DFT
    at `nfreq` frequencies uniform in [0.5, 1.5] f_res."""
    length = int(length) | 1
    mat = np.zeros((nz, ny, nx), np.uint8)
    table = []
    if slab is not None:
        x0, x1, er = slab
        mat[:, :, x0:x1] = 2
        table.append((float(er), 0.0))
    ci, cj, ck = nx // 2, ny // 2, nz // 2
    h = length // 2
    k0, k1 = max(ck - h, 1), min(ck + h, nz - 2)
    mat[k0:k1 + 1, cj, ci] = 1
    mat[ck, cj, ci] = 0
    mat = mat.reshape(-1)
    f_res = float(C0_F32) / (2.0 * length * dl)
    w = Workload(name, nx, ny, nz, mat, table, dl=dl, f0=2.0 * f_res, waveform=2, steps=steps,
                 rho=0.0, storage=storage)
    w.ports.append(([w.cell(ci, cj, ck)], 2, 1.0))
    w.dft_freqs = np.linspace(0.5 * f_res, 1.5 * f_res, nfreq)
    w.meta.update(f_res=f_res, length=length)
    return w


def precision_dipole(storage=0, steps=8000, nx=384, ny=384, nz=256):
    """384x384x256, half-wave dipole of 60 PEC nodes plus the 1-node gap."""
    return dipole(nx, ny, nz, 61, None, steps=steps, storage=storage, name="precision_dipole")


def random_dipole(rng, nx, ny, nz, steps, storage=0, name="instance"):
    """Dipole of length U[0.3,0.9]*nz with a random dielectric slab
    (eps_r ~ U[1,6]) beside it."""
    length = max(3, int(rng.uniform(0.3, 0.9) * nz))
    ci = nx // 2
    width = int(rng.integers(1, max(2, nx // 4)))
    x0 = int(rng.integers(0, max(1, ci - 1 - width)))
    slab = (x0, min(x0 + width, ci - 1), float(rng.uniform(1.0, 6.0)))
    if slab[1] <= slab[0]:
        slab = None
    return dipole(nx, ny, nz, length, slab, steps=steps, storage=storage, name=name)


def batched_instances(count=256, steps=1000, seed=4, lo=24, hi=96):
    rng = np.random.default_rng(seed)
    out = []
    for b in range(count):
        nx, ny, nz = (int(v) for v in rng.integers(lo, hi + 1, 3))
        out.append(random_dipole(rng, nx, ny, nz, steps, name=f"instance{b}"))
    return out


def request_stream(count=10000, rate=200.0, seed=5, edge_lo=32, edge_hi=256, steps_lo=500,
                   steps_hi=8000):
    """[(arrival_time_s, Workload)]: Poisson arrivals, cubic edge log-uniform,
    steps uniform, storage FP32 or BF16 with probability 0.5 each."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for r in range(count):
        t += rng.exponential(1.0 / rate)
        edge = int(round(math.exp(rng.uniform(math.log(edge_lo), math.log(edge_hi)))))
        steps = int(rng.integers(steps_lo, steps_hi + 1))
        storage = 0 if rng.random() < 0.5 else 1
        out.append((t, random_dipole(rng, edge, edge, edge, steps, storage, name=f"req{r}")))
    return out
