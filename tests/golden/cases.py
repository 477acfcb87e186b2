"""Small seeded grids for the golden vectors and the parity tests.

They exercise every case of the step: all six outer faces with rho in
{-1, 0, 0.3, 0.5, 1}, isolated and clustered PEC cells next to air and
dielectric, overlapping lossy dielectric boxes, ports with three gap cells,
a plane-wave source, all three standard waveforms and x extents that are not
a multiple of the kernels' vector width.
"""
from __future__ import annotations

import numpy as np

from emsolver_b200 import workloads


def small_cases():
    """Small grids that exercise every face, PEC, dielectric and source case."""
    cases = []

    def boxes(rng, nx, ny, nz, nbox, pec_frac):
        mat = np.zeros((nz, ny, nx), np.uint8)
        table = []
        for b in range(nbox):
            lo = [int(rng.integers(0, d)) for d in (nz, ny, nx)]
            hi = [int(rng.integers(l, d)) + 1 for l, d in zip(lo, (nz, ny, nx))]
            mat[lo[0]:hi[0], lo[1]:hi[1], lo[2]:hi[2]] = 2 + b
            table.append((float(np.float32(rng.uniform(1, 10))), float(np.float32(rng.uniform(0, 0.05)))))
        if pec_frac > 0:
            mat[rng.random((nz, ny, nx)) < pec_frac] = 1
        return mat.reshape(-1), table

    specs = [
        # name, dims, rho, nbox, pec, waveform, plane wave, steps, seed
        ("pec_diel_rho0", (7, 6, 5), 0.0, 3, 0.08, 2, False, 80, 1),
        ("pec_rho_m1_plane", (9, 8, 10), -1.0, 3, 0.08, 1, True, 80, 2),
        ("diel_rho_half_cw", (12, 5, 7), 0.5, 2, 0.05, 0, False, 80, 3),
        ("cube16_mixed", (16, 16, 16), 0.0, 4, 0.04, 2, True, 120, 4),
        ("odd_x_rho_pmc", (13, 9, 11), 1.0, 2, 0.06, 2, False, 100, 5),
        ("air_only_rho_03", (10, 12, 9), 0.3, 0, 0.0, 1, False, 90, 6),
    ]
    for name, (nx, ny, nz), rho, nbox, pec, wf, plane, steps, seed in specs:
        rng = np.random.default_rng(seed)
        mat, table = boxes(rng, nx, ny, nz, nbox, pec)
        w = workloads.Workload("small_" + name, nx, ny, nz, mat, table, dl=1e-3, f0=3e10,
                               waveform=wf, steps=steps, rho=rho)
        kk, jj, ii = np.unravel_index(np.arange(mat.size), (nz, ny, nx))
        inner = (ii > 0) & (ii < nx - 1) & (jj > 0) & (jj < ny - 1) & (kk > 0) & (kk < nz - 1)
        air = np.flatnonzero((mat == 0) & inner)
        for p in range(2):
            cells = [int(c) for c in rng.choice(air, 3)]
            w.ports.append((cells, int(rng.integers(0, 3)), float(np.float32(rng.uniform(-2, 2)))))
        for q in range(3):
            w.probes_cell.append(tuple(int(rng.integers(0, d)) for d in (nx, ny, nz)))
        if plane:
            w.meta["plane_wave"] = (2, nz // 2, 0, 0.7)
        cases.append(w)
    return cases


def mid_cases():
    """Grids that hold both interior tiles of the step kernel (no PEC, source
    or monitor nearby) and general ones: x extents that leave row padding, a
    PEC block and isolated PEC voxels, overlapping lossy dielectric boxes,
    three-cell ports and probes, outer faces with rho in {0, 0.3, -1}."""
    cases = []
    specs = [
        # name, dims, rho, nbox, pec, waveform, steps, seed
        ("mid_pec_diel", (45, 150, 20), 0.3, 4, 12, 2, 40, 11),
        ("mid_diel_rho_m1", (61, 120, 18), -1.0, 5, 0, 1, 36, 12),
        ("mid_air", (30, 200, 14), 0.0, 0, 0, 2, 30, 13),
    ]
    for name, (nx, ny, nz), rho, nbox, pec, wf, steps, seed in specs:
        rng = np.random.default_rng(seed)
        mat = np.zeros((nz, ny, nx), np.uint8)
        table = []
        for b in range(nbox):
            lo = [int(rng.integers(0, d)) for d in (nz, ny, nx)]
            hi = [min(d, l + int(rng.integers(4, d // 2 + 5))) for l, d in zip(lo, (nz, ny, nx))]
            mat[lo[0]:hi[0], lo[1]:hi[1], lo[2]:hi[2]] = 2 + b
            table.append((float(np.float32(rng.uniform(1, 10))), float(np.float32(rng.uniform(0, 0.05)))))
        if pec > 0:
            # a small PEC block and `pec` isolated PEC voxels
            k0, j0, i0 = (int(rng.integers(1, d - 4)) for d in (nz, ny, nx))
            mat[k0:k0 + 3, j0:j0 + 3, i0:i0 + 3] = 1
            for _ in range(pec):
                mat[tuple(int(rng.integers(0, d)) for d in (nz, ny, nx))] = 1
        mat = mat.reshape(-1)
        w = workloads.Workload(name, nx, ny, nz, mat, table, dl=1e-3, f0=3e10, waveform=wf,
                               steps=steps, rho=rho)
        kk, jj, ii = np.unravel_index(np.arange(mat.size), (nz, ny, nx))
        inner = (ii > 0) & (ii < nx - 1) & (jj > 0) & (jj < ny - 1) & (kk > 0) & (kk < nz - 1)
        air = np.flatnonzero((mat == 0) & inner)
        for p in range(2):
            cells = [int(c) for c in rng.choice(air, 3)]
            w.ports.append((cells, int(rng.integers(0, 3)), float(np.float32(rng.uniform(-2, 2)))))
        for q in range(3):
            w.probes_cell.append(tuple(int(rng.integers(0, d)) for d in (nx, ny, nz)))
        cases.append(w)
    return cases


def interior_tiles(w, V=4, block=256):
    """Number of interior tiles the step kernel finds in `w` with V nodes per
    thread (mirrors the host rule: no PEC node or PEC neighbour, no source or
    monitor node, not the partial last tile)."""
    return int((~_general_mask(w, V, block)).sum())


def staged_tiles(w, block=256):
    """Number of FP32 tiles (2 nodes per thread) that the staged kernel takes:
    the interior tiles (no PEC in reach, no source or monitor, not the partial
    last tile), outer faces included."""
    return int((~_general_mask(w, 2, block)).sum())


def stub_tile_counts(w, block=256):
    """(sparse, dense): FP32 staged tiles (2 nodes per thread) with
    stub-loaded nodes, split by the kernel's rule: sparse when at most a
    quarter of the tile's nodes are stub-loaded (their stubs are loaded
    directly instead of staged)."""
    nx, ny, nz = w.nx, w.ny, w.nz
    px = (nx + 7) // 8 * 8
    T = block * 2
    mat = np.full((nz, ny, px), 1, np.uint8)
    mat[:, :, :nx] = np.asarray(w.mat).reshape(nz, ny, nx)
    diel = (mat >= 2).reshape(-1)
    nb = (diel.size // 2 + block - 1) // block
    cnt = np.bincount(np.arange(diel.size) // T, weights=diel, minlength=nb)[:nb]
    staged = ~_general_mask(w, 2, block)
    sparse = staged & (cnt > 0) & (cnt * 4 <= T)
    dense = staged & (cnt * 4 > T)
    return int(sparse.sum()), int(dense.sum())


def _general_mask(w, V, block):
    """Per tile of `block` threads x V nodes: True when the tile is general."""
    nx, ny, nz = w.nx, w.ny, w.nz
    px = (nx + 7) // 8 * 8
    P = px * ny * nz
    T = block * V
    nb = (P // V + block - 1) // block
    gen = np.zeros(nb, bool)
    if (P // V) % block:
        gen[-1] = True
    mat = np.asarray(w.mat).reshape(nz, ny, nx)
    for k, j, i in zip(*np.nonzero(mat == 1)):
        n = (k * ny + j) * px + i
        for m in (n, n - 1 if i > 0 else -1, n + 1 if i < nx - 1 else -1, n - px, n + px, n - px * ny, n + px * ny):
            if 0 <= m < P:
                gen[m // T] = True
    spec = []
    for cells, _, _ in w.ports:
        for c in cells:
            spec.append(c)
            i, j, k = c % nx, (c // nx) % ny, c // (nx * ny)
            spec += [(k * ny + j2) * nx + i2 for i2, j2 in ((i, j - 1), (i, j + 1), (i - 1, j), (i + 1, j))
                     if 0 <= i2 < nx and 0 <= j2 < ny]
    for (i, j, k) in w.probes_cell:
        spec.append((k * ny + j) * nx + i)
    for c in spec:
        i, r = c % nx, c // nx
        gen[(r * px + i) // T] = True
    return gen


def surface_cases():
    """Dipole grids with every surface monitor on: PEC-surface currents, a
    Huygens box, an |E| cut plane and playback frames, DFT from a settle step."""
    out = []
    for name, dims, length, slab, steps, settle, huy, every, plane in (
        ("surface_dipole_slab", (24, 26, 30), 13, (2, 6, 3.0), 90, 20, 3, 7, (1, 13)),
        ("surface_dipole_odd", (21, 23, 27), 11, None, 70, 30, 2, 5, (2, 9)),
    ):
        w = workloads.dipole(*dims, length, slab=slab, steps=steps, nfreq=4, name=name)
        w.meta.update(settle_steps=settle, huy_offset=huy, record_every=every, field_plane=plane,
                      surface_monitors=True)
        out.append(w)
    return out


def fdtd_cases():
    """Yee FDTD grids: a dipole with a lossy slab and every monitor on (ports,
    probes, PEC-surface currents, Huygens box, cut plane, frames), and a
    plane wave through overlapping lossy boxes with a PEC plate."""
    out = []
    w = workloads.dipole(16, 18, 20, 9, slab=(2, 5, 3.0), steps=70, nfreq=4, name="fdtd_dipole")
    w.meta.update(settle_steps=10, huy_offset=2, record_every=9, field_plane=(1, 9), surface_monitors=True)
    w.probes_cell = [(4, 9, 10), (12, 3, 15)]
    out.append(w)
    rng = np.random.default_rng(31)
    nx, ny, nz = 17, 14, 19
    mat = np.zeros((nz, ny, nx), np.uint8)
    table = []
    for b in range(3):
        lo = [int(rng.integers(0, d - 3)) for d in (nz, ny, nx)]
        hi = [min(d, l + int(rng.integers(3, 9))) for l, d in zip(lo, (nz, ny, nx))]
        mat[lo[0]:hi[0], lo[1]:hi[1], lo[2]:hi[2]] = 2 + b
        table.append((float(np.float32(rng.uniform(1, 8))), float(np.float32(rng.uniform(0, 0.04)))))
    mat[12:14, 3:11, 4:13] = 1                      # PEC plate
    w = workloads.Workload("fdtd_planewave", nx, ny, nz, mat.reshape(-1), table, dl=1e-3, f0=2e10, waveform=1,
                           steps=60)
    w.meta["plane_wave"] = (2, 3, 0, 0.8)
    w.probes_cell = [(8, 7, 9), (2, 2, 16)]
    w.meta.update(settle_steps=5, record_every=11, field_plane=(2, 6), surface_monitors=True)
    out.append(w)
    return out
