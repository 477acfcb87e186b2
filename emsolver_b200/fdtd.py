"""FdtdSolver: the reference's Yee FDTD solver (FdtdSolver.h) on the B200.

The same IFieldSolver surface as ``TlmSolver`` (TlmSolver.h:148-192): setup
with a VoxelGridSpec, material table and TlmConfig, ports, plane waves,
probes, run / step, records, surface currents, Huygens far field, cut plane
and frames. Every call goes to the C ABI of include/fdtd_b200.h; there is no
CPU fallback.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import TLM_OK, TlmError
from .solver import MatProps, TlmConfig, VoxelGridSpec, _fp

FIELDS = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")


class FdtdSolver:
    def __init__(self, device: int = 0, variant: str | None = None):
        self._L = _lib.load(variant)
        h = C.c_void_p()
        self._h = None
        self._c(self._L.fdtd_create(C.byref(h), int(device)), none=True)
        self._h = h
        self._grid = None

    # -- plumbing
    def _c(self, st, none=False):
        if st != TLM_OK:
            msg = self._L.fdtd_last_error(None if none else self._h)
            raise TlmError(st, msg.decode() if msg else "")
        return st

    def close(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            self._L.fdtd_destroy(h)
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- IFieldSolver
    def setup(self, grid: VoxelGridSpec, materials, table: list[MatProps], cfg: TlmConfig):
        mat = np.ascontiguousarray(materials, dtype=np.uint8).reshape(-1)
        g = _lib.Grid(grid.nx, grid.ny, grid.nz, (C.c_float * 3)(*grid.origin), grid.dl)
        tab = (_lib.MatPropsC * max(len(table), 1))()
        for t, m in enumerate(table):
            tab[t].epsr = m.epsr
            tab[t].sigma = m.sigma
        c = cfg.to_c()
        self._c(self._L.fdtd_setup(self._h, C.byref(g), _fp(mat, C.c_uint8), mat.size, tab, len(table),
                                   C.byref(c)))
        self._grid = grid
        self._cfg = cfg

    def addPort(self, cells, polAxis: int, amp: float) -> int:
        c = np.ascontiguousarray(cells, dtype=np.uint64).reshape(-1)
        idx = C.c_int(-1)
        self._c(self._L.fdtd_add_port(self._h, _fp(c, C.c_uint64), c.size, int(polAxis), float(amp),
                                      C.byref(idx)))
        return idx.value

    def addPlaneWave(self, propAxis: int, planeIndex: int, polAxis: int, amp: float):
        self._c(self._L.fdtd_add_plane_wave(self._h, int(propAxis), int(planeIndex), int(polAxis), float(amp)))

    def addProbe(self, worldPos) -> int:
        idx = C.c_int(-1)
        x, y, z = (float(v) for v in worldPos)
        self._c(self._L.fdtd_add_probe(self._h, x, y, z, C.byref(idx)))
        return idx.value

    def setSourceTable(self, values):
        v = np.ascontiguousarray(values, dtype=np.float32).reshape(-1)
        self._c(self._L.fdtd_set_source_table(self._h, _fp(v, C.c_float), v.size))

    def step(self, n: int = 1):
        self._c(self._L.fdtd_step(self._h, int(n)))

    def run(self):
        self._c(self._L.fdtd_run(self._h))

    def currentStep(self) -> int:
        return self._L.fdtd_current_step(self._h)

    def timestep(self) -> float:
        return self._L.fdtd_timestep(self._h)

    def stream(self) -> int:
        st = C.c_void_p()
        self._c(self._L.fdtd_get_stream(self._h, C.byref(st)))
        return st.value or 0

    # -- state and records
    def field(self, which) -> np.ndarray:
        w = FIELDS.index(which) if isinstance(which, str) else int(which)
        n = C.c_size_t(0)
        self._c(self._L.fdtd_get_field(self._h, w, None, 0, C.byref(n)))
        out = np.zeros(n.value, np.float32)
        self._c(self._L.fdtd_get_field(self._h, w, _fp(out, C.c_float), out.size, C.byref(n)))
        return out

    def fields(self) -> dict:
        return {name: self.field(name) for name in FIELDS}

    def probe(self, idx: int):
        cap = max(self.currentStep(), 1)
        ex, ey, ez = (np.zeros(cap, np.float32) for _ in range(3))
        n = C.c_int(0)
        self._c(self._L.fdtd_get_probe(self._h, int(idx), _fp(ex, C.c_float), _fp(ey, C.c_float),
                                       _fp(ez, C.c_float), cap, C.byref(n)))
        return ex[:n.value], ey[:n.value], ez[:n.value]

    def port(self, idx: int):
        cap = max(self.currentStep(), 1)
        v, i = np.zeros(cap, np.float32), np.zeros(cap, np.float32)
        n = C.c_int(0)
        self._c(self._L.fdtd_get_port(self._h, int(idx), _fp(v, C.c_float), _fp(i, C.c_float), cap, C.byref(n)))
        return v[:n.value], i[:n.value]

    def getEnergyHistory(self, f64: bool = False):
        n = C.c_int(0)
        self._c(self._L.fdtd_get_energy_history(self._h, None, None, None, 0, C.byref(n)))
        steps = np.zeros(max(n.value, 1), np.int32)
        vals = np.zeros(max(n.value, 1), np.float64 if f64 else np.float32)
        if f64:
            self._c(self._L.fdtd_get_energy_history(self._h, _fp(steps, C.c_int), None, _fp(vals, C.c_double),
                                                    n.value, C.byref(n)))
        else:
            self._c(self._L.fdtd_get_energy_history(self._h, _fp(steps, C.c_int), _fp(vals, C.c_float), None,
                                                    n.value, C.byref(n)))
        return steps[:n.value], vals[:n.value]

    # -- surface monitors, cut plane, frames, far field (same shapes as TlmSolver)
    def faces(self):
        n = C.c_int(0)
        self._c(self._L.fdtd_get_surface_faces(self._h, None, None, None, None, 0, C.byref(n)))
        m = max(n.value, 1)
        cells, axis, sign = np.zeros(m, np.uint64), np.zeros(m, np.int32), np.zeros(m, np.int32)
        center = np.zeros((m, 3), np.float32)
        self._c(self._L.fdtd_get_surface_faces(self._h, _fp(cells, C.c_uint64), _fp(axis, C.c_int),
                                               _fp(sign, C.c_int), _fp(center, C.c_float), n.value, C.byref(n)))
        k = n.value
        return {"cells": cells[:k], "axis": axis[:k], "sign": sign[:k], "center": center[:k]}

    def getJsInstant(self):
        n = C.c_int(0)
        self._c(self._L.fdtd_get_js_instant(self._h, None, 0, C.byref(n)))
        out = np.zeros(max(n.value, 1), np.float32)
        self._c(self._L.fdtd_get_js_instant(self._h, _fp(out, C.c_float), n.value, C.byref(n)))
        return out[:n.value]

    def getJsDft(self, raw: bool = False):
        n, ns = C.c_int(0), C.c_int(0)
        self._c(self._L.fdtd_get_js_dft(self._h, None, None, None, 0, C.byref(n), C.byref(ns)))
        m = max(n.value, 1)
        mag, re, im = np.zeros(m, np.float32), np.zeros(2 * m, np.float32), np.zeros(2 * m, np.float32)
        self._c(self._L.fdtd_get_js_dft(self._h, _fp(mag, C.c_float), _fp(re, C.c_float), _fp(im, C.c_float),
                                        n.value, C.byref(n), C.byref(ns)))
        k = n.value
        if raw:
            return mag[:k], re[:2 * k].reshape(k, 2), im[:2 * k].reshape(k, 2), ns.value
        return mag[:k]

    def huygensFaces(self):
        n = C.c_int(0)
        self._c(self._L.fdtd_get_huygens_faces(self._h, None, None, None, None, 0, C.byref(n)))
        m = max(n.value, 1)
        cells, axis, sign = np.zeros(m, np.uint64), np.zeros(m, np.int32), np.zeros(m, np.int32)
        pos = np.zeros((m, 3), np.float32)
        self._c(self._L.fdtd_get_huygens_faces(self._h, _fp(cells, C.c_uint64), _fp(axis, C.c_int),
                                               _fp(sign, C.c_int), _fp(pos, C.c_float), n.value, C.byref(n)))
        k = n.value
        return {"cells": cells[:k], "axis": axis[:k], "out_sign": sign[:k], "pos": pos[:k]}

    def huygensDft(self):
        n, ns = C.c_int(0), C.c_int(0)
        self._c(self._L.fdtd_get_huygens_dft(self._h, None, 0, C.byref(n), C.byref(ns)))
        acc = np.zeros(max(n.value, 1) * 8, np.float32)
        self._c(self._L.fdtd_get_huygens_dft(self._h, _fp(acc, C.c_float), n.value, C.byref(n), C.byref(ns)))
        return acc[:8 * n.value].reshape(n.value, 8), ns.value

    def setFieldPlane(self, axis: int, index: int):
        self._c(self._L.fdtd_set_field_plane(self._h, int(axis), int(index)))

    def getFieldPlane(self):
        ax, idx, n1, n2 = (C.c_int(0) for _ in range(4))
        st = self._L.fdtd_get_field_plane(self._h, None, 0, C.byref(ax), C.byref(idx), C.byref(n1), C.byref(n2))
        if st != 0:
            return None
        out = np.zeros(n1.value * n2.value, np.float32)
        self._c(self._L.fdtd_get_field_plane(self._h, _fp(out, C.c_float), out.size, C.byref(ax), C.byref(idx),
                                             C.byref(n1), C.byref(n2)))
        return out.reshape(n2.value, n1.value), ax.value, idx.value

    def frameCount(self):
        n = C.c_int(0)
        self._c(self._L.fdtd_frame_count(self._h, C.byref(n)))
        return n.value

    def getFrame(self, idx: int):
        nj = C.c_int(0)
        self._c(self._L.fdtd_get_js_instant(self._h, None, 0, C.byref(nj)))
        g = self._grid
        big = max(g.nx * g.ny, g.nx * g.nz, g.ny * g.nz)
        js = np.zeros(max(nj.value, 1), np.float32)
        plane = np.zeros(big, np.float32)
        st, ax, pi, n1, n2 = (C.c_int(0) for _ in range(5))
        self._c(self._L.fdtd_get_frame(self._h, int(idx), C.byref(st), _fp(js, C.c_float), nj.value,
                                       _fp(plane, C.c_float), plane.size, C.byref(ax), C.byref(pi), C.byref(n1),
                                       C.byref(n2)))
        npl = n1.value * n2.value
        return {"step": st.value, "js": js[:nj.value],
                "plane": plane[:npl].reshape(n2.value, n1.value) if npl else None,
                "axis": ax.value, "index": pi.value}

    def computeFarField(self, nTheta: int = 37, nPhi: int = 73):
        U = np.zeros(nTheta * nPhi, np.float32)
        um, d, pt, pp = (C.c_float(0) for _ in range(4))
        self._c(self._L.fdtd_compute_far_field(self._h, int(nTheta), int(nPhi), _fp(U, C.c_float), C.byref(um),
                                               C.byref(d), C.byref(pt), C.byref(pp)))
        return {"U": U.reshape(nTheta, nPhi), "uMax": um.value, "directivity": d.value,
                "peakThetaDeg": pt.value, "peakPhiDeg": pp.value}


def build_fdtd(w, device: int = 0) -> FdtdSolver:
    """An FdtdSolver set up from a synthetic Workload the way the reference
    would be: setup, ports in order, plane wave, probes at cell centres."""
    s = FdtdSolver(device)
    grid = VoxelGridSpec(w.nx, w.ny, w.nz, tuple(w.origin), w.dl)
    cfg = TlmConfig(f0=w.f0, waveform=w.waveform, totalSteps=w.steps, settleSteps=w.meta.get("settle_steps", 0),
                    huyOffset=w.meta.get("huy_offset", 0), recordEvery=w.meta.get("record_every", 0),
                    surfaceMonitors=bool(w.meta.get("surface_monitors", False)), boundaryRho=w.rho)
    s.setup(grid, w.mat, [MatProps(e, g) for e, g in w.table], cfg)
    if w.waveform == 3 and w.sv is not None:
        s.setSourceTable(w.sv)
    for cells, pol, amp in w.ports:
        s.addPort(cells, pol, amp)
    if "plane_wave" in w.meta:
        s.addPlaneWave(*w.meta["plane_wave"])
    for (i, j, k) in w.probes_cell:
        s.addProbe(w.cell_center(i, j, k))
    if "field_plane" in w.meta:
        s.setFieldPlane(*w.meta["field_plane"])
    return s
