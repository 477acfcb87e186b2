"""Python mirror of the reference's TlmSolver interface over the C ABI.

Names, argument meaning and error behaviour follow TlmSolver.h:148-264 of
smilima/EMSolver (``setup``, ``addPort``, ``addPlaneWave``, ``addProbe``,
``run``, ``requestStop``, ``currentStep``, ``currentEnergy``, ``probe``,
``ports``, ``getEnergyHistory``, ``timestep``), so code written against the
reference reads the same. Every call goes to the CUDA library; there is no
CPU path.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from enum import IntEnum
import math
from typing import Sequence

import numpy as np

from . import _lib
from ._lib import check


class WaveformType(IntEnum):
    """TlmSolver.h:70, plus Table (per-step values from setSourceTable)."""
    CwRamped = 0
    GaussianSine = 1
    GaussianPulse = 2
    Table = 3


class Storage(IntEnum):
    F32 = _lib.STORE_F32
    BF16 = _lib.STORE_BF16
    F16 = _lib.STORE_F16
    F64 = _lib.STORE_F64
    BFP16 = _lib.STORE_BFP16


MAT_AIR, MAT_PEC, MAT_DIEL0 = 0, 1, 2


@dataclass
class VoxelGridSpec:
    """Geometry.h:85-113: uniform grid, cell index (k*ny + j)*nx + i."""
    nx: int
    ny: int
    nz: int
    origin: tuple = (0.0, 0.0, 0.0)
    dl: float = 1e-3

    def cellIndex(self, i, j, k):
        return (k * self.ny + j) * self.nx + i

    def inGrid(self, i, j, k):
        return 0 <= i < self.nx and 0 <= j < self.ny and 0 <= k < self.nz

    def cellCenter(self, i, j, k):
        """World position of a cell centre, in float32 like the reference."""
        f = np.float32
        o = [f(v) for v in self.origin]
        dl = f(self.dl)
        return tuple(float(o[a] + (f(c) + f(0.5)) * dl) for a, c in enumerate((i, j, k)))

    @property
    def ncells(self):
        return self.nx * self.ny * self.nz


@dataclass
class MatProps:
    """TlmSolver.h:61-65."""
    epsr: float = 1.0
    sigma: float = 0.0


@dataclass
class TlmConfig:
    """TlmSolver.h:113-123 plus the B200 extensions."""
    f0: float = 1e9
    waveform: int = WaveformType.CwRamped
    totalSteps: int = 2000
    settleSteps: int = 600
    boundaryRho: float = 0.0
    huyOffset: int = 0
    useGpu: bool = True
    recordEvery: int = 0
    storage: int = Storage.F32
    pulseScale: float = 0.0
    stepsPerLaunch: int = 0
    kernelVariant: int = 0
    rounding: int = 0          # 16-bit storage: 0 nearest, 1 stochastic
    generalTiles: bool = False  # True: no interior-tile fast path (cross-checks)
    surfaceMonitors: bool = False  # PEC-surface Js and Huygens-box DFT monitors
    noStaging: bool = False    # True: no shared-memory staging of FP32 interior tiles (cross-checks)
    stageWaitUs: int = 0       # staged tiles' wait limit in us (0 default ~2 s, < 0 first poll)
    nearField: int = 0         # FP16/BF16: radius of the FP32-residual box around PEC and ports (0 none)

    def to_c(self):
        c = _lib.ConfigC()
        c.f0 = self.f0
        c.waveform = int(self.waveform)
        c.total_steps = int(self.totalSteps)
        c.settle_steps = int(self.settleSteps)
        c.boundary_rho = self.boundaryRho
        c.huy_offset = int(self.huyOffset)
        c.use_gpu = 1
        c.record_every = int(self.recordEvery)
        c.storage = int(self.storage)
        c.pulse_scale = self.pulseScale
        c.steps_per_launch = int(self.stepsPerLaunch)
        c.kernel_variant = int(self.kernelVariant)
        c.rounding = int(self.rounding)
        c.general_tiles = 1 if self.generalTiles else 0
        c.surface_monitors = 1 if self.surfaceMonitors else 0
        c.no_staging = 1 if self.noStaging else 0
        c.stage_wait_us = int(self.stageWaitUs)
        c.near_field = int(self.nearField)
        return c


@dataclass
class TlmPort:
    """TlmSolver.h:81-87."""
    cells: list
    polAxis: int = 2
    amp: float = 1.0
    vRec: np.ndarray = field(default_factory=lambda: np.zeros(0, np.float32))
    iRec: np.ndarray = field(default_factory=lambda: np.zeros(0, np.float32))


@dataclass
class FieldProbe:
    """TlmSolver.h:136-141."""
    cell: int
    pos: tuple
    ex: np.ndarray
    ey: np.ndarray
    ez: np.ndarray


def _fp(a, t):
    return a.ctypes.data_as(C.POINTER(t))


class TlmSolver:
    """B200 SCN TLM solver with the reference's TlmSolver interface."""

    def __init__(self, device: int = 0, variant: str | None = None):
        self._L = _lib.load(variant)
        h = C.c_void_p()
        st = self._L.tlm_create(C.byref(h), device)
        if st != _lib.TLM_OK:
            raise _lib.TlmError(st, self._L.tlm_last_error(None).decode())
        self._h = h
        self._grid = None
        self._cfg = None
        self._probe_pos = []
        self._port_meta = []

    # -- lifetime -------------------------------------------------------
    def close(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            check(self._L, h, self._L.tlm_destroy(h))
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _c(self, status):
        return check(self._L, self._h, status)

    # -- setup ------------------------------------------------------------
    def setup(self, grid: VoxelGridSpec, materials, matTable: Sequence[MatProps] = (),
              cfg: TlmConfig | None = None):
        cfg = cfg or TlmConfig()
        mat = np.ascontiguousarray(materials, dtype=np.uint8).reshape(-1)
        g = _lib.Grid(grid.nx, grid.ny, grid.nz, (C.c_float * 3)(*grid.origin), grid.dl)
        tab = (_lib.MatPropsC * max(len(matTable), 1))()
        for t, m in enumerate(matTable):
            tab[t].epsr = m.epsr
            tab[t].sigma = m.sigma
        c = cfg.to_c()
        self._c(self._L.tlm_setup(self._h, C.byref(g), _fp(mat, C.c_uint8), mat.size, tab,
                                  len(matTable), C.byref(c)))
        self._grid = grid
        self._cfg = cfg
        self._probe_pos = []
        self._port_meta = []

    def addPort(self, cells, polAxis: int, amp: float) -> int:
        arr = np.ascontiguousarray(cells, dtype=np.uint64).reshape(-1)
        idx = C.c_int(-1)
        self._c(self._L.tlm_add_port(self._h, _fp(arr, C.c_uint64), arr.size, polAxis, amp,
                                     C.byref(idx)))
        self._port_meta.append((polAxis, amp))
        return idx.value

    def addPlaneWave(self, propAxis: int, planeIndex: int, polAxis: int, amp: float):
        self._c(self._L.tlm_add_plane_wave(self._h, propAxis, planeIndex, polAxis, amp))

    def addSourceCells(self, cells, polAxis: int, amp: float):
        """Soft sources cell by cell (the reference's SourceCell list)."""
        arr = np.ascontiguousarray(cells, dtype=np.uint64).reshape(-1)
        self._c(self._L.tlm_add_source_cells(self._h, _fp(arr, C.c_uint64), arr.size, polAxis, amp))

    def addProbe(self, worldPos) -> int:
        idx = C.c_int(-1)
        x, y, z = (float(v) for v in worldPos)
        self._c(self._L.tlm_add_probe(self._h, x, y, z, C.byref(idx)))
        if idx.value >= 0:
            self._probe_pos.append((x, y, z))
        return idx.value

    def addProbeCell(self, i: int, j: int, k: int) -> int:
        idx = C.c_int(-1)
        self._c(self._L.tlm_add_probe_cell(self._h, i, j, k, C.byref(idx)))
        if idx.value >= 0:
            self._probe_pos.append(self._grid.cellCenter(i, j, k))
        return idx.value

    def setSourceTable(self, sv):
        a = np.ascontiguousarray(sv, dtype=np.float32).reshape(-1)
        self._c(self._L.tlm_set_source_table(self._h, _fp(a, C.c_float), a.size))

    def setPortDft(self, freqs_hz):
        a = np.ascontiguousarray(freqs_hz, dtype=np.float64).reshape(-1)
        self._c(self._L.tlm_set_port_dft(self._h, _fp(a, C.c_double), a.size))

    # -- time loop ----------------------------------------------------------
    def step(self, n: int = 1):
        self._c(self._L.tlm_step(self._h, int(n)))

    def stepAsync(self, n: int = 1):
        self._c(self._L.tlm_step_async(self._h, int(n)))

    def sync(self):
        self._c(self._L.tlm_sync(self._h))

    def run(self) -> bool:
        """Blocking run to totalSteps; False if requestStop ended it early."""
        st = self._L.tlm_run(self._h)
        if st == _lib.TLM_ESTOPPED:
            return False
        self._c(st)
        return True

    def requestStop(self):
        self._L.tlm_request_stop(self._h)

    def isRunning(self):
        return bool(self._L.tlm_is_running(self._h))

    def isFinished(self):
        return bool(self._L.tlm_is_finished(self._h))

    def currentStep(self):
        return self._L.tlm_current_step(self._h)

    def totalSteps(self):
        return self._L.tlm_total_steps(self._h)

    def currentEnergy(self):
        return self._L.tlm_current_energy(self._h)

    def ranOnGpu(self):
        return True

    def gpuStatus(self):
        return self._L.tlm_version().decode()

    def solverName(self):
        return "TLM"

    def grid(self):
        return self._grid

    def cfg(self):
        return self._cfg

    def timestep(self):
        dt = C.c_float(0)
        self._c(self._L.tlm_timestep(self._h, C.byref(dt)))
        return dt.value

    # -- results --------------------------------------------------------------
    def probeCount(self):
        return self._L.tlm_probe_count(self._h)

    def probe(self, idx: int, f64: bool = False) -> FieldProbe:
        n = C.c_int(0)
        self._c(self._L.tlm_get_probe(self._h, idx, None, None, None, 0, C.byref(n)))
        t = np.float64 if f64 else np.float32
        ct = C.c_double if f64 else C.c_float
        ex, ey, ez = (np.zeros(n.value, t) for _ in range(3))
        fn = self._L.tlm_get_probe_f64 if f64 else self._L.tlm_get_probe
        self._c(fn(self._h, idx, _fp(ex, ct), _fp(ey, ct), _fp(ez, ct), n.value, C.byref(n)))
        cell = C.c_uint64(0)
        self._c(self._L.tlm_get_probe_cell(self._h, idx, C.byref(cell)))
        pos = self._probe_pos[idx] if idx < len(self._probe_pos) else None
        return FieldProbe(cell.value, pos, ex, ey, ez)

    def portCount(self):
        return self._L.tlm_port_count(self._h)

    def port(self, idx: int, f64: bool = False) -> TlmPort:
        n = C.c_int(0)
        self._c(self._L.tlm_get_port(self._h, idx, None, None, 0, C.byref(n)))
        t = np.float64 if f64 else np.float32
        ct = C.c_double if f64 else C.c_float
        v, i = np.zeros(n.value, t), np.zeros(n.value, t)
        fn = self._L.tlm_get_port_f64 if f64 else self._L.tlm_get_port
        self._c(fn(self._h, idx, _fp(v, ct), _fp(i, ct), n.value, C.byref(n)))
        nc = C.c_int(0)
        self._c(self._L.tlm_get_port_cells(self._h, idx, None, 0, C.byref(nc)))
        cells = np.zeros(max(nc.value, 1), np.uint64)
        self._c(self._L.tlm_get_port_cells(self._h, idx, _fp(cells, C.c_uint64), nc.value,
                                           C.byref(nc)))
        pol, amp = self._port_meta[idx] if idx < len(self._port_meta) else (2, 1.0)
        return TlmPort([int(c) for c in cells[:nc.value]], pol, amp, v, i)

    def ports(self):
        return [self.port(i) for i in range(self.portCount())]

    def portDft(self, idx: int):
        """(V(f), I(f)) complex128 arrays at the setPortDft frequencies."""
        n = C.c_int(0)
        self._c(self._L.tlm_get_port_dft(self._h, idx, None, None, None, None, 0, C.byref(n)))
        a = [np.zeros(n.value) for _ in range(4)]
        self._c(self._L.tlm_get_port_dft(self._h, idx, *(_fp(x, C.c_double) for x in a), n.value,
                                         C.byref(n)))
        return a[0] + 1j * a[1], a[2] + 1j * a[3]

    def getEnergyHistory(self, f64: bool = False):
        n = C.c_int(0)
        self._c(self._L.tlm_get_energy_history(self._h, None, None, None, 0, C.byref(n)))
        steps = np.zeros(n.value, np.int32)
        if f64:
            vals = np.zeros(n.value, np.float64)
            self._c(self._L.tlm_get_energy_history(self._h, _fp(steps, C.c_int), None,
                                                   _fp(vals, C.c_double), n.value, C.byref(n)))
        else:
            vals = np.zeros(n.value, np.float32)
            self._c(self._L.tlm_get_energy_history(self._h, _fp(steps, C.c_int),
                                                   _fp(vals, C.c_float), None, n.value,
                                                   C.byref(n)))
        return steps, vals

    def pulses(self, f64: bool = False):
        n = self._grid.ncells * 12
        if f64:
            out = np.zeros(n, np.float64)
            self._c(self._L.tlm_get_pulses_f64(self._h, _fp(out, C.c_double), n))
        else:
            out = np.zeros(n, np.float32)
            self._c(self._L.tlm_get_pulses(self._h, _fp(out, C.c_float), n))
        return out

    def setPulses(self, v):
        a = np.ascontiguousarray(v, dtype=np.float32).reshape(-1)
        self._c(self._L.tlm_set_pulses(self._h, _fp(a, C.c_float), a.size))

    # ---- surface monitors (TlmSolver.h:237-245), cut plane, frames, far field
    def faces(self):
        """PEC-surface faces (TlmSolver::faces): cells, axis, sign, centre [n, 3]."""
        n = C.c_int(0)
        self._c(self._L.tlm_get_surface_faces(self._h, None, None, None, None, 0, C.byref(n)))
        m = max(n.value, 1)
        cells, axis, sign = np.zeros(m, np.uint64), np.zeros(m, np.int32), np.zeros(m, np.int32)
        center = np.zeros((m, 3), np.float32)
        self._c(self._L.tlm_get_surface_faces(self._h, _fp(cells, C.c_uint64), _fp(axis, C.c_int),
                                              _fp(sign, C.c_int), _fp(center, C.c_float), n.value,
                                              C.byref(n)))
        k = n.value
        return {"cells": cells[:k], "axis": axis[:k], "sign": sign[:k], "center": center[:k]}

    def getJsInstant(self):
        n = C.c_int(0)
        self._c(self._L.tlm_get_js_instant(self._h, None, 0, C.byref(n)))
        out = np.zeros(max(n.value, 1), np.float32)
        self._c(self._L.tlm_get_js_instant(self._h, _fp(out, C.c_float), n.value, C.byref(n)))
        return out[:n.value]

    def getJsDft(self, raw: bool = False):
        """|Js| DFT magnitude per face (getJsDft after finalizeDft); with
        raw=True also (re [n, 2], im [n, 2], samples)."""
        n, ns = C.c_int(0), C.c_int(0)
        self._c(self._L.tlm_get_js_dft(self._h, None, None, None, 0, C.byref(n), C.byref(ns)))
        m = max(n.value, 1)
        mag, re, im = np.zeros(m, np.float32), np.zeros(2 * m, np.float32), np.zeros(2 * m, np.float32)
        self._c(self._L.tlm_get_js_dft(self._h, _fp(mag, C.c_float), _fp(re, C.c_float), _fp(im, C.c_float),
                                       n.value, C.byref(n), C.byref(ns)))
        k = n.value
        if raw:
            return mag[:k], re[:2 * k].reshape(k, 2), im[:2 * k].reshape(k, 2), ns.value
        return mag[:k]

    def huygensFaces(self):
        n = C.c_int(0)
        self._c(self._L.tlm_get_huygens_faces(self._h, None, None, None, None, 0, C.byref(n)))
        m = max(n.value, 1)
        cells, axis, sign = np.zeros(m, np.uint64), np.zeros(m, np.int32), np.zeros(m, np.int32)
        pos = np.zeros((m, 3), np.float32)
        self._c(self._L.tlm_get_huygens_faces(self._h, _fp(cells, C.c_uint64), _fp(axis, C.c_int),
                                              _fp(sign, C.c_int), _fp(pos, C.c_float), n.value, C.byref(n)))
        k = n.value
        return {"cells": cells[:k], "axis": axis[:k], "out_sign": sign[:k], "pos": pos[:k]}

    def huygensDft(self):
        """(accumulators [n, 8], samples)."""
        n, ns = C.c_int(0), C.c_int(0)
        self._c(self._L.tlm_get_huygens_dft(self._h, None, 0, C.byref(n), C.byref(ns)))
        acc = np.zeros(max(n.value, 1) * 8, np.float32)
        self._c(self._L.tlm_get_huygens_dft(self._h, _fp(acc, C.c_float), n.value, C.byref(n), C.byref(ns)))
        return acc[:8 * n.value].reshape(n.value, 8), ns.value

    def setFieldPlane(self, axis: int, index: int):
        self._c(self._L.tlm_set_field_plane(self._h, int(axis), int(index)))

    def getFieldPlane(self):
        """(plane [n2, n1], axis, index), or None before a plane exists."""
        ax, idx, n1, n2 = (C.c_int(0) for _ in range(4))
        st = self._L.tlm_get_field_plane(self._h, None, 0, C.byref(ax), C.byref(idx), C.byref(n1), C.byref(n2))
        if st != 0:
            return None
        out = np.zeros(n1.value * n2.value, np.float32)
        self._c(self._L.tlm_get_field_plane(self._h, _fp(out, C.c_float), out.size, C.byref(ax), C.byref(idx),
                                            C.byref(n1), C.byref(n2)))
        return out.reshape(n2.value, n1.value), ax.value, idx.value

    def frameCount(self):
        n = C.c_int(0)
        self._c(self._L.tlm_frame_count(self._h, C.byref(n)))
        return n.value

    def getFrame(self, idx: int):
        nj = C.c_int(0)
        self._c(self._L.tlm_get_js_instant(self._h, None, 0, C.byref(nj)))
        dims = sorted((self._grid.nx * self._grid.ny, self._grid.nx * self._grid.nz, self._grid.ny * self._grid.nz))
        js = np.zeros(max(nj.value, 1), np.float32)
        plane = np.zeros(dims[-1], np.float32)
        st, ax, pi, n1, n2 = (C.c_int(0) for _ in range(5))
        self._c(self._L.tlm_get_frame(self._h, int(idx), C.byref(st), _fp(js, C.c_float), nj.value,
                                      _fp(plane, C.c_float), plane.size, C.byref(ax), C.byref(pi), C.byref(n1),
                                      C.byref(n2)))
        npl = n1.value * n2.value
        return {"step": st.value, "js": js[:nj.value],
                "plane": plane[:npl].reshape(n2.value, n1.value) if npl else None,
                "axis": ax.value, "index": pi.value}

    def computeFarField(self, nTheta: int = 37, nPhi: int = 73):
        """FarFieldData (TlmSolver.h:103-110) as a dict."""
        U = np.zeros(nTheta * nPhi, np.float32)
        um, d, pt, pp = (C.c_float(0) for _ in range(4))
        self._c(self._L.tlm_compute_far_field(self._h, int(nTheta), int(nPhi), _fp(U, C.c_float), C.byref(um),
                                              C.byref(d), C.byref(pt), C.byref(pp)))
        return {"U": U.reshape(nTheta, nPhi), "uMax": um.value, "directivity": d.value,
                "peakThetaDeg": pt.value, "peakPhiDeg": pp.value}

    def stubs(self):
        n = self._grid.ncells * 3
        out = np.zeros(n, np.float32)
        self._c(self._L.tlm_get_stubs(self._h, _fp(out, C.c_float), n))
        return out

    def materials(self):
        out = np.zeros(self._grid.ncells, np.uint8)
        self._c(self._L.tlm_get_materials(self._h, _fp(out, C.c_uint8), out.size))
        return out

    def tables(self):
        n = C.c_int(0)
        y = np.zeros(256, np.float32)
        g = np.zeros(256, np.float32)
        self._c(self._L.tlm_get_tables(self._h, _fp(y, C.c_float), _fp(g, C.c_float), 256,
                                       C.byref(n)))
        return y[:n.value].copy(), g[:n.value].copy()

    def stream(self):
        s = C.c_void_p()
        self._c(self._L.tlm_get_stream(self._h, C.byref(s)))
        return s.value

    # -- z-slabs (tlm_set_slab) -------------------------------------------
    def setSlab(self, ghostLo: bool, ghostHi: bool):
        """Mark the first / last plane as ghost copies of the neighbouring
        slabs' planes (before the first step)."""
        self._c(self._L.tlm_set_slab(self._h, int(bool(ghostLo)), int(bool(ghostHi))))

    def haloBytes(self) -> int:
        b = C.c_size_t(0)
        self._c(self._L.tlm_halo_bytes(self._h, C.byref(b)))
        return b.value

    def haloPack(self, send_lo: int | None, send_hi: int | None):
        """Queue copies of the own boundary planes' outgoing z pulses into
        the device buffers at send_lo / send_hi (addresses, or None)."""
        self._c(self._L.tlm_halo_pack(self._h, send_lo, send_hi))

    def haloUnpack(self, recv_lo: int | None, recv_hi: int | None):
        self._c(self._L.tlm_halo_unpack(self._h, recv_lo, recv_hi))

    def slabStepBegin(self, send_lo: int | None, send_hi: int | None):
        """Step the own planes next to a ghost plane and pack their outgoing
        halo on the halo stream (the first half of an overlapped slab step)."""
        self._c(self._L.tlm_slab_step_begin(self._h, send_lo, send_hi))

    def slabStepEnd(self, recv_lo: int | None, recv_hi: int | None):
        """Unpack the received halo on the halo stream while the other own
        planes step (the second half)."""
        self._c(self._L.tlm_slab_step_end(self._h, recv_lo, recv_hi))

    def slabFlush(self):
        """Close the open launch window of slab steps (records, DFT, energy)."""
        self._c(self._L.tlm_slab_flush(self._h))

    def haloStream(self) -> int:
        """The cudaStream_t the halo messages of slab steps travel on."""
        s = C.c_void_p()
        self._c(self._L.tlm_get_halo_stream(self._h, C.byref(s)))
        return s.value

    def deviceBytes(self):
        b = C.c_size_t(0)
        self._c(self._L.tlm_device_bytes(self._h, C.byref(b)))
        return b.value

    def setKernelTiming(self, on: bool):
        self._c(self._L.tlm_set_kernel_timing(self._h, 1 if on else 0))

    def nearFieldBox(self):
        """((i0, j0, k0), (ni, nj, nk)) of the near-field box, or None."""
        b = (C.c_int * 6)()
        self._c(self._L.tlm_near_field_box(self._h, b))
        return None if b[3] == 0 else ((b[0], b[1], b[2]), (b[3], b[4], b[5]))

    def stepLaunches(self) -> int:
        """Kernels launched per step (not counting the window epilogue)."""
        n = C.c_int(0)
        self._c(self._L.tlm_step_launches(self._h, C.byref(n)))
        return n.value

    def kernelTime(self):
        ms = C.c_double(0)
        n = C.c_longlong(0)
        self._c(self._L.tlm_kernel_time(self._h, C.byref(ms), C.byref(n)))
        return ms.value, n.value

    # -- known-answer tests (TlmSolver.cpp:116-169) ---------------------------
    @staticmethod
    def ScatterUnitarityError(device: int = 0, variant: str | None = None) -> float:
        L = _lib.load(variant)
        e = C.c_float(0)
        check(L, None, L.tlm_scatter_unitarity_error(device, C.byref(e)))
        return e.value

    @staticmethod
    def DielScatterUnitarityError(epsr: float, device: int = 0, variant: str | None = None) -> float:
        L = _lib.load(variant)
        e = C.c_float(0)
        check(L, None, L.tlm_stub_unitarity_error(device, epsr, C.byref(e)))
        return e.value


def s11_from_dft(v: np.ndarray, i: np.ndarray, z0: float = 50.0):
    """Z = V/I and S11 = (Z - z0)/(Z + z0) (MainUnit.cpp:1830-1846)."""
    with np.errstate(divide="ignore", invalid="ignore"):
        z = np.where(np.abs(i) < 1e-30, 0.0, v / i)
    return z, (z - z0) / (z + z0)


__all__ = ["TlmSolver", "TlmConfig", "VoxelGridSpec", "MatProps", "TlmPort", "FieldProbe",
           "WaveformType", "Storage", "MAT_AIR", "MAT_PEC", "MAT_DIEL0", "s11_from_dft", "math"]
