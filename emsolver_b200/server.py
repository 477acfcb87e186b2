"""Continuous-batching request server for antenna solves (tlm_server_*).

Requests are complete solves (a ``Workload``). The native worker thread
admits them by HBM footprint into a running batch between launch windows,
keeps their state on the device, and retires each at its total step count;
requests arriving while others run join the batch at the next window.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import check
from .solver import TlmConfig

QUEUED, RUNNING, DONE, FAILED, CANCELLED = range(5)
STATE_NAMES = {QUEUED: "queued", RUNNING: "running", DONE: "done", FAILED: "failed",
               CANCELLED: "cancelled"}


def _p(a, t):
    return a.ctypes.data_as(C.POINTER(t))


class _Request:
    """A tlm_request built from a Workload; keeps the arrays alive."""

    def __init__(self, w, storage=None, rounding=0, near_field=None):
        self.mat = np.ascontiguousarray(w.mat, dtype=np.uint8).reshape(-1)
        self.tab = (_lib.MatPropsC * max(len(w.table), 1))()
        for t, (e, g) in enumerate(w.table):
            self.tab[t].epsr, self.tab[t].sigma = e, g
        cfg = TlmConfig(f0=w.f0, waveform=w.waveform, totalSteps=w.steps, settleSteps=0,
                        boundaryRho=w.rho, storage=w.storage if storage is None else storage,
                        rounding=rounding,
                        nearField=w.meta.get("near_field", 0) if near_field is None else near_field)
        self.sv = np.ascontiguousarray(w.sv if (w.waveform == 3 and w.sv is not None) else [],
                                       dtype=np.float32)
        self.cells = np.ascontiguousarray(
            np.concatenate([np.asarray(c, np.uint64) for c, _, _ in w.ports]) if w.ports
            else np.zeros(0, np.uint64), dtype=np.uint64)
        self.ncells = np.ascontiguousarray([len(c) for c, _, _ in w.ports], dtype=np.int32)
        self.pol = np.ascontiguousarray([p for _, p, _ in w.ports], dtype=np.int32)
        self.amp = np.ascontiguousarray([a for _, _, a in w.ports], dtype=np.float32)
        self.ijk = np.ascontiguousarray(np.asarray(w.probes_cell, np.int32).reshape(-1),
                                        dtype=np.int32)
        self.freqs = np.ascontiguousarray(w.dft_freqs if w.dft_freqs is not None else [],
                                          dtype=np.float64)
        r = _lib.RequestC()
        r.grid = _lib.Grid(w.nx, w.ny, w.nz, (C.c_float * 3)(*w.origin), w.dl)
        r.mat = _p(self.mat, C.c_uint8)
        r.n_cells = self.mat.size
        r.table = self.tab
        r.n_table = len(w.table)
        r.cfg = cfg.to_c()
        r.source_table = _p(self.sv, C.c_float)
        r.n_source = self.sv.size
        r.n_ports = len(w.ports)
        r.port_cells = _p(self.cells, C.c_uint64)
        r.port_ncells = _p(self.ncells, C.c_int)
        r.port_pol = _p(self.pol, C.c_int)
        r.port_amp = _p(self.amp, C.c_float)
        r.n_probes = len(w.probes_cell)
        r.probe_ijk = _p(self.ijk, C.c_int)
        r.n_freq = self.freqs.size
        r.freqs = _p(self.freqs, C.c_double)
        self.c = r


def footprint(w, storage=None, near_field=None) -> int:
    """Device bytes the solve holds while it runs (what admission counts)."""
    L = _lib.load()
    r = _Request(w, storage, near_field=near_field)
    b = C.c_size_t(0)
    check(L, None, L.tlm_request_footprint(C.byref(r.c), C.byref(b)))
    return b.value


class Server:
    def __init__(self, device: int = 0, hbm_budget: int = 0, steps_per_launch: int = 0,
                 variant: str | None = None):
        self._L = _lib.load(variant)
        h = C.c_void_p()
        st = self._L.tlm_server_create(C.byref(h), device, int(hbm_budget), int(steps_per_launch))
        if st != _lib.TLM_OK:
            raise _lib.TlmError(st, self._L.tlm_last_error(None).decode())
        self._s = h

    def _c(self, status):
        return check(self._L, None, status)

    ARRIVAL, LEAST_WORK = 0, 1

    def set_policy(self, order: int = 1, max_running_cells: int = 8 << 20, solo_cells: int = 1 << 20):
        """Admission order (LEAST_WORK first, or ARRIVAL), the cap on the
        running requests' padded cells (0: none), and the size from which a
        request runs on its own beside the batch (0: never)."""
        self._c(self._L.tlm_server_set_policy(self._s, int(order), int(max_running_cells), int(solo_cells)))

    def submit(self, w, storage=None, rounding=0, near_field=None) -> int:
        r = _Request(w, storage, rounding, near_field)
        rid = C.c_uint64(0)
        self._c(self._L.tlm_server_submit(self._s, C.byref(r.c), C.byref(rid)))
        return rid.value

    def poll(self, rid) -> int:
        st = C.c_int(0)
        self._c(self._L.tlm_server_poll(self._s, rid, C.byref(st)))
        return st.value

    def wait(self, rid, timeout: float = -1.0) -> int:
        st = C.c_int(0)
        self._c(self._L.tlm_server_wait(self._s, rid, float(timeout), C.byref(st)))
        return st.value

    def cancel(self, rid):
        self._c(self._L.tlm_server_cancel(self._s, rid))

    def result(self, rid, port: int = 0):
        """(V(f), I(f), latency_s) of a finished request."""
        n = C.c_int(0)
        lat = C.c_double(0)
        self._c(self._L.tlm_server_result(self._s, rid, port, None, None, None, None, 0,
                                          C.byref(n), C.byref(lat)))
        a = [np.zeros(n.value) for _ in range(4)]
        self._c(self._L.tlm_server_result(self._s, rid, port, *(_p(x, C.c_double) for x in a),
                                          n.value, C.byref(n), C.byref(lat)))
        return a[0] + 1j * a[1], a[2] + 1j * a[3], lat.value

    def port_records(self, rid, port: int = 0):
        n = C.c_int(0)
        self._c(self._L.tlm_server_port_records(self._s, rid, port, None, None, 0, C.byref(n)))
        v, i = np.zeros(n.value, np.float32), np.zeros(n.value, np.float32)
        self._c(self._L.tlm_server_port_records(self._s, rid, port, _p(v, C.c_float),
                                                _p(i, C.c_float), n.value, C.byref(n)))
        return v, i

    def release(self, rid):
        self._c(self._L.tlm_server_release(self._s, rid))

    def stats(self) -> dict:
        st = _lib.ServerStatsC()
        self._c(self._L.tlm_server_stats(self._s, C.byref(st)))
        return {k: getattr(st, k) for k, _ in _lib.ServerStatsC._fields_}

    def close(self):
        s = getattr(self, "_s", None)
        if s is not None and s.value:
            self._L.tlm_server_destroy(s)
        self._s = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
