"""ctypes wrappers for the oracle libraries (TEST INFRASTRUCTURE ONLY)."""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libtlmref.so")

_u8p = C.POINTER(C.c_uint8)
_f32p = C.POINTER(C.c_float)
_f64p = C.POINTER(C.c_double)
_i32p = C.POINTER(C.c_int)
_u64p = C.POINTER(C.c_uint64)


# The reference's source tree: $TLM_REFERENCE_SRC, else where this build
# environment mounts it. Absent (as on a machine that only runs tests), the
# prebuilt oracle/_ref/ is kept.
REF_SRC = os.environ.get("TLM_REFERENCE_SRC", "/root/reference")


def build_oracle(quiet: bool = True) -> None:
    """Compile liboracle.so (and the reference under _ref/ when its sources exist)."""
    cmd = ["make", "-C", HERE]
    if os.path.exists(os.path.join(REF_SRC, "TlmSolver.cpp")):
        cmd.append(f"REF={REF_SRC}")
    out = subprocess.run(cmd, capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + out.stdout + out.stderr)
    if not quiet:
        print(out.stdout)


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def _ptr(a, t):
    return a.ctypes.data_as(t)


def _setup_args(nx, ny, nz, origin, dl, mat, table):
    mat = np.ascontiguousarray(mat, dtype=np.uint8).reshape(-1)
    if mat.size != nx * ny * nz:
        raise ValueError("material map size mismatch")
    eps = np.ascontiguousarray([t[0] for t in table] or [1.0], dtype=np.float32)
    sig = np.ascontiguousarray([t[1] for t in table] or [0.0], dtype=np.float32)
    ox, oy, oz = (float(v) for v in origin)
    return mat, eps, sig, ox, oy, oz


class _SurfaceMonitors:
    """Js faces and DFT, Huygens-box DFT, |E| cut plane, playback frames and
    the far field (TlmSolver.cpp:303-348, 616-675, 715-763, 805-916), shared by
    ``Oracle`` and ``RefSolver``. Subclasses set ``_p`` (symbol prefix) and
    ``_rt``/``_rp`` (the library's real type and its pointer type)."""

    def _f(self, name):
        return getattr(self.L, self._p + name)

    def set_field_plane(self, axis, index):
        self._f("set_field_plane")(self.h, axis, index)

    def surface_faces(self):
        n = self._f("surface_faces")(self.h, None, None, None, None, 0)
        cells = np.empty(max(n, 1), np.uint64)
        axis = np.empty(max(n, 1), np.int32)
        sign = np.empty(max(n, 1), np.int32)
        center = np.empty((max(n, 1), 3), np.float32)
        self._f("surface_faces")(self.h, _ptr(cells, _u64p), _ptr(axis, _i32p), _ptr(sign, _i32p),
                                 _ptr(center, _f32p), n)
        return {"cells": cells[:n], "axis": axis[:n], "sign": sign[:n], "center": center[:n]}

    def js_instant(self):
        n = self._f("js_instant")(self.h, None, 0)
        out = np.empty(max(n, 1), self._rt)
        self._f("js_instant")(self.h, _ptr(out, self._rp), n)
        return out[:n].astype(self.dtype)

    def js_dft(self):
        """(re [nf, 2], im [nf, 2], magnitude as finalised after a run [nf], samples)."""
        n = self._f("js_dft")(self.h, None, None, None, 0, None)
        re = np.empty(max(2 * n, 2), self._rt)
        im = np.empty(max(2 * n, 2), self._rt)
        mag = np.empty(max(n, 1), self._rt)
        samples = C.c_int(0)
        self._f("js_dft")(self.h, _ptr(re, self._rp), _ptr(im, self._rp), _ptr(mag, self._rp), n,
                          C.byref(samples))
        return (re[:2 * n].reshape(n, 2).astype(self.dtype), im[:2 * n].reshape(n, 2).astype(self.dtype),
                mag[:n].astype(self.dtype), samples.value)

    def huygens_faces(self):
        n = self._f("huygens_faces")(self.h, None, None, None, None, 0)
        cells = np.empty(max(n, 1), np.uint64)
        axis = np.empty(max(n, 1), np.int32)
        sign = np.empty(max(n, 1), np.int32)
        pos = np.empty((max(n, 1), 3), np.float32)
        self._f("huygens_faces")(self.h, _ptr(cells, _u64p), _ptr(axis, _i32p), _ptr(sign, _i32p),
                                 _ptr(pos, _f32p), n)
        return {"cells": cells[:n], "axis": axis[:n], "out_sign": sign[:n], "pos": pos[:n]}

    def huygens_dft(self):
        """(accumulators [nh, 8]: E1 re/im, E2 re/im, eta0*H1 re/im, eta0*H2 re/im; samples)."""
        n = self._f("huygens_faces")(self.h, None, None, None, None, 0)
        acc = np.empty(max(8 * n, 8), self._rt)
        samples = C.c_int(0)
        self._f("huygens_dft")(self.h, _ptr(acc, self._rp), n, C.byref(samples))
        return acc[:8 * n].reshape(n, 8).astype(self.dtype), samples.value

    def field_plane(self):
        cap = 1 << 22
        buf = np.empty(cap, self._rt)
        ax, idx, n1, n2 = (C.c_int(0) for _ in range(4))
        rc = self._f("field_plane")(self.h, _ptr(buf, self._rp), cap, C.byref(ax), C.byref(idx),
                                    C.byref(n1), C.byref(n2))
        if rc != 0:
            return None
        return buf[:n1.value * n2.value].reshape(n2.value, n1.value).astype(self.dtype), ax.value, idx.value

    def frames(self):
        out = []
        nj = self._f("js_instant")(self.h, None, 0)
        for f in range(self._f("frame_count")(self.h)):
            js = np.empty(max(nj, 1), self._rt)
            plane = np.empty(1 << 22, self._rt)
            st, ax, pi, n1, n2 = (C.c_int(0) for _ in range(5))
            npl = self._f("get_frame")(self.h, f, C.byref(st), _ptr(js, self._rp), nj, _ptr(plane, self._rp),
                                       plane.size, C.byref(ax), C.byref(pi), C.byref(n1), C.byref(n2))
            out.append({"step": st.value, "js": js[:nj].astype(self.dtype),
                        "plane": plane[:max(npl, 0)].reshape(n2.value, n1.value).astype(self.dtype)
                        if npl > 0 else None, "axis": ax.value, "index": pi.value})
        return out

    def far_field(self, n_theta=37, n_phi=73):
        U = np.empty(n_theta * n_phi, self._rt)
        um, d, pt, pp = (self._rs(0) for _ in range(4))
        rc = self._f("far_field")(self.h, n_theta, n_phi, _ptr(U, self._rp), C.byref(um), C.byref(d),
                                  C.byref(pt), C.byref(pp))
        if rc != 0:
            return None
        return {"U": U.reshape(n_theta, n_phi).astype(self.dtype), "u_max": um.value,
                "directivity": d.value, "peak_theta_deg": pt.value, "peak_phi_deg": pp.value}


def _surface_signatures(L, p, rp, rs):
    getattr(L, p + "set_field_plane").argtypes = [C.c_void_p, C.c_int, C.c_int]
    for nm in ("surface_faces", "huygens_faces"):
        f = getattr(L, p + nm)
        f.restype = C.c_int
        f.argtypes = [C.c_void_p, _u64p, _i32p, _i32p, _f32p, C.c_int]
    f = getattr(L, p + "js_instant")
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, rp, C.c_int]
    f = getattr(L, p + "js_dft")
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, rp, rp, rp, C.c_int, _i32p]
    f = getattr(L, p + "huygens_dft")
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, rp, C.c_int, _i32p]
    f = getattr(L, p + "field_plane")
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, rp, C.c_size_t, _i32p, _i32p, _i32p, _i32p]
    f = getattr(L, p + "frame_count")
    f.restype = C.c_int
    f.argtypes = [C.c_void_p]
    f = getattr(L, p + "get_frame")
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, C.c_int, _i32p, rp, C.c_int, rp, C.c_size_t, _i32p, _i32p, _i32p, _i32p]
    f = getattr(L, p + "far_field")
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, C.c_int, C.c_int, rp, C.POINTER(rs), C.POINTER(rs), C.POINTER(rs),
                  C.POINTER(rs)]


class Oracle(_SurfaceMonitors):
    """The CPU restatement; ``fp64=False`` is bitwise the reference's float step."""

    _lib = None
    _p, _rt, _rp, _rs = "orc_", np.float64, _f64p, C.c_double

    @classmethod
    def lib(cls):
        if cls._lib is None:
            if not os.path.exists(ORACLE_SO):
                build_oracle()
            L = C.CDLL(ORACLE_SO)
            L.orc_create.restype = C.c_void_p
            L.orc_create.argtypes = [C.c_int]
            L.orc_destroy.argtypes = [C.c_void_p]
            L.orc_setup.restype = C.c_int
            L.orc_setup.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_float, C.c_float,
                                    C.c_float, C.c_float, _u8p, _f32p, _f32p, C.c_int, C.c_float,
                                    C.c_int, C.c_int, C.c_int, C.c_float]
            L.orc_add_port.restype = C.c_int
            L.orc_add_port.argtypes = [C.c_void_p, _u64p, C.c_int, C.c_int, C.c_float]
            L.orc_add_probe.restype = C.c_int
            L.orc_add_probe.argtypes = [C.c_void_p, C.c_float, C.c_float, C.c_float]
            L.orc_add_plane_wave.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_float]
            L.orc_waveform.restype = C.c_double
            L.orc_waveform.argtypes = [C.c_void_p, C.c_int]
            L.orc_dt.restype = C.c_double
            L.orc_dt.argtypes = [C.c_void_p]
            L.orc_steps.argtypes = [C.c_void_p, C.c_int, C.c_int, _f64p]
            for nm in ("orc_get_pulses", "orc_get_stubs"):
                getattr(L, nm).restype = C.c_size_t
                getattr(L, nm).argtypes = [C.c_void_p, _f64p, C.c_size_t]
            L.orc_set_pulses.restype = C.c_size_t
            L.orc_set_pulses.argtypes = [C.c_void_p, _f64p, C.c_size_t]
            L.orc_get_tables.restype = C.c_int
            L.orc_get_tables.argtypes = [C.c_void_p, _f64p, _f64p, C.c_int]
            L.orc_probe_count.restype = C.c_int
            L.orc_probe_count.argtypes = [C.c_void_p]
            L.orc_get_probe.restype = C.c_int
            L.orc_get_probe.argtypes = [C.c_void_p, C.c_int, _f64p, _f64p, _f64p, C.c_int, _u64p]
            L.orc_port_count.restype = C.c_int
            L.orc_port_count.argtypes = [C.c_void_p]
            L.orc_get_port.restype = C.c_int
            L.orc_get_port.argtypes = [C.c_void_p, C.c_int, _f64p, _f64p, C.c_int]
            L.orc_energy_history.restype = C.c_int
            L.orc_energy_history.argtypes = [C.c_void_p, _i32p, _f64p, C.c_int]
            L.orc_scatter_unitarity.restype = C.c_double
            L.orc_scatter_unitarity.argtypes = [C.c_int]
            L.orc_stub_unitarity.restype = C.c_double
            L.orc_stub_unitarity.argtypes = [C.c_int, C.c_double]
            L.orc_configure_surface.restype = C.c_int
            L.orc_configure_surface.argtypes = [C.c_void_p, C.c_int, C.c_int]
            _surface_signatures(L, "orc_", _f64p, C.c_double)
            cls._lib = L
        return cls._lib

    def __init__(self, fp64: bool = False):
        self.L = self.lib()
        self.fp64 = bool(fp64)
        self.h = self.L.orc_create(1 if fp64 else 0)
        self.n = 0
        self.step_index = 0
        self.dtype = np.float64 if fp64 else np.float32

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            self.L.orc_destroy(h)
            self.h = None

    def setup(self, nx, ny, nz, mat, table=(), origin=(0.0, 0.0, 0.0), dl=1e-3, f0=1e9,
              waveform=2, total_steps=2000, settle_steps=600, rho=0.0, huy_offset=0, record_every=0):
        mat, eps, sig, ox, oy, oz = _setup_args(nx, ny, nz, origin, dl, mat, table)
        rc = self.L.orc_setup(self.h, nx, ny, nz, ox, oy, oz, dl, _ptr(mat, _u8p), _ptr(eps, _f32p),
                              _ptr(sig, _f32p), len(table), f0, waveform, total_steps,
                              settle_steps, rho)
        if rc != 0:
            raise ValueError(f"oracle setup rejected the inputs (code {rc})")
        self.L.orc_configure_surface(self.h, huy_offset, record_every)
        self.n = nx * ny * nz
        self.step_index = 0

    def add_port(self, cells, pol, amp=1.0):
        c = np.ascontiguousarray(cells, dtype=np.uint64).reshape(-1)
        return self.L.orc_add_port(self.h, _ptr(c, _u64p), c.size, pol, amp)

    def add_probe(self, x, y, z):
        return self.L.orc_add_probe(self.h, x, y, z)

    def add_plane_wave(self, prop_axis, plane_index, pol_axis, amp=1.0):
        self.L.orc_add_plane_wave(self.h, prop_axis, plane_index, pol_axis, amp)

    def waveform(self, n):
        return self.L.orc_waveform(self.h, n)

    @property
    def dt(self):
        return self.L.orc_dt(self.h)

    def steps(self, count, sv=None):
        if sv is not None:
            sv = np.ascontiguousarray(sv, dtype=np.float64).reshape(-1)
            assert sv.size >= count
            self.L.orc_steps(self.h, self.step_index, count, _ptr(sv, _f64p))
        else:
            self.L.orc_steps(self.h, self.step_index, count, None)
        self.step_index += count

    def pulses(self):
        out = np.empty(self.n * 12, np.float64)
        self.L.orc_get_pulses(self.h, _ptr(out, _f64p), out.size)
        return out.astype(self.dtype)

    def set_pulses(self, v):
        v = np.ascontiguousarray(v, dtype=np.float64).reshape(-1)
        if self.L.orc_set_pulses(self.h, _ptr(v, _f64p), v.size) != v.size:
            raise ValueError("pulse array size mismatch")

    def stubs(self):
        n = self.L.orc_get_stubs(self.h, None, 0)
        out = np.empty(n, np.float64)
        if n:
            self.L.orc_get_stubs(self.h, _ptr(out, _f64p), n)
        return out.astype(self.dtype)

    def tables(self):
        y = np.empty(256, np.float64)
        g = np.empty(256, np.float64)
        n = self.L.orc_get_tables(self.h, _ptr(y, _f64p), _ptr(g, _f64p), 256)
        return y[:n].astype(self.dtype), g[:n].astype(self.dtype)

    def probe(self, idx):
        cap = self.step_index
        ex, ey, ez = (np.empty(max(cap, 1), np.float64) for _ in range(3))
        cell = C.c_uint64(0)
        n = self.L.orc_get_probe(self.h, idx, _ptr(ex, _f64p), _ptr(ey, _f64p), _ptr(ez, _f64p),
                                 cap, C.byref(cell))
        return (ex[:n].astype(self.dtype), ey[:n].astype(self.dtype), ez[:n].astype(self.dtype))

    def port(self, idx):
        cap = self.step_index
        v, i = (np.empty(max(cap, 1), np.float64) for _ in range(2))
        n = self.L.orc_get_port(self.h, idx, _ptr(v, _f64p), _ptr(i, _f64p), cap)
        return v[:n].astype(self.dtype), i[:n].astype(self.dtype)

    def energy_history(self):
        cap = self.step_index // 16 + 2
        st = np.empty(cap, np.int32)
        va = np.empty(cap, np.float64)
        n = self.L.orc_energy_history(self.h, _ptr(st, _i32p), _ptr(va, _f64p), cap)
        return st[:n].copy(), va[:n].copy()

    @classmethod
    def scatter_unitarity(cls, fp64=False):
        return cls.lib().orc_scatter_unitarity(1 if fp64 else 0)

    @classmethod
    def stub_unitarity(cls, epsr, fp64=False):
        return cls.lib().orc_stub_unitarity(1 if fp64 else 0, epsr)


class RefSolver(_SurfaceMonitors):
    """The reference's own TlmSolver (compiled headless), same methods as ``Oracle``."""

    _lib = None
    _p, _rt, _rp, _rs = "ref_", np.float32, _f32p, C.c_float

    @classmethod
    def lib(cls):
        if cls._lib is None:
            if not os.path.exists(REF_SO):
                raise FileNotFoundError(
                    "oracle/_ref/libtlmref.so is missing (it is built from the reference sources "
                    "by `make -C oracle`)")
            L = C.CDLL(REF_SO)
            L.ref_create.restype = C.c_void_p
            L.ref_destroy.argtypes = [C.c_void_p]
            L.ref_setup.restype = C.c_int
            L.ref_setup.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_float, C.c_float,
                                    C.c_float, C.c_float, _u8p, _f32p, _f32p, C.c_int, C.c_float,
                                    C.c_int, C.c_int, C.c_int, C.c_float]
            L.ref_add_port.restype = C.c_int
            L.ref_add_port.argtypes = [C.c_void_p, _u64p, C.c_int, C.c_int, C.c_float]
            L.ref_add_probe.restype = C.c_int
            L.ref_add_probe.argtypes = [C.c_void_p, C.c_float, C.c_float, C.c_float]
            L.ref_add_plane_wave.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_float]
            L.ref_steps.argtypes = [C.c_void_p, C.c_int, C.c_int]
            L.ref_steps_sv.argtypes = [C.c_void_p, C.c_int, C.c_int, _f32p]
            L.ref_run.argtypes = [C.c_void_p]
            L.ref_waveform.restype = C.c_float
            L.ref_waveform.argtypes = [C.c_void_p, C.c_int]
            L.ref_dt.restype = C.c_float
            L.ref_dt.argtypes = [C.c_void_p]
            L.ref_threads.restype = C.c_int
            L.ref_threads.argtypes = [C.c_void_p]
            L.ref_current_step.restype = C.c_int
            L.ref_current_step.argtypes = [C.c_void_p]
            for nm in ("ref_get_pulses", "ref_get_stubs"):
                getattr(L, nm).restype = C.c_size_t
                getattr(L, nm).argtypes = [C.c_void_p, _f32p, C.c_size_t]
            L.ref_set_pulses.restype = C.c_size_t
            L.ref_set_pulses.argtypes = [C.c_void_p, _f32p, C.c_size_t]
            L.ref_get_tables.restype = C.c_int
            L.ref_get_tables.argtypes = [C.c_void_p, _f32p, _f32p, C.c_int]
            L.ref_probe_count.restype = C.c_int
            L.ref_probe_count.argtypes = [C.c_void_p]
            L.ref_get_probe.restype = C.c_int
            L.ref_get_probe.argtypes = [C.c_void_p, C.c_int, _f32p, _f32p, _f32p, C.c_int, _u64p]
            L.ref_port_count.restype = C.c_int
            L.ref_port_count.argtypes = [C.c_void_p]
            L.ref_get_port.restype = C.c_int
            L.ref_get_port.argtypes = [C.c_void_p, C.c_int, _f32p, _f32p, C.c_int, _u64p, C.c_int,
                                       _i32p]
            L.ref_energy_history.restype = C.c_int
            L.ref_energy_history.argtypes = [C.c_void_p, _i32p, _f32p, C.c_int]
            L.ref_scatter_unitarity.restype = C.c_float
            L.ref_diel_unitarity.restype = C.c_float
            L.ref_diel_unitarity.argtypes = [C.c_float]
            L.ref_hw_concurrency.restype = C.c_uint
            L.ref_setup_ex.restype = C.c_int
            L.ref_setup_ex.argtypes = L.ref_setup.argtypes + [C.c_int, C.c_int]
            _surface_signatures(L, "ref_", _f32p, C.c_float)
            cls._lib = L
        return cls._lib

    def __init__(self):
        self.L = self.lib()
        self.h = self.L.ref_create()
        self.n = 0
        self.step_index = 0
        self.dtype = np.float32

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            self.L.ref_destroy(h)
            self.h = None

    @property
    def threads(self):
        return self.L.ref_threads(self.h)

    def setup(self, nx, ny, nz, mat, table=(), origin=(0.0, 0.0, 0.0), dl=1e-3, f0=1e9,
              waveform=2, total_steps=2000, settle_steps=600, rho=0.0, huy_offset=0, record_every=0):
        mat, eps, sig, ox, oy, oz = _setup_args(nx, ny, nz, origin, dl, mat, table)
        self.L.ref_setup_ex(self.h, nx, ny, nz, ox, oy, oz, dl, _ptr(mat, _u8p), _ptr(eps, _f32p),
                            _ptr(sig, _f32p), len(table), f0, waveform, total_steps, settle_steps, rho,
                            huy_offset, record_every)
        self.n = nx * ny * nz
        self.step_index = 0

    def add_port(self, cells, pol, amp=1.0):
        c = np.ascontiguousarray(cells, dtype=np.uint64).reshape(-1)
        return self.L.ref_add_port(self.h, _ptr(c, _u64p), c.size, pol, amp)

    def add_probe(self, x, y, z):
        return self.L.ref_add_probe(self.h, x, y, z)

    def add_plane_wave(self, prop_axis, plane_index, pol_axis, amp=1.0):
        self.L.ref_add_plane_wave(self.h, prop_axis, plane_index, pol_axis, amp)

    def waveform(self, n):
        return self.L.ref_waveform(self.h, n)

    @property
    def dt(self):
        return self.L.ref_dt(self.h)

    def steps(self, count, sv=None):
        if sv is not None:
            sv = np.ascontiguousarray(sv, dtype=np.float32).reshape(-1)
            assert sv.size >= count
            self.L.ref_steps_sv(self.h, self.step_index, count, _ptr(sv, _f32p))
        else:
            self.L.ref_steps(self.h, self.step_index, count)
        self.step_index += count

    def run(self):
        self.L.ref_run(self.h)
        self.step_index = self.L.ref_current_step(self.h)

    def pulses(self):
        out = np.empty(self.n * 12, np.float32)
        self.L.ref_get_pulses(self.h, _ptr(out, _f32p), out.size)
        return out

    def set_pulses(self, v):
        v = np.ascontiguousarray(v, dtype=np.float32).reshape(-1)
        if self.L.ref_set_pulses(self.h, _ptr(v, _f32p), v.size) != v.size:
            raise ValueError("pulse array size mismatch")

    def stubs(self):
        n = self.L.ref_get_stubs(self.h, None, 0)
        out = np.empty(n, np.float32)
        if n:
            self.L.ref_get_stubs(self.h, _ptr(out, _f32p), n)
        return out

    def tables(self):
        y = np.empty(256, np.float32)
        g = np.empty(256, np.float32)
        n = self.L.ref_get_tables(self.h, _ptr(y, _f32p), _ptr(g, _f32p), 256)
        return y[:n].copy(), g[:n].copy()

    def probe(self, idx):
        cap = self.step_index
        ex, ey, ez = (np.empty(max(cap, 1), np.float32) for _ in range(3))
        cell = C.c_uint64(0)
        n = self.L.ref_get_probe(self.h, idx, _ptr(ex, _f32p), _ptr(ey, _f32p), _ptr(ez, _f32p),
                                 cap, C.byref(cell))
        return ex[:n].copy(), ey[:n].copy(), ez[:n].copy()

    def port(self, idx):
        cap = self.step_index
        v, i = (np.empty(max(cap, 1), np.float32) for _ in range(2))
        nc = C.c_int(0)
        n = self.L.ref_get_port(self.h, idx, _ptr(v, _f32p), _ptr(i, _f32p), cap, None, 0,
                                C.byref(nc))
        return v[:n].copy(), i[:n].copy()

    def energy_history(self):
        cap = self.step_index // 16 + 2
        st = np.empty(cap, np.int32)
        va = np.empty(cap, np.float32)
        n = self.L.ref_energy_history(self.h, _ptr(st, _i32p), _ptr(va, _f32p), cap)
        return st[:n].copy(), va[:n].astype(np.float64)

    @classmethod
    def scatter_unitarity(cls):
        return cls.lib().ref_scatter_unitarity()

    @classmethod
    def stub_unitarity(cls, epsr):
        return cls.lib().ref_diel_unitarity(epsr)


class RefFdtd(_SurfaceMonitors):
    """The reference's own Yee FDTD solver (FdtdSolver.cpp, compiled headless)."""

    _lib = None
    _p, _rt, _rp, _rs = "fdr_", np.float32, _f32p, C.c_float

    @classmethod
    def lib(cls):
        if cls._lib is None:
            L = RefSolver.lib()
            L.fdr_create.restype = C.c_void_p
            L.fdr_destroy.argtypes = [C.c_void_p]
            L.fdr_setup.restype = C.c_int
            L.fdr_setup.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_float, C.c_float, C.c_float,
                                    C.c_float, _u8p, _f32p, _f32p, C.c_int, C.c_float, C.c_int, C.c_int,
                                    C.c_int, C.c_int, C.c_int]
            L.fdr_add_port.restype = C.c_int
            L.fdr_add_port.argtypes = [C.c_void_p, _u64p, C.c_int, C.c_int, C.c_float]
            L.fdr_add_probe.restype = C.c_int
            L.fdr_add_probe.argtypes = [C.c_void_p, C.c_float, C.c_float, C.c_float]
            L.fdr_add_plane_wave.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_float]
            L.fdr_steps.argtypes = [C.c_void_p, C.c_int, C.c_int]
            L.fdr_steps_sv.argtypes = [C.c_void_p, C.c_int, C.c_int, _f32p]
            L.fdr_dt.restype = C.c_float
            L.fdr_dt.argtypes = [C.c_void_p]
            L.fdr_get_field.restype = C.c_size_t
            L.fdr_get_field.argtypes = [C.c_void_p, C.c_int, _f32p, C.c_size_t]
            L.fdr_get_probe.restype = C.c_int
            L.fdr_get_probe.argtypes = [C.c_void_p, C.c_int, _f32p, _f32p, _f32p, C.c_int]
            L.fdr_get_port.restype = C.c_int
            L.fdr_get_port.argtypes = [C.c_void_p, C.c_int, _f32p, _f32p, C.c_int]
            L.fdr_energy_history.restype = C.c_int
            L.fdr_energy_history.argtypes = [C.c_void_p, _i32p, _f32p, C.c_int]
            _surface_signatures(L, "fdr_", _f32p, C.c_float)
            cls._lib = L
        return cls._lib

    def __init__(self):
        self.L = self.lib()
        self.h = self.L.fdr_create()
        self.n = 0
        self.step_index = 0
        self.dtype = np.float32

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            self.L.fdr_destroy(h)
            self.h = None

    def setup(self, nx, ny, nz, mat, table=(), origin=(0.0, 0.0, 0.0), dl=1e-3, f0=1e9,
              waveform=2, total_steps=2000, settle_steps=600, rho=0.0, huy_offset=0, record_every=0):
        mat, eps, sig, ox, oy, oz = _setup_args(nx, ny, nz, origin, dl, mat, table)
        self.L.fdr_setup(self.h, nx, ny, nz, ox, oy, oz, dl, _ptr(mat, _u8p), _ptr(eps, _f32p),
                         _ptr(sig, _f32p), len(table), f0, waveform, total_steps, settle_steps, huy_offset,
                         record_every)
        self.n = nx * ny * nz
        self.step_index = 0

    def add_port(self, cells, pol, amp=1.0):
        c = np.ascontiguousarray(cells, dtype=np.uint64).reshape(-1)
        return self.L.fdr_add_port(self.h, _ptr(c, _u64p), c.size, pol, amp)

    def add_probe(self, x, y, z):
        return self.L.fdr_add_probe(self.h, x, y, z)

    def add_plane_wave(self, prop_axis, plane_index, pol_axis, amp=1.0):
        self.L.fdr_add_plane_wave(self.h, prop_axis, plane_index, pol_axis, amp)

    @property
    def dt(self):
        return self.L.fdr_dt(self.h)

    def steps(self, count, sv=None):
        if sv is not None:
            sv = np.ascontiguousarray(sv, dtype=np.float32).reshape(-1)
            assert sv.size >= count
            self.L.fdr_steps_sv(self.h, self.step_index, count, _ptr(sv, _f32p))
        else:
            self.L.fdr_steps(self.h, self.step_index, count)
        self.step_index += count

    def fields(self):
        """Ex, Ey, Ez, Hx, Hy, Hz in the reference's Yee layouts (flat)."""
        out = {}
        for w, name in enumerate(("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")):
            n = self.L.fdr_get_field(self.h, w, None, 0)
            a = np.empty(n, np.float32)
            self.L.fdr_get_field(self.h, w, _ptr(a, _f32p), n)
            out[name] = a
        return out

    def probe(self, idx):
        cap = self.step_index
        ex, ey, ez = (np.empty(max(cap, 1), np.float32) for _ in range(3))
        n = self.L.fdr_get_probe(self.h, idx, _ptr(ex, _f32p), _ptr(ey, _f32p), _ptr(ez, _f32p), cap)
        return ex[:n].copy(), ey[:n].copy(), ez[:n].copy()

    def port(self, idx):
        cap = self.step_index
        v, i = (np.empty(max(cap, 1), np.float32) for _ in range(2))
        n = self.L.fdr_get_port(self.h, idx, _ptr(v, _f32p), _ptr(i, _f32p), cap)
        return v[:n].copy(), i[:n].copy()

    def energy_history(self):
        cap = self.step_index // 16 + 2
        st = np.empty(cap, np.int32)
        va = np.empty(cap, np.float32)
        n = self.L.fdr_energy_history(self.h, _ptr(st, _i32p), _ptr(va, _f32p), cap)
        return st[:n].copy(), va[:n].astype(np.float64)


class RefEmsim:
    """The reference's own SaveProject / LoadProject (ProjectIO.cpp, compiled
    headless into _ref/libtlmref.so) for checking the .emsim code."""

    _lib = None

    @classmethod
    def lib(cls):
        if cls._lib is None:
            L = RefSolver.lib()
            L.ref_emsim_resave.restype = C.c_int
            L.ref_emsim_resave.argtypes = [C.c_char_p, C.c_char_p, C.c_char_p, C.c_int]
            L.ref_emsim_write_sample.restype = C.c_int
            L.ref_emsim_write_sample.argtypes = [C.c_char_p, C.c_int, C.c_int]
            L.ref_emsim_summary.restype = C.c_int
            L.ref_emsim_summary.argtypes = [C.c_char_p, C.POINTER(C.c_int64), C.c_char_p, C.c_int]
            cls._lib = L
        return cls._lib

    @classmethod
    def write_sample(cls, path, seed, playback=True):
        """A project with every section filled from `seed`, written by SaveProject."""
        if cls.lib().ref_emsim_write_sample(str(path).encode(), int(seed), int(bool(playback))) != 1:
            raise OSError(f"reference SaveProject failed for {path}")

    @classmethod
    def resave(cls, src, dst):
        """LoadProject(src) then SaveProject(dst): "" on success, else the
        reference's load error."""
        err = C.create_string_buffer(256)
        r = cls.lib().ref_emsim_resave(str(src).encode(), str(dst).encode(), err, 256)
        if r == -1:
            raise OSError(f"reference SaveProject failed for {dst}")
        return "" if r == 1 else err.value.decode()

    @classmethod
    def summary(cls, path):
        """Section sizes as LoadProject reads them (see ref_emsim_summary)."""
        out = (C.c_int64 * 12)()
        err = C.create_string_buffer(256)
        if cls.lib().ref_emsim_summary(str(path).encode(), out, err, 256) != 1:
            raise OSError(err.value.decode())
        keys = ("settings", "objects", "faces", "face_vals", "plane_vals", "pattern_u", "pages",
                "page0_curves", "playback_valid", "playback_faces", "frames", "frame0_js")
        return dict(zip(keys, list(out)))
