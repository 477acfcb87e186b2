"""The .emsim project file (the reference's ProjectIO.h / ProjectIO.cpp,
format version 2) through the C ABI of include/emsim_b200.h.

``load_project(path)`` mirrors ``LoadProject`` (raising ``EmsimError`` with
the reference's message), ``Project.save(path)`` mirrors ``SaveProject``.
Sections read back as plain Python values and numpy arrays; ``capture``
fills the result and playback sections from a solver the way the reference's
main window does before saving a finished run.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import (EmsimCaptureC, EmsimCurveC, EmsimFaceC, EmsimFrameC, EmsimObjectC, EmsimResultC,
                   EmsimToolbarC, Grid, TLM_OK)

TOOLBAR_FIELDS = ("solver", "excitation", "waveform", "currents", "db_range", "gpu", "show_model", "db_scale",
                  "plane_on", "mesh_on")


class EmsimError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(message)
        self.status = status


def _arr(ptr, n, dtype, shape=None):
    if not n or not ptr:
        a = np.zeros(0, dtype)
    else:
        a = np.ctypeslib.as_array(ptr, shape=(n,)).astype(dtype, copy=True)
    return a.reshape(shape) if shape else a


def _vecs(ptr, n):
    return _arr(ptr, 3 * n, np.float32, (-1, 3)) if n else np.zeros((0, 3), np.float32)


def _ptr(a, ctype):
    return a.ctypes.data_as(C.POINTER(ctype)) if a is not None and a.size else None


def _faces_to_c(faces):
    n = len(faces["cells"]) if faces else 0
    arr = (EmsimFaceC * max(n, 1))()
    for i in range(n):
        arr[i].air_cell = int(faces["cells"][i])
        arr[i].center[:] = [float(v) for v in faces["center"][i]]
        arr[i].axis = int(faces["axis"][i])
        arr[i].sign = int(faces["sign"][i])
    return arr, n


def _faces_from_c(ptr, n):
    cells = np.zeros(n, np.int32)
    center = np.zeros((n, 3), np.float32)
    axis = np.zeros(n, np.int8)
    sign = np.zeros(n, np.int8)
    for i in range(n):
        f = ptr[i]
        cells[i], axis[i], sign[i] = f.air_cell, f.axis, f.sign
        center[i] = list(f.center)
    return {"cells": cells, "center": center, "axis": axis, "sign": sign}


def _grid_dict(g):
    return {"nx": g.nx, "ny": g.ny, "nz": g.nz, "origin": tuple(g.origin), "dl": g.dl}


def _grid_c(d):
    g = Grid()
    g.nx, g.ny, g.nz = int(d["nx"]), int(d["ny"]), int(d["nz"])
    g.origin[:] = [float(v) for v in d["origin"]]
    g.dl = float(d["dl"])
    return g


class Project:
    """One project in memory (ProjectData, ProjectIO.h:46-57)."""

    def __init__(self, _handle=None):
        self._L = _lib.load()
        if _handle is None:
            h = C.c_void_p()
            st = self._L.emsim_new(C.byref(h))
            if st != TLM_OK:
                raise EmsimError(st, "out of host memory")
            _handle = h
        self._h = _handle

    def close(self):
        if self._h:
            self._L.emsim_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _c(self, st):
        if st != TLM_OK:
            raise EmsimError(st, (self._L.emsim_last_error(self._h) or b"").decode())

    # -- file -----------------------------------------------------------
    def save(self, path):
        """SaveProject (ProjectIO.cpp:137-191): format version 2."""
        self._c(self._L.emsim_save(self._h, str(path).encode()))

    @property
    def file_version(self):
        return self._L.emsim_file_version(self._h)

    # -- settings and toolbar --------------------------------------------
    @property
    def settings(self):
        out = []
        for i in range(self._L.emsim_setting_count(self._h)):
            k, v = C.c_char_p(), C.c_char_p()
            self._c(self._L.emsim_get_setting(self._h, i, C.byref(k), C.byref(v)))
            out.append((k.value.decode(), v.value.decode()))
        return out

    def add_setting(self, key, value):
        self._c(self._L.emsim_add_setting(self._h, key.encode(), value.encode()))

    def clear_settings(self):
        self._c(self._L.emsim_clear_settings(self._h))

    @property
    def toolbar(self):
        t = EmsimToolbarC()
        self._c(self._L.emsim_get_toolbar(self._h, C.byref(t)))
        return {f: getattr(t, f) for f in TOOLBAR_FIELDS}

    def set_toolbar(self, **kw):
        t = EmsimToolbarC()
        self._c(self._L.emsim_get_toolbar(self._h, C.byref(t)))
        for k, v in kw.items():
            setattr(t, k, int(v))
        self._c(self._L.emsim_set_toolbar(self._h, C.byref(t)))

    # -- objects ---------------------------------------------------------
    @property
    def objects(self):
        out = []
        for i in range(self._L.emsim_object_count(self._h)):
            o = EmsimObjectC()
            self._c(self._L.emsim_get_object(self._h, i, C.byref(o)))
            params = []
            for p in range(o.n_params):
                nm, val = C.c_char_p(), C.c_double()
                self._c(self._L.emsim_get_object_param(self._h, i, p, C.byref(nm), C.byref(val)))
                params.append((nm.value.decode(), val.value))
            out.append({"kind": o.kind, "name": o.name.decode(), "position": tuple(o.position),
                        "rot_deg": tuple(o.rot_deg), "dielectric": bool(o.dielectric), "epsr": o.epsr,
                        "sigma": o.sigma, "design_freq_hz": o.design_freq_hz, "is_stl": bool(o.is_stl),
                        "stl_verts": _arr(o.stl_verts, o.n_stl_verts, np.float32),
                        "stl_idx": _arr(o.stl_idx, o.n_stl_idx, np.int32), "params": params})
        return out

    def add_object(self, kind, name, position=(0, 0, 0), rot_deg=(0, 0, 0), dielectric=False, epsr=4.0,
                   sigma=0.0, design_freq_hz=1e9, stl_verts=None, stl_idx=None, params=()):
        verts = None if stl_verts is None else np.ascontiguousarray(stl_verts, np.float32).ravel()
        idx = None if stl_idx is None else np.ascontiguousarray(stl_idx, np.int32).ravel()
        o = EmsimObjectC()
        o.kind, o.name = int(kind), name.encode()
        o.position[:], o.rot_deg[:] = [float(v) for v in position], [float(v) for v in rot_deg]
        o.dielectric, o.epsr, o.sigma, o.design_freq_hz = int(bool(dielectric)), epsr, sigma, design_freq_hz
        o.is_stl = int(verts is not None)
        o.n_stl_verts, o.stl_verts = (0 if verts is None else verts.size), _ptr(verts, C.c_float)
        o.n_stl_idx, o.stl_idx = (0 if idx is None else idx.size), _ptr(idx, C.c_int32)
        i = C.c_int()
        self._c(self._L.emsim_add_object(self._h, C.byref(o), C.byref(i)))
        for k, v in params:
            self._c(self._L.emsim_add_object_param(self._h, i.value, k.encode(), float(v)))
        return i.value

    def clear_objects(self):
        self._c(self._L.emsim_clear_objects(self._h))

    # -- result ----------------------------------------------------------
    @property
    def result(self):
        r = EmsimResultC()
        self._c(self._L.emsim_get_result(self._h, C.byref(r)))
        p = r.pattern
        return {"faces": _faces_from_c(r.faces, r.n_faces), "face_vals": _arr(r.face_vals, r.n_face_vals, np.float32),
                "face_dl": r.face_dl, "tri_v": _vecs(r.tri_v, r.n_tri_v),
                "tri_idx": _arr(r.tri_idx, r.n_tri_idx, np.int32), "tri_mag": _arr(r.tri_mag, r.n_tri_mag, np.float32),
                "wire_pts": _vecs(r.wire_pts, r.n_wire_pts), "wire_mag": _arr(r.wire_mag, r.n_wire_mag, np.float32),
                "has_plane": bool(r.has_plane), "plane_grid": _grid_dict(r.plane_grid), "plane_axis": r.plane_axis,
                "plane_index": r.plane_index, "plane_n1": r.plane_n1, "plane_n2": r.plane_n2,
                "plane_vals": _arr(r.plane_vals, r.n_plane_vals, np.float32), "has_pattern": bool(r.has_pattern),
                "pattern": {"n_theta": p.n_theta, "n_phi": p.n_phi, "U": _arr(p.U, p.n_u, np.float32),
                            "u_max": p.u_max, "directivity": p.directivity, "peak_theta_deg": p.peak_theta_deg,
                            "peak_phi_deg": p.peak_phi_deg},
                "pat_center": tuple(r.pat_center), "pat_scale": r.pat_scale, "domain_lo": tuple(r.domain_lo),
                "domain_hi": tuple(r.domain_hi), "domain_visible": bool(r.domain_visible),
                "probe_markers": _vecs(r.probe_markers, r.n_probe_markers)}

    def set_result(self, **kw):
        """Replace the result section; keys as `result` returns them, missing
        ones take GLResult's defaults."""
        r = EmsimResultC()
        self._L.emsim_result_default(C.byref(r))
        keep = []

        def arr(key, dtype):
            a = kw.get(key)
            if a is None:
                return None, 0
            a = np.ascontiguousarray(a, dtype)
            keep.append(a)
            return a, a.size

        faces, nf = _faces_to_c(kw.get("faces"))
        r.faces, r.n_faces = (faces if nf else None), nf
        for key, ctype, dtype, vec in (("face_vals", C.c_float, np.float32, False),
                                       ("tri_v", C.c_float, np.float32, True),
                                       ("tri_idx", C.c_int32, np.int32, False),
                                       ("tri_mag", C.c_float, np.float32, False),
                                       ("wire_pts", C.c_float, np.float32, True),
                                       ("wire_mag", C.c_float, np.float32, False),
                                       ("plane_vals", C.c_float, np.float32, False),
                                       ("probe_markers", C.c_float, np.float32, True)):
            a, n = arr(key, dtype)
            setattr(r, key, _ptr(a, ctype))
            setattr(r, "n_" + key, n // 3 if vec else n)
        for key in ("face_dl", "plane_axis", "plane_index", "plane_n1", "plane_n2", "pat_scale"):
            if key in kw:
                setattr(r, key, kw[key])
        for key in ("has_plane", "has_pattern", "domain_visible"):
            if key in kw:
                setattr(r, key, int(bool(kw[key])))
        for key in ("pat_center", "domain_lo", "domain_hi"):
            if key in kw:
                getattr(r, key)[:] = [float(v) for v in kw[key]]
        if "plane_grid" in kw:
            r.plane_grid = _grid_c(kw["plane_grid"])
        if "pattern" in kw:
            pt = kw["pattern"]
            r.pattern.n_theta, r.pattern.n_phi = pt["n_theta"], pt["n_phi"]
            U = np.ascontiguousarray(pt["U"], np.float32)
            keep.append(U)
            r.pattern.U, r.pattern.n_u = _ptr(U, C.c_float), U.size
            for k in ("u_max", "directivity", "peak_theta_deg", "peak_phi_deg"):
                setattr(r.pattern, k, pt.get(k, 0.0))
        self._c(self._L.emsim_set_result(self._h, C.byref(r)))

    # -- plot pages ------------------------------------------------------
    @property
    def pages(self):
        out = []
        for i in range(self._L.emsim_page_count(self._h)):
            t, x, y, nc = C.c_char_p(), C.c_char_p(), C.c_char_p(), C.c_int()
            self._c(self._L.emsim_get_page(self._h, i, C.byref(t), C.byref(x), C.byref(y), C.byref(nc)))
            curves = []
            for c in range(nc.value):
                cv = EmsimCurveC()
                self._c(self._L.emsim_get_curve(self._h, i, c, C.byref(cv)))
                curves.append({"name": cv.name.decode(), "color": cv.color, "x": _arr(cv.x, cv.n_x, np.float64),
                               "y": _arr(cv.y, cv.n_y, np.float64)})
            out.append({"title": t.value.decode(), "x_label": x.value.decode(), "y_label": y.value.decode(),
                        "curves": curves})
        return out

    def add_page(self, title, x_label, y_label, curves=()):
        i = C.c_int()
        self._c(self._L.emsim_add_page(self._h, title.encode(), x_label.encode(), y_label.encode(), C.byref(i)))
        for c in curves:
            self.add_curve(i.value, c["name"], c["x"], c["y"], c.get("color", 0))
        return i.value

    def add_curve(self, page, name, x, y, color=0):
        x = np.ascontiguousarray(x, np.float64)
        y = np.ascontiguousarray(y, np.float64)
        cv = EmsimCurveC(name.encode(), int(color), x.size, _ptr(x, C.c_double), y.size, _ptr(y, C.c_double))
        self._c(self._L.emsim_add_curve(self._h, page, C.byref(cv)))

    def clear_pages(self):
        self._c(self._L.emsim_clear_pages(self._h))

    # -- playback --------------------------------------------------------
    @property
    def playback(self):
        valid, g, dt = C.c_int(), Grid(), C.c_float()
        fp, nf, nfr = C.POINTER(EmsimFaceC)(), C.c_uint32(), C.c_uint32()
        self._c(self._L.emsim_get_playback(self._h, C.byref(valid), C.byref(g), C.byref(dt), C.byref(fp),
                                           C.byref(nf), C.byref(nfr)))
        frames = []
        for i in range(nfr.value):
            f = EmsimFrameC()
            self._c(self._L.emsim_get_frame(self._h, i, C.byref(f)))
            frames.append({"step": f.step, "plane_axis": f.plane_axis, "plane_index": f.plane_index,
                           "plane_n1": f.plane_n1, "plane_n2": f.plane_n2,
                           "js": _arr(f.js, f.n_js, np.float32), "plane": _arr(f.plane, f.n_plane, np.float32)})
        return {"valid": bool(valid.value), "grid": _grid_dict(g), "dt": dt.value,
                "faces": _faces_from_c(fp, nf.value), "frames": frames}

    def set_playback(self, grid, dt, faces):
        arr, n = _faces_to_c(faces)
        self._c(self._L.emsim_set_playback(self._h, C.byref(_grid_c(grid)), float(dt), arr, n))

    def add_frame(self, step, js, plane=None, plane_axis=-1, plane_index=0, plane_n1=0, plane_n2=0):
        js = np.ascontiguousarray(js, np.float32)
        pl = None if plane is None else np.ascontiguousarray(plane, np.float32)
        f = EmsimFrameC(int(step), int(plane_axis), int(plane_index), int(plane_n1), int(plane_n2), js.size,
                        _ptr(js, C.c_float), 0 if pl is None else pl.size, _ptr(pl, C.c_float))
        self._c(self._L.emsim_add_frame(self._h, C.byref(f)))

    def clear_playback(self):
        self._c(self._L.emsim_clear_playback(self._h))

    # -- from a solver ---------------------------------------------------
    def capture(self, solver, js_dft=True, n_theta=0, n_phi=0, playback=True):
        """Result and playback of a finished run (MainUnit.cpp:1025-1057,
        2026-2043, 2275-2302) from a TlmSolver or FdtdSolver."""
        from .fdtd import FdtdSolver
        c = EmsimCaptureC(int(bool(js_dft)), int(n_theta), int(n_phi), int(bool(playback)))
        fn = self._L.emsim_from_fdtd if isinstance(solver, FdtdSolver) else self._L.emsim_from_tlm
        self._c(fn(self._h, solver._h, C.byref(c)))


def load_project(path) -> Project:
    """LoadProject (ProjectIO.cpp:194-248); EmsimError carries its message."""
    L = _lib.load()
    h = C.c_void_p()
    err = C.create_string_buffer(256)
    st = L.emsim_load(str(path).encode(), C.byref(h), err, 256)
    if st != TLM_OK:
        raise EmsimError(st, err.value.decode())
    return Project(h)
