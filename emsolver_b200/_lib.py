"""ctypes binding of the in-tree C ABI (include/tlm_b200.h, fdtd_b200.h,
emsim_b200.h).

The library is loaded from this package directory. There is no fallback: if
``libtlm_b200.so`` is missing or cannot be loaded, importing the binding
raises, and every compute call fails unless a CUDA device is present.
Set ``TLM_B200_VARIANT=checked`` to load the bounds-checked build instead.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))

TLM_OK, TLM_EINVAL, TLM_ENOMEM, TLM_ECUDA, TLM_ETIMEOUT, TLM_ESTOPPED, TLM_ESTATE, TLM_ENODEV, \
    TLM_EBUSY = range(9)
STATUS_NAMES = {0: "TLM_OK", 1: "TLM_EINVAL", 2: "TLM_ENOMEM", 3: "TLM_ECUDA", 4: "TLM_ETIMEOUT",
                5: "TLM_ESTOPPED", 6: "TLM_ESTATE", 7: "TLM_ENODEV", 8: "TLM_EBUSY"}

STORE_F32, STORE_BF16, STORE_F16, STORE_F64, STORE_BFP16 = range(5)
WAVE_CW_RAMPED, WAVE_GAUSSIAN_SINE, WAVE_GAUSSIAN_PULSE, WAVE_TABLE = range(4)


class TlmError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


class Grid(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("origin", C.c_float * 3),
                ("dl", C.c_float)]


class MatPropsC(C.Structure):
    _fields_ = [("epsr", C.c_float), ("sigma", C.c_float)]


class ConfigC(C.Structure):
    _fields_ = [("f0", C.c_float), ("waveform", C.c_int), ("total_steps", C.c_int),
                ("settle_steps", C.c_int), ("boundary_rho", C.c_float), ("huy_offset", C.c_int),
                ("use_gpu", C.c_int), ("record_every", C.c_int), ("storage", C.c_int),
                ("pulse_scale", C.c_float), ("steps_per_launch", C.c_int),
                ("kernel_variant", C.c_int), ("rounding", C.c_int), ("general_tiles", C.c_int),
                ("surface_monitors", C.c_int), ("no_staging", C.c_int), ("stage_wait_us", C.c_int),
                ("near_field", C.c_int)]


class EmsimFaceC(C.Structure):
    _fields_ = [("air_cell", C.c_int32), ("center", C.c_float * 3), ("axis", C.c_int8), ("sign", C.c_int8)]


class EmsimToolbarC(C.Structure):
    _fields_ = [(n, C.c_int) for n in ("solver", "excitation", "waveform", "currents", "db_range", "gpu",
                                       "show_model", "db_scale", "plane_on", "mesh_on")]


class EmsimObjectC(C.Structure):
    _fields_ = [("kind", C.c_int), ("name", C.c_char_p), ("position", C.c_float * 3), ("rot_deg", C.c_float * 3),
                ("dielectric", C.c_int), ("epsr", C.c_float), ("sigma", C.c_float),
                ("design_freq_hz", C.c_double), ("is_stl", C.c_int), ("n_stl_verts", C.c_uint32),
                ("stl_verts", C.POINTER(C.c_float)), ("n_stl_idx", C.c_uint32), ("stl_idx", C.POINTER(C.c_int32)),
                ("n_params", C.c_uint32)]


class EmsimPatternC(C.Structure):
    _fields_ = [("n_theta", C.c_int), ("n_phi", C.c_int), ("n_u", C.c_uint32), ("U", C.POINTER(C.c_float)),
                ("u_max", C.c_float), ("directivity", C.c_float), ("peak_theta_deg", C.c_float),
                ("peak_phi_deg", C.c_float)]


class EmsimResultC(C.Structure):
    _fields_ = [("n_faces", C.c_uint32), ("faces", C.POINTER(EmsimFaceC)),
                ("n_face_vals", C.c_uint32), ("face_vals", C.POINTER(C.c_float)), ("face_dl", C.c_float),
                ("n_tri_v", C.c_uint32), ("tri_v", C.POINTER(C.c_float)),
                ("n_tri_idx", C.c_uint32), ("tri_idx", C.POINTER(C.c_int32)),
                ("n_tri_mag", C.c_uint32), ("tri_mag", C.POINTER(C.c_float)),
                ("n_wire_pts", C.c_uint32), ("wire_pts", C.POINTER(C.c_float)),
                ("n_wire_mag", C.c_uint32), ("wire_mag", C.POINTER(C.c_float)),
                ("has_plane", C.c_int), ("plane_grid", Grid), ("plane_axis", C.c_int), ("plane_index", C.c_int),
                ("plane_n1", C.c_int), ("plane_n2", C.c_int),
                ("n_plane_vals", C.c_uint32), ("plane_vals", C.POINTER(C.c_float)),
                ("has_pattern", C.c_int), ("pattern", EmsimPatternC), ("pat_center", C.c_float * 3),
                ("pat_scale", C.c_float), ("domain_lo", C.c_float * 3), ("domain_hi", C.c_float * 3),
                ("domain_visible", C.c_int), ("n_probe_markers", C.c_uint32),
                ("probe_markers", C.POINTER(C.c_float))]


class EmsimCurveC(C.Structure):
    _fields_ = [("name", C.c_char_p), ("color", C.c_uint32), ("n_x", C.c_uint32), ("x", C.POINTER(C.c_double)),
                ("n_y", C.c_uint32), ("y", C.POINTER(C.c_double))]


class EmsimFrameC(C.Structure):
    _fields_ = [("step", C.c_int), ("plane_axis", C.c_int), ("plane_index", C.c_int), ("plane_n1", C.c_int),
                ("plane_n2", C.c_int), ("n_js", C.c_uint32), ("js", C.POINTER(C.c_float)),
                ("n_plane", C.c_uint32), ("plane", C.POINTER(C.c_float))]


class EmsimCaptureC(C.Structure):
    _fields_ = [("js_dft", C.c_int), ("n_theta", C.c_int), ("n_phi", C.c_int), ("playback", C.c_int)]


class BatchTuningC(C.Structure):
    _fields_ = [("kernel_variant", C.c_int), ("steps_per_launch", C.c_int),
                ("blocks_per_sm", C.c_int), ("use_graphs", C.c_int), ("overlap", C.c_int),
                ("ms_per_step", C.c_double)]


class RequestC(C.Structure):
    _fields_ = [("grid", Grid), ("mat", C.POINTER(C.c_uint8)), ("n_cells", C.c_size_t),
                ("table", C.POINTER(MatPropsC)), ("n_table", C.c_int), ("cfg", ConfigC),
                ("source_table", C.POINTER(C.c_float)), ("n_source", C.c_int),
                ("n_ports", C.c_int), ("port_cells", C.POINTER(C.c_uint64)),
                ("port_ncells", C.POINTER(C.c_int)), ("port_pol", C.POINTER(C.c_int)),
                ("port_amp", C.POINTER(C.c_float)), ("n_probes", C.c_int),
                ("probe_ijk", C.POINTER(C.c_int)), ("n_freq", C.c_int),
                ("freqs", C.POINTER(C.c_double))]


class ServerStatsC(C.Structure):
    _fields_ = [("completed", C.c_longlong), ("failed", C.c_longlong), ("cancelled", C.c_longlong),
                ("queued", C.c_longlong), ("running", C.c_longlong),
                ("latency_p50_s", C.c_double), ("latency_p99_s", C.c_double),
                ("latency_mean_s", C.c_double), ("solves_per_s", C.c_double),
                ("hbm_used_bytes", C.c_size_t), ("hbm_budget_bytes", C.c_size_t),
                ("windows", C.c_longlong), ("busy_s", C.c_double), ("gpu_window_s", C.c_double),
                ("setup_s", C.c_double), ("retire_s", C.c_double), ("mean_running_cells", C.c_double)]


_h = C.c_void_p
_st = C.c_int
_P = C.POINTER

# name -> (restype, argtypes): every symbol include/tlm_b200.h declares.
SIGNATURES = {
    "tlm_version": (C.c_char_p, []),
    "tlm_config_default": (None, [_P(ConfigC)]),
    "tlm_create": (_st, [_P(_h), C.c_int]),
    "tlm_destroy": (_st, [_h]),
    "tlm_last_error": (C.c_char_p, [_h]),
    "tlm_setup": (_st, [_h, _P(Grid), _P(C.c_uint8), C.c_size_t, _P(MatPropsC), C.c_int,
                        _P(ConfigC)]),
    "tlm_add_port": (_st, [_h, _P(C.c_uint64), C.c_int, C.c_int, C.c_float, _P(C.c_int)]),
    "tlm_add_plane_wave": (_st, [_h, C.c_int, C.c_int, C.c_int, C.c_float]),
    "tlm_add_source_cells": (_st, [_h, _P(C.c_uint64), C.c_int, C.c_int, C.c_float]),
    "tlm_add_probe": (_st, [_h, C.c_float, C.c_float, C.c_float, _P(C.c_int)]),
    "tlm_add_probe_cell": (_st, [_h, C.c_int, C.c_int, C.c_int, _P(C.c_int)]),
    "tlm_set_source_table": (_st, [_h, _P(C.c_float), C.c_int]),
    "tlm_set_port_dft": (_st, [_h, _P(C.c_double), C.c_int]),
    "tlm_step": (_st, [_h, C.c_int]),
    "tlm_step_async": (_st, [_h, C.c_int]),
    "tlm_sync": (_st, [_h]),
    "tlm_run": (_st, [_h]),
    "tlm_request_stop": (_st, [_h]),
    "tlm_current_step": (C.c_int, [_h]),
    "tlm_current_energy": (C.c_float, [_h]),
    "tlm_is_running": (C.c_int, [_h]),
    "tlm_is_finished": (C.c_int, [_h]),
    "tlm_total_steps": (C.c_int, [_h]),
    "tlm_timestep": (_st, [_h, _P(C.c_float)]),
    "tlm_probe_count": (C.c_int, [_h]),
    "tlm_get_probe": (_st, [_h, C.c_int, _P(C.c_float), _P(C.c_float), _P(C.c_float), C.c_int,
                            _P(C.c_int)]),
    "tlm_get_probe_f64": (_st, [_h, C.c_int, _P(C.c_double), _P(C.c_double), _P(C.c_double),
                                C.c_int, _P(C.c_int)]),
    "tlm_get_probe_cell": (_st, [_h, C.c_int, _P(C.c_uint64)]),
    "tlm_port_count": (C.c_int, [_h]),
    "tlm_get_port": (_st, [_h, C.c_int, _P(C.c_float), _P(C.c_float), C.c_int, _P(C.c_int)]),
    "tlm_get_port_f64": (_st, [_h, C.c_int, _P(C.c_double), _P(C.c_double), C.c_int,
                               _P(C.c_int)]),
    "tlm_get_port_cells": (_st, [_h, C.c_int, _P(C.c_uint64), C.c_int, _P(C.c_int)]),
    "tlm_get_port_dft": (_st, [_h, C.c_int, _P(C.c_double), _P(C.c_double), _P(C.c_double),
                               _P(C.c_double), C.c_int, _P(C.c_int)]),
    "tlm_get_energy_history": (_st, [_h, _P(C.c_int), _P(C.c_float), _P(C.c_double), C.c_int,
                                     _P(C.c_int)]),
    "tlm_get_pulses": (_st, [_h, _P(C.c_float), C.c_size_t]),
    "tlm_get_pulses_f64": (_st, [_h, _P(C.c_double), C.c_size_t]),
    "tlm_set_pulses": (_st, [_h, _P(C.c_float), C.c_size_t]),
    "tlm_get_stubs": (_st, [_h, _P(C.c_float), C.c_size_t]),
    "tlm_get_materials": (_st, [_h, _P(C.c_uint8), C.c_size_t]),
    "tlm_get_tables": (_st, [_h, _P(C.c_float), _P(C.c_float), C.c_int, _P(C.c_int)]),
    "tlm_waveform_value": (_st, [C.c_int, C.c_float, C.c_float, C.c_int, _P(C.c_float)]),
    "tlm_scatter_unitarity_error": (_st, [C.c_int, _P(C.c_float)]),
    "tlm_stub_unitarity_error": (_st, [C.c_int, C.c_float, _P(C.c_float)]),
    "tlm_get_surface_faces": (_st, [_h, _P(C.c_uint64), _P(C.c_int), _P(C.c_int), _P(C.c_float), C.c_int,
                                    _P(C.c_int)]),
    "tlm_get_js_instant": (_st, [_h, _P(C.c_float), C.c_int, _P(C.c_int)]),
    "tlm_get_js_dft": (_st, [_h, _P(C.c_float), _P(C.c_float), _P(C.c_float), C.c_int, _P(C.c_int),
                             _P(C.c_int)]),
    "tlm_get_huygens_faces": (_st, [_h, _P(C.c_uint64), _P(C.c_int), _P(C.c_int), _P(C.c_float), C.c_int,
                                    _P(C.c_int)]),
    "tlm_get_huygens_dft": (_st, [_h, _P(C.c_float), C.c_int, _P(C.c_int), _P(C.c_int)]),
    "tlm_set_field_plane": (_st, [_h, C.c_int, C.c_int]),
    "tlm_get_field_plane": (_st, [_h, _P(C.c_float), C.c_size_t, _P(C.c_int), _P(C.c_int), _P(C.c_int),
                                  _P(C.c_int)]),
    "tlm_frame_count": (_st, [_h, _P(C.c_int)]),
    "tlm_get_frame": (_st, [_h, C.c_int, _P(C.c_int), _P(C.c_float), C.c_int, _P(C.c_float), C.c_size_t,
                            _P(C.c_int), _P(C.c_int), _P(C.c_int), _P(C.c_int)]),
    "tlm_compute_far_field": (_st, [_h, C.c_int, C.c_int, _P(C.c_float), _P(C.c_float), _P(C.c_float),
                                    _P(C.c_float), _P(C.c_float)]),
    # Yee FDTD (include/fdtd_b200.h)
    "fdtd_create": (_st, [_P(_h), C.c_int]),
    "fdtd_destroy": (_st, [_h]),
    "fdtd_last_error": (C.c_char_p, [_h]),
    "fdtd_setup": (_st, [_h, _P(Grid), _P(C.c_uint8), C.c_size_t, _P(MatPropsC), C.c_int, _P(ConfigC)]),
    "fdtd_add_port": (_st, [_h, _P(C.c_uint64), C.c_int, C.c_int, C.c_float, _P(C.c_int)]),
    "fdtd_add_plane_wave": (_st, [_h, C.c_int, C.c_int, C.c_int, C.c_float]),
    "fdtd_add_probe": (_st, [_h, C.c_float, C.c_float, C.c_float, _P(C.c_int)]),
    "fdtd_set_source_table": (_st, [_h, _P(C.c_float), C.c_int]),
    "fdtd_step": (_st, [_h, C.c_int]),
    "fdtd_run": (_st, [_h]),
    "fdtd_current_step": (C.c_int, [_h]),
    "fdtd_get_stream": (_st, [_h, _P(C.c_void_p)]),
    "fdtd_timestep": (C.c_float, [_h]),
    "fdtd_get_field": (_st, [_h, C.c_int, _P(C.c_float), C.c_size_t, _P(C.c_size_t)]),
    "fdtd_get_probe": (_st, [_h, C.c_int, _P(C.c_float), _P(C.c_float), _P(C.c_float), C.c_int, _P(C.c_int)]),
    "fdtd_get_port": (_st, [_h, C.c_int, _P(C.c_float), _P(C.c_float), C.c_int, _P(C.c_int)]),
    "fdtd_get_energy_history": (_st, [_h, _P(C.c_int), _P(C.c_float), _P(C.c_double), C.c_int, _P(C.c_int)]),
    "fdtd_get_surface_faces": (_st, [_h, _P(C.c_uint64), _P(C.c_int), _P(C.c_int), _P(C.c_float), C.c_int,
                                     _P(C.c_int)]),
    "fdtd_get_js_instant": (_st, [_h, _P(C.c_float), C.c_int, _P(C.c_int)]),
    "fdtd_get_js_dft": (_st, [_h, _P(C.c_float), _P(C.c_float), _P(C.c_float), C.c_int, _P(C.c_int),
                              _P(C.c_int)]),
    "fdtd_get_huygens_faces": (_st, [_h, _P(C.c_uint64), _P(C.c_int), _P(C.c_int), _P(C.c_float), C.c_int,
                                     _P(C.c_int)]),
    "fdtd_get_huygens_dft": (_st, [_h, _P(C.c_float), C.c_int, _P(C.c_int), _P(C.c_int)]),
    "fdtd_set_field_plane": (_st, [_h, C.c_int, C.c_int]),
    "fdtd_get_field_plane": (_st, [_h, _P(C.c_float), C.c_size_t, _P(C.c_int), _P(C.c_int), _P(C.c_int),
                                   _P(C.c_int)]),
    "fdtd_frame_count": (_st, [_h, _P(C.c_int)]),
    "fdtd_get_frame": (_st, [_h, C.c_int, _P(C.c_int), _P(C.c_float), C.c_int, _P(C.c_float), C.c_size_t,
                             _P(C.c_int), _P(C.c_int), _P(C.c_int), _P(C.c_int)]),
    "fdtd_compute_far_field": (_st, [_h, C.c_int, C.c_int, _P(C.c_float), _P(C.c_float), _P(C.c_float),
                                     _P(C.c_float), _P(C.c_float)]),
    "tlm_step_planes_noalloc": (_st, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                      C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_float,
                                      C.c_int, C.c_void_p, C.c_void_p]),
    "tlm_kernel_variants": (C.c_int, [C.c_int]),
    "tlm_kernel_variant_info": (_st, [C.c_int, C.c_int, _P(C.c_int), _P(C.c_int)]),
    "tlm_batch_create": (_st, [_P(_h), C.c_int]),
    "tlm_batch_destroy": (_st, [_h]),
    "tlm_batch_attach": (_st, [_h, _h]),
    "tlm_batch_detach": (_st, [_h, _h]),
    "tlm_batch_size": (C.c_int, [_h]),
    "tlm_batch_active": (C.c_int, [_h]),
    "tlm_batch_step": (_st, [_h, C.c_int]),
    "tlm_batch_run": (_st, [_h]),
    "tlm_batch_launch_window": (_st, [_h, _P(C.c_int)]),
    "tlm_batch_sync": (_st, [_h]),
    "tlm_batch_set_tuning": (_st, [_h, _P(BatchTuningC)]),
    "tlm_batch_get_tuning": (_st, [_h, _P(BatchTuningC)]),
    "tlm_batch_autotune": (_st, [_h, C.c_int, _P(BatchTuningC)]),
    "tlm_batch_get_stream": (_st, [_h, _P(C.c_void_p)]),
    "tlm_server_create": (_st, [_P(_h), C.c_int, C.c_size_t, C.c_int]),
    "tlm_server_set_policy": (_st, [C.c_void_p, C.c_int, C.c_longlong, C.c_longlong]),
    "tlm_server_destroy": (_st, [_h]),
    "tlm_server_submit": (_st, [_h, _P(RequestC), _P(C.c_uint64)]),
    "tlm_server_poll": (_st, [_h, C.c_uint64, _P(C.c_int)]),
    "tlm_server_wait": (_st, [_h, C.c_uint64, C.c_double, _P(C.c_int)]),
    "tlm_server_cancel": (_st, [_h, C.c_uint64]),
    "tlm_server_result": (_st, [_h, C.c_uint64, C.c_int, _P(C.c_double), _P(C.c_double),
                                _P(C.c_double), _P(C.c_double), C.c_int, _P(C.c_int),
                                _P(C.c_double)]),
    "tlm_server_port_records": (_st, [_h, C.c_uint64, C.c_int, _P(C.c_float), _P(C.c_float),
                                      C.c_int, _P(C.c_int)]),
    "tlm_server_release": (_st, [_h, C.c_uint64]),
    "tlm_server_stats": (_st, [_h, _P(ServerStatsC)]),
    "tlm_request_footprint": (_st, [_P(RequestC), _P(C.c_size_t)]),
    "tlm_get_stream": (_st, [_h, _P(C.c_void_p)]),
    "tlm_get_grid": (_st, [_h, _P(Grid)]),
    "tlm_set_slab": (_st, [_h, C.c_int, C.c_int]),
    "tlm_halo_bytes": (_st, [_h, _P(C.c_size_t)]),
    "tlm_halo_pack": (_st, [_h, C.c_void_p, C.c_void_p]),
    "tlm_halo_unpack": (_st, [_h, C.c_void_p, C.c_void_p]),
    "fdtd_get_grid": (_st, [_h, _P(Grid)]),
    "emsim_new": (_st, [_P(_h)]),
    "emsim_load": (_st, [C.c_char_p, _P(_h), C.c_char_p, C.c_size_t]),
    "emsim_save": (_st, [_h, C.c_char_p]),
    "emsim_free": (None, [_h]),
    "emsim_last_error": (C.c_char_p, [_h]),
    "emsim_file_version": (C.c_int, [_h]),
    "emsim_setting_count": (C.c_int, [_h]),
    "emsim_get_setting": (_st, [_h, C.c_int, _P(C.c_char_p), _P(C.c_char_p)]),
    "emsim_add_setting": (_st, [_h, C.c_char_p, C.c_char_p]),
    "emsim_clear_settings": (_st, [_h]),
    "emsim_get_toolbar": (_st, [_h, _P(EmsimToolbarC)]),
    "emsim_set_toolbar": (_st, [_h, _P(EmsimToolbarC)]),
    "emsim_object_count": (C.c_int, [_h]),
    "emsim_get_object": (_st, [_h, C.c_int, _P(EmsimObjectC)]),
    "emsim_get_object_param": (_st, [_h, C.c_int, C.c_int, _P(C.c_char_p), _P(C.c_double)]),
    "emsim_add_object": (_st, [_h, _P(EmsimObjectC), _P(C.c_int)]),
    "emsim_add_object_param": (_st, [_h, C.c_int, C.c_char_p, C.c_double]),
    "emsim_clear_objects": (_st, [_h]),
    "emsim_result_default": (None, [_P(EmsimResultC)]),
    "emsim_get_result": (_st, [_h, _P(EmsimResultC)]),
    "emsim_set_result": (_st, [_h, _P(EmsimResultC)]),
    "emsim_page_count": (C.c_int, [_h]),
    "emsim_get_page": (_st, [_h, C.c_int, _P(C.c_char_p), _P(C.c_char_p), _P(C.c_char_p), _P(C.c_int)]),
    "emsim_get_curve": (_st, [_h, C.c_int, C.c_int, _P(EmsimCurveC)]),
    "emsim_add_page": (_st, [_h, C.c_char_p, C.c_char_p, C.c_char_p, _P(C.c_int)]),
    "emsim_add_curve": (_st, [_h, C.c_int, _P(EmsimCurveC)]),
    "emsim_clear_pages": (_st, [_h]),
    "emsim_get_playback": (_st, [_h, _P(C.c_int), _P(Grid), _P(C.c_float), _P(_P(EmsimFaceC)),
                                 _P(C.c_uint32), _P(C.c_uint32)]),
    "emsim_set_playback": (_st, [_h, _P(Grid), C.c_float, _P(EmsimFaceC), C.c_uint32]),
    "emsim_get_frame": (_st, [_h, C.c_uint32, _P(EmsimFrameC)]),
    "emsim_add_frame": (_st, [_h, _P(EmsimFrameC)]),
    "emsim_clear_playback": (_st, [_h]),
    "emsim_from_tlm": (_st, [_h, _h, _P(EmsimCaptureC)]),
    "emsim_from_fdtd": (_st, [_h, _h, _P(EmsimCaptureC)]),
    "tlm_device_bytes": (_st, [_h, _P(C.c_size_t)]),
    "tlm_set_kernel_timing": (_st, [_h, C.c_int]),
    "tlm_kernel_time": (_st, [_h, _P(C.c_double), _P(C.c_longlong)]),
    "tlm_slab_step_begin": (_st, [_h, C.c_void_p, C.c_void_p]),
    "tlm_slab_step_end": (_st, [_h, C.c_void_p, C.c_void_p]),
    "tlm_slab_flush": (_st, [_h]),
    "tlm_get_halo_stream": (_st, [_h, _P(C.c_void_p)]),
    "tlm_step_launches": (_st, [_h, _P(C.c_int)]),
    "tlm_near_field_box": (_st, [_h, _P(C.c_int)]),
}


def library_path(variant: str | None = None) -> str:
    variant = variant or os.environ.get("TLM_B200_VARIANT", "")
    name = "libtlm_b200_checked.so" if variant == "checked" else "libtlm_b200.so"
    return os.path.join(HERE, name)


_LIBS: dict = {}


def load(variant: str | None = None):
    """Load (once) and return the C library with its prototypes set."""
    path = library_path(variant)
    if path in _LIBS:
        return _LIBS[path]
    if not os.path.exists(path):
        raise ImportError(f"{path} is not built; run emsolver_b200.build.build() "
                          "(there is no CPU fallback)")
    lib = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _LIBS[path] = lib
    return lib


def check(lib, h, status):
    if status != TLM_OK:
        msg = lib.tlm_last_error(h)
        raise TlmError(status, msg.decode() if msg else "")
    return status
