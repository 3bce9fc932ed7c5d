"""ctypes mirror of include/supra_b200.h and the loader of the native library.

This is the binding a Python caller of the C ABI uses (the same role as a ctypes stub in a
SUPRA-side integration). The CUDA library is loaded from supra_b200/lib/libsupra_b200.so; there is
no fallback: if it is missing or fails to load, load_library() raises.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

import numpy as np

SB_OK = 0
SB_ERR_INVALID_ARG = -1
SB_ERR_CUDA = -2
SB_ERR_UNSUPPORTED = -3
SB_ERR_NO_MEMORY = -4
SB_ERR_TIMEOUT = -5
SB_ERR_NOT_READY = -6

SB_INT16 = 1
SB_FLOAT32 = 2
SB_UINT8 = 3
SB_COMPLEX64 = 4
SB_UINT16 = 5

SB_WINDOW_RECTANGULAR = 0
SB_WINDOW_HANN = 1
SB_WINDOW_HAMMING = 2
SB_WINDOW_GAUSS = 3

WINDOW_NAMES = {"Rectangular": 0, "Hann": 1, "Hamming": 2, "Gauss": 3}

# numpy views of the structs (byte layout identical to the C structs and to SUPRA's
# ScanlineRxParameters3D, SupraLib/USImageProperties.h:43-95)
TX_DTYPE = np.dtype([
    ("first", "<u2", (2,)),
    ("last", "<u2", (2,)),
    ("tx_idx", "<u2"),
    ("pad", "<u2", (3,)),
    ("initial_delay", "<f8"),
])
SCANLINE_DTYPE = np.dtype([
    ("position", "<f8", (3,)),
    ("direction", "<f8", (3,)),
    ("tx_weights", "<f8", (4,)),
    ("tx", TX_DTYPE, (4,)),
    ("max_element_distance", "<f8", (2,)),
])
assert TX_DTYPE.itemsize == 24 and SCANLINE_DTYPE.itemsize == 192


class sb_tx_params(C.Structure):
    _fields_ = [
        ("first_active_element", C.c_uint16 * 2),
        ("last_active_element", C.c_uint16 * 2),
        ("tx_scanline_idx", C.c_uint16),
        ("_pad", C.c_uint16 * 3),
        ("initial_delay_s", C.c_double),
    ]


class sb_scanline_rx(C.Structure):
    _fields_ = [
        ("position", C.c_double * 3),
        ("direction", C.c_double * 3),
        ("tx_weights", C.c_double * 4),
        ("tx", sb_tx_params * 4),
        ("max_element_distance", C.c_double * 2),
    ]


assert C.sizeof(sb_scanline_rx) == 192


class sb_geometry(C.Structure):
    _fields_ = [
        ("num_elements", C.c_uint32),
        ("element_layout", C.c_uint32 * 2),
        ("num_channels", C.c_uint32),
        ("num_samples", C.c_uint32),
        ("num_tx", C.c_uint32),
        ("num_rx", C.c_uint32),
        ("rx_layout", C.c_uint32 * 2),
        ("num_depths", C.c_uint32),
        ("sampling_frequency_hz", C.c_double),
        ("element_x_mm", C.POINTER(C.c_float)),
        ("element_y_mm", C.POINTER(C.c_float)),
        ("depths_mm", C.POINTER(C.c_float)),
        ("scanlines", C.c_void_p),
        ("element_to_channel", C.POINTER(C.c_int32)),
    ]


class sb_mv_stats(C.Structure):
    _fields_ = [
        ("systems", C.c_uint64),
        ("fp64_systems", C.c_uint64),
        ("max_condition_estimate", C.c_float),
    ]


class sb_batch_frame(C.Structure):
    _fields_ = [("probe", C.c_void_p), ("rf", C.c_void_p), ("iq_out", C.c_void_p)]


class sb_batch_params(C.Structure):
    _fields_ = [
        ("f_number", C.c_double),
        ("speed_of_sound_mm_s", C.c_double),
        ("window_type", C.c_int),
        ("window_parameter", C.c_float),
        ("mixing_frequency_hz", C.c_double),
        ("cutoff_frequency_hz", C.c_double),
        ("lowpass_length", C.c_uint32),
        ("decimation", C.c_uint32),
        ("ctas_per_sm", C.c_int32),
        ("depth_tile", C.c_int32),
        ("frames_per_pack", C.c_int32),
        ("staged", C.c_int32),
    ]


class sb_record(C.Structure):
    _fields_ = [("is_image", C.c_int), ("dtype", C.c_int), ("state", C.c_int), ("size", C.c_uint32 * 3),
                ("data", C.c_void_p)]


_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libsupra_b200.so")

_lib: Optional[C.CDLL] = None

_vp = C.c_void_p
_u32 = C.c_uint32
_i32 = C.c_int32
_int = C.c_int
_f32 = C.c_float
_f64 = C.c_double
_sz = C.c_size_t

_SIGNATURES = {
    "sb_last_error": (C.c_char_p, []),
    "sb_version": (_int, [C.POINTER(_int), C.POINTER(_int)]),
    "sb_window_lut": (_int, [_int, _f32, _u32, _vp]),
    "sb_fir_design": (_int, [_u32, _int, _int, _f64, _f64, _f64, _vp]),
    "sb_das_plan_create": (_int, [C.POINTER(sb_geometry), C.POINTER(_vp)]),
    "sb_das_plan_destroy": (_int, [_vp]),
    "sb_das_run": (_int, [_vp, _vp, _int, _vp, _int, _f64, _f64, _int, _f32, _int, _i32, _vp]),
    "sb_das_run_beamformer": (_int, [_vp, _int, _vp, _int, _vp, _int, _f64, _f64, _int, _f32, _int, _i32, _vp]),
    "sb_temporal_filter_run": (_int, [_vp, _u32, _vp, _int, _vp, _int, C.c_uint64, _vp]),
    "sb_selftest_bounded_wait": (_int, [_u32, _int, C.POINTER(_int), _vp]),
    "sb_selftest_sqrt": (_int, [_u32, C.c_uint64, C.POINTER(C.c_uint64), C.POINTER(_u32), _vp]),
    "sb_analytic_plan_create": (_int, [_u32, C.POINTER(_vp)]),
    "sb_analytic_plan_destroy": (_int, [_vp]),
    "sb_analytic_env_run": (_int, [_vp, _vp, _int, _vp, _int, _u32, _vp]),
    "sb_das_run_static": (_int, [C.POINTER(sb_geometry), _vp, _int, _vp, _int, _f64, _f64, _int, _f32, _int, _i32,
                                 _vp]),
    "sb_rawdelay_run": (_int, [_vp, _vp, _int, _vp, _int, _f64, _f64, _int, _f32, _vp]),
    "sb_hilbert_plan_create": (_int, [_u32, C.POINTER(_vp)]),
    "sb_hilbert_plan_destroy": (_int, [_vp]),
    "sb_hilbert_env_run": (_int, [_vp, _vp, _int, _vp, _int, _u32, _u32, _vp]),
    "sb_logcompress_run": (_int, [_vp, _int, _vp, _int, _sz, _f64, _f64, _f64, _vp]),
    "sb_iq_plan_create": (_int, [_f64, _f64, _u32, _u32, _u32, _vp, _vp, _vp, C.POINTER(_vp)]),
    "sb_iq_plan_destroy": (_int, [_vp]),
    "sb_iq_magnitude_run": (_int, [_vp, _vp, _int, _vp, _int, _u32, _u32, _u32, _vp]),
    "sb_iq_complex_run": (_int, [_vp, _int, _vp, _u32, _u32, _f64, _f64, _f64, _u32, _u32, _vp]),
    "sb_scan_plan_create": (_int, [_vp, _u32, _u32, _u32, _f64, _f64, C.POINTER(_vp)]),
    "sb_scan_plan_destroy": (_int, [_vp]),
    "sb_scan_image_size": (_int, [_vp, _vp]),
    "sb_scan_copy_tables": (_int, [_vp, _vp, _vp, _vp, _vp, _vp]),
    "sb_scan_tables_2d_host": (_int, [_vp, _u32, _u32, _f64, _f64, _vp, _vp, _vp, _vp, _vp]),
    "sb_scan_run": (_int, [_vp, _vp, _int, _vp, _int, _vp]),
    "sb_env_log_scan_run": (_int, [_vp, _vp, _vp, _vp, _int, _f64, _f64, _f64, _vp]),
    "sb_mv_run": (_int, [_vp, _int, _vp, _int, _u32, _u32, _u32, _u32, _u32, _f64, _int, _f32, _f32,
                         C.POINTER(sb_mv_stats), _vp]),
    "sb_mv_pcg_run": (_int, [_vp, _int, _vp, _int, _u32, _u32, _u32, _u32, _u32, _u32, _f64, _f64, _int, _f32, _vp]),
    "sb_batch_plan_create": (_int, [_vp, _u32, C.POINTER(sb_batch_params), C.POINTER(_vp)]),
    "sb_batch_plan_destroy": (_int, [_vp]),
    "sb_batch_run": (_int, [_vp, _int, _vp]),
    "sb_batch_set_rf_outputs": (_int, [_vp, _vp]),
    "sb_batch_autotune": (_int, [_vp, C.c_char_p, C.POINTER(_i32), C.POINTER(_i32), C.POINTER(_i32),
                                 C.POINTER(_i32), _vp]),
    "sb_check_device_errors": (_int, [_int]),
    "sb_hilbert_env_adjoint": (_int, [_vp, _vp, _vp, _vp, _u32, _u32, _vp]),
    "sb_das_forward_apod": (_int, [_vp, _vp, _vp, _vp, _u32, _f64, _f64, _int, _f32, _vp]),
    "sb_das_adjoint": (_int, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _u32, _f64, _f64, _int, _f32, _vp]),
    "sb_convert_run": (_int, [_vp, _int, _vp, _int, _sz, _vp]),
    "sb_node_create": (_int, [C.c_char_p, C.c_char_p, C.POINTER(_vp)]),
    "sb_node_destroy": (_int, [_vp]),
    "sb_node_set_param": (_int, [_vp, C.c_char_p, C.c_char_p]),
    "sb_node_get_param": (_int, [_vp, C.c_char_p, C.c_char_p, _sz]),
    "sb_node_param_count": (_int, [_vp]),
    "sb_node_param_info": (_int, [_vp, _int, C.c_char_p, C.c_char_p, C.c_char_p, C.c_char_p, _sz]),
    "sb_node_type_count": (_int, []),
    "sb_node_type_name": (_int, [_int, C.c_char_p, _sz]),
    "sb_node_process_raw": (_int, [_vp, C.POINTER(sb_geometry), _vp, _int, _int, _u32, _u32, _u32, _f64, _f64, _vp,
                                   C.POINTER(sb_record)]),
    "sb_node_process_last": (_int, [_vp, _vp, C.POINTER(sb_record)]),
    "sb_graph_process_next": (_int, [_vp, _f64, _vp, C.POINTER(_int), C.POINTER(sb_record)]),
    "sb_mock_meta_read": (_int, [C.c_char_p, C.POINTER(_vp)]),
    "sb_mock_meta_destroy": (_int, [_vp]),
    "sb_mock_meta_geometry": (_int, [_vp, C.POINTER(sb_geometry), C.POINTER(_f64), C.POINTER(_f64)]),
    "sb_mock_write_json": (_int, [C.c_char_p, C.POINTER(sb_geometry), _f64, _f64]),
    "sb_mock_reader_create": (_int, [_vp, C.c_char_p, _int, _int, C.POINTER(_vp)]),
    "sb_mock_reader_info": (_int, [_vp, C.POINTER(C.c_uint64), C.POINTER(_u32), C.POINTER(C.c_uint64)]),
    "sb_mock_reader_next": (_int, [_vp, _vp, _vp, C.POINTER(_int)]),
    "sb_mock_reader_destroy": (_int, [_vp]),
    "sb_node_process_image": (_int, [_vp, C.POINTER(sb_geometry), _vp, _int, _int, C.POINTER(_u32), _f64, _f64, _vp,
                                     C.POINTER(sb_record)]),
    "sb_graph_create_xml": (_int, [C.c_char_p, C.POINTER(_vp)]),
    "sb_graph_destroy": (_int, [_vp]),
    "sb_graph_chain": (_int, [_vp, C.c_char_p, _sz]),
    "sb_graph_node_get_param": (_int, [_vp, C.c_char_p, C.c_char_p, C.c_char_p, _sz]),
    "sb_graph_process_raw": (_int, [_vp, C.POINTER(sb_geometry), _vp, _int, _u32, _u32, _u32, _f64, _f64, _vp,
                                    C.POINTER(sb_record)]),
}

EXPORTED = tuple(_SIGNATURES)


class SupraError(RuntimeError):
    def __init__(self, fn: str, code: int, msg: str):
        super().__init__(f"{fn} failed with status {code}: {msg}")
        self.code = code


def load_library(path: Optional[str] = None) -> C.CDLL:
    """Load libsupra_b200.so and attach the ABI signatures. Raises OSError if it is missing."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise OSError(f"supra_b200 CUDA library not built: {p} (run __graft_entry__.build())")
    lib = C.CDLL(p)
    for name, (res, args) in _SIGNATURES.items():
        if not hasattr(lib, name):
            continue
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


def check(fn_name: str, status: int) -> None:
    if status != SB_OK:
        lib = load_library()
        msg = lib.sb_last_error()
        raise SupraError(fn_name, status, msg.decode() if msg else "")


def call(name: str, *args) -> int:
    lib = load_library()
    st = getattr(lib, name)(*args)
    check(name, st)
    return st
