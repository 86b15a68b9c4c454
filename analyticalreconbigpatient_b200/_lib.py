"""ctypes binding of libhelixrecon.so (the C ABI declared in include/helixrecon.h).

There is no fallback: if the library is missing or cannot be loaded, every
call raises. Device pointers are passed as integers (e.g. ``tensor.data_ptr()``).
"""
from __future__ import annotations

import ctypes
import os

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "libhelixrecon.so")

HR_OK = 0
HR_ERR_INVALID_ARGUMENT, HR_ERR_CUDA, HR_ERR_OUT_OF_MEMORY, HR_ERR_NO_DEVICE, HR_ERR_UNSUPPORTED = 1, 2, 3, 4, 5
HR_FORM_PLAIN, HR_FORM_FP64, HR_FORM_FAST = 0, 1, 2
HR_LAYOUT_ROWS, HR_LAYOUT_REBIN = 0, 1
HR_SLAB_BLOCKS, HR_SLAB_ROUND_ROBIN = 0, 1

_i = ctypes.c_int
_f = ctypes.c_float
_d = ctypes.c_double
_p = ctypes.c_void_p


class HelixError(RuntimeError):
    """A library call returned a non-zero hr_status."""

    def __init__(self, status: int, message: str):
        super().__init__(f"helixrecon status {status}: {message}")
        self.status = status


class BpGeom(ctypes.Structure):
    _fields_ = ([(n, _i) for n in ("N_2pi", "XN", "YN", "ZN", "YL", "ZL", "PN")]
                + [(n, _d) for n in ("XNC", "YNC", "ZNC", "dx", "dy", "dz", "YLC", "ZLC", "dYL", "dZL", "h", "BetaS",
                                     "DeltaFai", "N_pi", "HSCoef", "SO", "SD", "k1")])

    @classmethod
    def from_dict(cls, g: dict) -> "BpGeom":
        return cls(**{k: g[k] for k, _ in cls._fields_})


class ReconDesc(ctypes.Structure):
    _fields_ = ([("YL", _i), ("ZL", _i), ("ViewN", _i)]
                + [(n, _f) for n in ("YLC", "dYA", "DeltaTheta", "PLC", "DeltaT", "DeltaFai", "SO")]
                + [("view0", _i)] + [(n, _f) for n in ("fPLC", "fZLC", "fdYL", "fdZL", "fSO")]
                + [("bp", BpGeom), ("w", _p), ("form", _i)])


class SlabWindow(ctypes.Structure):
    _fields_ = [(n, _i) for n in ("slab", "first_slice", "n_slices", "bp_view0", "bp_views", "fan_view0", "fan_views",
                                  "shared_views")]


class GeHeader(ctypes.Structure):
    _fields_ = ([("raw", _f * 18)] + [(n, _d) for n in ("Source2DetDis", "Source2IsoDis", "DetCellPitch",
                                                         "BeginViewAngle")]
                + [(n, _i) for n in ("NumberOfViewPerRotation", "TotalViewNumber", "NumberOfDetChannelPerRow",
                                     "NumberOfDetectorRow")]
                + [(n, _d) for n in ("IsoChannelLocation", "SliceHeigh", "HelicalPitch")])


class GeOptions(ctypes.Structure):
    _fields_ = [("k1", _d), ("delta", _i), ("HSCoef", _d)]


# name -> (restype, argtypes)
_SIGS = {
    "hr_last_error": (ctypes.c_char_p, []),
    "hr_version": (_i, []),
    "hr_view_weights": (_i, [_p, _i, _d, _i]),
    "ParallelRebinningCBCurve_GPU": (None, [_p, _p, _i, _i, _i] + [_f] * 7),
    "filtering": (None, [_p, _p, _i, _i, _i] + [_f] * 5),
    "ParallekFDKHelical3DWeighting_GPU_float": (None, [_p, _p, _p, _i, _i, _i, _i] + [_f] * 6 + [_i] * 3 + [_f] * 12),
    "ParallekFDKHelical3DWeighting_GPU_double": (None, [_p, _p, _p, _i, _i, _i, _i] + [_d] * 6 + [_i] * 3 + [_d] * 12),
    "ParallelFDKHelical3DWeighting": (None, [_p, _p, _d, _d, _i, _i] + [_d] * 6 + [_i, _i, _d, _i, _i, _i] + [_d] * 3
                                      + [_i, _d, _d, _i]),
    "hr_rebin_host": (_i, [_p, _p, _i, _i, _i] + [_f] * 7),
    "hr_filter_host": (_i, [_p, _p, _i, _i, _i] + [_f] * 5),
    "hr_bp_host_float": (_i, [_p, _p, _p, _i, _i, _i, _i] + [_f] * 6 + [_i] * 3 + [_f] * 12),
    "hr_bp_host_double": (_i, [_p, _p, _p, _i, _i, _i, _i] + [_d] * 6 + [_i] * 3 + [_d] * 12),
    "hr_bp_host_reference": (_i, [_p, _p, _d, _d, _i, _i] + [_d] * 6 + [_i, _i, _d, _i, _i, _i] + [_d] * 3
                             + [_i, _d, _d, _i]),
    "hr_rebin_plan_create": (_i, [ctypes.POINTER(_p), _i, _i, _i] + [_f] * 7),
    "hr_rebin_execute": (_i, [_p, _p, _p, _p]),
    "hr_rebin_plan_destroy": (None, [_p]),
    "hr_filter_plan_create": (_i, [ctypes.POINTER(_p), _i, _i, _i] + [_f] * 5),
    "hr_filter_execute": (_i, [_p, _p, _p, _i, _i, _p]),
    "hr_filter_plan_destroy": (None, [_p]),
    "hr_bp_plan_create": (_i, [ctypes.POINTER(_p), ctypes.POINTER(BpGeom), _p, _i]),
    "hr_bp_execute": (_i, [_p, _p, _p, _p]),
    "hr_bp_plan_destroy": (None, [_p]),
    "hr_project_ellipsoids": (_i, [_p, _i, _i, _i] + [_d] * 9 + [_p, _i, _p]),
    "hr_pack_bf16_pairs": (_i, [_p, _p, ctypes.c_longlong, _i, _p]),
    "hr_filter_tc_plan_create": (_i, [ctypes.POINTER(_p), _i, _i, _i] + [_f] * 5),
    "hr_filter_tc_execute": (_i, [_p, _p, _p, _i, _i, _p]),
    "hr_filter_tc_check": (_i, [_p]),
    "hr_filter_tc_test_stall": (_i, [_p, _i, ctypes.c_uint]),
    "hr_filter_tc_device_bytes": (ctypes.c_size_t, [_p]),
    "hr_filter_tc_plan_destroy": (None, [_p]),
    "hr_recon_check": (_i, [_p]),
    "hr_slab_plan_create": (_i, [ctypes.POINTER(_p), ctypes.POINTER(ReconDesc), _i]),
    "hr_slab_execute": (_i, [_p, _p, _p, _i, _i]),
    "hr_slab_describe": (_i, [_p, ctypes.c_char_p, _i]),
    "hr_slab_device_bytes": (ctypes.c_size_t, [_p]),
    "hr_slab_plan_destroy": (None, [_p]),
    "hr_slab_windows": (_i, [ctypes.POINTER(ReconDesc), _i, _i, _i, _i, _p, _i, ctypes.POINTER(_i)]),
    "hr_rebin_fan_views": (_i, [_i, _i] + [_f] * 7 + [_i, _i, ctypes.POINTER(_i), ctypes.POINTER(_i)]),
    "hr_recon_stream_schedule": (_i, [ctypes.POINTER(ReconDesc), _i, _i, _p, _i, ctypes.POINTER(_i)]),
    "hr_slab_plan_create_part": (_i, [ctypes.POINTER(_p), ctypes.POINTER(ReconDesc), _i, _i, _i, _i]),
    "hr_slab_execute_range": (_i, [_p, _p, _p, _i, _i, _i]),
    "hr_slab_fan_range": (_i, [_p, ctypes.POINTER(_i), ctypes.POINTER(_i), ctypes.POINTER(ctypes.c_size_t)]),
    "hr_recon_describe": (_i, [_p, ctypes.c_char_p, _i]),
    "hr_bp_autotune": (_i, [_p, _p, _p, _p]),
    "hr_bp_describe": (_i, [_p, ctypes.c_char_p, _i]),
    "hr_bp_select": (_i, [_p, _i]),
    "hr_bp_plain_noalloc": (_i, [_p, _p, _p, ctypes.POINTER(BpGeom), _p]),
    "hr_batch_plan_create": (_i, [ctypes.POINTER(_p), ctypes.POINTER(ReconDesc), _i]),
    "hr_batch_execute": (_i, [_p, _p, _p, _p]),
    "hr_batch_execute_host": (_i, [_p, _p, _p]),
    "hr_batch_select": (_i, [_p, _i]),
    "hr_batch_backproject": (_i, [_p, _p, _p]),
    "hr_batch_describe": (_i, [_p, ctypes.c_char_p, _i]),
    "hr_batch_check": (_i, [_p]),
    "hr_batch_device_bytes": (ctypes.c_size_t, [_p]),
    "hr_batch_plan_destroy": (None, [_p]),
    "hr_add_poisson_noise": (_i, [_p, ctypes.c_longlong, _d, ctypes.c_ulonglong, _p]),
    "hr_cnn_param_count": (ctypes.c_size_t, []),
    "hr_cnn_create": (_i, [ctypes.POINTER(_p), _p]),
    "hr_cnn_get_params": (_i, [_p, _p]),
    "hr_cnn_get_grads": (_i, [_p, _p]),
    "hr_cnn_train_step": (_i, [_p, _p, _p, _p, _i, _i, _i, _f, _f, _p, _p]),
    "hr_cnn_forward": (_i, [_p, _p, _p, _p, ctypes.c_longlong, ctypes.c_longlong, _i, _i, _i, _f, _p]),
    "hr_cnn_apply_volume": (_i, [_p, _p, _p, _i, _i, _i, _f, _i, _p]),
    "hr_cnn_pack_input": (_i, [_p, _p, _i, _i, _i, _i, _i, _f, _p]),
    "hr_cnn_check": (_i, [_p]),
    "hr_cnn_test_stall": (_i, [_p, _i, ctypes.c_uint]),
    "hr_cnn_destroy": (None, [_p]),
    "hr_ge_parse_header": (_i, [_p, ctypes.POINTER(GeHeader)]),
    "hr_ge_read_header": (_i, [ctypes.c_char_p, ctypes.POINTER(GeHeader)]),
    "hr_ge_segments": (_i, [ctypes.POINTER(GeHeader), _i, ctypes.POINTER(_i), ctypes.POINTER(_i)]),
    "hr_ge_segment_views": (_i, [ctypes.POINTER(GeHeader), _i, _i, ctypes.POINTER(_i), ctypes.POINTER(_i)]),
    "hr_ge_read_segment": (_i, [ctypes.c_char_p, ctypes.POINTER(GeHeader), _i, _i, _p, ctypes.POINTER(_i)]),
    "hr_ge_segment_desc": (_i, [ctypes.POINTER(GeHeader), _i, _i, _d, _i, _i, _i, ctypes.POINTER(GeOptions), _i,
                                ctypes.POINTER(ReconDesc), _p]),
    "hr_ge_reconstruct": (_i, [ctypes.c_char_p, ctypes.c_char_p, _i, _d, _i, _i, _i, ctypes.POINTER(GeOptions), _i,
                               _p]),
    "hr_accumulate": (_i, [_p, _p, ctypes.c_longlong, _p]),
    "hr_recon_plan_create": (_i, [ctypes.POINTER(_p), ctypes.POINTER(ReconDesc)]),
    "hr_recon_execute": (_i, [_p, _p, _p, _p]),
    "hr_recon_execute_host": (_i, [_p, _p, _p]),
    "hr_recon_device_bytes": (ctypes.c_size_t, [_p]),
    "hr_recon_plan_destroy": (None, [_p]),
}

_lib = None


def load() -> ctypes.CDLL:
    """Load the library (once). Raises if it is missing: there is no CPU path."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is not built; run `python -m analyticalreconbigpatient_b200.build`")
        lib = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


def exported_symbols() -> list[str]:
    return list(_SIGS)


def check(status: int) -> None:
    if status != HR_OK:
        msg = load().hr_last_error()
        raise HelixError(status, msg.decode() if msg else "")


def call(name: str, *args):
    """Call a status-returning entry and raise HelixError on failure."""
    check(getattr(load(), name)(*args))
