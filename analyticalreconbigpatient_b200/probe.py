"""Device probe for the texture-sampling backprojection's roofline.

libhelixprobe.so (csrc/probe.cu) measures the rate at which the texture units
return bilinear samples of an FP16 layered texture -- the format the texture
backprojection variants sample -- with every lane active on a cache-resident
texture. It is a measurement tool beside the product library, not part of its
C ABI: the benchmark divides the texture backprojection's samples per second by
this rate.
"""
from __future__ import annotations

import ctypes
import os

_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libhelixprobe.so")
_lib = None


def _load() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(_PATH):
            raise ImportError(f"{_PATH} is not built; run `python -m analyticalreconbigpatient_b200.build`")
        lib = ctypes.CDLL(_PATH)
        lib.hr_texture_sample_rate.restype = ctypes.c_int
        lib.hr_texture_sample_rate.argtypes = [ctypes.POINTER(ctypes.c_double), ctypes.c_void_p]
        lib.hr_last_error.restype = ctypes.c_char_p
        _lib = lib
    return _lib


def texture_sample_rate(stream: int = 0) -> float:
    """Bilinear samples per second of the whole device (synchronises the stream)."""
    lib = _load()
    rate = ctypes.c_double(0.0)
    st = lib.hr_texture_sample_rate(ctypes.byref(rate), stream)
    if st != 0:
        raise RuntimeError(f"hr_texture_sample_rate failed ({st}): {lib.hr_last_error().decode()}")
    return rate.value
