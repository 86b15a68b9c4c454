"""GE raw scans: the 18-float header, segment reads and the segment-by-segment
reconstruction driver of the reference's MATLAB code (analyticalRecon.m,
readBigPatientData.m, GetHeadofGeDataSet.m, analyticalReconBigPatient.m),
implemented in libhelixrecon.so (hr_ge_*); plus a writer that stores a
synthetic fan scan in the same format."""
from __future__ import annotations

import ctypes
import math

import numpy as np

from . import _lib
from .geometry import Scan

FIELDS = {2: "Source2DetDis", 3: "Source2IsoDis", 4: "DetCellPitch", 5: "BeginViewAngle",
          8: "NumberOfViewPerRotation", 9: "TotalViewNumber", 10: "NumberOfDetChannelPerRow",
          11: "IsoChannelLocation", 12: "NumberOfDetectorRow", 13: "SliceHeigh", 14: "HelicalPitch"}


def read_header(path: str) -> _lib.GeHeader:
    h = _lib.GeHeader()
    _lib.check(_lib.load().hr_ge_read_header(path.encode(), ctypes.byref(h)))
    return h


def segments(h: _lib.GeHeader, seg_length: int) -> tuple[int, int]:
    """(overlap in views, number of segments)."""
    ov, num = ctypes.c_int(), ctypes.c_int()
    _lib.check(_lib.load().hr_ge_segments(ctypes.byref(h), seg_length, ctypes.byref(ov), ctypes.byref(num)))
    return ov.value, num.value


def read_segment(path: str, h: _lib.GeHeader, seg_length: int, seg_ind: int) -> np.ndarray:
    """Segment seg_ind (1-based) as fan data [views][YL][ZL], channels flipped."""
    out = np.empty((seg_length, h.NumberOfDetChannelPerRow, h.NumberOfDetectorRow), dtype=np.float32)
    dl = ctypes.c_int()
    _lib.check(_lib.load().hr_ge_read_segment(path.encode(), ctypes.byref(h), seg_length, seg_ind,
                                              out.ctypes.data, ctypes.byref(dl)))
    return out[:dl.value]


def segment_desc(h: _lib.GeHeader, seg_length: int, seg_ind: int, objR: float, XN: int, YN: int, ZN: int,
                 form: int = _lib.HR_FORM_PLAIN, k1: float = 5.0, delta: int = 60, HSCoef: float = 0.68):
    """(hr_recon_desc, weight table) of one segment."""
    d = _lib.ReconDesc()
    w = np.zeros(h.NumberOfViewPerRotation, dtype=np.float64)
    opt = _lib.GeOptions(k1=k1, delta=delta, HSCoef=HSCoef)
    _lib.check(_lib.load().hr_ge_segment_desc(ctypes.byref(h), seg_length, seg_ind, objR, XN, YN, ZN,
                                              ctypes.byref(opt), form, ctypes.byref(d), w.ctypes.data))
    return d, w


def reconstruct(proj_path: str, head_path: str, seg_length: int, objR: float, XN: int, YN: int, ZN: int,
                form: int = _lib.HR_FORM_PLAIN, k1: float = 5.0, delta: int = 60, HSCoef: float = 0.68) -> np.ndarray:
    """analyticalRecon: every segment reconstructed on the GPU and summed; [YN][XN][ZN] float32."""
    out = np.empty((YN, XN, ZN), dtype=np.float32)
    opt = _lib.GeOptions(k1=k1, delta=delta, HSCoef=HSCoef)
    _lib.check(_lib.load().hr_ge_reconstruct(proj_path.encode(), head_path.encode(), seg_length, objR, XN, YN, ZN,
                                             ctypes.byref(opt), form, out.ctypes.data))
    return out


def write_scan(proj_path: str, head_path: str, fan: np.ndarray, scan: Scan) -> np.ndarray:
    """Stores fan data [views][YL][ZL] of a synthetic scan (post-flip channels,
    the projector's convention) as a GE pair of files: the header (18 floats)
    and the raw projections [view][row][channel] with the channels in scanner
    order (flipped back). Returns the header floats."""
    raw = np.zeros(18, dtype=np.float32)
    raw[2], raw[3] = scan.SD, scan.SO
    raw[4] = scan.det_pitch
    raw[5] = (math.pi - scan.BetaS) * 180.0 / math.pi
    raw[8], raw[9] = scan.N_2pi, scan.views
    raw[10], raw[12] = scan.YL, scan.ZL
    raw[11] = scan.YL - scan.YLC1                          # the driver mirrors it back
    raw[13] = scan.row_height * scan.SO / scan.SD          # slice height at iso
    raw[14] = scan.pitch * scan.ZL                         # table feed / slice height
    raw.tofile(head_path)
    data = np.ascontiguousarray(np.asarray(fan, dtype=np.float32)[:, ::-1, :].transpose(0, 2, 1))
    data.tofile(proj_path)
    return raw
