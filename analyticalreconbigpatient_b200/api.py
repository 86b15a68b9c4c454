"""Reference-facing functions with the names, argument meaning and array
layouts of the reference's three MEX functions (the calls its MATLAB driver
makes), running on the B200 through libhelixrecon.so. Arrays are numpy, C
order, i.e. the MATLAB dimensions reversed.

* ParallelRebinningCBCurve   src/ParallelRebinningCBCurve.cpp:101-129
* reWeigAdFiltr_GPU          src/reWeigAdFiltr_GPU.cpp:36-63
* Parallel_FDK_Helical_3DWeighting  src/Parallel_FDK_Helical_3DWeighting.cpp:204-269

Errors raise (TypeError/ValueError for bad arguments, HelixError for a failed
library call) where the reference exits the process or prints and continues.
``useGPU`` is accepted for signature compatibility; every path runs on the GPU
(useGPU == 0 selects the FP64 data path for the backprojection, matching the
reference's double-precision CPU branch).
"""
from __future__ import annotations

import numpy as np

from . import _lib


def _c(a: np.ndarray, dtype) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=dtype)


def weight_table(N_2pi: int, HSCoef: float = 0.68, delta: int = 60) -> np.ndarray:
    """View weight w[N_2pi] (src/Parallel_FDK_Helical_3DWeighting.cpp:156-170)."""
    w = np.zeros(int(N_2pi), dtype=np.float64)
    _lib.call("hr_view_weights", w.ctypes.data, int(N_2pi), float(HSCoef), int(delta))
    return w


def ParallelRebinningCBCurve(Proj, YL, ZL, ViewN, YLC, dYA, DeltaTheta, PLC, DeltaT, DeltaFai, SO, useGPU=1):
    """Fan -> parallel rebinning. ``Proj``: single [ViewN][YL][ZL] (MATLAB
    [ZL,YL,ViewN]); ``YLC``, ``PLC`` 1-based as the MEX receives them (it
    subtracts 1 in single precision, :122)."""
    YL, ZL, ViewN = int(YL), int(ZL), int(ViewN)
    Proj = _c(Proj, np.float32)
    if Proj.size != YL * ZL * ViewN:
        raise ValueError(f"Proj has {Proj.size} elements, expected YL*ZL*ViewN = {YL * ZL * ViewN}")
    f = np.float32
    out = np.empty((ViewN, YL, ZL), dtype=np.float32)
    _lib.call("hr_rebin_host", out.ctypes.data, Proj.ctypes.data, YL, ZL, ViewN, float(f(YLC) - f(1)), float(f(dYA)),
              float(f(DeltaTheta)), float(f(PLC) - f(1)), float(f(DeltaT)), float(f(DeltaFai)), float(f(SO)))
    return out


def reWeigAdFiltr_GPU(Proj, PLC, ZLC, dYL, dZL, SO):
    """Preweight + ramp filter. ``Proj``: single [ViewN][ZL][YL] (MATLAB
    [YL,ZL,ViewN]); sizes come from its shape as the MEX takes them from the
    dims (:48-51). ``PLC``, ``ZLC`` as passed by the driver (already minus 1)."""
    Proj = np.asarray(Proj)
    if Proj.ndim != 3:
        raise ValueError("reWeigAdFiltr_GPU: Proj must be 3-D [ViewN][ZL][YL]")
    ViewN, ZL, YL = Proj.shape
    Proj = _c(Proj, np.float32)
    out = np.empty_like(Proj)
    _lib.call("hr_filter_host", out.ctypes.data, Proj.ctypes.data, YL, ZL, ViewN, float(np.float32(PLC)),
              float(np.float32(ZLC)), float(np.float32(dYL)), float(np.float32(dZL)), float(np.float32(SO)))
    return out


def Parallel_FDK_Helical_3DWeighting(ScanGeom: dict, fpwd, ctimage: np.ndarray, useGPU: int = 1) -> None:
    """3D-weighted helical backprojection into ``ctimage`` in place (the MEX
    writes into its third input, :253). ``ScanGeom`` has the driver's struct
    fields ScDet=[SO DO YL ZL DecWidth DecHeigh YLC ZLC h], Proj=[BetaS BetaE
    ViewN N_2pi], Obj=[ObjR XN YN ZN XC YC ZC], Rec=[delta HSCoef k1] with
    1-based centres; ``fpwd``: [PN][ZL][YL]; ``ctimage``: float64 C-contiguous
    with XN*YN*ZN elements, filled [YN][XN][ZN] (z fastest)."""
    if not isinstance(ctimage, np.ndarray) or ctimage.dtype != np.float64 or not ctimage.flags["C_CONTIGUOUS"]:
        raise TypeError("ctimage must be a C-contiguous float64 numpy array (written in place)")
    sc, pj, ob, rc = (np.asarray(ScanGeom[k], dtype=np.float64).ravel() for k in ("ScDet", "Proj", "Obj", "Rec"))
    SO, DO = sc[0], sc[1]
    YL, ZL = int(sc[2] + 0.5), int(sc[3] + 0.5)
    DecWidth, DecHeigh = sc[4], sc[5]
    YLC = (YL - 1) * 0.5  # the MEX ignores ScDet(7) (:229)
    ZLC = sc[7] - 1.0
    h = sc[8] * DecHeigh
    BetaS, PN, N_2pi = pj[0], int(pj[2]), int(pj[3])
    ObjR = ob[0]
    XN, YN, ZN = int(ob[1] + 0.5), int(ob[2] + 0.5), int(ob[3] + 0.5)
    XNC, YNC, ZNC = ob[4] - 1.0, ob[5] - 1.0, ob[6] - 1.0
    delta, HSCoef, k1 = int(rc[0] + 0.5), rc[1], rc[2] * sc[8]
    fp = _c(fpwd, np.float64)
    if fp.size != YL * ZL * PN:
        raise ValueError(f"fpwd has {fp.size} elements, expected YL*ZL*PN = {YL * ZL * PN}")
    if ctimage.size != XN * YN * ZN:
        raise ValueError(f"ctimage has {ctimage.size} elements, expected XN*YN*ZN = {XN * YN * ZN}")
    _lib.call("hr_bp_host_reference", ctimage.ctypes.data, fp.ctypes.data, SO, DO, YL, ZL, DecWidth, DecHeigh, YLC,
              ZLC, h, BetaS, PN, N_2pi, ObjR, XN, YN, ZN, XNC, YNC, ZNC, delta, HSCoef, k1, int(useGPU))


def ParallekFDKHelical3DWeighting_GPU_float(fp, w, g: dict) -> np.ndarray:
    """Lower-level FP32 entry with explicit (possibly anisotropic) dx, dy, dz.
    ``g`` holds the float arguments of ParallelFDKHelical3DWeightingGPU.h:16-24."""
    fp = _c(fp, np.float32)
    w = _c(w, np.float32)
    out = np.empty((g["YN"], g["XN"], g["ZN"]), dtype=np.float32)
    i = lambda k: int(g[k])
    f = lambda k: float(np.float32(g[k]))
    _lib.call("hr_bp_host_float", out.ctypes.data, fp.ctypes.data, w.ctypes.data, i("N_2pi"), i("XN"), i("YN"),
              i("ZN"), f("XNC"), f("YNC"), f("ZNC"), f("dx"), f("dy"), f("dz"), i("YL"), i("ZL"), i("PN"), f("YLC"),
              f("ZLC"), f("dYL"), f("dZL"), f("h"), f("BetaS"), f("DeltaFai"), f("N_pi"), f("HSCoef"), f("SO"),
              f("SD"), f("k1"))
    return out


def ParallekFDKHelical3DWeighting_GPU_double(fp, w, g: dict) -> np.ndarray:
    """Lower-level FP64 entry (ParallelFDKHelical3DWeightingGPU.h:4-13)."""
    fp = _c(fp, np.float64)
    w = _c(w, np.float64)
    out = np.empty((g["YN"], g["XN"], g["ZN"]), dtype=np.float64)
    i = lambda k: int(g[k])
    d = lambda k: float(g[k])
    _lib.call("hr_bp_host_double", out.ctypes.data, fp.ctypes.data, w.ctypes.data, i("N_2pi"), i("XN"), i("YN"),
              i("ZN"), d("XNC"), d("YNC"), d("ZNC"), d("dx"), d("dy"), d("dz"), i("YL"), i("ZL"), i("PN"), d("YLC"),
              d("ZLC"), d("dYL"), d("dZL"), d("h"), d("BetaS"), d("DeltaFai"), d("N_pi"), d("HSCoef"), d("SO"),
              d("SD"), d("k1"))
    return out
