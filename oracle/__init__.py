"""CPU oracle for the helical cone-beam FBP chain -- TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__.smoke()`` and the CPU-baseline legs of
``bench.py`` may import this package, and only as the checker. The product
library never routes through it.

Two layers:

* ``libhelix_oracle.so`` (helix_oracle.c): a project-written CPU restatement of
  the reference's rebinning (src/ParallelRebinningCBCurve.cpp:22-97),
  preweight + ramp filter (src/analyticalReconBigPatient.m:107-134 with
  src/filtering.cu:15-25,187-207), view-weight table
  (src/Parallel_FDK_Helical_3DWeighting.cpp:156-170) and 3D-weighted helical
  backprojection (src/Parallel_FDK_Helical_3DWeighting.cpp:42-113), plus an
  analytic FP64 ellipsoid projector as the data source.
* ``_ref/libref_cpu.so``: the reference's own CPU functions compiled from its
  sources by oracle/Makefile (the parity pin for the restatement), and
  ``_ref/libref_gpu.so``: the reference's own .cu files (cuFFT filter) used on a
  GPU host to make the filter's golden vectors.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "libhelix_oracle.so")
REF_CPU_SO = os.path.join(HERE, "_ref", "libref_cpu.so")
REF_GPU_SO = os.path.join(HERE, "_ref", "libref_gpu.so")

_c_int = ctypes.c_int
_c_f = ctypes.c_float
_c_d = ctypes.c_double
_vp = ctypes.c_void_p

_lib = None
_ref = None
_ref_gpu = None


def build() -> None:
    """Compile the oracle (and, where the reference sources exist, _ref/)."""
    subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)


def _ptr(a: np.ndarray) -> int:
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            build()
        L = ctypes.CDLL(ORACLE_SO)
        L.hxo_rebin_f32.argtypes = [_vp, _vp, _c_int, _c_int, _c_int] + [_c_f] * 7
        L.hxo_rebin_f32.restype = None
        L.hxo_rebin_f64.argtypes = [_vp, _vp, _c_int, _c_int, _c_int] + [_c_d] * 7 + [_c_int]
        L.hxo_rebin_f64.restype = None
        L.hxo_weight_table.argtypes = [_vp, _c_int, _c_d, _c_int]
        L.hxo_weight_table.restype = None
        L.hxo_filter_f64.argtypes = [_vp, _vp, _c_int, _c_int, _c_int] + [_c_d] * 5 + [_c_int]
        L.hxo_filter_f64.restype = None
        L.hxo_bp_f64.argtypes = ([_vp, _vp, _c_int, _c_int, _vp, _c_int, _c_int, _c_int, _c_int]
                                 + [_c_d] * 6 + [_c_int, _c_int, _c_int] + [_c_d] * 12
                                 + [_vp, ctypes.c_int64, _c_int])
        L.hxo_bp_f64.restype = _c_int
        L.hxo_project_ellipsoids.argtypes = ([_vp, _c_int, _c_int, _c_int] + [_c_d] * 9 + [_vp, _c_int, _c_int])
        L.hxo_project_ellipsoids.restype = None
        _lib = L
    return _lib


def ref_available() -> bool:
    return os.path.exists(REF_CPU_SO)


def ref() -> ctypes.CDLL:
    """The reference's own CPU functions (compiled from its sources)."""
    global _ref
    if _ref is None:
        if not os.path.exists(REF_CPU_SO):
            raise FileNotFoundError(f"{REF_CPU_SO} missing: run `make -C oracle ref` where the reference sources exist")
        L = ctypes.CDLL(REF_CPU_SO)
        L.ref_rebin_cpu_f32.argtypes = [_vp, _vp, _c_int, _c_int, _c_int] + [_c_f] * 7
        L.ref_rebin_cpu_f32.restype = None
        L.ref_rebin_cpu_f64.argtypes = [_vp, _vp, _c_int, _c_int, _c_int] + [_c_d] * 7
        L.ref_rebin_cpu_f64.restype = None
        L.ref_bp_cpu_f64.argtypes = ([_vp, _vp, _vp, _c_int, _c_int, _c_int, _c_int] + [_c_d] * 6
                                     + [_c_int, _c_int, _c_int] + [_c_d] * 12)
        L.ref_bp_cpu_f64.restype = None
        L.ref_ParallelFDKHelical3DWeighting.argtypes = (
            [_vp, _vp, _c_d, _c_d, _c_int, _c_int] + [_c_d] * 6 + [_c_int, _c_int, _c_d, _c_int, _c_int, _c_int]
            + [_c_d] * 3 + [_c_int, _c_d, _c_d, _c_int])
        L.ref_ParallelFDKHelical3DWeighting.restype = None
        _ref = L
    return _ref


def ref_gpu() -> ctypes.CDLL:
    """The reference's own GPU entry points (needs a CUDA device)."""
    global _ref_gpu
    if _ref_gpu is None:
        L = ctypes.CDLL(REF_GPU_SO)
        L.ref_gpu_filtering.argtypes = [_vp, _vp, _c_int, _c_int, _c_int] + [_c_f] * 5
        L.ref_gpu_filtering.restype = None
        L.ref_gpu_ParallelRebinningCBCurve_GPU.argtypes = [_vp, _vp, _c_int, _c_int, _c_int] + [_c_f] * 7
        L.ref_gpu_ParallelRebinningCBCurve_GPU.restype = None
        _ref_gpu = L
    return _ref_gpu


# --------------------------------------------------------------------------
# Rebinning. Layout [ViewN][YL][ZL] (ZL fastest) in and out.
# --------------------------------------------------------------------------
def rebin_f32(proj, YL, ZL, ViewN, YLC, dYA, DeltaTheta, PLC, DeltaT, DeltaFai, SO):
    proj = np.ascontiguousarray(proj, dtype=np.float32)
    out = np.empty_like(proj)
    lib().hxo_rebin_f32(_ptr(out), _ptr(proj), YL, ZL, ViewN, YLC, dYA, DeltaTheta, PLC, DeltaT, DeltaFai, SO)
    return out


def ref_rebin_f32(proj, YL, ZL, ViewN, YLC, dYA, DeltaTheta, PLC, DeltaT, DeltaFai, SO):
    proj = np.ascontiguousarray(proj, dtype=np.float32)
    out = np.empty_like(proj)
    ref().ref_rebin_cpu_f32(_ptr(out), _ptr(proj), YL, ZL, ViewN, YLC, dYA, DeltaTheta, PLC, DeltaT, DeltaFai, SO)
    return out


def rebin_f64(proj, YL, ZL, ViewN, YLC, dYA, DeltaTheta, PLC, DeltaT, DeltaFai, SO, nthreads=0):
    proj = np.ascontiguousarray(proj, dtype=np.float64)
    out = np.empty_like(proj)
    lib().hxo_rebin_f64(_ptr(out), _ptr(proj), YL, ZL, ViewN, YLC, dYA, DeltaTheta, PLC, DeltaT, DeltaFai, SO,
                        nthreads or os.cpu_count())
    return out


# --------------------------------------------------------------------------
# Filter. Layout [ViewN][ZL][YL] (YL fastest).
# --------------------------------------------------------------------------
def filter_f64(proj, YL, ZL, ViewN, PLC, ZLC, dYL, dZL, SO, nthreads=0):
    """Direct FP64 Toeplitz restatement (see helix_oracle.c)."""
    proj = np.ascontiguousarray(proj, dtype=np.float64)
    out = np.empty_like(proj)
    lib().hxo_filter_f64(_ptr(out), _ptr(proj), YL, ZL, ViewN, PLC, ZLC, dYL, dZL, SO, nthreads or os.cpu_count())
    return out


def filter_fft_f64(proj, YL, ZL, ViewN, PLC, ZLC, dYL, dZL, SO):
    """Second FP64 restatement, step for step the MATLAB CPU branch
    (src/analyticalReconBigPatient.m:107-134): preweight, NN = 2^ceil(log2(3 YL))
    wrapped kernel HS, ifft(fft(HS) .* fft(p, NN)), real part of the first YL."""
    p = np.asarray(proj, dtype=np.float64).reshape(ViewN, ZL, YL)
    j = np.arange(YL, dtype=np.float64)
    k = np.arange(ZL, dtype=np.float64)
    t = (j - PLC) * dYL
    b = (k - ZLC) * dZL
    wt = SO * SO / np.sqrt(SO ** 4 + (SO * b[:, None]) ** 2 - (b[:, None] * t[None, :]) ** 2)
    p = p * wt[None, :, :]
    n = np.arange(-YL, YL + 1, dtype=np.float64)
    hsl = -2.0 / ((np.pi ** 2) * (4 * n * n - 1)) / dYL
    NN = int(2 ** np.ceil(np.log(YL * 3) / np.log(2)))
    HS = np.zeros(NN)
    HS[: YL + 1] = hsl[YL: 2 * YL + 1]
    HS[NN - YL:] = hsl[:YL]
    FtS = np.fft.fft(HS)
    FtP = np.fft.fft(p, NN, axis=-1)
    return np.real(np.fft.ifft(FtS * FtP, axis=-1)[..., :YL])


# --------------------------------------------------------------------------
# Backprojection. fp layout [view][ZL][YL]; volume [YN][XN][ZN] (z fastest).
# --------------------------------------------------------------------------
def weight_table(N_2pi, HSCoef=0.68, delta=60):
    w = np.zeros(N_2pi, dtype=np.float64)
    lib().hxo_weight_table(_ptr(w), N_2pi, HSCoef, delta)
    return w


BP_KEYS = ("N_2pi", "XN", "YN", "ZN", "XNC", "YNC", "ZNC", "dx", "dy", "dz", "YL", "ZL", "PN", "YLC", "ZLC", "dYL",
           "dZL", "h", "BetaS", "DeltaFai", "N_pi", "HSCoef", "SO", "SD", "k1")


def bp_f64(fp, w, g, fp_view0=0, vox=None, nthreads=0):
    """FP64 backprojection restatement. ``g`` maps BP_KEYS to values. ``fp`` may
    hold only a window of views starting at ``fp_view0``. ``vox``: optional int64
    linear voxel indices ((yi*XN+xi)*ZN+zi); returns those voxels only."""
    fp = np.ascontiguousarray(fp, dtype=np.float64)
    w = np.ascontiguousarray(w, dtype=np.float64)
    nviews = fp.size // (g["ZL"] * g["YL"])
    if vox is None:
        out = np.zeros(g["XN"] * g["YN"] * g["ZN"], dtype=np.float64)
        vptr, nv = None, 0
    else:
        vox = np.ascontiguousarray(vox, dtype=np.int64)
        out = np.zeros(vox.size, dtype=np.float64)
        vptr, nv = _ptr(vox), vox.size
    rc = lib().hxo_bp_f64(_ptr(out), _ptr(fp), fp_view0, nviews, _ptr(w), g["N_2pi"], g["XN"], g["YN"], g["ZN"],
                          g["XNC"], g["YNC"], g["ZNC"], g["dx"], g["dy"], g["dz"], g["YL"], g["ZL"], g["PN"],
                          g["YLC"], g["ZLC"], g["dYL"], g["dZL"], g["h"], g["BetaS"], g["DeltaFai"], g["N_pi"],
                          g["HSCoef"], g["SO"], g["SD"], g["k1"], vptr, nv, nthreads or os.cpu_count())
    if rc != 0:
        raise ValueError("oracle backprojection needs views outside the supplied window")
    return out


def ref_bp_f64(fp, w, g):
    """The reference's own ParallelFDKHelical3DWeightingCPU (full volume)."""
    fp = np.ascontiguousarray(fp, dtype=np.float64)
    w = np.ascontiguousarray(w, dtype=np.float64)
    out = np.zeros(g["XN"] * g["YN"] * g["ZN"], dtype=np.float64)
    ref().ref_bp_cpu_f64(_ptr(out), _ptr(fp), _ptr(w), *[g[k] for k in BP_KEYS])
    return out


# --------------------------------------------------------------------------
# Analytic projector (data source).
# --------------------------------------------------------------------------
def project_ellipsoids(objects, YL, ZL, ViewN, SO, SD, dYA, YLC0, dZL, ZLC0, BetaS, dBeta, h, nthreads=0):
    """FP64 line integrals, output float32 [ViewN][YL][ZL]."""
    obj = np.ascontiguousarray(objects, dtype=np.float64).reshape(-1, 17)
    out = np.empty((ViewN, YL, ZL), dtype=np.float32)
    lib().hxo_project_ellipsoids(_ptr(out), YL, ZL, ViewN, SO, SD, dYA, YLC0, dZL, ZLC0, BetaS, dBeta, h, _ptr(obj),
                                 obj.shape[0], nthreads or os.cpu_count())
    return out
