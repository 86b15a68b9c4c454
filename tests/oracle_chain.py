"""Test helpers: the CPU reference chain (oracle) restricted to the views that
a set of z slices needs, so that full-size scans can be checked on a few
slices in seconds."""
from __future__ import annotations

import math

import numpy as np

import oracle

MARGIN = 80  # fan views beyond the rebinned window (half fan = 76 views at 984/rot)


def slice_windows(scan, zis):
    g = scan.bp_geom()
    half = math.ceil(g["N_pi"] * g["HSCoef"])
    lo, hi = g["PN"], -1
    for zi in zis:
        z = (zi - g["ZNC"]) * g["dz"]
        s0 = math.ceil((2.0 * 3.14159265358979 * z / g["h"] - g["BetaS"]) / g["DeltaFai"] - 0.5)
        lo = min(lo, max(0, s0 - half))
        hi = max(hi, min(g["PN"] - 1, s0 + half))
    return lo, hi


def reference_slices(scan, fan, zis, fp64_rebin=True, xy_step=1, rebinned=None):
    """FP64 oracle for whole slices ``zis``; ``fan`` is the host fan data
    [views][YL][ZL]. Each slice is computed from its own view window.

    The FP64 rebinning of a window equals that of the whole scan (the index
    arithmetic is shift-invariant in double). The reference's FP32 rebinning is
    not: it forms Theta = i*DeltaTheta in float, so its rounding depends on the
    absolute view index. For the reference CPU path pass ``rebinned``, the FP32
    rebinning of the whole scan ([views][YL][ZL]); ``fp64_rebin=False`` without
    it rebins the window in FP32 (an approximation of that path).
    Returns the values (slice by slice, every ``xy_step``-th column of [YN][XN])
    and their linear voxel indices."""
    w = oracle.weight_table(scan.N_2pi, scan.HSCoef, scan.delta)
    vals, voxs = [], []
    for zi in zis:
        lo, hi = slice_windows(scan, [zi])
        # parallel views lo..hi (backprojection numbering) are rebinned views
        # crop_front + lo ..; rebin a fan window around them (shift-invariant
        # because DeltaTheta == DeltaFai, which the driver's arguments guarantee)
        if rebinned is not None:
            reb, k0 = rebinned, scan.crop_front + lo
        else:
            a0 = max(0, scan.crop_front + lo - MARGIN)
            a1 = min(scan.views, scan.crop_front + hi + MARGIN + 1)
            sub = np.ascontiguousarray(fan[a0:a1])
            ra = dict(scan.rebin_args(), ViewN=a1 - a0)
            reb = oracle.rebin_f64(sub, **ra) if fp64_rebin else oracle.rebin_f32(sub, **ra)
            k0 = scan.crop_front + lo - a0
        rows = np.ascontiguousarray(reb[k0: k0 + hi - lo + 1].transpose(0, 2, 1), dtype=np.float64)
        filt = oracle.filter_f64(rows, **dict(scan.filter_args(), ViewN=hi - lo + 1))
        vox = np.array([(yi * scan.XN + xi) * scan.ZN + zi for yi in range(0, scan.YN, xy_step)
                        for xi in range(0, scan.XN, xy_step)], dtype=np.int64)
        vals.append(oracle.bp_f64(filt, w, scan.bp_geom(), fp_view0=lo, vox=vox))
        voxs.append(vox)
    return np.concatenate(vals), np.concatenate(voxs)


def hu_rmse(a, b, water_level):
    """RMSE in Hounsfield units, with the reconstructed water level as the
    calibration (HU = 1000 (mu - mu_w)/mu_w)."""
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    return float(1000.0 * np.sqrt(np.mean((a - b) ** 2)) / water_level)
