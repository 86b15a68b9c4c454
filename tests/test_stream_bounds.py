"""CPU tests of the host arithmetic behind the streamed host execution
(hr_recon_execute_host streams the fan data in by ranges of views): the fan
views that the rebinning of a range of output views reads (hr_rebin_fan_views)
must contain every fan view its bilinear taps touch, so that a chunk is never
rebinned before its data have arrived, and must stay tight (a view or two of
slack), so that rebinning starts early. The taps are recomputed here by brute
force over every channel and view with the rebinning's own float arithmetic
(src/ParallelRebinningCBCurve.cpp:37-85 with T = float, the CPU clamp rule)."""
import ctypes

import numpy as np
import pytest

from analyticalreconbigpatient_b200 import _lib, geometry as G


def taps_range(a, i0, i1):
    f = np.float32
    j = np.arange(a["YL"], dtype=np.float32)
    t = (j - f(a["PLC"])) * f(a["DeltaT"])
    beta = np.arcsin((t / f(a["SO"])).astype(np.float64)).astype(np.float32)
    i = np.arange(i0, i1).astype(np.float32)
    fai_index = (i[:, None] * f(a["DeltaTheta"]) + beta[None, :]) / f(a["DeltaFai"])
    FI = np.ceil(fai_index).astype(np.int64)
    last = a["ViewN"] - 1
    XU = np.where(FI <= 0, 0, np.where(FI > last, last, FI))
    XB = np.where(FI <= 0, 0, np.where(FI > last, last, FI - 1))
    return int(XB.min()), int(XU.max())


def fan_views(a, i0, i1):
    f0, f1 = ctypes.c_int(), ctypes.c_int()
    _lib.check(_lib.load().hr_rebin_fan_views(a["YL"], a["ViewN"], a["YLC"], a["dYA"], a["DeltaTheta"], a["PLC"],
                                              a["DeltaT"], a["DeltaFai"], a["SO"], i0, i1, ctypes.byref(f0),
                                              ctypes.byref(f1)))
    return f0.value, f1.value


@pytest.mark.parametrize("scan", [G.Scan(ZL=64, pitch=0.984, rotations=20), G.Scan(ZL=16, pitch=0.9375, rotations=4),
                                  G.Scan(ZL=16, YL=200, det_pitch=1.0239 * 888 / 200, N_2pi=240, rotations=5)],
                         ids=["c2", "c1", "coarse"])
def test_rebin_fan_views_cover_every_tap_and_stay_tight(scan):
    a = scan.rebin_args()
    V = a["ViewN"]
    rng = np.random.default_rng(3)
    ranges = [(0, 1), (0, min(V, 1024)), (V - 1, V), (max(0, V - 700), V)]
    ranges += [(int(x), int(min(V, x + n))) for x, n in zip(rng.integers(0, V - 1, 12), rng.integers(1, 1500, 12))]
    for i0, i1 in ranges:
        lo, hi = taps_range(a, i0, i1)
        f0, f1 = fan_views(a, i0, i1)
        assert f0 <= lo and hi <= f1, (i0, i1, lo, hi, f0, f1)
        assert lo - f0 <= 3 and f1 - hi <= 3, (i0, i1, lo, hi, f0, f1)


def test_rebin_fan_views_rejects_bad_ranges():
    a = G.Scan(ZL=16, pitch=0.9375, rotations=2).rebin_args()
    f0, f1 = ctypes.c_int(), ctypes.c_int()
    lib = _lib.load()
    for i0, i1 in ((5, 5), (-1, 3), (0, a["ViewN"] + 1)):
        st = lib.hr_rebin_fan_views(a["YL"], a["ViewN"], a["YLC"], a["dYA"], a["DeltaTheta"], a["PLC"], a["DeltaT"],
                                    a["DeltaFai"], a["SO"], i0, i1, ctypes.byref(f0), ctypes.byref(f1))
        assert st == _lib.HR_ERR_INVALID_ARGUMENT
        assert b"hr_rebin_fan_views" in lib.hr_last_error()
