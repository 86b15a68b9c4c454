"""CPU tests of the host arithmetic behind the streamed host execution
(hr_recon_execute_host streams the fan data in by ranges of views): the fan
views that the rebinning of a range of output views reads (hr_rebin_fan_views)
must contain every fan view its bilinear taps touch, so that a chunk is never
rebinned before its data have arrived, and must stay tight (a view or two of
slack), so that rebinning starts early. The taps are recomputed here by brute
force over every channel and view with the rebinning's own float arithmetic
(src/ParallelRebinningCBCurve.cpp:37-85 with T = float, the CPU clamp rule)."""
import ctypes
import math

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


def block_windows(scan, nz):
    """Each z block's union of its slices' clamped [s1, s2] view windows (the
    backprojection's own central-view rule, ..._3DWeighting.cpp:61-70), or None."""
    g = scan.bp_geom()
    half = math.ceil(g["N_pi"] * g["HSCoef"])
    out = []
    for b in range((g["ZN"] + nz - 1) // nz):
        lo, hi = None, None
        for zi in range(b * nz, min(g["ZN"], (b + 1) * nz)):
            z = (zi - g["ZNC"]) * g["dz"]
            s0 = math.ceil((2.0 * 3.14159265358979 * z / g["h"] - g["BetaS"]) / g["DeltaFai"] - 0.5)
            s1, s2 = s0 - half, s0 + half
            if s1 < g["PN"] and s2 > 0:
                lo = max(0, s1) if lo is None else min(lo, max(0, s1))
                hi = min(g["PN"] - 1, s2) if hi is None else max(hi, min(g["PN"] - 1, s2))
        out.append(None if lo is None else (lo, hi))
    return out


def schedule(scan, nz, chunk):
    from analyticalreconbigpatient_b200.pipeline import recon_desc, view_weights

    w = view_weights(scan)
    d = recon_desc(scan, w, _lib.HR_FORM_FAST)
    lib = _lib.load()
    n = ctypes.c_int()
    _lib.check(lib.hr_recon_stream_schedule(ctypes.byref(d), nz, chunk, None, 0, ctypes.byref(n)))
    out = (ctypes.c_int * (3 * n.value))()
    _lib.check(lib.hr_recon_stream_schedule(ctypes.byref(d), nz, chunk, out, n.value, ctypes.byref(n)))
    return [tuple(out[3 * j: 3 * j + 3]) for j in range(n.value)]


@pytest.mark.parametrize("nz", [16, 8, 4])
@pytest.mark.parametrize("scan,chunk", [
    (G.Scan(ZL=64, pitch=0.984, rotations=6, XN=32, YN=32, ZN=1, dx=8.0, dy=8.0, dz=0.625), 1024),
    (G.Scan(ZL=64, pitch=0.984, rotations=6, XN=32, YN=32, ZN=1, dx=8.0, dy=8.0, dz=3.92), 700),
    (G.Scan(ZL=16, pitch=0.9375, rotations=8, XN=16, YN=16, ZN=1, dx=8.0, dy=8.0, dz=1.0), 256)],
    ids=["thin", "thick", "c1-like"])
def test_stream_schedule_launches_a_range_only_after_its_views_are_filtered(scan, chunk, nz):
    """The streamed host execution backprojects z-block ranges on one stream
    after waiting for the filtering of chunks 0..ready: every view of every
    block's window must lie in those chunks (a later one would be read before
    it is written: a race the device tests could miss). The ranges cover every
    z block once, in z order, starting with one block and ending with at most
    eight (one range when the scan has at most eight blocks)."""
    scan = G.Scan(**{**scan.__dict__, "ZN": scan.fully_sampled_slices() + 5})  # a few partial end slices
    ranges = schedule(scan, nz, chunk)
    wins = block_windows(scan, nz)
    PN = scan.PN
    assert ranges and ranges[0][0] == 0 and ranges[-1][1] == len(wins)
    if len(wins) > 8:
        assert ranges[0][1] == 1 and ranges[-1][1] - ranges[-1][0] <= 8
    else:
        assert len(ranges) == 1  # a scan of at most eight blocks is one range
    for (a0, a1, _), (b0, _, _) in zip(ranges, ranges[1:]):
        assert a1 == b0 and a0 < a1
    last_chunk = (PN - 1) // min(chunk, PN)
    for b0, b1, ready in ranges:
        assert 0 <= ready <= last_chunk
        for b in range(b0, b1):
            if wins[b] is not None:
                assert wins[b][1] // min(chunk, PN) <= ready, (b, wins[b], ready)
