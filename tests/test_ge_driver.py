"""The GE reader and segment driver (hr_ge_*): header field map, segment
arithmetic and raw reads on the CPU against restatements of the MATLAB files;
on the GPU, the summed segment reconstruction against the oracle run segment
by segment on the same arguments."""
import math
import os

import numpy as np
import pytest

from analyticalreconbigpatient_b200 import _lib, api, ge, geometry as G


def tiny_scan(views_per_rot=120, rotations=3):
    # 96 channels spanning the full detector's fan, 8 rows, helix centred on z = 0
    return G.tiny(YL=96, ZL=8, N_2pi=views_per_rot, rotations=rotations, iso_channel=48.75)


def header_floats(sc):
    raw = np.zeros(18, dtype=np.float32)
    raw[2], raw[3], raw[4] = sc.SD, sc.SO, sc.det_pitch
    raw[5] = (math.pi - sc.BetaS) * 180 / math.pi
    raw[8], raw[9], raw[10], raw[11], raw[12] = sc.N_2pi, sc.views, sc.YL, sc.YL - sc.YLC1, sc.ZL
    raw[13] = sc.row_height * sc.SO / sc.SD
    raw[14] = sc.pitch * sc.ZL
    return raw


def test_header_field_map(tmp_path):
    raw = np.arange(18, dtype=np.float32) * 1.5 + 3.0
    raw[2], raw[3], raw[4] = 949.0, 541.0, 1.0239
    raw[8], raw[9], raw[10], raw[12] = 984, 19680, 888, 64
    p = str(tmp_path / "head.dat")
    raw.tofile(p)
    h = ge.read_header(p)
    for i, name in ge.FIELDS.items():
        assert getattr(h, name) == pytest.approx(float(raw[i]), rel=1e-7), name
    assert list(h.raw) == pytest.approx(list(raw))
    bad = raw.copy()
    bad[3] = 2000.0  # source-iso beyond source-detector
    bad.tofile(p)
    with pytest.raises(_lib.HelixError, match="implausible"):
        ge.read_header(p)


@pytest.mark.parametrize("total,seg", [(19680, 4000), (19680, 19680), (3000, 1000), (360, 150)])
def test_segment_arithmetic(total, seg):
    sc = tiny_scan() if total == 360 else G.Scan(ZL=64, pitch=0.984, rotations=total / 984)
    raw = header_floats(sc)
    raw[9] = total
    h = _lib.GeHeader()
    _lib.check(_lib.load().hr_ge_parse_header(raw.ctypes.data, h))
    ov, num = ge.segments(h, seg)
    # analyticalRecon.m:15-17
    so = math.atan(h.DetCellPitch / h.Source2DetDis / 2) * h.NumberOfDetChannelPerRow
    exp_ov = math.ceil(so * h.NumberOfViewPerRotation / (2 * math.pi)) + 1
    assert ov == exp_ov == sc.seg_overlap
    assert num == max(1, math.ceil((total - seg) / (seg - 2 * ov)) + 1)
    covered = 0
    for s in range(1, num + 1):
        first, dl = ctypes_views(h, seg, s)
        assert first == (seg - 2 * ov) * (s - 1)
        assert dl == (seg if s < num else total - first)
        covered = first + dl
    assert covered == total


def ctypes_views(h, seg, s):
    import ctypes

    f, d = ctypes.c_int(), ctypes.c_int()
    _lib.check(_lib.load().hr_ge_segment_views(ctypes.byref(h), seg, s, ctypes.byref(f), ctypes.byref(d)))
    return f.value, d.value


def test_read_segment_flips_channels_and_transposes(tmp_path):
    sc = tiny_scan()
    rng = np.random.default_rng(0)
    fan = rng.random((sc.views, sc.YL, sc.ZL), dtype=np.float32)
    pp, hp = str(tmp_path / "proj.dat"), str(tmp_path / "head.dat")
    ge.write_scan(pp, hp, fan, sc)
    # the file is [view][row][channel] in scanner channel order
    raw = np.fromfile(pp, dtype=np.float32).reshape(sc.views, sc.ZL, sc.YL)
    assert np.array_equal(raw[5, 3, ::-1], fan[5, :, 3])
    h = ge.read_header(hp)
    ov, num = ge.segments(h, 150)
    for s in range(1, num + 1):
        first, dl = ctypes_views(h, 150, s)
        got = ge.read_segment(pp, h, 150, s)
        assert got.shape == (dl, sc.YL, sc.ZL)
        assert np.array_equal(got, fan[first:first + dl])


def expected_desc(h, seg_length, s, objR, XN, YN, ZN, k1=5.0, delta=60, HSCoef=0.68):
    """analyticalReconBigPatient.m:30-146 and the MEX field mapping, restated."""
    ov, num = ge.segments(h, seg_length)
    first, DLength = ctypes_views(h, seg_length, s)
    f = np.float32
    SO = h.Source2IsoDis
    DO = h.Source2DetDis - h.Source2IsoDis
    YL, ZL = h.NumberOfDetChannelPerRow, h.NumberOfDetectorRow
    YLC = YL - h.IsoChannelLocation
    ZLC = (1 + ZL) * 0.5
    DetHei = h.SliceHeigh * (DO + SO) / SO
    DecAngle = math.atan(h.DetCellPitch / (SO + DO) / 2) * YL * 2
    DecHeigh = DetHei * ZL
    N_2pi = h.NumberOfViewPerRotation
    hn = h.HelicalPitch / ZL * SO / (DO + SO)
    ViewN = DLength
    BetaS = math.pi - h.BeginViewAngle * math.pi / 180 + (s - 1) * (seg_length - 2 * ov) * 2 * math.pi / N_2pi
    BetaE = BetaS + ViewN * 2 * math.pi / N_2pi
    e = dict(YL=YL, ZL=ZL, ViewN=ViewN, YLC=float(f(YLC) - f(1)), dYA=float(f(DecAngle / YL)),
             DeltaFai=float(f((BetaE - BetaS) / (ViewN - 1))), DeltaT=float(f(math.tan(DecAngle * 0.5) * SO * 3 / YL)),
             PLC=float(f((1 + YL) * 0.5) - f(1)), SO=float(f(SO)))
    e["DeltaTheta"] = e["DeltaFai"]
    dv = 2 * math.pi / N_2pi
    if s == 1:
        view0, ViewN = 0, ViewN - ov
    elif s == num:
        view0, ViewN, BetaS = ov, ViewN - ov, BetaS + ov * dv
    else:
        view0, ViewN, BetaS = ov, ViewN - 2 * ov, BetaS + ov * dv
    DecWidth = math.tan(DecAngle * 0.5) * SO * 2 * 1.5
    e.update(view0=view0, fPLC=float(f((1 + YL) * 0.5 - 1)), fZLC=float(f(ZLC - 1)), fdYL=float(f(DecWidth / YL)),
             fdZL=float(f(DecHeigh / ZL)), fSO=float(f(SO)))
    bp = dict(N_2pi=N_2pi, XN=XN, YN=YN, ZN=ZN, YL=YL, ZL=ZL, PN=ViewN, XNC=(XN + 1) / 2 - 1, YNC=(YN + 1) / 2 - 1,
              ZNC=9.0, dx=2 * objR / XN, dy=2 * objR / YN, dz=2 * objR / ZN, YLC=(YL - 1) / 2, ZLC=ZLC - 1,
              dYL=DecWidth / YL, dZL=DecHeigh / ZL, h=hn * DecHeigh, BetaS=BetaS, DeltaFai=2 * math.pi / N_2pi,
              N_pi=N_2pi / 2, HSCoef=HSCoef, SO=SO, SD=SO + DO, k1=k1 * hn)
    return e, bp


@pytest.mark.parametrize("seg_length", [150, 360])
def test_segment_descriptions_follow_the_matlab_driver(seg_length):
    sc = tiny_scan()
    raw = header_floats(sc)
    h = _lib.GeHeader()
    _lib.check(_lib.load().hr_ge_parse_header(raw.ctypes.data, h))
    _, num = ge.segments(h, seg_length)
    for s in range(1, num + 1):
        d, w = ge.segment_desc(h, seg_length, s, 6.0, 16, 16, 18)
        e, bp = expected_desc(h, seg_length, s, 6.0, 16, 16, 18)
        for k, v in e.items():
            assert getattr(d, k) == pytest.approx(v, rel=1e-12, abs=0), (s, k)
        for k, v in bp.items():
            assert getattr(d.bp, k) == pytest.approx(v, rel=1e-12, abs=1e-12), (s, k)
        np.testing.assert_array_equal(w, api.weight_table(h.NumberOfViewPerRotation, 0.68, 60))


@pytest.mark.gpu
def test_segment_driver_matches_the_oracle_segment_by_segment(cuda, tmp_path):
    import oracle
    from conftest import rel_l2

    sc = tiny_scan()
    fan = np.random.default_rng(3).random((sc.views, sc.YL, sc.ZL), dtype=np.float32)
    pp, hp = str(tmp_path / "proj.dat"), str(tmp_path / "head.dat")
    ge.write_scan(pp, hp, fan, sc)
    h = ge.read_header(hp)
    seg, objR, XN, YN, ZN = 150, 6.0, 16, 16, 18
    got = ge.reconstruct(pp, hp, seg, objR, XN, YN, ZN)
    _, num = ge.segments(h, seg)
    assert num == 3
    ref = np.zeros(XN * YN * ZN)
    for s in range(1, num + 1):
        d, w = ge.segment_desc(h, seg, s, objR, XN, YN, ZN)
        p = ge.read_segment(pp, h, seg, s)
        r = oracle.rebin_f32(p, d.YL, d.ZL, d.ViewN, d.YLC, d.dYA, d.DeltaTheta, d.PLC, d.DeltaT, d.DeltaFai, d.SO)
        r = r[d.view0:d.view0 + d.bp.PN].transpose(0, 2, 1)  # [PN][ZL][YL]
        f = oracle.filter_f64(r, d.YL, d.ZL, d.bp.PN, d.fPLC, d.fZLC, d.fdYL, d.fdZL, d.fSO)
        g = {k: getattr(d.bp, k) for k in oracle.BP_KEYS}
        ref += oracle.bp_f64(f, w, g)
    assert np.count_nonzero(ref) > ref.size // 2
    assert rel_l2(got.ravel(), ref) < 1e-5
