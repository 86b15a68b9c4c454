"""CPU tests: the oracle restatement pinned to the reference's own outputs.

The reference has no tests or fixtures of its own, so the pins are (a) golden
vectors produced by the reference's compiled CPU functions and its cuFFT
filter (tests/golden/make_golden.py) and (b) the compiled reference called
live where oracle/_ref/ exists.
"""
import glob
import os

import numpy as np
import pytest

import oracle
from analyticalreconbigpatient_b200 import geometry as G, phantom as P
from conftest import rel_l2

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _rebin_cases():
    return sorted(glob.glob(os.path.join(GOLDEN, "rebin_*.npz")))


def _bp_cases():
    return sorted(glob.glob(os.path.join(GOLDEN, "bp_*.npz")))


def load_rebin(path):
    d = np.load(path)
    YL, ZL, ViewN = (int(v) for v in d["sizes"])
    a = [float(v) for v in d["args"]]
    args = dict(YL=YL, ZL=ZL, ViewN=ViewN, YLC=a[0], dYA=a[1], DeltaTheta=a[2], PLC=a[3], DeltaT=a[4],
                DeltaFai=a[5], SO=a[6])
    return d["proj"], d["out"], args


def load_bp(path):
    d = np.load(path)
    g = {}
    for k, v in zip(d["geom_keys"], d["geom"]):
        k = str(k)
        g[k] = int(v) if k in ("N_2pi", "XN", "YN", "ZN", "YL", "ZL", "PN") else float(v)
    return d["fp"], d["w"], g, d["vol"]


def test_golden_present():
    assert len(_rebin_cases()) >= 3 and len(_bp_cases()) >= 3


@pytest.mark.parametrize("path", _rebin_cases(), ids=os.path.basename)
def test_rebin_f32_restatement_bit_exact_to_reference_golden(path):
    proj, out, args = load_rebin(path)
    mine = oracle.rebin_f32(proj, **args)
    np.testing.assert_array_equal(mine.view(np.uint32), out.view(np.uint32))


@pytest.mark.parametrize("path", _rebin_cases(), ids=os.path.basename)
def test_rebin_f64_close_to_reference_f32(path):
    proj, out, args = load_rebin(path)
    mine = oracle.rebin_f64(proj, **args)
    assert rel_l2(mine, out) < 1e-5


@pytest.mark.parametrize("path", _bp_cases(), ids=os.path.basename)
def test_bp_restatement_matches_reference_golden(path):
    fp, w, g, vol = load_bp(path)
    mine = oracle.bp_f64(fp.astype(np.float64), w, g)
    np.testing.assert_allclose(mine, vol, rtol=1e-12, atol=1e-12 * np.abs(vol).max())


@pytest.mark.parametrize("path", _bp_cases()[:1], ids=os.path.basename)
def test_bp_voxel_subset_and_view_window(path):
    fp, w, g, vol = load_bp(path)
    rng = np.random.default_rng(5)
    vox = rng.choice(vol.size, size=200, replace=False).astype(np.int64)
    sub = oracle.bp_f64(fp.astype(np.float64), w, g, vox=vox)
    np.testing.assert_array_equal(sub, oracle.bp_f64(fp.astype(np.float64), w, g)[vox])
    # a window of views that misses needed ones is refused
    with pytest.raises(ValueError):
        oracle.bp_f64(fp[:5].astype(np.float64), w, g, fp_view0=0)


@pytest.mark.skipif(not oracle.ref_available(), reason="compiled reference not present")
def test_restatement_matches_live_reference_random_geometry():
    rng = np.random.default_rng(11)
    for trial in range(3):
        sc = G.tiny(YL=int(rng.integers(40, 90)), ZL=int(rng.integers(3, 9)), iso_channel=float(rng.uniform(20, 30)),
                    beta_start=float(rng.uniform(-5, 5)), pitch=float(rng.uniform(0.4, 1.4)), delta=5,
                    XN=10, YN=9, ZN=7, dx=20.0, dy=21.0, dz=float(rng.uniform(0.5, 2.0)))
        ra = sc.rebin_args()
        proj = rng.random((ra["ViewN"], ra["YL"], ra["ZL"]), dtype=np.float32)
        a = oracle.rebin_f32(proj, **ra)
        b = oracle.ref_rebin_f32(proj, **ra)
        np.testing.assert_array_equal(a.view(np.uint32), b.view(np.uint32))
        g = sc.bp_geom()
        w = oracle.weight_table(sc.N_2pi, sc.HSCoef, sc.delta)
        fp = rng.standard_normal((g["PN"], g["ZL"], g["YL"]))
        np.testing.assert_array_equal(oracle.bp_f64(fp, w, g), oracle.ref_bp_f64(fp, w, g))


def test_filter_toeplitz_equals_matlab_fft_restatement():
    sc = G.tiny(YL=80, ZL=5)
    fa = sc.filter_args()
    rng = np.random.default_rng(3)
    p = rng.standard_normal((fa["ViewN"], fa["ZL"], fa["YL"]))
    a = oracle.filter_f64(p, **fa)
    b = oracle.filter_fft_f64(p, **fa)
    assert rel_l2(a, b) < 1e-12


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "filter_*.npz"))), ids=os.path.basename)
def test_filter_restatement_matches_reference_cufft_golden(path):
    d = np.load(path)
    YL, ZL, ViewN = (int(v) for v in d["sizes"])
    PLC, ZLC, dYL, dZL, SO = (float(v) for v in d["args"])
    mine = oracle.filter_f64(d["proj"].astype(np.float64), YL, ZL, ViewN, PLC, ZLC, dYL, dZL, SO)
    # the reference runs cuFFT in FP32 with --use_fast_math
    assert rel_l2(mine, d["out"]) < 2e-6


def test_filter_ramp_kernel_dc_and_shape():
    # a constant row is nearly annihilated inside (ramp has ~zero DC gain)
    sc = G.tiny(YL=256, ZL=1)
    fa = sc.filter_args()
    p = np.ones((1, 1, 256))
    out = oracle.filter_f64(p, **{**fa, "ViewN": 1, "ZL": 1})
    assert abs(out[0, 0, 128]) < 0.02 * abs(out[0, 0, 0])


def test_weight_table_shape():
    w = oracle.weight_table(984, 0.68, 60)
    half = int(np.ceil(492 * 0.68))
    assert half == 335
    nz = np.nonzero(w)[0]
    assert nz[0] == 492 - half and nz[-1] == 492 + half  # 671 views
    assert np.all(w[nz[0] + 60: nz[-1] - 59] == 1.0)
    np.testing.assert_allclose(w[nz[0]: nz[0] + 60], w[nz[-1] - 59: nz[-1] + 1][::-1], rtol=1e-12)
    assert 0 < w[nz[0]] < 1e-3


def test_projector_water_cylinder_chord():
    sc = G.tiny(YL=65, ZL=3, iso_channel=33.0)  # channel 32 is the central ray
    obj = P.water_cylinder(radius=100.0, half_length=5000.0)
    proj = oracle.project_ellipsoids(obj, **P.projector_args(sc))
    slope = (0 - (sc.ZLC1 - 1)) * sc.row_height / sc.SD
    expect = 200.0 * G.MU_WATER * np.sqrt(1 + slope ** 2)
    np.testing.assert_allclose(proj[:, 32, 0], expect, rtol=1e-6)
    # rays that miss the cylinder are zero
    assert np.all(proj[:, 0, :] == 0.0)


def test_projector_ellipsoid_matches_sphere_formula():
    # a sphere: chord = 2 sqrt(r^2 - d^2) for a ray at distance d from the centre
    sc = G.tiny(YL=33, ZL=1, iso_channel=17.0, rotations=0.25)
    r = 60.0
    obj = np.array([[0, 0, 0, sc.h * sc.BetaS / (2 * np.pi), r, r, r, 1, 0, 0, 0, 1, 0, 0, 0, 1, 1.0]])
    proj = oracle.project_ellipsoids(obj, **{**P.projector_args(sc), "ZL": 1, "ZLC0": 0.0})
    gam = (np.arange(33) - 16.0) * sc.dYA
    d = sc.SO * np.abs(np.sin(gam))
    expect = np.where(d < r, 2 * np.sqrt(np.maximum(r * r - d * d, 0)), 0)
    np.testing.assert_allclose(proj[0, :, 0], expect, rtol=1e-5, atol=1e-4)


def test_windowed_oracle_chain_equals_full_chain():
    """The helper that rebins/filters only the views a few slices need gives
    the same FP64 result as the whole-scan chain."""
    from oracle_chain import reference_slices

    sc = G.Scan(ZL=8, pitch=0.9375, rotations=4, XN=12, YN=12, ZN=40, dx=16.0, dy=16.0, dz=0.8, YL=160,
                det_pitch=1.0239 * 888 / 160, N_2pi=240, delta=15)
    obj = P.random_ellipsoids(5, 6, (-10.0, 10.0), body=(120.0, 90.0), semi_axes=(10, 50))
    fan = oracle.project_ellipsoids(obj, **P.projector_args(sc))
    zis = [3, 20, 37]
    vals, vox = reference_slices(sc, fan, zis)
    reb = oracle.rebin_f64(fan, **sc.rebin_args())
    rows = np.ascontiguousarray(reb.transpose(0, 2, 1)[sc.crop_front: sc.views - sc.crop_back])
    filt = oracle.filter_f64(rows, **sc.filter_args())
    w = oracle.weight_table(sc.N_2pi, sc.HSCoef, sc.delta)
    full = oracle.bp_f64(filt, w, sc.bp_geom(), vox=vox)
    assert rel_l2(vals, full) < 1e-10
