"""CPU tests of the host-side geometry derivation and phantom generation."""
import math

import numpy as np
import pytest

from analyticalreconbigpatient_b200 import geometry as G, phantom as P


def test_full_config_derived_scalars():
    sc = G.config("full")
    assert sc.views == 19680
    assert sc.seg_overlap == 77  # half fan in views + 1 (analyticalRecon.m:15-16)
    assert sc.PN == 19680 - 2 * 77
    np.testing.assert_allclose(sc.h, 0.984 * 64 * 1.0963 * 541 / 949, rtol=1e-12)  # table feed at iso
    np.testing.assert_allclose(sc.k1, 5 * 0.984 * 541 / 949, rtol=1e-12)
    assert abs(sc.k1 - 2.80) < 0.01
    np.testing.assert_allclose(sc.dYA, 2 * math.atan(1.0239 / (2 * 949)), rtol=1e-12)
    g = sc.bp_geom()
    assert g["YLC"] == (888 - 1) / 2 and g["ZLC"] == (64 - 1) / 2
    assert math.ceil(g["N_pi"] * g["HSCoef"]) == 335
    # every slice of the fully sampled grid sees the full 671-view window
    assert sc.ZN >= 1200
    assert np.all(sc.window_per_slice() == 671)
    assert sc.updates() == 512 * 512 * sc.ZN * 671


def test_small_config_updates_counts_clamped_windows():
    sc = G.config("small")
    win = sc.window_per_slice()
    assert win.max() == 671 and win.min() > 0
    # brute force against the backprojection's own window rule
    g = sc.bp_geom()
    tot = 0
    for zi in range(sc.ZN):
        z = (zi - g["ZNC"]) * g["dz"]
        s0 = math.ceil((2.0 * G.PI_TRUNC * z / g["h"] - g["BetaS"]) / g["DeltaFai"] - 0.5)
        s1, s2 = s0 - 335, s0 + 335
        if s1 < g["PN"] and s2 > 0:
            tot += min(s2, g["PN"] - 1) - max(s1, 0) + 1
    assert sc.updates() == tot * 256 * 256


def test_rebin_args_follow_the_matlab_driver():
    sc = G.config("small")
    ra = sc.rebin_args()
    f = np.float32
    # DeltaFai = (BetaE - BetaS)/(ViewN - 1), BetaE = BetaS + ViewN 2pi/N_2pi (Q4 of the reference)
    assert ra["DeltaFai"] == float(f(2 * math.pi / 984 * 3936 / 3935))
    assert ra["DeltaTheta"] == ra["DeltaFai"]
    assert ra["PLC"] == float(f(444.5) - f(1.0))
    assert ra["DeltaT"] == float(f(math.tan(sc.DecAngle / 2) * 541 * 3 / 888))
    fa = sc.filter_args()
    assert fa["dYL"] == float(f(sc.DecWidth / 888)) and fa["ViewN"] == sc.PN


def test_splitmix64_known_answer():
    # first outputs of SplitMix64 seeded with 0 (published reference values)
    r = P.SplitMix64(0)
    assert r.next_u64() == 0xE220A8397B1DCDAF
    assert r.next_u64() == 0x6E789E6AA1B965F4


def test_random_phantom_is_seeded_and_bounded():
    a = P.random_ellipsoids(7, 60, (-300.0, 300.0))
    b = P.random_ellipsoids(7, 60, (-300.0, 300.0))
    c = P.random_ellipsoids(8, 60, (-300.0, 300.0))
    assert np.array_equal(a, b) and not np.array_equal(a, c)
    assert a.shape == (61, 17) and a[0, 0] == 1  # body cylinder first
    ell = a[1:]
    assert np.all((ell[:, 4:7] >= 5) & (ell[:, 4:7] <= 120))
    mu = ell[:, 16] + G.MU_WATER
    assert np.all((mu >= 0.010) & (mu <= 0.030))
    assert np.all((ell[:, 1] / 180) ** 2 + (ell[:, 2] / 140) ** 2 <= 0.85 ** 2 + 1e-12)
    for row in ell:
        R = row[7:16].reshape(3, 3)
        np.testing.assert_allclose(R @ R.T, np.eye(3), atol=1e-12)
        assert abs(np.linalg.det(R) - 1) < 1e-12


def test_shepp_logan_scaled():
    ph = P.shepp_logan(fov=400.0)
    assert ph.shape == (10, 17)
    np.testing.assert_allclose(ph[0, 4:6], [0.69 * 200, 0.92 * 200])
    np.testing.assert_allclose(ph[0, 16] + ph[1, 16], 1.02 * G.MU_WATER)


@pytest.mark.parametrize("name", ["small", "full", "halfview"])
def test_configs_build(name):
    sc = G.config(name)
    assert sc.PN > 2 * math.ceil(sc.N_2pi / 2 * sc.HSCoef)
    assert sc.updates() > 0


def test_bigpatient_geometry_spans_the_scan():
    sc = G.config("bigpatient")
    assert sc.views == 196800 and sc.ZN == 2000
    assert abs(sc.ZN * sc.dz - sc.h * (sc.PN - 2 * 335) / 984) < 1e-6 * sc.ZN * sc.dz
    assert np.all(sc.window_per_slice() == 671)
