"""GPU tests of the fast (chosen) form: BF16 filtered data, fast
backprojection. Its error is stated in HU against the FP64 oracle, with the
water level of the same geometry as the HU calibration (the reference's 3D
weight scales the reconstructed level with the pitch)."""
import numpy as np
import pytest
import torch

from analyticalreconbigpatient_b200 import _lib, geometry as G, phantom as P
from analyticalreconbigpatient_b200.pipeline import HelicalRecon, project
from conftest import rel_l2
from oracle_chain import hu_rmse, reference_slices

pytestmark = pytest.mark.gpu

HU_BUDGET = 1.0


def recon(scan, fan, form):
    rec = HelicalRecon(scan, form=form)
    vol = rec.run(fan)
    torch.cuda.synchronize()
    out = vol.cpu().numpy()
    rec.close()
    return out


def water_level(scan):
    fan = project(scan, P.water_cylinder(radius=120.0, half_length=1e5))
    v = recon(scan, fan, _lib.HR_FORM_PLAIN)
    c = scan.XN // 2
    r = max(2, int(40.0 / scan.dx))
    return float(v[c - r: c + r, c - r: c + r, :].mean())


@pytest.mark.parametrize("cfg", ["small", "full"])
def test_fast_and_plain_hu_rmse_vs_fp64_oracle(cuda, cfg):
    sc = G.config(cfg)
    zlo = sc.h * sc.BetaS / (2 * np.pi)
    zhi = sc.h * (sc.BetaS + sc.views * sc.dBeta) / (2 * np.pi)
    obj = P.shepp_logan() if cfg == "small" else P.random_ellipsoids(1000, 60, (zlo, zhi))
    fan = project(sc, obj)
    fast = recon(sc, fan, _lib.HR_FORM_FAST)
    plain = recon(sc, fan, _lib.HR_FORM_PLAIN)
    wl = water_level(sc)
    assert 0.8 * G.MU_WATER < wl < 1.05 * G.MU_WATER
    fan_h = fan.cpu().numpy()
    del fan
    # full: the first and last slices (windows clamped to the scan's views) and two inner ones
    zis = [sc.ZN // 2] if cfg == "small" else [0, sc.ZN // 3, 2 * sc.ZN // 3, sc.ZN - 1]
    step = 1 if cfg == "small" else 2
    ref, vox = reference_slices(sc, fan_h, zis, xy_step=step)
    # the reference CPU path rebins the whole scan in FP32 (bit-identical to the GPU rebinning)
    import oracle

    reb32 = oracle.rebin_f32(fan_h, **sc.rebin_args())
    refpath, _ = reference_slices(sc, fan_h, zis, xy_step=step, rebinned=reb32)
    del reb32
    hu_fast = hu_rmse(fast.ravel()[vox], ref, wl)
    hu_plain = hu_rmse(plain.ravel()[vox], ref, wl)
    e_path = rel_l2(plain.ravel()[vox], refpath)
    e_f64 = rel_l2(plain.ravel()[vox], ref)
    n = vox.size // len(zis)
    per_slice = [rel_l2(plain.ravel()[vox[i * n:(i + 1) * n]], refpath[i * n:(i + 1) * n]) for i in range(len(zis))]
    print(f"[{cfg}] HU RMSE vs FP64 oracle: fast {hu_fast:.4f}  plain {hu_plain:.5f}  "
          f"(water level {wl:.6f}, {vox.size} voxels); plain rel L2 vs reference path {e_path:.3e} "
          f"(by slice {', '.join(f'z{z}: {e:.2e}' for z, e in zip(zis, per_slice))}), vs FP64 oracle {e_f64:.3e}")
    assert hu_plain < 0.05
    assert hu_fast < HU_BUDGET
    assert e_path < 1e-5 and max(per_slice) < 1e-5


def test_fast_backprojection_matches_plain_on_the_same_data(cuda):
    """With identical BF16-representable filtered data the two backprojections
    differ only by FP32 arithmetic and approximate SFU functions."""
    from analyticalreconbigpatient_b200.pipeline import StagePlans

    sc = G.Scan(ZL=16, pitch=0.9375, rotations=3, XN=64, YN=64, ZN=24, dx=4.0, dy=4.0, dz=1.0)
    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(0)
    filt = torch.tensor(rng.standard_normal((sc.PN, sc.ZL, sc.YL)).astype(np.float32), device=dev)
    filt = filt.to(torch.bfloat16).to(torch.float32)  # make the data exactly BF16
    plain = StagePlans(sc, _lib.HR_FORM_PLAIN)
    fast = StagePlans(sc, _lib.HR_FORM_FAST)
    pairs = torch.empty((sc.PN, sc.ZL, sc.YL), dtype=torch.int32, device=dev)
    fast.pack(pairs, filt)
    v1 = torch.empty((sc.YN, sc.XN, sc.ZN), dtype=torch.float32, device=dev)
    v2 = torch.empty_like(v1)
    plain.backproject(v1, filt)
    fast.backproject(v2, pairs)
    torch.cuda.synchronize()
    a, b = v1.cpu().numpy(), v2.cpu().numpy()
    plain.close()
    fast.close()
    assert rel_l2(b, a) < 2e-4
    assert np.array_equal(a == 0, b == 0)


def test_pack_pairs_layout(cuda):
    dev = torch.device("cuda", 0)
    x = torch.randn(7, 33, device=dev)
    out = torch.empty((7, 33), dtype=torch.int32, device=dev)
    _lib.check(_lib.load().hr_pack_bf16_pairs(out.data_ptr(), x.data_ptr(), 7, 33, 0))
    torch.cuda.synchronize()
    o = out.cpu().numpy().view(np.uint32)
    lo = (o & 0xFFFF).astype(np.uint32) << 16
    hi = o & 0xFFFF0000
    xb = x.to(torch.bfloat16).to(torch.float32).cpu().numpy()
    np.testing.assert_array_equal(lo.view(np.float32), xb)
    np.testing.assert_array_equal(hi[:, :-1].view(np.float32), xb[:, 1:])
    assert np.all(hi[:, -1] == 0)


@pytest.mark.parametrize("pixel", [5.0, 0.9766])
def test_every_fast_variant_gives_the_same_volume(cuda, pixel):
    """The autotuner's candidates differ only in work distribution: the same
    FP32 operations per (voxel, view) in the same view order, so identical bits.
    Coarse 5 mm voxels spread a CTA's taps over the whole detector; 0.98 mm
    voxels (the clinical 500 mm / 512 grid) keep them within a few channels."""
    from analyticalreconbigpatient_b200.pipeline import StagePlans

    sc = G.Scan(ZL=16, pitch=0.9375, rotations=3, XN=40, YN=48, ZN=37, dx=pixel, dy=pixel, dz=1.0)
    rng = np.random.default_rng(3)
    filt = torch.tensor(rng.standard_normal((sc.PN, sc.ZL, sc.YL)).astype(np.float32), device=cuda)
    fast = StagePlans(sc, _lib.HR_FORM_FAST)
    pairs = torch.empty((sc.PN, sc.ZL, sc.YL), dtype=torch.int32, device=cuda)
    fast.pack(pairs, filt)
    lib = _lib.load()
    vols = []
    nvar = 22
    for v in range(nvar):
        _lib.check(lib.hr_bp_select(fast._bp, v))
        vol = torch.full((sc.YN, sc.XN, sc.ZN), float("nan"), device=cuda)
        fast.backproject(vol, pairs)
        torch.cuda.synchronize()
        vols.append(vol.cpu().numpy())
    desc = fast.autotune(torch.empty_like(vol), pairs)
    assert "autotuned" in desc
    fast.close()
    for v in (1, 2, 3, 4, 5, 8, 10):
        assert np.array_equal(vols[v], vols[0]), v
    for v in (6, 7, 9):  # packed FP32x2 rounds like FP32, but FMA contraction may differ
        assert rel_l2(vols[v], vols[0]) < 1e-6, v
    # texture variants: the hardware blends with 1.8 fixed-point weights, an
    # error of up to 1/256 of the neighbour difference per tap (largest, about
    # 0.5 % of the volume, on white-noise data like these)
    for v in (11, 12, 13, 14, 15):
        assert rel_l2(vols[v], vols[0]) < 1e-2, (v, rel_l2(vols[v], vols[0]))
    assert np.array_equal(vols[11], vols[12]) and np.array_equal(vols[11], vols[13])
    assert np.array_equal(vols[14], vols[15])
    # segmented view loops (16: 8 slices per thread, 17: 4; 18, 19: two views per iteration in narrow
    # segments): same operations per slice and view, in the same order
    assert np.array_equal(vols[16], vols[11]) and np.array_equal(vols[17], vols[13])
    assert np.array_equal(vols[18], vols[11]) and np.array_equal(vols[19], vols[13])
    # 20, 21: the code of 16 and 19 with registers bounded for 6 CTAs per SM
    assert np.array_equal(vols[20], vols[16]) and np.array_equal(vols[21], vols[19])
    assert np.isfinite(vols[0]).all()


def test_two_view_segments_equal_one_view_at_thick_slices(cuda):
    """At 4 mm slices most segments hold a few slices, so the two-view loop of
    variants 18-19 (8 / 4 slices per thread) runs for most views (odd segment
    lengths included); it must give the one-view loop's bits (variants 16-17
    and 11 / 13, the same operations per slice and view in the same order)."""
    from analyticalreconbigpatient_b200.pipeline import StagePlans

    sc = G.Scan(ZL=16, pitch=0.9375, rotations=6, XN=48, YN=40, ZN=1, dx=0.98, dy=0.98, dz=4.0)
    sc = G.replace(sc, ZN=sc.fully_sampled_slices())
    assert sc.ZN >= 8, sc.ZN
    rng = np.random.default_rng(5)
    filt = torch.tensor(rng.standard_normal((sc.PN, sc.ZL, sc.YL)).astype(np.float32), device=cuda)
    fast = StagePlans(sc, _lib.HR_FORM_FAST)
    pairs = torch.empty((sc.PN, sc.ZL, sc.YL), dtype=torch.int32, device=cuda)
    fast.pack(pairs, filt)
    lib = _lib.load()
    vols = {}
    for v in (11, 13, 16, 17, 18, 19, 20, 21):
        _lib.check(lib.hr_bp_select(fast._bp, v))
        vol = torch.full((sc.YN, sc.XN, sc.ZN), float("nan"), device=cuda)
        fast.backproject(vol, pairs)
        torch.cuda.synchronize()
        vols[v] = vol.cpu().numpy()
    fast.close()
    assert np.isfinite(vols[11]).all() and np.count_nonzero(vols[11]) > vols[11].size // 2
    for a, b in ((18, 11), (16, 11), (19, 13), (17, 13), (20, 11), (21, 13)):
        assert np.array_equal(vols[a], vols[b]), (a, b)


@pytest.mark.parametrize("gain", [2.0**18, 2.0**-100])
def test_fp16_texture_scales_any_data_range(cuda, gain):
    """The FP16 texture copy is scaled by a power of two chosen from the data's
    largest magnitude: data far outside FP16's range (overflow at 65504,
    underflow below 6e-8) give the volume of the unit-range data times the gain
    (a power of two, so the BF16 samples scale exactly)."""
    from analyticalreconbigpatient_b200.pipeline import StagePlans

    sc = G.Scan(ZL=16, pitch=0.9375, rotations=3, XN=24, YN=24, ZN=21, dx=2.0, dy=2.0, dz=1.0)
    rng = np.random.default_rng(5)
    filt = torch.tensor(rng.standard_normal((sc.PN, sc.ZL, sc.YL)).astype(np.float32), device=cuda)
    fast = StagePlans(sc, _lib.HR_FORM_FAST)
    lib = _lib.load()
    out = {}
    for name, g in (("unit", 1.0), ("scaled", gain)):
        pairs = torch.empty((sc.PN, sc.ZL, sc.YL), dtype=torch.int32, device=cuda)
        fast.pack(pairs, filt * g)
        for v in (11, 14):
            _lib.check(lib.hr_bp_select(fast._bp, v))
            vol = torch.full((sc.YN, sc.XN, sc.ZN), float("nan"), device=cuda)
            fast.backproject(vol, pairs)
            torch.cuda.synchronize()
            out[name, v] = vol.cpu().numpy().astype(np.float64)
    fast.close()
    assert rel_l2(out["unit", 11], out["unit", 14]) < 1e-3
    assert rel_l2(out["scaled", 11] / gain, out["unit", 11]) < 1e-6
    assert rel_l2(out["scaled", 14] / gain, out["unit", 14]) < 1e-6


def test_texture_sample_rate_probe(cuda):
    """The texture-rate probe (the roofline of the texture variants) returns a
    device-wide bilinear sample rate of the right order for a B200: 148 SMs,
    up to four samples per SM per clock at ~2 GHz."""
    from analyticalreconbigpatient_b200 import probe

    rate = probe.texture_sample_rate()
    assert 1e11 < rate < 4e12, rate
