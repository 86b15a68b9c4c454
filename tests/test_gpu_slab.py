"""GPU tests of the slab-batched pipeline for long scans (hr_slab_plan).

A slab reconstructs its slices from its own view window; the result must
match the whole-scan fast chain to within BF16 rounding noise (the window's
rebinning measures view angles from its own first view, which can move a
BF16 rounding), and host- and device-resident buffers must give the same
bits."""
import numpy as np
import pytest
import torch

from analyticalreconbigpatient_b200 import _lib, geometry as G, phantom as P
from analyticalreconbigpatient_b200.pipeline import HelicalRecon, SlabRecon, project

pytestmark = pytest.mark.gpu


def whole(scan, fan):
    rec = HelicalRecon(scan, form=_lib.HR_FORM_FAST)
    v = rec.run(fan).clone()
    torch.cuda.synchronize()
    rec.close()
    return v.cpu().numpy()


@pytest.mark.parametrize("slab,dz", [(16, 1.0), (8, 2.5)])
def test_slabs_match_whole_scan_fast_chain(cuda, slab, dz):
    sc = G.Scan(ZL=16, pitch=0.9375, rotations=6, XN=96, YN=96, ZN=1, dx=3.0, dy=3.0, dz=dz)
    sc = G.Scan(**{**sc.__dict__, "ZN": sc.fully_sampled_slices() + 3})  # a few partially sampled end slices
    zlo, zhi = sc.h * sc.BetaS / (2 * np.pi), -sc.h * sc.BetaS / (2 * np.pi)
    fan = project(sc, P.random_ellipsoids(11, 20, (zlo, zhi), body=(130.0, 100.0), semi_axes=(5, 40)))
    ref = whole(sc, fan)
    rec = SlabRecon(sc, slab_slices=slab)
    vol = torch.full((sc.YN, sc.XN, sc.ZN), float("nan"), device=cuda)
    rec.run(fan, vol)
    desc = rec.describe()
    got = vol.cpu().numpy()
    assert np.isfinite(got).all(), desc
    scale = np.abs(ref).max()
    err = np.sqrt(np.mean((got - ref) ** 2)) / G.MU_WATER * 1000.0  # HU
    assert err < 0.05, (err, desc)
    assert np.abs(got - ref).max() < 0.01 * scale
    # host-resident buffers (pinned fan, pageable volume): identical bits
    fan_h = fan.cpu().pin_memory()
    vol_h = torch.zeros((sc.YN, sc.XN, sc.ZN))
    rec.run(fan_h, vol_h)
    assert np.array_equal(vol_h.numpy(), got)
    rec.close()



@pytest.mark.parametrize("assign", [_lib.HR_SLAB_BLOCKS, _lib.HR_SLAB_ROUND_ROBIN])
def test_parts_of_one_scan_compose_the_whole(cuda, assign):
    """The slabs of one scan split between plans (part p of 3, as ranks on three
    GPUs would hold them; here run one after the other on one GPU): every plan
    writes only its own slices, each from only its own fan views, and together
    they give the single plan's volume bit for bit (same kernel variant)."""
    import os

    from analyticalreconbigpatient_b200.pipeline import slab_windows

    sc = G.Scan(ZL=16, pitch=0.9375, rotations=6, XN=64, YN=64, ZN=1, dx=4.0, dy=4.0, dz=1.5)
    sc = G.Scan(**{**sc.__dict__, "ZN": sc.fully_sampled_slices() + 2})
    zlo, zhi = sc.h * sc.BetaS / (2 * np.pi), -sc.h * sc.BetaS / (2 * np.pi)
    fan = project(sc, P.random_ellipsoids(12, 20, (zlo, zhi), body=(110.0, 90.0), semi_axes=(5, 40)))
    os.environ["HELIXRECON_BP_VARIANT"] = "11"
    try:
        whole_plan = SlabRecon(sc, slab_slices=8)
        ref = torch.full((sc.YN, sc.XN, sc.ZN), float("nan"), device=cuda)
        whole_plan.run(fan, ref)
        first, count, nbytes = whole_plan.fan_range()
        whole_plan.close()
        per_view = sc.YL * sc.ZL * 4
        # each fan view crosses from the caller's buffer once (overlaps are copied on the device)
        assert nbytes == count * per_view and first + count <= sc.views
        got = torch.full_like(ref, float("nan"))
        for part in range(3):
            rec = SlabRecon(sc, slab_slices=8, part=part, nparts=3, assign=assign)
            f0, n, _ = rec.fan_range()
            only_mine = fan[f0: f0 + n].clone()  # the part's views and nothing else
            rec.run(only_mine, got, fan_view0=f0)
            assert f"part {part} of 3" in rec.describe()
            rec.close()
    finally:
        del os.environ["HELIXRECON_BP_VARIANT"]
    wins = [w for p in range(3) for w in slab_windows(sc, 8, p, 3, assign)]
    assert sorted(w["slab"] for w in wins) == list(range(-(-sc.ZN // 8)))
    assert torch.isfinite(got).all()
    assert torch.equal(got, ref)
