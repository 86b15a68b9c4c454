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

