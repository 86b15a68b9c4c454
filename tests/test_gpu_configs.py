"""Parity of the big-patient slab pipeline and of the uneven batch at their own
geometries (not only at the c2 geometry the fast form was first pinned on).

* Big patient: the 888x64 detector at pitch 0.984, a 512x512 grid of
  0.9766 mm pixels and the 3.92 mm slices of the 200-rotation workload, in
  slabs of 64 slices, on a 16-rotation scan (three slabs: a first, a middle and
  a last one). Whole slices -- the first and last of the volume, both sides of
  each slab boundary, the middle -- against the FP64 oracle, each from its own
  view window. The reference reconstructs long scans by summing overlapping
  view segments (src/analyticalRecon.m:15-25, crop at
  src/analyticalReconBigPatient.m:80-93); the slabs replace that loop.
* Uneven batch: scans of pitch 0.5 and 1.375, 16/32/64 rows, thin slices, with
  Poisson noise at I0 = 2e5 photons per ray, through one batch plan; each
  scan's volume against the same scan's plain FP32 solo reconstruction (the
  drop-in path), as the batch workload states its error.
"""
import math

import numpy as np
import pytest
import torch

from analyticalreconbigpatient_b200 import _lib, geometry as G, phantom as P
from analyticalreconbigpatient_b200.pipeline import BatchRecon, HelicalRecon, SlabRecon, add_poisson_noise, project
from oracle_chain import hu_rmse, reference_slices

pytestmark = pytest.mark.gpu

HU_BUDGET = 1.0


def _plain(scan, fan):
    rec = HelicalRecon(scan, form=_lib.HR_FORM_PLAIN)
    v = rec.run(fan).cpu().numpy()
    rec.close()
    torch.cuda.empty_cache()
    return v


def _water_level(scan):
    fan = project(scan, P.water_cylinder(radius=120.0, half_length=1e6))
    v = _plain(scan, fan)
    c = scan.XN // 2
    r = max(2, int(40.0 / scan.dx))
    return float(v[c - r: c + r, c - r: c + r, :].mean())


def bigpatient_scan(rotations=16):
    """The big-patient workload's detector, pitch, grid and slice thickness
    (3.92 mm) on a shorter helix; the slices span its fully sampled range."""
    dz = G.config("bigpatient").dz
    sc = G.Scan(ZL=64, pitch=0.984, rotations=rotations, XN=512, YN=512, ZN=1, dx=0.9766, dy=0.9766, dz=dz)
    return G.replace(sc, ZN=sc.fully_sampled_slices())


def test_bigpatient_slabs_vs_fp64_oracle(cuda):
    sc = bigpatient_scan()
    slab = 64
    assert abs(sc.dz - 3.92) < 0.01 and sc.ZN > 2 * slab, (sc.dz, sc.ZN)
    zlo = sc.h * sc.BetaS / (2 * np.pi)
    zhi = sc.h * (sc.BetaS + sc.views * sc.dBeta) / (2 * np.pi)
    objs = P.random_ellipsoids(3016, 40, (zlo, zhi), body=(250.0, 175.0), body_half_length=0.5 * (zhi - zlo) + 200.0)
    fan = project(sc, objs)
    rec = SlabRecon(sc, slab_slices=slab)
    vol = torch.full((sc.YN, sc.XN, sc.ZN), float("nan"), device=cuda)
    rec.run(fan, vol)
    desc = rec.describe()
    rec.close()
    got = vol.cpu().numpy()
    del vol
    assert np.isfinite(got).all(), desc
    assert desc.startswith(f"{-(-sc.ZN // slab)} slabs"), desc
    wl = _water_level(sc)
    fan_h = fan.cpu().numpy()
    del fan
    torch.cuda.empty_cache()
    zis = sorted({0, slab - 1, slab, sc.ZN // 2, 2 * slab - 1, 2 * slab, sc.ZN - 1})
    ref, vox = reference_slices(sc, fan_h, zis, xy_step=2)
    n = vox.size // len(zis)
    per_slice = [hu_rmse(got.ravel()[vox[i * n:(i + 1) * n]], ref[i * n:(i + 1) * n], wl) for i in range(len(zis))]
    total = hu_rmse(got.ravel()[vox], ref, wl)
    print(f"[bigpatient 3.92 mm, {desc.split(';')[0]}] HU RMSE vs FP64 oracle by slice "
          + ", ".join(f"z{z}: {h:.3f}" for z, h in zip(zis, per_slice)) + f"; all {total:.3f} (water {wl:.6f})")
    assert max(per_slice) < HU_BUDGET, per_slice
    assert np.count_nonzero(ref) > ref.size // 2


def batch_config_scans():
    """Six scans of the uneven batch's kinds: pitch 0.5 and 1.375, 16, 32 and
    64 rows, 256^2 (1.953 mm) or 512^2 (0.9766 mm) grids and slices thinner
    than 0.625 mm, 2-4 rotations."""
    out = []
    for rot, ZL, pitch, N, ZN in ((2, 16, 0.5, 256, 40), (3, 32, 1.375, 256, 120), (2, 64, 1.375, 512, 160),
                                  (4, 16, 1.375, 512, 100), (3, 64, 0.5, 256, 200), (2, 32, 0.5, 512, 48)):
        d = 500.0 / N
        sc = G.Scan(ZL=ZL, pitch=pitch, rotations=rot, XN=N, YN=N, ZN=ZN, dx=d, dy=d, dz=0.625)
        half = math.ceil(sc.N_2pi / 2.0 * sc.HSCoef)
        span = sc.h * (sc.PN - 2 * half) / sc.N_2pi
        out.append(G.replace(sc, dz=min(0.625, span / ZN)))
    return out


@pytest.mark.parametrize("variant", [None, 0, 9])
def test_batch_vs_plain_solo_with_noise(cuda, variant):
    """variant None: what the batch autotuner chooses; 0: persistent launch,
    register gathers; 9: persistent launch, FP16 texture taps."""
    scans = batch_config_scans()
    assert {s.pitch for s in scans} == {0.5, 1.375} and {s.ZL for s in scans} == {16, 32, 64}
    assert all(s.dz < 0.625 for s in scans)
    fans = []
    for i, sc in enumerate(scans):
        zlo = sc.h * sc.BetaS / (2 * np.pi)
        zhi = sc.h * (sc.BetaS + sc.views * sc.dBeta) / (2 * np.pi)
        f = project(sc, P.random_ellipsoids(5100 + i, 30, (zlo, zhi)))
        add_poisson_noise(f, 2e5, 7100 + i)
        fans.append(f)
    rec = BatchRecon(scans)
    if variant is not None:
        rec.select(variant)
    vols = [torch.full((s.YN, s.XN, s.ZN), float("nan"), device=cuda) for s in scans]
    rec.run(fans, vols)
    torch.cuda.synchronize()
    rec.check()
    desc = rec.describe()
    got = [v.cpu().numpy() for v in vols]
    rec.close()
    del vols
    torch.cuda.empty_cache()
    hus = []
    for sc, fan, g in zip(scans, fans, got):
        ref = _plain(sc, fan)
        assert np.isfinite(g).all(), desc
        hus.append(float(np.sqrt(np.mean((g.astype(np.float64) - ref) ** 2)) / G.MU_WATER * 1000.0))
    print(f"[batch variant {variant}] HU RMSE vs plain solo by scan: " + ", ".join(f"{h:.3f}" for h in hus)
          + f" ({desc})")
    assert max(hus) < HU_BUDGET, (hus, desc)
