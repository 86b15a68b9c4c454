"""GPU tests of the uneven-batch persistent launch (hr_batch_plan) and of the
Poisson photon-noise generator that feeds it.

A scan reconstructed inside the batch must equal the same scan reconstructed
alone with the same backprojection kernel body (the persistent kernel runs the
solo kernel's per-column code on the same tables): identical up to the FMA
contraction choices of the two compiled kernels (rel L2 < 1e-6), and replaying
the captured graph, or capturing a new one for other buffers, changes nothing."""
import math
import os

import numpy as np
import pytest
import torch

from analyticalreconbigpatient_b200 import _lib, geometry as G, phantom as P
from analyticalreconbigpatient_b200.pipeline import BatchRecon, HelicalRecon, add_poisson_noise, project
from conftest import rel_l2

pytestmark = pytest.mark.gpu


def uneven_scans():
    base = dict(YL=200, det_pitch=1.0239 * 888 / 200, N_2pi=240)
    return [G.Scan(**base, ZL=8, pitch=0.9375, rotations=3, XN=40, YN=40, ZN=10, dx=6.0, dy=6.0, dz=1.0),
            G.Scan(**base, ZL=16, pitch=0.5, rotations=5, XN=64, YN=48, ZN=23, dx=4.0, dy=4.0, dz=0.8),
            G.Scan(**base, ZL=4, pitch=1.375, rotations=2, XN=24, YN=24, ZN=3, dx=9.0, dy=9.0, dz=0.5),
            G.Scan(**base, ZL=32, pitch=0.9375, rotations=4, XN=56, YN=56, ZN=41, dx=4.5, dy=4.5, dz=0.7)]


def fans_for(scans, noise=False):
    out = []
    for i, sc in enumerate(scans):
        zlo, zhi = sc.h * sc.BetaS / (2 * math.pi), -sc.h * sc.BetaS / (2 * math.pi)
        fan = project(sc, P.random_ellipsoids(100 + i, 15, (zlo, zhi), body=(90.0, 70.0), semi_axes=(5, 40)))
        if noise:
            add_poisson_noise(fan, 2e5, 1000 + i)
        out.append(fan)
    return out


def solo(scan, fan, fast_variant):
    os.environ["HELIXRECON_BP_VARIANT"] = str(fast_variant)
    try:
        rec = HelicalRecon(scan, form=_lib.HR_FORM_FAST)
    finally:
        del os.environ["HELIXRECON_BP_VARIANT"]
    v = rec.run(fan).clone()
    torch.cuda.synchronize()
    rec.close()
    return v.cpu().numpy()


# slices per thread -> the solo per-slice variant with the same kernel body
NZ_TO_FAST = {16: 0, 8: 3, 4: 8}
# batch variants with texture taps: the solo FP16 texture variants
NZ_TO_TEX = {8: 11, 4: 13}
TEXTURED = (6, 7, 8, 9, 10, 12, 13, 14, 15, 16)


PER_SCAN = 11  # each scan's own kernel on a stream of its own


@pytest.mark.parametrize("bv", [0, 1, 2, 3, 5, 6, 7, 9, PER_SCAN, 12, 13, 15, 16])
def test_batch_equals_each_scan_alone(cuda, bv):
    scans = uneven_scans()
    fans = fans_for(scans, noise=True)
    rec = BatchRecon(scans)
    rec.select(bv)
    vols = [torch.full((s.YN, s.XN, s.ZN), float("nan"), device=cuda) for s in scans]
    rec.run(fans, vols)
    torch.cuda.synchronize()
    rec.check()
    desc = rec.describe()
    if bv == PER_SCAN:
        solo_variants = [int(t) for t in desc.split("variant by scan:")[1].split("(")[0].split()]
        assert len(solo_variants) == len(scans), desc
    else:
        nzs = [int(t) for t in desc.split("slices per thread by scan:")[1].split("(")[0].split()]
        assert len(nzs) == len(scans) and set(nzs) <= ({8, 4} if bv in TEXTURED else {16, 8, 4}), desc
        assert ("FP16 textures" in desc) == (bv in TEXTURED), desc
        solo_variants = [(NZ_TO_TEX if bv in TEXTURED else NZ_TO_FAST)[nz] for nz in nzs]
    for sc, fan, v, sv in zip(scans, fans, vols, solo_variants):
        got = v.cpu().numpy()
        ref = solo(sc, fan, sv)
        assert np.isfinite(got).all(), rec.describe()
        assert np.count_nonzero(ref) > ref.size // 2
        assert rel_l2(got, ref) < 1e-6, (sc, rec.describe())
    rec.close()


@pytest.mark.parametrize("bv", [3, PER_SCAN])
def test_batch_graph_replay_and_new_buffers(cuda, bv):
    scans = uneven_scans()[:3]
    fans = fans_for(scans)
    rec = BatchRecon(scans)
    rec.select(bv)
    desc = rec.describe()
    assert "3 scans" in desc and ("persistent launch" in desc) == (bv != PER_SCAN), desc
    vols = [torch.zeros((s.YN, s.XN, s.ZN), device=cuda) for s in scans]
    rec.run(fans, vols)
    first = [v.clone() for v in vols]
    for v in vols:
        v.fill_(float("nan"))
    rec.run(fans, vols)  # graph replay
    other = [torch.zeros_like(v) for v in vols]
    fans2 = [f.clone() for f in fans]
    rec.run(fans2, other)  # new addresses: a new graph
    torch.cuda.synchronize()
    for a, b, c in zip(first, vols, other):
        assert torch.equal(a, b) and torch.equal(a, c)
    with pytest.raises(ValueError):
        rec.run(fans[:2], vols[:2])
    rec.close()


@pytest.mark.parametrize("bv,pinned", [(PER_SCAN, True), (15, True), (9, False)])
def test_batch_host_entry_equals_device_entry(cuda, bv, pinned):
    """hr_batch_execute_host (fans streamed in through the two staging buffers,
    volumes copied out per scan or after the persistent launch) gives the
    device entry's volumes bit for bit, from page-locked or pageable memory,
    and again on a second call (buffers kept with the plan)."""
    scans = uneven_scans()
    fans = fans_for(scans, noise=True)
    rec = BatchRecon(scans)
    rec.select(bv)
    vols = [torch.empty((s.YN, s.XN, s.ZN), device=cuda) for s in scans]
    rec.run(fans, vols)
    torch.cuda.synchronize()
    ref = [v.cpu() for v in vols]
    h_fans = [f.cpu().pin_memory() if pinned else f.cpu() for f in fans]
    for rep in range(2):
        h_vols = [torch.full(r.shape, float("nan")).pin_memory() if pinned else torch.full(r.shape, float("nan"))
                  for r in ref]
        rec.run_host(h_fans, h_vols)
        for a, b in zip(h_vols, ref):
            assert torch.equal(a, b), (bv, rep, rec.describe())
    with pytest.raises(TypeError):
        rec.run_host(fans, h_vols)  # device fans
    rec.close()


def test_batch_autotuner_reports_every_variant(cuda):
    rec = BatchRecon(uneven_scans()[:2])
    desc = rec.describe()
    assert "autotuned" in desc and all(f"v{v}=" in desc for v in range(12)), desc
    rec.close()


@pytest.mark.parametrize("p", [0.5, 2.0, 7.0, 10.0, 12.5])
def test_poisson_noise_moments(cuda, p):
    # both branches of the sampler (lam >= 10: PTRS; lam < 10: product of uniforms)
    I0 = 2e5
    lam = I0 * math.exp(-p)
    n = 1 << 20
    x = torch.full((n,), p, dtype=torch.float32, device=cuda)
    add_poisson_noise(x, I0, 7)
    N = np.rint(I0 * np.exp(-x.double().cpu().numpy()))
    # the generator reports max(N, 1): E = lam + P0, E[X^2] = lam + lam^2 + P0
    p0 = math.exp(-lam)
    mu = lam + p0
    var_true = lam + lam * lam + p0 - mu * mu
    mean, var = N.mean(), N.var()
    assert abs(mean - mu) < 5 * math.sqrt(var_true / n), (mean, mu)
    # spread of the sample variance ~ sqrt((mu4 - var^2) / n), with mu4 <= var + 3 var^2 + lam for these laws
    assert abs(var - var_true) < 5 * math.sqrt((var_true + 2 * var_true ** 2 + lam) / n), (var, var_true)
    # seeded and launch-independent: the same seed gives the same bits
    y = torch.full((n,), p, dtype=torch.float32, device=cuda)
    add_poisson_noise(y, I0, 7)
    assert torch.equal(x, y)
    z = torch.full((n,), p, dtype=torch.float32, device=cuda)
    add_poisson_noise(z, I0, 8)
    assert not torch.equal(x, z)


def test_poisson_noise_small_counts_follow_the_pmf(cuda):
    I0, lam = 1e5, 3.0
    p = math.log(I0 / lam)
    n = 1 << 20
    x = torch.full((n,), p, dtype=torch.float32, device=cuda)
    add_poisson_noise(x, I0, 11)
    N = np.rint(I0 * np.exp(-x.double().cpu().numpy())).astype(np.int64)
    # N = 0 is reported as 1 photon (log of zero counts is clamped)
    counts = np.bincount(N, minlength=12)[:12].astype(np.float64)
    pmf = np.array([math.exp(-lam) * lam ** k / math.factorial(k) for k in range(12)])
    expect = pmf * n
    expect[1] += expect[0]
    expect[0] = 0.0
    for k in range(1, 10):
        assert abs(counts[k] - expect[k]) < 6 * math.sqrt(expect[k]), (k, counts[k], expect[k])
