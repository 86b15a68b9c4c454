"""GPU tests of the streamed host execution of the whole-chain plan
(hr_recon_execute_host, fast form).

The fan data cross the host link in chunks of views; each chunk is rebinned
and filtered as soon as it has arrived (the same bits as the whole-scan
launches), the backprojection runs in z-block ranges as their view windows
complete, and every range's slices are copied out while later ranges compute.
Against the device entry (hr_recon_execute on the same plan):

* register-gather variants read the BF16 data directly: identical bits;
* texture variants sample an FP16 copy filled range by range with a scale taken
  from the first chunk (2^4 of headroom): the same samples up to that power of
  two except for values in FP16's subnormal range, so the volumes agree to
  FP32 rounding;
* when a later chunk outgrows that scale the copy is refilled whole with the
  scan's own scale: identical bits to the device entry again.
Short chunks (HELIXRECON_STREAM_CHUNK) give small scans several chunks and
backprojection ranges; 0 turns streaming off (the serial copy-in, chain,
copy-out path)."""
import contextlib
import os

import numpy as np
import pytest
import torch

from analyticalreconbigpatient_b200 import _lib, geometry as G, phantom as P
from analyticalreconbigpatient_b200.pipeline import HelicalRecon, project
from conftest import rel_l2

pytestmark = pytest.mark.gpu


@contextlib.contextmanager
def env(**kw):
    old = {k: os.environ.get(k) for k in kw}
    os.environ.update({k: str(v) for k, v in kw.items()})
    try:
        yield
    finally:
        for k, v in old.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v


def scan_and_fan(rotations=8, dz=1.0, seed=21):
    sc = G.Scan(ZL=16, pitch=0.9375, rotations=rotations, XN=96, YN=96, ZN=1, dx=3.0, dy=3.0, dz=dz)
    sc = G.Scan(**{**sc.__dict__, "ZN": sc.fully_sampled_slices() + 3})  # a few partially sampled end slices
    zlo, zhi = sc.h * sc.BetaS / (2 * np.pi), -sc.h * sc.BetaS / (2 * np.pi)
    fan = project(sc, P.random_ellipsoids(seed, 20, (zlo, zhi), body=(130.0, 100.0), semi_axes=(5, 40)))
    return sc, fan


def plan(sc, **kw):
    with env(**kw):
        return HelicalRecon(sc, form=_lib.HR_FORM_FAST)


def device_volume(rec, fan):
    v = rec.run(fan).clone()
    torch.cuda.synchronize()
    return v.cpu().numpy()


def host_volume(rec, fan, pinned):
    s = rec.scan
    fan_h = fan.cpu().pin_memory() if pinned else fan.cpu()
    vol_h = torch.full((s.YN, s.XN, s.ZN), float("nan"))
    if pinned:
        vol_h = vol_h.pin_memory()
    rec.run_host(fan_h, vol_h)
    return vol_h.numpy().copy()


@pytest.mark.parametrize("chunk", [256, 700, 0])
def test_streamed_host_entry_matches_the_device_entry(cuda, chunk):
    sc, fan = scan_and_fan()
    assert sc.PN > 2 * 700
    rec = plan(sc, HELIXRECON_STREAM_CHUNK=chunk)
    ref = device_volume(rec, fan)
    desc = rec.describe()
    scale = np.abs(ref).max()
    for pinned in (True, False, True):  # the last call repeats the first on the plan's kept buffers
        got = host_volume(rec, fan, pinned)
        assert np.isfinite(got).all(), (chunk, pinned, desc)
        if chunk == 0 or "texture" not in desc:
            assert np.array_equal(got, ref), (chunk, pinned, desc)
        else:
            assert rel_l2(got, ref) < 1e-6, (chunk, pinned, desc)
            assert np.abs(got - ref).max() < 1e-6 * scale, (chunk, pinned, desc)
    # a host fan into a device volume (the copies take their direction from the addresses)
    vol_d = torch.full((sc.YN, sc.XN, sc.ZN), float("nan"), device=cuda)
    rec.run_host(fan.cpu().pin_memory(), vol_d)
    assert np.array_equal(vol_d.cpu().numpy(), got), (chunk, desc)
    rec.close()


def test_streamed_host_entry_is_exact_with_register_gathers(cuda):
    sc, fan = scan_and_fan(rotations=6, dz=2.5, seed=5)
    rec = plan(sc, HELIXRECON_STREAM_CHUNK=300, HELIXRECON_BP_VARIANT=3)  # 8 slices per thread, BF16 gathers
    ref = device_volume(rec, fan)
    got = host_volume(rec, fan, pinned=True)
    assert np.array_equal(got, ref), rec.describe()
    rec.close()


def test_streamed_texture_copy_is_refilled_when_later_views_outgrow_the_first_chunk(cuda):
    sc, fan = scan_and_fan(seed=33)
    fan = fan.clone()
    fan[fan.shape[0] // 2:] *= 4096.0  # later views 2^12 larger: beyond the first chunk's 2^4 of headroom
    rec = plan(sc, HELIXRECON_STREAM_CHUNK=256)
    desc = rec.describe()
    ref = device_volume(rec, fan)
    got = host_volume(rec, fan, pinned=True)
    assert np.array_equal(got, ref), desc  # (texture variants: the whole copy refilled with the scan's own scale)
    # and a scan within the headroom afterwards is streamed again on the same plan
    fan2 = scan_and_fan(seed=34)[1]
    ref2 = device_volume(rec, fan2)
    got2 = host_volume(rec, fan2, pinned=True)
    assert rel_l2(got2, ref2) < 1e-6, desc
    rec.close()
