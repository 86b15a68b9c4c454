"""The allocation-free backprojection entry (hr_bp_plain_noalloc).

It exists for callers that cannot call cudaMalloc -- code running under CUDA
graph capture, streaming pipelines that must not allocate (cudaMalloc and
cudaFree synchronise the device), hosts whose allocator owns all device
memory. Its scratch (the per-view table) is a fixed array inside the library.
The test calls it through the C ABI twice in a row, on two different scans,
and checks each result against the plan-based plain entry (hr_bp_execute)
within the plain form's tolerance. This file sorts last so that a run stopping
at the first failure has run every other test first.
"""
import ctypes

import numpy as np
import pytest
import torch

from analyticalreconbigpatient_b200 import _lib, geometry as G
from conftest import rel_l2

pytestmark = pytest.mark.gpu

PLAIN_TOL = 1e-5


def _case(scan, seed, dev):
    rng = np.random.default_rng(seed)
    w = np.zeros(scan.N_2pi)
    _lib.call("hr_view_weights", w.ctypes.data, scan.N_2pi, scan.HSCoef, scan.delta)
    fp = torch.tensor(rng.standard_normal((scan.PN, scan.ZL, scan.YL)).astype(np.float32), device=dev)
    return _lib.BpGeom.from_dict(scan.bp_geom()), w, fp


def _plan_result(geom, w, fp, shape, dev):
    lib = _lib.load()
    plan = ctypes.c_void_p()
    _lib.check(lib.hr_bp_plan_create(ctypes.byref(plan), ctypes.byref(geom), w.ctypes.data, _lib.HR_FORM_PLAIN))
    vol = torch.empty(shape, dtype=torch.float32, device=dev)
    _lib.check(lib.hr_bp_execute(plan, vol.data_ptr(), fp.data_ptr(), 0))
    torch.cuda.synchronize()
    lib.hr_bp_plan_destroy(plan)
    return vol.cpu().numpy()


def test_no_alloc_entry_matches_plan_entry_on_two_calls(cuda):
    lib = _lib.load()
    scans = [G.Scan(ZL=16, pitch=0.9375, rotations=3, XN=48, YN=40, ZN=20, dx=5.0, dy=5.5, dz=1.0),
             G.Scan(ZL=8, pitch=1.2, rotations=2.5, XN=32, YN=36, ZN=13, dx=6.0, dy=6.0, dz=2.0, beta_start=40.0,
                    delta=40)]
    for seed, sc in enumerate(scans):
        geom, w, fp = _case(sc, seed, cuda)
        d_w = torch.tensor(w.astype(np.float32), device=cuda)
        vol = torch.full((sc.YN, sc.XN, sc.ZN), float("nan"), dtype=torch.float32, device=cuda)
        _lib.check(lib.hr_bp_plain_noalloc(vol.data_ptr(), fp.data_ptr(), d_w.data_ptr(), ctypes.byref(geom), 0))
        torch.cuda.synchronize()
        mine = vol.cpu().numpy()
        ref = _plan_result(geom, w, fp, (sc.YN, sc.XN, sc.ZN), cuda)
        assert np.isfinite(mine).all()
        assert rel_l2(mine, ref) < PLAIN_TOL, seed
        assert np.array_equal(mine == 0, ref == 0)


def test_no_alloc_entry_rejects_too_many_views(cuda):
    lib = _lib.load()
    sc = G.Scan(ZL=16, pitch=0.9375, rotations=40, XN=8, YN=8, ZN=8)  # 39360 fan views > 32768
    geom = _lib.BpGeom.from_dict(sc.bp_geom())
    x = torch.zeros(16, device=cuda)
    st = lib.hr_bp_plain_noalloc(x.data_ptr(), x.data_ptr(), x.data_ptr(), ctypes.byref(geom), 0)
    assert st == 1
    assert b"32768" in lib.hr_last_error()
