"""The allocation-free backprojection entry (hr_bp_plain_noalloc).

It exists for callers that cannot call cudaMalloc: pipelines that must not
allocate once running (cudaMalloc and cudaFree synchronise the device), hosts
whose pooling allocator owns all device memory, services held to a fixed
memory budget. Its scratch (the per-view table) is a fixed array inside the
library, filled from the same host-computed table as the plan's. The tests call
it through the C ABI twice in a row, on two different scans, and on a scan of
nearly the array's maximum number of views, and require the volume to equal the
plan-based plain entry's (hr_bp_execute) bit for bit (the plain form's index
selection is exact, so no tolerance is needed). This file sorts last so that a
run stopping at the first failure has run every other test first.
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


def _noalloc_result(geom, w, fp, shape, dev):
    lib = _lib.load()
    d_w = torch.tensor(w.astype(np.float32), device=dev)
    vol = torch.full(shape, float("nan"), dtype=torch.float32, device=dev)
    _lib.check(lib.hr_bp_plain_noalloc(vol.data_ptr(), fp.data_ptr(), d_w.data_ptr(), ctypes.byref(geom), 0))
    torch.cuda.synchronize()
    return vol.cpu().numpy()


def test_no_alloc_entry_matches_plan_entry_on_two_calls(cuda):
    scans = [G.Scan(ZL=16, pitch=0.9375, rotations=3, XN=48, YN=40, ZN=20, dx=5.0, dy=5.5, dz=1.0),
             G.Scan(ZL=8, pitch=1.2, rotations=2.5, XN=32, YN=36, ZN=13, dx=6.0, dy=6.0, dz=2.0, beta_start=40.0,
                    delta=40)]
    for seed, sc in enumerate(scans):
        geom, w, fp = _case(sc, seed, cuda)
        shape = (sc.YN, sc.XN, sc.ZN)
        mine = _noalloc_result(geom, w, fp, shape, cuda)
        ref = _plan_result(geom, w, fp, shape, cuda)
        assert np.isfinite(mine).all()
        assert rel_l2(mine, ref) < PLAIN_TOL, seed
        assert np.array_equal(mine, ref), (seed, int(np.sum(mine != ref)))


def test_no_alloc_entry_bit_exact_on_many_views(cuda):
    # 30 rotations: 29,520 fan views (near the 32,768-view limit), source angles
    # up to ~95 rad, slices spread over the whole helix
    sc = G.Scan(ZL=16, pitch=0.9375, rotations=30, XN=24, YN=24, ZN=28, dx=12.0, dy=12.0, dz=9.5)
    geom, w, fp = _case(sc, 7, cuda)
    assert sc.PN > 29000
    shape = (sc.YN, sc.XN, sc.ZN)
    mine = _noalloc_result(geom, w, fp, shape, cuda)
    ref = _plan_result(geom, w, fp, shape, cuda)
    assert np.count_nonzero(ref) > ref.size // 2
    assert np.array_equal(mine, ref), int(np.sum(mine != ref))


def test_no_alloc_entry_rejects_too_many_views(cuda):
    lib = _lib.load()
    sc = G.Scan(ZL=16, pitch=0.9375, rotations=40, XN=8, YN=8, ZN=8)  # 39360 fan views > 32768
    geom = _lib.BpGeom.from_dict(sc.bp_geom())
    x = torch.zeros(16, device=cuda)
    st = lib.hr_bp_plain_noalloc(x.data_ptr(), x.data_ptr(), x.data_ptr(), ctypes.byref(geom), 0)
    assert st == 1
    assert b"32768" in lib.hr_last_error()
