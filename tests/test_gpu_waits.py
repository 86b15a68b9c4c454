"""Bounded device waits: a tensor-core pipeline whose wait runs out returns
with an error flag instead of hanging, and the device stays usable.

The tensor-core filter's TMA producer is told (hr_filter_tc_test_stall) to
leave one K block unloaded, so the MMA issuer's wait on that stage's barrier
can only run out (a barrier nothing completes). No fault, trap or endless
loop is involved: every wait has a poll limit. The test checks that the
execution returns, that hr_filter_tc_check reports the timeout (and clears
it), that no CTA wrote its tile, and that the next normal executions on the
same device -- which allocate tensor memory on every SM again, so aborted CTAs
must have freed theirs -- give the bit-identical result of a run before it.
The reference checks nothing (src/reWeigAdFiltr_GPU.cpp:41-46 calls exit).
"""
import ctypes
import time

import numpy as np
import pytest
import torch

from analyticalreconbigpatient_b200 import _lib, geometry as G

pytestmark = pytest.mark.gpu


def test_filter_tc_wait_runs_out_and_device_stays_usable(cuda):
    lib = _lib.load()
    sc = G.Scan(ZL=16, pitch=0.9375)
    fa = sc.filter_args()
    nv = 24  # 384 rows: 3 row tiles x 8 column tiles, 14 K blocks of 64 channels
    rng = np.random.default_rng(11)
    rows = torch.tensor(rng.standard_normal((nv, sc.ZL, sc.YL)).astype(np.float32), device=cuda)
    plan = ctypes.c_void_p()
    _lib.check(lib.hr_filter_tc_plan_create(ctypes.byref(plan), sc.YL, sc.ZL, nv, fa["PLC"], fa["ZLC"], fa["dYL"],
                                            fa["dZL"], fa["SO"]))
    try:
        ref = torch.empty((nv, sc.ZL, sc.YL), dtype=torch.int32, device=cuda)
        _lib.check(lib.hr_filter_tc_execute(plan, ref.data_ptr(), rows.data_ptr(), _lib.HR_LAYOUT_ROWS, 0, 0))
        torch.cuda.synchronize()
        _lib.check(lib.hr_filter_tc_check(plan))
        # the stalled execution: every CTA's wait on K block 5 runs out
        _lib.check(lib.hr_filter_tc_test_stall(plan, 5, 2000))
        out = torch.full_like(ref, -1)
        t = time.perf_counter()
        _lib.check(lib.hr_filter_tc_execute(plan, out.data_ptr(), rows.data_ptr(), _lib.HR_LAYOUT_ROWS, 0, 0))
        torch.cuda.synchronize()  # returns: the kernel ended by itself
        elapsed = time.perf_counter() - t
        st = lib.hr_filter_tc_check(plan)
        assert st == _lib.HR_ERR_CUDA, st
        assert b"timed out" in lib.hr_last_error()
        assert elapsed < 30.0, elapsed
        assert bool((out == -1).all()), "an aborted CTA wrote its tile"
        assert lib.hr_filter_tc_check(plan) == 0  # the check cleared the flag
        # normal operation again, twice, on the same device and plan
        _lib.check(lib.hr_filter_tc_test_stall(plan, -1, 0))
        for _ in range(2):
            again = torch.full_like(ref, -1)
            _lib.check(lib.hr_filter_tc_execute(plan, again.data_ptr(), rows.data_ptr(), _lib.HR_LAYOUT_ROWS, 0, 0))
            torch.cuda.synchronize()
            _lib.check(lib.hr_filter_tc_check(plan))
            assert torch.equal(again, ref)
    finally:
        lib.hr_filter_tc_check(plan)
        lib.hr_filter_tc_plan_destroy(plan)
