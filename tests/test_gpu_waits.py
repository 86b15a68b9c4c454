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


def test_cnn_wait_runs_out_and_device_stays_usable(cuda):
    """The learned correction's conv kernels: every CTA leaves one of its input
    rows unloaded, so its MMA issuer's wait runs out; forward and training calls
    return, hr_cnn_check reports (and clears) the timeout, and normal calls
    afterwards reproduce the results of a run before the stall bit for bit."""
    from analyticalreconbigpatient_b200 import learned as L
    from analyticalreconbigpatient_b200.geometry import MU_WATER

    lib = _lib.load()
    rng = np.random.default_rng(5)
    B, H, W = 2, 24, 256
    u = np.zeros((B, H, W, 16), dtype=np.float32)
    u[..., :5] = rng.standard_normal((B, H, W, 5)).astype(np.float32) * 0.3
    xb = torch.from_numpy(u).to(cuda).to(torch.bfloat16).view(torch.int16).contiguous()
    base = torch.full((B, H, W), MU_WATER, device=cuda)
    from oracle import cnn_oracle as C

    net = L.Corrector(C.init_params(4, zero_last=False), device=cuda)  # a non-zero residual
    ref = net.forward(xb, base).clone()
    torch.cuda.synchronize()
    net.check()
    _lib.check(lib.hr_cnn_test_stall(net._net, 3, 2000))
    t = time.perf_counter()
    net.forward(xb, base)
    torch.cuda.synchronize()
    elapsed = time.perf_counter() - t
    assert lib.hr_cnn_check(net._net) == _lib.HR_ERR_CUDA
    assert b"timed out" in lib.hr_last_error()
    assert elapsed < 60.0, elapsed
    assert lib.hr_cnn_check(net._net) == 0
    _lib.check(lib.hr_cnn_test_stall(net._net, -1, 0))
    for _ in range(2):
        again = net.forward(xb, base).clone()
        torch.cuda.synchronize()
        net.check()
        assert torch.equal(again, ref)
