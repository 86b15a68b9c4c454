"""GPU tests of the tensor-core (tcgen05) split-BF16 Toeplitz ramp filter.

Its output is BF16 channel pairs; the check is against the FP64 oracle filter
(the reference's math, pinned to the reference's own cuFFT output): the error
must be the BF16 storage rounding (2^-9 relative) and nothing more.
"""
import ctypes

import numpy as np
import pytest
import torch

import oracle
from analyticalreconbigpatient_b200 import _lib, geometry as G
from conftest import rel_l2

pytestmark = pytest.mark.gpu


def run_tc(fa, data, layout, view0=0):
    lib = _lib.load()
    plan = ctypes.c_void_p()
    _lib.check(lib.hr_filter_tc_plan_create(ctypes.byref(plan), fa["YL"], fa["ZL"], fa["ViewN"], fa["PLC"],
                                            fa["ZLC"], fa["dYL"], fa["dZL"], fa["SO"]))
    dev = torch.device("cuda", 0)
    x = torch.tensor(data, device=dev)
    pairs = torch.full((fa["ViewN"], fa["ZL"], fa["YL"]), -1, dtype=torch.int32, device=dev)
    _lib.check(lib.hr_filter_tc_execute(plan, pairs.data_ptr(), x.data_ptr(), layout, view0, 0))
    torch.cuda.synchronize()
    _lib.check(lib.hr_filter_tc_check(plan))
    lib.hr_filter_tc_plan_destroy(plan)
    w = pairs.cpu().numpy().view(np.uint32)
    lo = ((w & 0xFFFF) << 16).view(np.float32)
    hi = (w & 0xFFFF0000).view(np.float32)
    return lo, hi


def bf16_round(x):
    return torch.tensor(x, dtype=torch.float32).to(torch.bfloat16).to(torch.float32).numpy()


@pytest.mark.parametrize("YL,ZL,views", [(888, 64, 6), (90, 5, 37), (300, 16, 9), (888, 16, 12)])
def test_tc_filter_matches_fp64_oracle(cuda, YL, ZL, views):
    sc = G.tiny(YL=YL, ZL=ZL)
    fa = dict(sc.filter_args(), ViewN=views)
    rng = np.random.default_rng(YL + ZL)
    rows = rng.standard_normal((views, ZL, YL)).astype(np.float32)
    lo, hi = run_tc(fa, rows, _lib.HR_LAYOUT_ROWS)
    ref = oracle.filter_f64(rows.astype(np.float64), **fa)
    # pairs: high half of word j is the low half of word j+1
    np.testing.assert_array_equal(hi[..., :-1], lo[..., 1:])
    assert np.all(hi[..., -1] == 0)
    err = rel_l2(lo, ref)
    assert err < 2.5e-3, err  # BF16 storage: 2^-9 relative rounding
    # the value before storage is ~1e-5 accurate, so it rounds to bf16(ref) almost always
    same = np.mean(lo == bf16_round(ref))
    assert same > 0.97, same


def test_tc_filter_reads_the_rebinning_layout_with_a_view_offset(cuda):
    sc = G.tiny(YL=888, ZL=64, det_pitch=1.0239)
    fa = dict(sc.filter_args(), ViewN=5)
    rng = np.random.default_rng(7)
    reb = rng.standard_normal((9, 888, 64)).astype(np.float32)  # [views][YL][ZL]
    lo, _ = run_tc(fa, reb, _lib.HR_LAYOUT_REBIN, view0=3)
    rows = np.ascontiguousarray(reb[3:8].transpose(0, 2, 1)).astype(np.float64)
    ref = oracle.filter_f64(rows, **fa)
    assert rel_l2(lo, ref) < 2.5e-3
