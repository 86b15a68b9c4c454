"""GPU parity of each stage through the C ABI against the reference's outputs
(golden vectors from its compiled code) and the oracle.

Tolerances: rebinning is bit-exact to the reference CPU path; the FP32 filter
and backprojection must agree with the FP64 references within 1e-5 relative
L2 (plain form), the FP64 backprojection within 1e-12.
"""
import ctypes
import glob
import os

import numpy as np
import pytest

import oracle
from analyticalreconbigpatient_b200 import _lib, api, geometry as G, phantom as P
from conftest import rel_l2
from test_oracle import GOLDEN, load_bp, load_rebin

pytestmark = pytest.mark.gpu

PLAIN_TOL = 1e-5


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "rebin_*.npz"))), ids=os.path.basename)
def test_rebin_bit_exact_to_reference_golden(cuda, path):
    proj, out, a = load_rebin(path)
    mine = np.empty_like(out)
    _lib.load().ParallelRebinningCBCurve_GPU(mine.ctypes.data, proj.ctypes.data, a["YL"], a["ZL"], a["ViewN"],
                                             a["YLC"], a["dYA"], a["DeltaTheta"], a["PLC"], a["DeltaT"],
                                             a["DeltaFai"], a["SO"])
    np.testing.assert_array_equal(mine.view(np.uint32), out.view(np.uint32))


@pytest.mark.parametrize("ZL", [16, 6, 1])
def test_rebin_bit_exact_small_config_and_odd_rows(cuda, ZL):
    sc = G.config("small") if ZL == 16 else G.tiny(ZL=ZL, YL=200, det_pitch=1.0239 * 888 / 200, iso_channel=100.75)
    ra = sc.rebin_args()
    rng = np.random.default_rng(ZL)
    proj = rng.random((ra["ViewN"], ra["YL"], ra["ZL"]), dtype=np.float32)
    mine = api.ParallelRebinningCBCurve(proj, ra["YL"], ra["ZL"], ra["ViewN"], ra["YLC"] + 1, ra["dYA"],
                                        ra["DeltaTheta"], ra["PLC"] + 1, ra["DeltaT"], ra["DeltaFai"], ra["SO"], 1)
    ref = oracle.rebin_f32(proj, **ra)
    np.testing.assert_array_equal(mine.view(np.uint32), ref.view(np.uint32))


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "filter_*.npz"))), ids=os.path.basename)
def test_filter_vs_reference_cufft_golden(cuda, path):
    d = np.load(path)
    YL, ZL, ViewN = (int(v) for v in d["sizes"])
    PLC, ZLC, dYL, dZL, SO = (float(v) for v in d["args"])
    proj = d["proj"]  # keep the array alive across the C call
    mine = np.empty_like(proj)
    _lib.load().filtering(mine.ctypes.data, proj.ctypes.data, YL, ZL, ViewN, PLC, ZLC, dYL, dZL, SO)
    assert rel_l2(mine, d["out"]) < PLAIN_TOL


@pytest.mark.parametrize("cfg", ["tiny", "small"])
def test_filter_vs_fp64_oracle(cuda, cfg):
    sc = G.tiny(YL=150, ZL=7) if cfg == "tiny" else G.config("small")
    fa = sc.filter_args()
    rng = np.random.default_rng(1)
    nv = min(fa["ViewN"], 300)
    p = rng.standard_normal((nv, fa["ZL"], fa["YL"])).astype(np.float32)
    mine = api.reWeigAdFiltr_GPU(p, fa["PLC"], fa["ZLC"], fa["dYL"], fa["dZL"], fa["SO"])
    ref = oracle.filter_f64(p.astype(np.float64), fa["YL"], fa["ZL"], nv, fa["PLC"], fa["ZLC"], fa["dYL"], fa["dZL"],
                            fa["SO"])
    assert rel_l2(mine, ref) < PLAIN_TOL
    # every row individually, too
    err = np.linalg.norm(mine - ref, axis=-1) / np.maximum(np.linalg.norm(ref, axis=-1), 1e-30)
    assert err.max() < 1e-5


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "bp_*.npz"))), ids=os.path.basename)
def test_bp_float_entry_vs_reference_golden(cuda, path):
    fp, w, g, vol = load_bp(path)
    mine = api.ParallekFDKHelical3DWeighting_GPU_float(fp, w.astype(np.float32), g)
    # the float entry receives float32 geometry; compare with the reference run on the same rounded values
    g32 = {k: (int(v) if isinstance(v, int) else float(np.float32(v))) for k, v in g.items()}
    ref = oracle.ref_bp_f64(fp.astype(np.float64), w.astype(np.float32).astype(np.float64), g32) \
        if oracle.ref_available() else oracle.bp_f64(fp.astype(np.float64), w.astype(np.float32).astype(np.float64), g32)
    assert rel_l2(mine.ravel(), ref) < PLAIN_TOL
    assert np.abs(mine.ravel() - ref).max() < 1e-4 * np.abs(ref).max()
    assert np.array_equal(mine.ravel() == 0, ref == 0)


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "bp_*.npz"))), ids=os.path.basename)
def test_bp_double_entry_vs_reference_golden(cuda, path):
    fp, w, g, vol = load_bp(path)
    mine = api.ParallekFDKHelical3DWeighting_GPU_double(fp.astype(np.float64), w, g)
    np.testing.assert_allclose(mine.ravel(), vol, rtol=1e-11, atol=1e-12 * np.abs(vol).max())


def test_bp_high_level_entry_both_branches(cuda):
    # ParallelFDKHelical3DWeighting derives dx=dy=dz=2 ObjR/N and w itself
    rng = np.random.default_rng(4)
    SO, DO, YL, ZL, N_2pi, PN = 541.0, 408.0, 60, 5, 60, 150
    DecWidth, DecHeigh = 600.0, 5 * 1.0963
    h, BetaS, ObjR, XN, YN, ZN = 9.0, -4.0, 120.0, 12, 10, 14
    XNC, YNC, ZNC, delta, HSCoef, k1 = 5.5, 4.5, 6.0, 5, 0.68, 2.5
    fp = rng.standard_normal((PN, ZL, YL))
    args = (SO, DO, YL, ZL, DecWidth, DecHeigh, (YL - 1) / 2, (ZL - 1) / 2, h, BetaS, PN, N_2pi, ObjR, XN, YN, ZN,
            XNC, YNC, ZNC, delta, HSCoef, k1)
    ref = np.zeros(XN * YN * ZN)
    if not oracle.ref_available():
        pytest.skip("compiled reference not present")
    oracle.ref().ref_ParallelFDKHelical3DWeighting(ref.ctypes.data, fp.ctypes.data, *args, 0)
    assert np.count_nonzero(ref) > 100
    for use_gpu, tol in ((0, 1e-11), (1, PLAIN_TOL)):
        mine = np.zeros(XN * YN * ZN)
        _lib.load().ParallelFDKHelical3DWeighting(mine.ctypes.data, fp.ctypes.data, *args, use_gpu)
        assert rel_l2(mine, ref) < tol, use_gpu


def test_scan_geom_mex_mirror(cuda):
    sc = G.tiny(delta=8, XN=12, YN=10, ZN=12, dx=0.5, dy=0.6, dz=0.5)
    g = sc.bp_geom()
    rng = np.random.default_rng(9)
    fp = rng.standard_normal((g["PN"], g["ZL"], g["YL"]))
    ObjR = sc.dx * sc.XN / 2
    sc2 = G.tiny(delta=8, XN=sc.XN, YN=sc.YN, ZN=sc.ZN, dx=ObjR * 2 / sc.XN, dy=ObjR * 2 / sc.YN,
                 dz=ObjR * 2 / sc.ZN)
    g2 = sc2.bp_geom()
    scan_geom = {"ScDet": [sc.SO, sc.DO, sc.YL, sc.ZL, sc.DecWidth, sc.DecHeigh, 0.0, sc.ZLC1, sc.h_norm],
                 "Proj": [g["BetaS"], 0.0, g["PN"], sc.N_2pi],
                 "Obj": [ObjR, sc.XN, sc.YN, sc.ZN, g2["XNC"] + 1, g2["YNC"] + 1, g2["ZNC"] + 1],
                 "Rec": [sc.delta, sc.HSCoef, sc.mk1]}
    ct = np.zeros(sc.XN * sc.YN * sc.ZN)
    api.Parallel_FDK_Helical_3DWeighting(scan_geom, fp, ct, 0)
    w = oracle.weight_table(sc.N_2pi, sc.HSCoef, sc.delta)
    ref = oracle.bp_f64(fp, w, g2)
    assert np.count_nonzero(ref) > ref.size // 2
    np.testing.assert_allclose(ct, ref, rtol=1e-10, atol=1e-12 * np.abs(ref).max())


def test_projector_gpu_matches_cpu_oracle(cuda):
    import torch

    from analyticalreconbigpatient_b200.pipeline import project

    sc = G.tiny(YL=120, ZL=8, rotations=1.5)
    obj = np.concatenate([P.random_ellipsoids(3, 8, (-5.0, 5.0), body=(150.0, 110.0), semi_axes=(10, 60)),
                          P.shepp_logan(fov=300.0)])
    gpu = project(sc, obj).cpu().numpy()
    cpu = oracle.project_ellipsoids(obj, **P.projector_args(sc))
    np.testing.assert_allclose(gpu, cpu, rtol=2e-6, atol=1e-6 * np.abs(cpu).max())


def test_errors_are_raised_not_swallowed(cuda):
    with pytest.raises(_lib.HelixError):
        api.reWeigAdFiltr_GPU(np.zeros((2, 2, 3000), np.float32), 0, 0, 1, 1, 541)
    with pytest.raises(ValueError):
        api.ParallelRebinningCBCurve(np.zeros(10, np.float32), 8, 4, 10, 1, 0.01, 0.1, 1, 1, 0.1, 541, 1)


def test_filter_refuses_overlapping_buffers(cuda):
    import torch

    sc = G.tiny(YL=64, ZL=4)
    fa = sc.filter_args()
    plan = ctypes.c_void_p()
    lib = _lib.load()
    _lib.check(lib.hr_filter_plan_create(ctypes.byref(plan), fa["YL"], fa["ZL"], 10, fa["PLC"], fa["ZLC"], fa["dYL"],
                                         fa["dZL"], fa["SO"]))
    x = torch.zeros((11, fa["ZL"], fa["YL"]), device=cuda)
    assert lib.hr_filter_execute(plan, x.data_ptr(), x.data_ptr(), 0, 0, 0) == 1
    assert lib.hr_filter_execute(plan, x[1:].data_ptr(), x.data_ptr(), 0, 0, 0) == 1
    y = torch.zeros_like(x)
    assert lib.hr_filter_execute(plan, y.data_ptr(), x.data_ptr(), 0, 1, 0) == 0
    torch.cuda.synchronize()
    lib.hr_filter_plan_destroy(plan)


@pytest.mark.parametrize("kernel", ["0", "1"])
@pytest.mark.parametrize("ZL,YL", [(16, 888), (7, 888), (8, 1000)])
def test_filter_2048_both_layouts_vs_fp64_oracle(cuda, ZL, YL, kernel, monkeypatch):
    """888 channels transform with 2048 points (the register-resident kernels:
    two warps per row pair, or one with HELIXRECON_FILTER2048=1): both input
    layouts against the FP64 oracle, every row within 1e-5 (odd ZL: row pairs
    that straddle two views; 1000 channels: no samples pruned), and the two
    layouts give the same bits."""
    import torch

    monkeypatch.setenv("HELIXRECON_FILTER2048", kernel)
    sc = G.Scan(ZL=ZL, YL=YL, pitch=0.9375)
    fa = sc.filter_args()
    nv = 37
    rng = np.random.default_rng(7)
    rows = rng.standard_normal((nv + 3, ZL, sc.YL)).astype(np.float32)  # [v][ZL][YL]
    dev = torch.device("cuda", 0)
    lib = _lib.load()
    fplan = ctypes.c_void_p()
    _lib.check(lib.hr_filter_plan_create(ctypes.byref(fplan), fa["YL"], ZL, nv, fa["PLC"], fa["ZLC"], fa["dYL"],
                                         fa["dZL"], fa["SO"]))
    d_rows = torch.tensor(rows, device=dev)
    d_reb = torch.tensor(np.ascontiguousarray(rows.transpose(0, 2, 1)), device=dev)  # [v][YL][ZL]
    out_r = torch.empty((nv, ZL, sc.YL), device=dev)
    out_b = torch.empty_like(out_r)
    _lib.check(lib.hr_filter_execute(fplan, out_r.data_ptr(), d_rows.data_ptr(), _lib.HR_LAYOUT_ROWS, 3, 0))
    _lib.check(lib.hr_filter_execute(fplan, out_b.data_ptr(), d_reb.data_ptr(), _lib.HR_LAYOUT_REBIN, 3, 0))
    torch.cuda.synchronize()
    lib.hr_filter_plan_destroy(fplan)
    got_r, got_b = out_r.cpu().numpy(), out_b.cpu().numpy()
    assert np.array_equal(got_r, got_b)
    ref = oracle.filter_f64(rows[3:].astype(np.float64), sc.YL, ZL, nv, fa["PLC"], fa["ZLC"], fa["dYL"], fa["dZL"],
                            fa["SO"])
    err = np.linalg.norm(got_r - ref, axis=-1) / np.maximum(np.linalg.norm(ref, axis=-1), 1e-30)
    assert err.max() < 1e-5, err.max()

