"""GPU end-to-end tests of the device-resident pipeline (rebin -> filter -> BP)
against the CPU reference path and the FP64 oracle, plus known-answer tests.

"Reference path" = the reference CPU's own arithmetic: float rebinning
(bit-identical to ParallelRebinningCBCurve_CPU<float>), the MATLAB filter in
FP64, the double backprojection (bit-identical to
ParallelFDKHelical3DWeightingCPU). "FP64 oracle" = the same chain with an FP64
rebinning.
"""
import os

import numpy as np
import pytest

import oracle
from analyticalreconbigpatient_b200 import _lib, geometry as G, phantom as P
from conftest import rel_l2

pytestmark = pytest.mark.gpu

PLAIN_TOL = 1e-5


def reference_chain(scan, fan, vox, fp64_rebin=False):
    ra = scan.rebin_args()
    reb = oracle.rebin_f64(fan, **ra) if fp64_rebin else oracle.rebin_f32(fan, **ra)
    rows = np.ascontiguousarray(reb.transpose(0, 2, 1)[scan.crop_front: scan.views - scan.crop_back],
                                dtype=np.float64)
    filt = oracle.filter_f64(rows, **scan.filter_args())
    w = oracle.weight_table(scan.N_2pi, scan.HSCoef, scan.delta)
    return oracle.bp_f64(filt, w, scan.bp_geom(), vox=vox)


def run_gpu(scan, objects, form=_lib.HR_FORM_PLAIN):
    import torch

    from analyticalreconbigpatient_b200.pipeline import HelicalRecon, project

    fan = project(scan, objects)
    rec = HelicalRecon(scan, form=form)
    vol = rec.run(fan)
    torch.cuda.synchronize()
    out = vol.cpu().numpy()
    fan_h = fan.cpu().numpy()
    rec.close()
    return fan_h, out


def pick_voxels(scan, n, seed=0, full_slices=()):
    rng = np.random.default_rng(seed)
    v = set(rng.choice(scan.XN * scan.YN * scan.ZN, size=n, replace=False).tolist())
    for zi in full_slices:
        for yi in range(scan.YN):
            for xi in range(0, scan.XN, 2):
                v.add((yi * scan.XN + xi) * scan.ZN + zi)
    return np.array(sorted(v), dtype=np.int64)


def test_small_config_plain_vs_reference_path_and_fp64_oracle(cuda):
    sc = G.config("small")
    fan, vol = run_gpu(sc, P.shepp_logan())
    vox = pick_voxels(sc, 3000, full_slices=(0, sc.ZN // 2, sc.ZN - 1))
    ref = reference_chain(sc, fan, vox)
    mine = vol.ravel()[vox]
    assert rel_l2(mine, ref) < PLAIN_TOL
    f64 = reference_chain(sc, fan, vox, fp64_rebin=True)
    assert rel_l2(mine, f64) < 5 * PLAIN_TOL


def test_water_cylinder_known_answer(cuda):
    sc = G.Scan(ZL=16, pitch=0.9375, rotations=3, XN=96, YN=96, ZN=16, dx=3.0, dy=3.0, dz=1.0)
    fan, vol = run_gpu(sc, P.water_cylinder(radius=110.0, half_length=4000.0))
    core = vol[38:58, 38:58, :]
    # flat interior
    assert core.std() / core.mean() < 2e-3
    # the reference's 3D weight (conjugate offset of 0.5 mm instead of h/2)
    # scales the level; the GPU level equals the reference path's
    vox = pick_voxels(sc, 400, seed=1)
    ref = reference_chain(sc, fan, vox)
    assert rel_l2(vol.ravel()[vox], ref) < PLAIN_TOL
    ratio = core.mean() / G.MU_WATER
    assert 0.85 < ratio < 0.95
    # outside the body it is air
    assert abs(vol[2:6, 2:6, :]).mean() < 0.05 * core.mean()


def test_offcentre_sphere_lands_at_its_position(cuda):
    sc = G.Scan(ZL=16, pitch=0.9375, rotations=3, XN=64, YN=64, ZN=20, dx=3.0, dy=3.0, dz=1.0)
    cx, cy, cz, r = 40.0, -30.0, 2.0, 5.0
    sphere = np.array([[0, cx, cy, cz, r, r, r, 1, 0, 0, 0, 1, 0, 0, 0, 1, 0.02]])
    water = P.water_cylinder(radius=110.0, half_length=4000.0)
    _, v1 = run_gpu(sc, np.concatenate([water, sphere]))
    _, v0 = run_gpu(sc, water)
    d = v1 - v0
    g = sc.bp_geom()
    yi, xi, zi = np.meshgrid(np.arange(sc.YN), np.arange(sc.XN), np.arange(sc.ZN), indexing="ij")
    x, y, z = (xi - g["XNC"]) * g["dx"], (yi - g["YNC"]) * g["dy"], (zi - g["ZNC"]) * g["dz"]
    m = np.where(d > 0.5 * d.max(), d, 0.0)
    c = [(m * a).sum() / m.sum() for a in (x, y, z)]
    assert abs(c[0] - cx) < 0.5 * sc.dx and abs(c[1] - cy) < 0.5 * sc.dy and abs(c[2] - cz) < 0.5 * sc.dz, c


def test_out_of_memory_is_reported_and_the_device_stays_usable(cuda):
    import torch
    from analyticalreconbigpatient_b200.pipeline import HelicalRecon

    # 1200 rotations of the 888 x 64 detector: the rebinned buffer alone would take 268 GB
    huge = G.Scan(ZL=64, pitch=0.984, rotations=1200, XN=64, YN=64, ZN=4, dx=4.0, dy=4.0, dz=1.0)
    with pytest.raises(_lib.HelixError) as exc:
        HelicalRecon(huge, form=_lib.HR_FORM_PLAIN)
    assert exc.value.status == _lib.HR_ERR_OUT_OF_MEMORY, exc.value
    sc = G.tiny()
    rec = HelicalRecon(sc)
    fan = torch.zeros((sc.views, sc.YL, sc.ZL), device=cuda)
    vol = rec.run(fan)
    torch.cuda.synchronize()
    assert float(vol.abs().max()) == 0.0
    rec.close()


def test_log_variable_prints_plan_choices(cuda):
    import subprocess
    import sys

    code = ("from analyticalreconbigpatient_b200 import _lib, geometry as G\n"
            "from analyticalreconbigpatient_b200.pipeline import HelicalRecon\n"
            "HelicalRecon(G.tiny(YL=200, ZL=8), form=_lib.HR_FORM_FAST).close()\n")
    env = dict(os.environ, HELIXRECON_LOG="1")
    r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert "[helixrecon] recon plan:" in r.stderr and "autotuned" in r.stderr, r.stderr
    env["HELIXRECON_LOG"] = "0"
    r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=300)
    assert "[helixrecon]" not in r.stderr
