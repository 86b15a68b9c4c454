"""Generates the golden vectors under tests/golden/ from the reference itself.

* rebin_*.npz, bp_*.npz: the reference's own CPU functions
  (ParallelRebinningCBCurve_CPU<float>, ParallelFDKHelical3DWeightingCPU)
  compiled from its sources by oracle/Makefile (oracle/_ref/libref_cpu.so).
  Run where the reference sources exist:  python tests/golden/make_golden.py
* filter_*.npz: the reference's own cuFFT filter (src/filtering.cu, built
  unmodified into oracle/_ref/libref_gpu.so); needs a CUDA device:
  python tests/golden/make_golden.py --filter [--out DIR]

Inputs are seeded and stored with the outputs so that a check does not depend
on regenerating them bit-for-bit elsewhere.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from analyticalreconbigpatient_b200 import geometry as G  # noqa: E402


def small_scan(**kw) -> G.Scan:
    base = dict(YL=64, det_pitch=1.0239 * 888 / 64, ZL=4, N_2pi=48, pitch=0.9375, rotations=2.5, XN=16, YN=16, ZN=6,
                dx=15.0, dy=15.0, dz=1.2, delta=4)
    base.update(kw)
    return G.Scan(**base)


CASES = {
    # name: scan kwargs
    "centred": dict(),
    "offcentre": dict(iso_channel=33.25, beta_start=1.3, ZL=6, pitch=0.5),
    "wide": dict(YL=72, det_pitch=1.0239 * 888 / 72, ZL=4, N_2pi=40, rotations=3, XN=12, YN=20, ZN=8, dx=18.0,
                 dy=14.0, dz=2.0, z_centre=3.0),
}


def make_cpu() -> None:
    for name, kw in CASES.items():
        sc = small_scan(**kw)
        rng = np.random.default_rng(len(name) * 7919 + 17)
        ra = sc.rebin_args()
        proj = rng.random((ra["ViewN"], ra["YL"], ra["ZL"]), dtype=np.float32)
        out = oracle.ref_rebin_f32(proj, **ra)
        np.savez_compressed(os.path.join(HERE, f"rebin_{name}.npz"), proj=proj, out=out,
                            args=np.array([ra[k] for k in ("YLC", "dYA", "DeltaTheta", "PLC", "DeltaT", "DeltaFai",
                                                           "SO")], dtype=np.float32),
                            sizes=np.array([ra["YL"], ra["ZL"], ra["ViewN"]], dtype=np.int64))
        g = sc.bp_geom()
        w = oracle.weight_table(sc.N_2pi, sc.HSCoef, sc.delta)
        fp = rng.standard_normal((g["PN"], g["ZL"], g["YL"])).astype(np.float32).astype(np.float64)
        vol = oracle.ref_bp_f64(fp, w, g)
        np.savez_compressed(os.path.join(HERE, f"bp_{name}.npz"), fp=fp.astype(np.float32), w=w, vol=vol,
                            geom_keys=np.array(oracle.BP_KEYS), geom=np.array([g[k] for k in oracle.BP_KEYS],
                                                                               dtype=np.float64))
        print("wrote", name, "rebin", proj.shape, "bp", vol.shape)


def make_filter(out_dir: str = HERE) -> None:
    import ctypes  # noqa: F401

    L = oracle.ref_gpu()
    for name, kw in CASES.items():
        sc = small_scan(**kw)
        fa = sc.filter_args()
        rng = np.random.default_rng(len(name) * 104729 + 3)
        proj = rng.standard_normal((fa["ViewN"], fa["ZL"], fa["YL"])).astype(np.float32)
        out = np.zeros_like(proj)
        L.ref_gpu_filtering(out.ctypes.data, proj.ctypes.data, fa["YL"], fa["ZL"], fa["ViewN"], fa["PLC"], fa["ZLC"],
                            fa["dYL"], fa["dZL"], fa["SO"])
        np.savez_compressed(os.path.join(out_dir, f"filter_{name}.npz"), proj=proj, out=out,
                            args=np.array([fa[k] for k in ("PLC", "ZLC", "dYL", "dZL", "SO")], dtype=np.float32),
                            sizes=np.array([fa["YL"], fa["ZL"], fa["ViewN"]], dtype=np.int64))
        print("wrote filter", name, proj.shape, float(np.abs(out).max()))


if __name__ == "__main__":
    if "--filter" in sys.argv:
        # --out DIR: where to write (a GPU host may only return some folders)
        make_filter(sys.argv[sys.argv.index("--out") + 1] if "--out" in sys.argv else HERE)
    else:
        make_cpu()
