"""One scan split by z slabs between ranks, on CPU ranks (gloo, world size 2).

The multi-GPU path of the big-patient workload gives each rank a part of the
scan's z slabs (hr_slab_plan_create_part); a rank reconstructs its slabs from
only its own fan windows and writes only their slices, with no exchange. The
reference's only way to split a long scan is its sequential segment loop
(src/analyticalRecon.m:20-25), whose segments are summed into one volume.

Here each rank takes its slab windows from the library's own window arithmetic
(hr_slab_windows, the same code the GPU plans use; host arithmetic, no GPU)
and reconstructs its slabs through the FP64 oracle from nothing but the fan
views of each window. The union of both ranks' slabs, gathered over gloo, must
equal the single-rank whole-scan oracle reconstruction: a window too short, a
margin too small or a wrong view offset would change the result.
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from analyticalreconbigpatient_b200 import _lib, geometry as G

SLAB = 4


def toy_scan():
    sc = G.tiny(rotations=8, ZN=1, dz=1.5)
    return G.replace(sc, ZN=sc.fully_sampled_slices() + 2)  # two partially sampled end slices


def toy_fan(sc):
    import oracle
    from analyticalreconbigpatient_b200 import phantom as P

    zlo = sc.h * sc.BetaS / (2 * np.pi)
    zhi = sc.h * (sc.BetaS + sc.views * sc.dBeta) / (2 * np.pi)
    objs = P.random_ellipsoids(77, 12, (zlo, zhi), body=(130.0, 100.0), semi_axes=(10, 60))
    ra = sc.rebin_args()
    return oracle.project_ellipsoids(objs, sc.YL, sc.ZL, sc.views, sc.SO, sc.SD, sc.dYA, sc.YLC1 - 1.0, sc.dZL,
                                     sc.ZLC1 - 1.0, sc.BetaS, sc.dBeta, sc.h, nthreads=2), ra


def slab_recon(sc, fan_window, win):
    """FP64 oracle reconstruction of one slab from its fan window only."""
    import oracle

    ra = dict(sc.rebin_args(), ViewN=win["fan_views"])
    reb = oracle.rebin_f64(fan_window, **ra, nthreads=2)
    m = sc.crop_front  # the margin on both sides of the backprojection window
    rows = np.ascontiguousarray(reb[m: m + win["bp_views"]].transpose(0, 2, 1))
    filt = oracle.filter_f64(rows, **dict(sc.filter_args(), ViewN=win["bp_views"]), nthreads=2)
    g = sc.bp_geom()
    gs = dict(g, ZN=win["n_slices"], ZNC=g["ZNC"] - win["first_slice"], PN=win["bp_views"],
              BetaS=g["BetaS"] + win["bp_view0"] * g["DeltaFai"])
    w = oracle.weight_table(sc.N_2pi, sc.HSCoef, sc.delta)
    return oracle.bp_f64(filt, w, gs, nthreads=2).reshape(sc.YN, sc.XN, win["n_slices"])


def whole_recon(sc, fan):
    import oracle

    reb = oracle.rebin_f64(fan, **sc.rebin_args(), nthreads=2)
    rows = np.ascontiguousarray(reb[sc.crop_front: sc.crop_front + sc.PN].transpose(0, 2, 1))
    filt = oracle.filter_f64(rows, **sc.filter_args(), nthreads=2)
    w = oracle.weight_table(sc.N_2pi, sc.HSCoef, sc.delta)
    return oracle.bp_f64(filt, w, sc.bp_geom(), nthreads=2).reshape(sc.YN, sc.XN, sc.ZN)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, assign, out):
    import torch.distributed as dist
    from datetime import timedelta

    from analyticalreconbigpatient_b200.pipeline import slab_windows

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    try:
        sc = toy_scan()
        fan, _ = toy_fan(sc)
        wins = slab_windows(sc, SLAB, rank, world, assign)
        mine = []
        for win in wins:
            a0, n = win["fan_view0"], win["fan_views"]
            assert 0 <= a0 and a0 + n <= sc.views
            mine.append((win, slab_recon(sc, np.ascontiguousarray(fan[a0: a0 + n]), win)))
        gathered = [None] * world
        dist.all_gather_object(gathered, mine)
        if rank == 0:
            out.put(gathered)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("assign", [_lib.HR_SLAB_BLOCKS, _lib.HR_SLAB_ROUND_ROBIN])
def test_two_ranks_split_one_scan_by_slabs(assign):
    sc = toy_scan()
    nslabs = -(-sc.ZN // SLAB)
    assert nslabs >= 4, sc.ZN
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, assign, q)) for r in range(2)]
    for p in procs:
        p.start()
    gathered = q.get(timeout=300)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    vol = np.full((sc.YN, sc.XN, sc.ZN), np.nan)
    owner = {}
    for rank, part in enumerate(gathered):
        assert part, rank  # every rank has work
        for win, v in part:
            k = win["slab"]
            assert k not in owner, k
            owner[k] = rank
            assert win["first_slice"] == k * SLAB
            vol[:, :, win["first_slice"]: win["first_slice"] + win["n_slices"]] = v
    assert sorted(owner) == list(range(nslabs))
    if assign == _lib.HR_SLAB_ROUND_ROBIN:
        assert all(owner[k] == k % 2 for k in owner)
    else:
        assert [owner[k] for k in range(nslabs)] == sorted(owner[k] for k in range(nslabs))
    fan, _ = toy_fan(sc)
    ref = whole_recon(sc, fan)
    assert np.isfinite(vol).all()
    err = float(np.linalg.norm(vol - ref) / np.linalg.norm(ref))
    assert err < 1e-9, err


def test_slab_windows_arithmetic():
    """Windows of one part: every slice's clamped view window lies inside its
    slab's backprojection window, the fan window adds the half-fan margin on
    both sides, and consecutive slabs of a part share their overlapping views."""
    from analyticalreconbigpatient_b200.pipeline import slab_windows

    for sc, S in ((toy_scan(), SLAB), (G.config("full"), 128), (G.config("bigpatient"), 64)):
        g = sc.bp_geom()
        half = int(np.ceil(g["N_pi"] * g["HSCoef"]))
        zi = np.arange(sc.ZN, dtype=np.float64)
        s0 = np.ceil((2.0 * G.PI_TRUNC * (zi - g["ZNC"]) * g["dz"] / g["h"] - g["BetaS"]) / g["DeltaFai"] - 0.5)
        s1, s2 = np.maximum(s0 - half, 0), np.minimum(s0 + half, sc.PN - 1)
        for nparts in (1, 2, 3):
            for assign in (_lib.HR_SLAB_BLOCKS, _lib.HR_SLAB_ROUND_ROBIN):
                covered = []
                for part in range(nparts):
                    wins = slab_windows(sc, S, part, nparts, assign)
                    prev = None
                    for w in wins:
                        z = np.arange(w["first_slice"], w["first_slice"] + w["n_slices"])
                        covered.extend(z.tolist())
                        assert (s1[z] >= w["bp_view0"]).all() and (s2[z] <= w["bp_view0"] + w["bp_views"] - 1).all()
                        # fan view0 = crop + bp view0 - margin, and the margin is the crop
                        assert w["fan_view0"] == w["bp_view0"]
                        assert w["fan_views"] == w["bp_views"] + 2 * sc.crop_front
                        assert 0 <= w["fan_view0"] and w["fan_view0"] + w["fan_views"] <= sc.views
                        if prev is None:
                            assert w["shared_views"] == 0
                        else:
                            assert w["shared_views"] == max(0, prev["fan_view0"] + prev["fan_views"] - w["fan_view0"])
                        prev = w
                assert sorted(covered) == list(range(sc.ZN)), (sc.ZN, nparts, assign)
    # more parts than slabs is refused
    with pytest.raises(_lib.HelixError):
        slab_windows(toy_scan(), 10_000, 0, 2)
