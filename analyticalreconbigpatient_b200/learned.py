"""Learned artifact correction of half-view reconstructions (2.5D residual CNN).

The network and its kernels live in libhelixrecon.so (hr_cnn_*): forward and
backward-data convolutions on the tensor cores, weight gradients and Adam on
the CUDA cores. This module holds the parameter initialisation, the training
data the plain method produces from seeded phantoms, the training loop and
the evaluation in HU.

Training pairs: a full-view scan (984 views/rotation) of a seeded random
ellipsoid phantom with Poisson noise is reconstructed with the plain FP32
chain; the half-view scan is every second view of the same noisy data (492
views/rotation) reconstructed the same way. The network maps 5 adjacent
half-view slices to a correction of the centre slice; the full-view slice is
the target. A slice depends only on the views within its 3D-weighting window,
so the pairs come from short (2-rotation) scans whose central slices see the
same view windows as the slices of a 10-rotation scan.
"""
from __future__ import annotations

import ctypes
import math
from dataclasses import replace

import numpy as np
import torch

from . import _lib
from .geometry import MU_WATER, Scan

CIN = (16, 32, 32, 32, 32, 32, 32, 32)
COUT = (32, 32, 32, 32, 32, 32, 32, 16)


def param_count() -> int:
    return int(_lib.load().hr_cnn_param_count())


def init_params(seed: int) -> np.ndarray:
    """He-normal weights over the real input channels (5 slices at layer 1),
    zero biases, zero padded channels, and a zero last layer: the untrained
    network returns its centre slice unchanged."""
    rng = np.random.default_rng(seed)
    p = np.zeros(sum(9 * ci * co + co for ci, co in zip(CIN, COUT)), dtype=np.float32)
    o = 0
    for l, (ci, co) in enumerate(zip(CIN, COUT)):
        w = p[o:o + 9 * ci * co].reshape(co, 9, ci)
        if l < 7:
            ci_real = 5 if l == 0 else ci
            w[:, :, :ci_real] = rng.standard_normal((co, 9, ci_real)) * math.sqrt(2.0 / (9 * ci_real))
        o += 9 * ci * co + co
    return p


class Corrector:
    """The network on one device (parameters, Adam state, work buffers)."""

    def __init__(self, params: np.ndarray | None = None, seed: int = 0, device: int | torch.device = 0):
        self.device = torch.device("cuda", device) if isinstance(device, int) else device
        p = init_params(seed) if params is None else np.ascontiguousarray(params, dtype=np.float32)
        if p.size != param_count():
            raise ValueError(f"expected {param_count()} parameters, got {p.size}")
        self._net = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            _lib.check(_lib.load().hr_cnn_create(ctypes.byref(self._net), p.ctypes.data))

    # ---- parameters ---------------------------------------------------------
    def params(self) -> np.ndarray:
        out = np.empty(param_count(), dtype=np.float32)
        _lib.check(_lib.load().hr_cnn_get_params(self._net, out.ctypes.data))
        return out

    def grads(self) -> np.ndarray:
        out = np.empty(param_count(), dtype=np.float32)
        _lib.check(_lib.load().hr_cnn_get_grads(self._net, out.ctypes.data))
        return out

    # ---- data -----------------------------------------------------------------
    def pack_input(self, out: torch.Tensor, vol: torch.Tensor, z0: int, nz: int, mu_w: float = MU_WATER) -> None:
        """Network input [nz][YN][XN][16] (BF16 bits as int16) of slices z0.. of vol [YN][XN][ZN]."""
        YN, XN, ZN = vol.shape
        _lib.check(_lib.load().hr_cnn_pack_input(out.data_ptr(), vol.data_ptr(), XN, YN, ZN, z0, nz, mu_w,
                                                 torch.cuda.current_stream(self.device).cuda_stream))

    # ---- training / inference ----------------------------------------------------
    def train_step(self, x: torch.Tensor, base: torch.Tensor, target: torch.Tensor, lr: float,
                   mu_w: float = MU_WATER) -> float:
        """x [B][H][W][16] int16 (BF16 bits); base/target float32 [B][H][W]. Returns the loss
        (mean squared error in units of mu_w, before the update); lr = 0 only computes gradients."""
        B, H, W = base.shape
        loss = ctypes.c_float()
        _lib.check(_lib.load().hr_cnn_train_step(self._net, x.data_ptr(), base.data_ptr(), target.data_ptr(), B, H,
                                                 W, mu_w, lr, ctypes.byref(loss),
                                                 torch.cuda.current_stream(self.device).cuda_stream))
        return float(loss.value)

    def forward(self, x: torch.Tensor, base: torch.Tensor, mu_w: float = MU_WATER) -> torch.Tensor:
        B, H, W = base.shape
        out = torch.empty_like(base)
        _lib.check(_lib.load().hr_cnn_forward(self._net, out.data_ptr(), x.data_ptr(), base.data_ptr(), H * W, 1,
                                              B, H, W, mu_w, torch.cuda.current_stream(self.device).cuda_stream))
        return out

    def apply_volume(self, vol: torch.Tensor, out: torch.Tensor | None = None, mu_w: float = MU_WATER,
                     chunk: int = 32) -> torch.Tensor:
        """Corrects every slice of a reconstructed volume [YN][XN][ZN]."""
        YN, XN, ZN = vol.shape
        if out is None:
            out = torch.empty_like(vol)
        _lib.check(_lib.load().hr_cnn_apply_volume(self._net, out.data_ptr(), vol.data_ptr(), XN, YN, ZN, mu_w,
                                                   chunk, torch.cuda.current_stream(self.device).cuda_stream))
        return out

    def check(self) -> None:
        _lib.check(_lib.load().hr_cnn_check(self._net))

    def close(self) -> None:
        if self._net:
            _lib.load().hr_cnn_destroy(self._net)
            self._net = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---- training pairs from the plain method ------------------------------------------
def pair_scans(grid: int = 512, pixel: float = 0.9766, slices: int = 20, rotations: int = 2,
               ZL: int = 64) -> tuple[Scan, Scan]:
    """(full-view, half-view) scans of the same helix: 984 and 492 views per
    rotation, the half-view views being every second full-view view."""
    full = Scan(ZL=ZL, pitch=0.984, rotations=rotations, N_2pi=984, XN=grid, YN=grid, ZN=slices, dx=pixel, dy=pixel,
                dz=0.625)
    full = replace(full, beta_start=full.BetaS)
    half = replace(full, N_2pi=492)
    assert half.views * 2 == full.views
    return full, half


class PairSet:
    """Half-view input volumes and full-view target slices of seeded phantoms,
    resident on the device: inputs [n][YN][XN][ZN] FP32, targets [n][S][YN][XN]
    FP32 for the S = ZN - 4 slices with a full 5-slice context. I0: photons per
    ray of the Poisson noise added before the log (0: noiseless data)."""

    def __init__(self, seeds, grid: int = 512, pixel: float = 0.9766, slices: int = 20, I0: float = 1e5,
                 n_ellipsoids: int = 60, device: int = 0):
        from . import phantom as P
        from .pipeline import HelicalRecon, add_poisson_noise, project

        self.full, self.half = pair_scans(grid, pixel, slices)
        self.device = torch.device("cuda", device)
        seeds = list(seeds)
        S = slices - 4
        f, h = self.full, self.half
        self.inputs = torch.empty((len(seeds), h.YN, h.XN, h.ZN), dtype=torch.float32, device=self.device)
        self.targets = torch.empty((len(seeds), S, f.YN, f.XN), dtype=torch.float32, device=self.device)
        rf = HelicalRecon(f, form=_lib.HR_FORM_PLAIN, device=self.device)
        rh = HelicalRecon(h, form=_lib.HR_FORM_PLAIN, device=self.device)
        zlo = f.h * f.BetaS / (2 * np.pi)
        zhi = f.h * (f.BetaS + f.views * f.dBeta) / (2 * np.pi)
        scale = grid * pixel / 500.0  # phantoms scale with the field of view
        vol_f = torch.empty((f.YN, f.XN, f.ZN), dtype=torch.float32, device=self.device)
        for k, seed in enumerate(seeds):
            objs = P.random_ellipsoids(seed, n_ellipsoids, (zlo, zhi), body=(180.0 * scale, 140.0 * scale),
                                       semi_axes=(5.0 * scale, 120.0 * scale))
            fan = project(f, objs, device=self.device.index)
            if I0 > 0:
                add_poisson_noise(fan, I0, 0x5EED0000 + seed)
            rf.run(fan, vol_f)
            half_fan = fan[::2].contiguous()
            rh.run(half_fan, self.inputs[k])
            self.targets[k].copy_(vol_f[:, :, 2:2 + S].permute(2, 0, 1))
            del fan, half_fan
        torch.cuda.synchronize()
        rf.close()
        rh.close()
        self.S = S

    def __len__(self) -> int:
        return self.inputs.shape[0]

    def batch(self, net: Corrector, idx, zs, x: torch.Tensor, base: torch.Tensor, target: torch.Tensor):
        """Fills x/base/target for samples (phantom idx[i], centre slice 2 + zs[i])."""
        for i, (k, z) in enumerate(zip(idx, zs)):
            net.pack_input(x[i:i + 1], self.inputs[k], 2 + int(z), 1)
            base[i].copy_(self.inputs[k][:, :, 2 + int(z)])
            target[i].copy_(self.targets[k][int(z)])


def hu_rmse(a: torch.Tensor, b: torch.Tensor) -> float:
    return float(torch.sqrt(torch.mean((a.double() - b.double()) ** 2))) / MU_WATER * 1000.0


def train(net: Corrector, data: PairSet, steps: int, batch: int = 8, lr: float = 1e-3, seed: int = 0,
          log_every: int = 0) -> list[float]:
    """Adam on random (phantom, slice) samples; cosine learning-rate decay."""
    rng = np.random.default_rng(seed)
    H, W = data.half.YN, data.half.XN
    x = torch.empty((batch, H, W, 16), dtype=torch.int16, device=data.device)
    base = torch.empty((batch, H, W), dtype=torch.float32, device=data.device)
    target = torch.empty_like(base)
    losses = []
    for s in range(steps):
        idx = rng.integers(0, len(data), batch)
        zs = rng.integers(0, data.S, batch)
        data.batch(net, idx, zs, x, base, target)
        step_lr = lr * 0.5 * (1.0 + math.cos(math.pi * s / max(steps, 1)))
        losses.append(net.train_step(x, base, target, step_lr))
        if log_every and s % log_every == 0:
            print(f"step {s} loss {losses[-1]:.3e} ({math.sqrt(losses[-1]) * 1000:.2f} HU)", flush=True)
    net.check()
    return losses


def evaluate(net: Corrector, data: PairSet, chunk: int = 8) -> dict:
    """HU RMSE against the full-view slices, with and without the network."""
    H, W = data.half.YN, data.half.XN
    x = torch.empty((chunk, H, W, 16), dtype=torch.int16, device=data.device)
    sq_net = sq_plain = 0.0
    n = 0
    for k in range(len(data)):
        for z0 in range(0, data.S, chunk):
            nz = min(chunk, data.S - z0)
            net.pack_input(x, data.inputs[k], 2 + z0, nz)
            base = data.inputs[k][:, :, 2 + z0:2 + z0 + nz].permute(2, 0, 1).contiguous()
            pred = net.forward(x[:nz], base)
            tgt = data.targets[k][z0:z0 + nz]
            sq_net += float(torch.sum((pred.double() - tgt.double()) ** 2))
            sq_plain += float(torch.sum((base.double() - tgt.double()) ** 2))
            n += pred.numel()
    return {"hu_rmse_learned": math.sqrt(sq_net / n) / MU_WATER * 1000.0,
            "hu_rmse_half_view": math.sqrt(sq_plain / n) / MU_WATER * 1000.0, "slices": n // (H * W)}


def error_scales(net: Corrector, data: PairSet, sigma: float = 8.0, chunk: int = 8) -> dict:
    """Where the remaining error lives: the half-view and the learned errors
    (against the full-view slices) split into a smooth part (Gaussian blur of
    sigma pixels, wider than the network's 17 x 17 in-plane receptive field)
    and the rest, each as an HU RMSE. Error the network cannot see around a
    pixel shows up in the smooth part."""
    H, W = data.half.YN, data.half.XN
    r = int(math.ceil(3 * sigma))
    g = torch.exp(-0.5 * (torch.arange(-r, r + 1, dtype=torch.float64, device=data.device) / sigma) ** 2)
    g = (g / g.sum()).float()
    gx, gy = g.view(1, 1, 1, -1), g.view(1, 1, -1, 1)

    def blur(e):  # e: [n][H][W]
        e = e.unsqueeze(1)
        e = torch.nn.functional.conv2d(torch.nn.functional.pad(e, (r, r, 0, 0), mode="replicate"), gx)
        e = torch.nn.functional.conv2d(torch.nn.functional.pad(e, (0, 0, r, r), mode="replicate"), gy)
        return e.squeeze(1)

    x = torch.empty((chunk, H, W, 16), dtype=torch.int16, device=data.device)
    acc = {k: 0.0 for k in ("half_low", "half_high", "learned_low", "learned_high")}
    n = 0
    for k in range(len(data)):
        for z0 in range(0, data.S, chunk):
            nz = min(chunk, data.S - z0)
            net.pack_input(x, data.inputs[k], 2 + z0, nz)
            base = data.inputs[k][:, :, 2 + z0:2 + z0 + nz].permute(2, 0, 1).contiguous()
            pred = net.forward(x[:nz], base)
            tgt = data.targets[k][z0:z0 + nz]
            for name, e in (("half", base - tgt), ("learned", pred - tgt)):
                lo = blur(e)
                acc[name + "_low"] += float(torch.sum(lo.double() ** 2))
                acc[name + "_high"] += float(torch.sum((e - lo).double() ** 2))
            n += pred.numel()
    return {f"hu_rmse_{k}": math.sqrt(v / n) / MU_WATER * 1000.0 for k, v in acc.items()} | {"sigma_px": sigma}


def main(argv=None) -> None:
    """Train on seeded phantoms and evaluate on held-out ones from the command line:
    python -m analyticalreconbigpatient_b200.learned --phantoms 200 --steps 600 --eval 20 [--save params.npy]"""
    import argparse
    import json
    import time

    ap = argparse.ArgumentParser(description=main.__doc__)
    ap.add_argument("--phantoms", type=int, default=200)
    ap.add_argument("--steps", type=int, default=600)
    ap.add_argument("--eval", type=int, default=20)
    ap.add_argument("--batch", type=int, default=8)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--grid", type=int, default=512)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--i0", type=float, default=1e5, help="photons per ray before the log (0: noiseless)")
    ap.add_argument("--save", default=None, help="write the trained parameters (.npy)")
    ap.add_argument("--scales", action="store_true",
                    help="also split the remaining error into a smooth part and the rest (error_scales)")
    a = ap.parse_args(argv)
    pixel = 0.9766 * 512 / a.grid
    t0 = time.perf_counter()
    train_set = PairSet(range(1, 1 + a.phantoms), grid=a.grid, pixel=pixel, I0=a.i0)
    t1 = time.perf_counter()
    net = Corrector(seed=a.seed)
    losses = train(net, train_set, steps=a.steps, batch=a.batch, lr=a.lr, seed=a.seed)
    torch.cuda.synchronize()
    t2 = time.perf_counter()
    del train_set
    test_set = PairSet(range(100001, 100001 + a.eval), grid=a.grid, pixel=pixel, I0=a.i0)
    ev = evaluate(net, test_set)
    if a.scales:
        ev |= error_scales(net, test_set)
    if a.save:
        np.save(a.save, net.params())
    print(json.dumps({"data_s": t1 - t0, "train_s": t2 - t1, "loss_first": float(np.mean(losses[:20])),
                      "loss_last": float(np.mean(losses[-20:])), **ev}), flush=True)
    net.close()


if __name__ == "__main__":
    main()
