"""GPU tests of the learned correction network (hr_cnn_*): forward output and
parameter gradients of the tensor-core / CUDA-core kernels against the CPU
oracle (which rounds to BF16 where the kernels store BF16), and a small
training run that must beat the half-view reconstruction it corrects."""
import numpy as np
import pytest
import torch

from analyticalreconbigpatient_b200 import learned as L
from analyticalreconbigpatient_b200.geometry import MU_WATER
from conftest import rel_l2
from oracle import cnn_oracle as C

pytestmark = pytest.mark.gpu


def bf16_bits(a: np.ndarray) -> np.ndarray:
    u = np.asarray(a, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) >> 16
    return u.astype(np.uint16)


def problem(B, H, W, seed=0):
    rng = np.random.default_rng(seed)
    params = C.init_params(seed, zero_last=False)
    params[C.param_count() - 16] = 0.01  # a non-zero residual bias
    u = np.zeros((B, H, W, 16), dtype=np.float32)
    u[..., :5] = rng.standard_normal((B, H, W, 5)).astype(np.float32) * 0.3
    base = (MU_WATER * (1.0 + rng.standard_normal((B, H, W)) * 0.05)).astype(np.float32)
    target = (base + MU_WATER * rng.standard_normal((B, H, W)) * 0.01).astype(np.float32)
    return params, u, base, target


@pytest.mark.parametrize("B,H,W", [(2, 5, 150), (1, 3, 128), (3, 4, 40)])
def test_forward_and_gradients_match_the_oracle(cuda, B, H, W):
    params, u, base, target = problem(B, H, W, seed=B * 100 + W)
    net = L.Corrector(params)
    x = torch.from_numpy(bf16_bits(u).view(np.int16)).to(cuda)
    tb, tt = torch.from_numpy(base).to(cuda), torch.from_numpy(target).to(cuda)
    pred = net.forward(x, tb).cpu().numpy()
    loss = net.train_step(x, tb, tt, lr=0.0)
    grads = net.grads()
    net.check()
    xr = C.bf16(u)
    opred, _, _ = C.forward(params, xr, base, MU_WATER)
    oloss, ograds = C.loss_and_grads(params, xr, base, target, MU_WATER)
    assert rel_l2(pred - base, opred - base) < 1e-3
    assert abs(loss - oloss) < 1e-3 * oloss
    o = 0
    for l, (ci, co) in enumerate(zip(C.CIN, C.COUT)):
        n = 9 * ci * co + co
        g, og = grads[o:o + n], ograds[o:o + n]
        assert np.linalg.norm(og) > 0, l
        assert rel_l2(g, og) < 1e-2, (l, rel_l2(g, og))
        o += n


def test_adam_step_updates_parameters(cuda):
    params, u, base, target = problem(2, 4, 64, seed=3)
    net = L.Corrector(params)
    x = torch.from_numpy(bf16_bits(u).view(np.int16)).to(cuda)
    tb, tt = torch.from_numpy(base).to(cuda), torch.from_numpy(target).to(cuda)
    l0 = net.train_step(x, tb, tt, lr=1e-3)
    p1 = net.params()
    # the first Adam step moves every parameter with a non-zero gradient by ~lr
    g = net.grads()
    moved = np.abs(p1 - params)
    nz = np.abs(g) > 1e-12
    assert np.all(moved[~nz] == 0)
    assert np.median(moved[nz]) == pytest.approx(1e-3, rel=0.05)
    for _ in range(20):
        l1 = net.train_step(x, tb, tt, lr=1e-3)
    assert l1 < l0


def test_training_beats_the_half_view_reconstruction(cuda):
    # 128^2 grid over the same 500 mm field; short scans; 14 training + 3 held-out phantoms
    train = L.PairSet(range(1, 15), grid=128, pixel=500.0 / 128, slices=12)
    test = L.PairSet(range(1001, 1004), grid=128, pixel=500.0 / 128, slices=12)
    net = L.Corrector(seed=0)
    before = L.evaluate(net, test)
    assert before["hu_rmse_learned"] == pytest.approx(before["hu_rmse_half_view"], rel=1e-6)  # starts as identity
    losses = L.train(net, train, steps=300, batch=8, lr=2e-3)
    after = L.evaluate(net, test)
    assert np.mean(losses[-30:]) < 0.8 * np.mean(losses[:30])
    assert after["hu_rmse_learned"] < 0.9 * after["hu_rmse_half_view"], after
    # whole-volume inference equals the per-slice forward on the interior slices
    vol = test.inputs[0]
    out = net.apply_volume(vol)
    x = torch.empty((4, vol.shape[0], vol.shape[1], 16), dtype=torch.int16, device=cuda)
    net.pack_input(x, vol, 2, 4)
    ref = net.forward(x, vol[:, :, 2:6].permute(2, 0, 1).contiguous())
    assert torch.equal(out[:, :, 2:6].permute(2, 0, 1), ref)
    net.close()
