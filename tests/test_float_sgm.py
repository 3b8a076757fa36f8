"""Differentiable float32 SGM: CUDA forward/backward vs a plain-PyTorch reference (autograd) and
FP64 finite differences, on 64x48x32 crops of a seeded scene (Hamming cost + U(0,0.5) jitter)."""
import numpy as np
import pytest
import torch

from fasterstereocuda_b200 import scenes
from fasterstereocuda_b200.float_sgm import reference_sgm


def jittered_cost(oracle_mod, W, H, D, B=1, seed=70):
    vols = []
    rng = np.random.Generator(np.random.PCG64(seed))
    for b in range(B):
        L, R, _ = scenes.planar_pair(seed + b, W, H, dmin=2.0, dmax=D - 6.0)
        cfg = oracle_mod.Config(width=W, height=H, disp_range=D, do_lr_check=0, do_median=0)
        c = oracle_mod.match(cfg, L, R, dump=True)["cost"].astype(np.float64)
        vols.append(c + rng.uniform(0.0, 0.5, size=c.shape))
    return np.stack(vols)


def fd_check(f, x, idx, g_analytic, h=1e-6):
    """central differences of the scalar f at flat indices idx of x (float64, modified in place)"""
    fd = []
    flat = x.view(-1)
    for i in idx:
        old = flat[i].item()
        flat[i] = old + h
        fp = f().item()
        flat[i] = old - h
        fm = f().item()
        flat[i] = old
        fd.append((fp - fm) / (2 * h))
    fd = np.array(fd)
    ga = g_analytic.reshape(-1)[idx]
    return np.linalg.norm(ga - fd) / max(np.linalg.norm(fd), 1e-12)


def test_reference_autograd_matches_fp64_finite_differences(oracle_mod):
    """CPU: the PyTorch restatement's autograd gradient equals central differences in FP64."""
    c = torch.tensor(jittered_cost(oracle_mod, 14, 11, 32), dtype=torch.float64, requires_grad=True)
    p1 = torch.full(c.shape[:-1], 10.0, dtype=torch.float64, requires_grad=True)
    p2 = torch.full(c.shape[:-1], 150.0, dtype=torch.float64, requires_grad=True)
    w = torch.randn(c.shape[:-1], dtype=torch.float64, generator=torch.Generator().manual_seed(0))
    (reference_sgm(c, p1, p2) * w).sum().backward()
    with torch.no_grad():
        f = lambda: (reference_sgm(c, p1, p2) * w).sum()  # noqa: E731
        gc = c.grad.numpy()
        idx = np.argsort(-np.abs(gc.reshape(-1)))[:20]
        assert fd_check(f, c, idx, gc) < 1e-6
        g1 = p1.grad.numpy()
        idx = np.argsort(-np.abs(g1.reshape(-1)))[:8]
        assert fd_check(f, p1, idx, g1) < 1e-6


@pytest.mark.gpu
def test_forward_matches_reference(oracle_mod):
    c64 = torch.tensor(jittered_cost(oracle_mod, 64, 48, 32, B=2), dtype=torch.float64)
    p1 = torch.full(c64.shape[:-1], 10.0, dtype=torch.float64)
    p2 = torch.full(c64.shape[:-1], 150.0, dtype=torch.float64)
    from fasterstereocuda_b200.float_sgm import float_sgm
    d = float_sgm(c64.float().cuda(), p1.float().cuda(), p2.float().cuda()).cpu().double()
    ref = reference_sgm(c64, p1, p2)
    assert torch.allclose(d, ref, rtol=1e-4, atol=1e-4), (d - ref).abs().max()


@pytest.mark.gpu
@pytest.mark.parametrize("D", [32, 64])
def test_backward_matches_fp64_finite_differences_and_autograd(oracle_mod, D):
    from fasterstereocuda_b200.float_sgm import float_sgm
    c64 = torch.tensor(jittered_cost(oracle_mod, 64, 48, D), dtype=torch.float64)
    gen = torch.Generator().manual_seed(1)
    p1 = (10.0 + torch.rand(c64.shape[:-1], generator=gen, dtype=torch.float64))
    p2 = (150.0 + 10 * torch.rand(c64.shape[:-1], generator=gen, dtype=torch.float64))
    w = torch.randn(c64.shape[:-1], generator=gen, dtype=torch.float64)
    # kernel gradients (float32)
    c = c64.float().cuda().requires_grad_()
    q1 = p1.float().cuda().requires_grad_()
    q2 = p2.float().cuda().requires_grad_()
    (float_sgm(c, q1, q2) * w.float().cuda()).sum().backward()
    gk = [c.grad.cpu().double().numpy(), q1.grad.cpu().double().numpy(), q2.grad.cpu().double().numpy()]
    # autograd reference (FP64)
    cr, r1, r2 = (t.clone().requires_grad_() for t in (c64, p1, p2))
    (reference_sgm(cr, r1, r2) * w).sum().backward()
    gr = [cr.grad.numpy(), r1.grad.numpy(), r2.grad.numpy()]
    for a, b, name in zip(gk, gr, ("cost", "p1", "p2")):
        rel = np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-12)
        assert rel < 1e-3, (name, rel)
    # FP64 finite differences on the largest entries
    with torch.no_grad():
        xs = [c64.clone(), p1.clone(), p2.clone()]
        f = lambda: (reference_sgm(xs[0], xs[1], xs[2]) * w).sum()  # noqa: E731
        for k, n in ((0, 24), (1, 8), (2, 8)):
            idx = np.argsort(-np.abs(gk[k].reshape(-1)))[:n]
            assert fd_check(f, xs[k], idx, gk[k]) < 1e-3, k


@pytest.mark.gpu
@pytest.mark.parametrize("D", [32, 64])
def test_ragged_sizes_match_autograd_and_repeat(oracle_mod, D):
    """Line counts that leave part of a warp idle and scanlines ending inside a segment: forward
    and gradients against the FP64 autograd reference; a second run gives the same bits."""
    from fasterstereocuda_b200.float_sgm import float_sgm
    c64 = torch.tensor(jittered_cost(oracle_mod, 37, 29, D, B=2, seed=91), dtype=torch.float64)
    gen = torch.Generator().manual_seed(3)
    p1 = 8.0 + 4 * torch.rand(c64.shape[:-1], generator=gen, dtype=torch.float64)
    p2 = 100.0 + 60 * torch.rand(c64.shape[:-1], generator=gen, dtype=torch.float64)
    w = torch.randn(c64.shape[:-1], generator=gen, dtype=torch.float64)

    def run():
        c = c64.float().cuda().requires_grad_()
        q1 = p1.float().cuda().requires_grad_()
        q2 = p2.float().cuda().requires_grad_()
        d = float_sgm(c, q1, q2)
        (d * w.float().cuda()).sum().backward()
        return [t.detach().cpu() for t in (d, c.grad, q1.grad, q2.grad)]
    first, again = run(), run()
    for a, b in zip(first, again):
        assert torch.equal(a, b)
    cr, r1, r2 = (t.clone().requires_grad_() for t in (c64, p1, p2))
    dr = reference_sgm(cr, r1, r2)
    assert torch.allclose(first[0].double(), dr.detach(), rtol=1e-4, atol=1e-4), (first[0].double() - dr).abs().max()
    (dr * w).sum().backward()
    for a, b, name in zip(first[1:], (cr.grad, r1.grad, r2.grad), ("cost", "p1", "p2")):
        rel = (a.double() - b).norm() / max(b.norm(), 1e-12)
        assert rel < 1e-3, (name, rel)


@pytest.mark.gpu
def test_fitting_penalty_maps_reduces_l1(oracle_mod):
    """Demo: fit per-pixel P1/P2 maps to the ground-truth disparity under an L1 loss."""
    from fasterstereocuda_b200.float_sgm import float_sgm
    W, H, D = 128, 96, 64
    L, R, gt = scenes.planar_pair(80, W, H, dmin=4.0, dmax=50.0)
    cfg = oracle_mod.Config(width=W, height=H, disp_range=D, do_lr_check=0, do_median=0)
    cost = torch.tensor(oracle_mod.match(cfg, L, R, dump=True)["cost"], dtype=torch.float32).cuda()[None]
    cost = cost + torch.rand(cost.shape, generator=torch.Generator(device="cuda").manual_seed(0), device="cuda") * 0.5
    gt = torch.tensor(gt).cuda()[None]
    lp1 = torch.full((1, H, W), np.log(10.0), device="cuda", requires_grad=True)
    lp2 = torch.full((1, H, W), np.log(150.0), device="cuda", requires_grad=True)
    opt = torch.optim.Adam([lp1, lp2], lr=0.05)
    losses = []
    inner = (slice(None), slice(8, H - 8), slice(8, W - 8))
    for _ in range(40):
        opt.zero_grad()
        disp = float_sgm(cost, lp1.exp(), lp2.exp())
        loss = (disp[inner] - gt[inner]).abs().mean()
        loss.backward()
        opt.step()
        losses.append(loss.item())
    assert losses[-1] < losses[0] * 0.98, losses[::10]
