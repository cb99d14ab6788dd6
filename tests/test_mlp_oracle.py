"""The warm-start MLP oracle pinned on the CPU: bf16 rounding and Adam against
PyTorch, the backward pass against finite differences, the wall distance
against dense sampling of the triangle."""
import numpy as np
import pytest
import torch

from oracle import mlp_oracle as mo


def _problem(seed=0, n=7):
    rng = np.random.default_rng(seed)
    w = mo.init_like_kernel(rng)
    x = np.column_stack([rng.uniform(-1, 1, (n, 7)), np.ones(n)])
    t = rng.standard_normal((n, 5))
    return w, x, t


def test_bf16_rounding_matches_torch():
    rng = np.random.default_rng(1)
    v = np.concatenate([rng.standard_normal(10000).astype(np.float32) * 10.0 ** rng.integers(-6, 6, 10000),
                        np.array([0.0, -0.0, 1.0, 1.00390625, 1.01171875, 65504.0], np.float32)]).astype(np.float32)
    ref = torch.from_numpy(v).to(torch.bfloat16).to(torch.float32).numpy()
    assert np.array_equal(mo.bf16(v), ref)


def test_exact_gradient_matches_finite_differences():
    w, x, t = _problem()
    loss, g = mo.loss_and_grad(w, x, t, mode="exact")
    rng = np.random.default_rng(2)
    pad = mo.padding_mask()
    idx = []
    for lo, hi in ((mo.OFF_W1, mo.OFF_W2), (mo.OFF_W2, mo.OFF_W3), (mo.OFF_W3, mo.OFF_W4), (mo.OFF_W4, mo.N_PARAMS)):
        cand = [i for i in range(lo, hi) if not pad[i]]
        idx += list(rng.choice(cand, 12, replace=False))
    h = 1e-6
    for i in idx:
        wp, wm = w.copy(), w.copy()
        wp[i] += h
        wm[i] -= h
        fd = (mo.loss_and_grad(wp, x, t)[0] - mo.loss_and_grad(wm, x, t)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(g[i])) + 1e-8, (i, fd, g[i])
    # padding weights get no gradient
    assert np.all(g[pad] == 0)


def test_exact_gradient_matches_torch_autograd():
    w, x, t = _problem(seed=5, n=33)
    loss, g = mo.loss_and_grad(w, x, t, mode="exact")
    w1, w2, w3, w4 = (torch.tensor(m, dtype=torch.float64, requires_grad=True) for m in mo.split(w))
    xp = torch.zeros((x.shape[0], 16), dtype=torch.float64)
    xp[:, :8] = torch.from_numpy(x)
    a = torch.nn.functional.silu(xp @ w1.T)
    a = torch.nn.functional.silu(a @ w2.T)
    a = torch.nn.functional.silu(a @ w3.T)
    y = (a @ w4.T)[:, :5]
    lt = torch.mean((y - torch.from_numpy(t)) ** 2)
    lt.backward()
    gt = np.concatenate([m.grad.numpy().ravel() for m in (w1, w2, w3, w4)])
    gt[mo.padding_mask()] = 0.0
    assert abs(lt.item() - loss) < 1e-12
    np.testing.assert_allclose(g, gt, rtol=1e-10, atol=1e-14)


def test_kernel_mode_is_close_to_exact():
    w, x, t = _problem(seed=3, n=256)
    le, ge = mo.loss_and_grad(w, x, t, mode="exact")
    lk, gk = mo.loss_and_grad(w, x, t, mode="kernel")
    assert abs(lk - le) < 2e-2 * le
    cos = ge @ gk / np.linalg.norm(ge) / np.linalg.norm(gk)
    assert cos > 0.999


def test_adam_matches_torch():
    w, x, t = _problem(seed=4, n=16)
    wt = torch.tensor(w, requires_grad=True)
    opt = torch.optim.Adam([wt], lr=1e-3, betas=(0.9, 0.999), eps=1e-8)
    m = np.zeros_like(w)
    v = np.zeros_like(w)
    ww = w.copy()
    pad = mo.padding_mask()
    for step in range(1, 6):
        _, g = mo.loss_and_grad(ww, x, t)
        ww, m, v = mo.adam_step(ww, m, v, g, step)
        opt.zero_grad()
        wt.grad = torch.from_numpy(g.copy())
        opt.step()
    # torch's CPU Adam may take a vectorised path (FMA contraction depends on
    # the tensor's alignment): allow ulp-level differences over 5 steps; a
    # formula difference shows at 1e-4 and above
    np.testing.assert_allclose(ww[~pad], wt.detach().numpy()[~pad], rtol=1e-9, atol=1e-13)


def test_point_triangle_distance_against_sampling():
    rng = np.random.default_rng(6)
    for _ in range(20):
        a, b, c = rng.standard_normal((3, 3))
        p = rng.standard_normal((50, 3)) * 2
        d = mo.point_triangle_distance(p, a, b, c)
        u, v = np.meshgrid(np.linspace(0, 1, 301), np.linspace(0, 1, 301))
        keep = u + v <= 1
        q = a + u[keep][:, None] * (b - a) + v[keep][:, None] * (c - a)
        brute = np.min(np.linalg.norm(p[:, None, :] - q[None, :, :], axis=2), axis=1)
        assert np.all(d <= brute + 1e-12)
        assert np.all(brute - d < 0.02 * (np.linalg.norm(b - a) + np.linalg.norm(c - a)))
