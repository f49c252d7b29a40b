"""The closure's training step on the device against torch: the Adam update (k_adam) against
torch.optim.Adam driven by the same gradients over two steps, and the cell loss and its output gradient (the
transpose of the divergence, k_loss_grad) against autograd of the same loss written in torch.

The sample is a real capture (a 16^3 coarse turbulence problem and its 32^3 fine run). The loss-gradient test
feeds autograd's dL/d(output) through the device's own backward (gam_closure_backward_host), so the two
parameter gradients differ only where the output gradient differs; the output gradient is rounded to BF16 on
both routes, which bounds the agreement at about 1e-2 relative L2."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
G = 4


def _captured_sample(n=16, seed=7):
    """A closure with one captured sample, the net input of that sample (host float, the device's
    normalisation), and the host restriction residual."""
    from kaiju_b200 import gamera as gm, turbulence as tu, closure_train as ct
    c = gm.Closure(n, n, n, seed=0)
    c.set_params(c.params() * 4.0)
    c.reserve(1)
    fine = tu.turbulence_problem(2 * n, seed=seed)
    coarse = tu.coarse_problem(n)
    coarse.restrict_from(fine, gm.GAM_SYNC_OSTATE)
    ta = fine.status()["time"]
    fine.step(); fine.step()
    tb = fine.status()["time"]
    coarse.restrict_from(fine, gm.GAM_SYNC_STATE)
    c.in_mean, c.in_std = ct.primitive_stats(coarse)
    flux_scale = np.full(8, 2e-3)
    c.set_norm(c.in_mean, c.in_std, flux_scale, np.full(5, 1e-3))
    fine.step(); fine.step()
    tc = fine.status()["time"]
    coarse.set_scalars(tb, tc - tb, 0.0, 1, tb, ta)
    gas, b = coarse.fetch("gas"), coarse.fetch("bxyz")
    c.capture(0, coarse, fine)
    # the net input as k_closure_input forms it: normalised primitives of State n, ghosts included
    rho = gas[..., 0]
    v = gas[..., 1:4] / rho[..., None]
    P = (5.0 / 3.0 - 1.0) * (gas[..., 4] - 0.5 * rho * (v * v).sum(-1))
    w = np.concatenate([rho[..., None], v, P[..., None], b], axis=-1)
    mean = np.asarray(c.in_mean, dtype=np.float32).astype(np.float64)
    std = np.asarray(c.in_std, dtype=np.float32).astype(np.float64)
    x = ((w - mean) / std).astype(np.float32)
    fg = fine.fetch("gas")[G:-G, G:-G, G:-G]
    res = fg.reshape(n, 2, n, 2, n, 2, 5).mean(axis=(1, 3, 5)) - coarse.fetch("gas")[G:-G, G:-G, G:-G]
    fine.close(); coarse.close()
    return c, x, res.astype(np.float32), tc - tb, flux_scale


def test_adam_matches_torch():
    torch = pytest.importorskip("torch")
    c, x, res, dt, fs = _captured_sample()
    p0 = c.params().astype(np.float32)
    lr = 1e-3
    t = torch.tensor(p0, dtype=torch.float32, requires_grad=True)
    opt = torch.optim.Adam([t], lr=lr, betas=(0.9, 0.999), eps=1e-8)
    for step in range(2):
        c.train([0], lr)
        g = c.grads().astype(np.float32)
        assert np.linalg.norm(g) > 0
        t.grad = torch.tensor(g)
        opt.step()
        dev = c.params()
        ref = t.detach().numpy()
        # every parameter moves by about lr; the two agree to float rounding of that move
        assert np.max(np.abs(dev - ref)) <= 1e-3 * lr + 4 * np.finfo(np.float32).eps * np.max(np.abs(ref)), step
        assert np.max(np.abs(dev - p0)) > 0.5 * lr
    c.close()


def test_cell_loss_gradient_matches_autograd():
    torch = pytest.importorskip("torch")
    c, x, res, dt, fs = _captured_sample()
    n = res.shape[0]
    p0 = c.params()
    out = torch.tensor(c.forward_host(x), dtype=torch.float32, requires_grad=True)   # (n, n, n, 24)
    # uniform periodic unit cube: face area h^2, volume h^3
    h = 1.0 / n
    A, V = h * h, h * h * h
    fsT = torch.tensor(fs, dtype=torch.float32)
    dU = [torch.zeros((n, n, n)) for _ in range(5)]
    for d in range(3):
        for v in range(8):
            corr = out[..., d * 8 + v] * fsT[v] * A   # lower d-face of each cell; the upper face is the next cell's
            div = corr - torch.roll(corr, shifts=-1, dims=d)
            u = v if v < 5 else v - 4
            dU[u] = dU[u] + div
    r = torch.tensor(res)
    loss = torch.zeros(())
    for v in range(5):
        e = (float(dt) / V * dU[v] - r[..., v]) / 1e-3
        loss = loss + (e * e).mean()
    loss.backward()
    gout = out.grad.numpy().copy()
    # the device's training pass: its loss and its parameter gradient at p0
    dev_loss = c.train([0], 1e-6)
    g_train = c.grads().copy()
    assert dev_loss == pytest.approx(float(loss), rel=1e-3)
    c.set_params(p0)
    g_auto = c.backward_host(x, gout)
    rel = np.linalg.norm(g_train - g_auto) / np.linalg.norm(g_auto)
    assert rel < 1e-2, rel
    c.close()
