"""The closure's training step on the device against torch: the Adam update (k_adam) against
torch.optim.Adam driven by the same gradients over two steps, and the cell loss and its output gradient (the
transpose of the divergence, k_loss_grad) against autograd of the same loss written in torch.

The sample is a real capture (a 16^3 coarse turbulence problem and its 32^3 fine run). The loss-gradient test
feeds autograd's dL/d(output) through the device's own backward (gam_closure_backward_host), so the two
parameter gradients differ only where the output gradient differs; the output gradient is rounded to BF16 on
both routes, which bounds the agreement at about 1e-2 relative L2. It runs with and without the EMF outputs
(the face magnetic-flux residual through the curl of the EMF corrections)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
G = 4


def _captured_sample(n=16, seed=7, emf=False):
    """A closure with one captured sample, the net input of that sample (host float, the device's
    normalisation), the host restriction residuals (gas, and with emf the face magnetic fluxes), the sample's
    dt and the flux and EMF scales."""
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
    emf_scale = np.array([3e-3, 2e-3, 4e-3]) if emf else np.zeros(3)
    if emf:
        c.set_norm_emf(emf_scale, np.full(3, 1e-4))
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
    # magnetic flux of each active coarse cell's lower faces: the 2 x 2 fine sub-faces minus the coarse flux
    fm, cm = fine.fetch("magflux"), coarse.fetch("magflux")
    s = slice(G, G + 2 * n, 2)
    f0 = fm[s, s, s, 0] + fm[s, G + 1:G + 2 * n:2, s, 0] + fm[s, s, G + 1:G + 2 * n:2, 0] + \
        fm[s, G + 1:G + 2 * n:2, G + 1:G + 2 * n:2, 0]
    f1 = fm[s, s, s, 1] + fm[G + 1:G + 2 * n:2, s, s, 1] + fm[s, s, G + 1:G + 2 * n:2, 1] + \
        fm[G + 1:G + 2 * n:2, s, G + 1:G + 2 * n:2, 1]
    f2 = fm[s, s, s, 2] + fm[G + 1:G + 2 * n:2, s, s, 2] + fm[s, G + 1:G + 2 * n:2, s, 2] + \
        fm[G + 1:G + 2 * n:2, G + 1:G + 2 * n:2, s, 2]
    resb = np.stack([f0, f1, f2], axis=-1) - cm[G:G + n, G:G + n, G:G + n, :]
    fine.close(); coarse.close()
    return c, x, res.astype(np.float32), resb.astype(np.float32), tc - tb, flux_scale, emf_scale


def test_adam_matches_torch():
    torch = pytest.importorskip("torch")
    c, x, res, resb, dt, fs, es = _captured_sample()
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


@pytest.mark.parametrize("emf", [False, True])
def test_cell_loss_gradient_matches_autograd(emf):
    """With emf the net's EMF outputs correct the edge EMFs and the loss adds the face magnetic-flux residual
    through the curl (E2Flux's stencil) on the periodic grid."""
    torch = pytest.importorskip("torch")
    c, x, res, resb, dt, fs, es = _captured_sample(emf=emf)
    n = res.shape[0]
    p0 = c.params()
    out = torch.tensor(c.forward_host(x), dtype=torch.float32, requires_grad=True)   # (n, n, n, 27)
    # uniform periodic unit cube: face area h^2, volume h^3, edge length h
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
    if emf:
        Ei, Ej, Ek = (out[..., 24 + q] * float(es[q]) * h for q in range(3))
        up = lambda a, d: torch.roll(a, shifts=-1, dims=d)
        df = [up(Ek, 1) - Ek - up(Ej, 2) + Ej, up(Ei, 2) - Ei - up(Ek, 0) + Ek, up(Ej, 0) - Ej - up(Ei, 1) + Ei]
        rb = torch.tensor(resb)
        for d in range(3):
            e = (-float(dt) * df[d] - rb[..., d]) / 1e-4
            loss = loss + (e * e).mean()
    loss.backward()
    gout = out.grad.numpy().copy()
    # the device's training pass: its loss and its parameter gradient at p0
    dev_loss = c.train([0], 1e-6)
    g_train = c.grads().copy()
    assert dev_loss == pytest.approx(float(loss.detach()), rel=1e-3)
    c.set_params(p0)
    g_auto = c.backward_host(x, gout)
    rel = np.linalg.norm(g_train - g_auto) / np.linalg.norm(g_auto)
    assert rel < 1e-2, rel
    c.close()
