"""The closure network's CPU oracle: its torch form follows the device's tap convention (checked against an
explicit loop over the taps), and its gradients against finite differences (no GPU needed)."""
import numpy as np


def test_torch_form_matches_tap_loop():
    import torch
    import torch.nn.functional as F
    from oracle import closure_oracle as co
    rng = np.random.default_rng(0)
    cin, cout = 3, 4
    W = rng.normal(size=(27, cout, cin))
    b = rng.normal(size=cout)
    x = rng.normal(size=(7, 6, 5, cin))
    ref = co.conv_loop(W, b, x)
    Wt = torch.from_numpy(np.ascontiguousarray(W.reshape(3, 3, 3, cout, cin).transpose(3, 4, 0, 1, 2)))
    y = F.conv3d(torch.from_numpy(np.ascontiguousarray(x.transpose(3, 2, 1, 0)))[None], Wt, torch.from_numpy(b))
    got = y[0].numpy().transpose(3, 2, 1, 0)
    assert np.allclose(got, ref, rtol=1e-12, atol=1e-12)


def test_oracle_shapes_and_gradient():
    from oracle import closure_oracle as co
    rng = np.random.default_rng(1)
    n = sum(27 * ci * cout + cout for ci, cout in co.LAYERS)
    p = (rng.normal(size=n) * 0.1).astype(np.float32)
    x = rng.normal(size=(10, 9, 9, 8)).astype(np.float32)
    y = co.net_forward(p, x)
    nout = co.LAYERS[-1][1]
    assert nout == 27 and y.shape == (2, 1, 1, nout)
    g = rng.normal(size=y.shape).astype(np.float32)
    grads = co.net_grads(p, x, g)
    assert grads.shape == (n,)
    # the bias of the output layer enters every output once: its gradient is the sum of gout
    assert np.allclose(grads[-nout:], g.reshape(-1, nout).sum(axis=0), rtol=1e-5, atol=1e-5)
