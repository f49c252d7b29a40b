"""The closure network's tensor-core kernels (tcgen05 implicit GEMMs) against the CPU oracle: forward
outputs and parameter gradients on random inputs and weights. Both sides round to BF16 at the same
points; the remaining differences are FP32 summation order (which moves a value near a BF16 rounding
boundary to the neighbouring BF16 value, 2^-8 relative in that element) and BF16 rounding of the backward's
intermediate gradients. Measured on a B200: 3.6e-4..4.5e-4 relative L2 forward, 1.3e-3..4.6e-3 per gradient
block; the bounds are 2e-3 (forward) and 1.5e-2 (gradients)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _rand_case(shape, seed):
    from kaiju_b200 import gamera as gm
    Nip, Njp, Nkp = shape
    c = gm.Closure(Nip, Njp, Nkp, seed=seed)
    rng = np.random.default_rng(seed)
    p = c.params()
    p *= 4.0   # larger weights than the initial scale: the output and gradients are far from zero
    c.set_params(p)
    x = rng.normal(size=(Nip + 8, Njp + 8, Nkp + 8, 8)).astype(np.float32)
    return c, p, x


@pytest.mark.parametrize("shape", [(16, 8, 8), (32, 16, 12), (128, 4, 4)])
def test_forward_matches_oracle(shape):
    from oracle import closure_oracle as co
    c, p, x = _rand_case(shape, 3)
    y = c.forward_host(x)
    ref = co.net_forward(p, x)
    rel = np.linalg.norm(y - ref) / np.linalg.norm(ref)
    assert rel < 2e-3, rel
    c.close()


@pytest.mark.parametrize("shape", [(16, 8, 8), (32, 16, 12)])
def test_gradients_match_oracle(shape):
    from kaiju_b200 import gamera as gm
    from oracle import closure_oracle as co
    c, p, x = _rand_case(shape, 5)
    rng = np.random.default_rng(7)
    gout = rng.normal(size=shape + (gm.CLOSURE_OUT,)).astype(np.float32)
    g = c.backward_host(x, gout)
    ref = co.net_grads(p, x, gout)
    o = 0
    for cin, cout in co.LAYERS:
        for n in (27 * cin * cout, cout):
            a, b = g[o:o + n], ref[o:o + n]
            rel = np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30)
            assert rel < 1.5e-2, (cin, cout, n, rel)
            o += n
    c.close()
