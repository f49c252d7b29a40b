"""CPU restatement of the learned flux closure's network, for the tests only (test infrastructure: the
product never imports it). The closure has no counterpart in the reference; this file is its oracle,
written with torch on the CPU in FP32, with the device's BF16 roundings reproduced: the input, the weights,
the hidden pre-activations and the GELU outputs are rounded to BF16, the output layer stays FP32.

Parameter layout (the device's): for each layer, W[27][cout][cin] with tap t = (di+1) + 3(dj+1) + 9(dk+1)
applied as out(i,j,k) += W[t] . in(i+di, j+dj, k+dk), then b[cout]. Layers 8 -> 32 -> 32 -> 32 -> 27,
GELU (the erf form) after the first three. Arrays use the solver's Fortran layout: inputs (Ni,Nj,Nk,8)
with 4 ghost layers, outputs (Nip,Njp,Nkp,27) on the active cells (each layer is a "valid" 3x3x3
convolution, so 4 layers consume exactly the 4 ghost layers).
"""
from __future__ import annotations

import numpy as np

LAYERS = ((8, 32), (32, 32), (32, 32), (32, 27))


def unpack(params: np.ndarray):
    """[(W as torch weight [cout][cin][kd][kh][kw], b)] per layer."""
    import torch
    out, o = [], 0
    for cin, cout in LAYERS:
        n = 27 * cout * cin
        W = np.asarray(params[o:o + n], dtype=np.float32).reshape(3, 3, 3, cout, cin)   # [dk][dj][di]
        o += n
        b = np.asarray(params[o:o + cout], dtype=np.float32)
        o += cout
        out.append((torch.from_numpy(np.ascontiguousarray(W.transpose(3, 4, 0, 1, 2))), torch.from_numpy(b.copy())))
    return out


def _bf16(t):
    import torch
    return t.to(torch.bfloat16).to(torch.float32)


def _to_torch(x: np.ndarray):
    """(Ni,Nj,Nk,C) Fortran -> [1, C, Nk, Nj, Ni]"""
    import torch
    return torch.from_numpy(np.ascontiguousarray(np.asarray(x, dtype=np.float32).transpose(3, 2, 1, 0)))[None]


def _from_torch(y) -> np.ndarray:
    return np.asfortranarray(y[0].detach().numpy().transpose(3, 2, 1, 0))


def forward_graph(params, x, requires_grad=False):
    import torch
    import torch.nn.functional as F
    layers = unpack(params)
    if requires_grad:
        layers = [(W.requires_grad_(True), b.requires_grad_(True)) for W, b in layers]
    h = _bf16(_to_torch(x))
    for l, (W, b) in enumerate(layers):
        z = F.conv3d(h, _bf16(W), b)
        if l < len(layers) - 1:
            h = _bf16(F.gelu(z))
        else:
            h = z
    return h, layers


def net_forward(params: np.ndarray, x: np.ndarray) -> np.ndarray:
    import torch
    with torch.no_grad():
        y, _ = forward_graph(params, x)
    return _from_torch(y)


def net_grads(params: np.ndarray, x: np.ndarray, gout: np.ndarray) -> np.ndarray:
    """d/dparams of sum(out * gout), flattened in the device's parameter order."""
    y, layers = forward_graph(params, x, requires_grad=True)
    g = _to_torch(gout)
    (y * g).sum().backward()
    parts = []
    for W, b in layers:
        parts.append(W.grad.numpy().transpose(2, 3, 4, 0, 1).reshape(-1))
        parts.append(b.grad.numpy())
    return np.concatenate(parts).astype(np.float32)


def conv_loop(W: np.ndarray, b: np.ndarray, x: np.ndarray) -> np.ndarray:
    """One layer by explicit loops over the taps (numpy, FP64): W[27][cout][cin], x (Ni,Nj,Nk,cin) ->
    (Ni-2, Nj-2, Nk-2, cout). Pins the tap convention of the torch form."""
    Ni, Nj, Nk, _ = x.shape
    cout = W.shape[1]
    out = np.zeros((Ni - 2, Nj - 2, Nk - 2, cout))
    for t in range(27):
        di, dj, dk = t % 3 - 1, (t // 3) % 3 - 1, t // 9 - 1
        xs = x[1 + di:Ni - 1 + di, 1 + dj:Nj - 1 + dj, 1 + dk:Nk - 1 + dk, :]
        out += np.einsum("ijkc,oc->ijko", xs, W[t])
    return out + b
