"""The allocation-free DivB entry point agrees with the handle-based one and with the oracle.

gam_divb_noalloc serves callers that cannot allocate device memory (device arrays owned by another
runtime, or code where an allocation would synchronise the device): it takes device copies of
State%magFlux (and of Grid%bFlux0 when the problem has a background field) and a device output word, and
keeps its only scratch in a static device array. This test calls it through the C ABI twice in a row on
problems of different size (the second call runs over scratch the first one left behind) and checks each
total against gam_gpu_divb of the same state and against the oracle's DivB on that state; a dipole
background case checks the bFlux0 term, and its NULL-bFlux0 call equals the magFlux-only sum.
It runs last (file name) so a failure here does not hide the other GPU tests.
"""
import ctypes as C

import numpy as np
import pytest

from helpers import device_to_oracle, oracle_and_gpu

pytestmark = pytest.mark.gpu
TOL = 1e-10


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a.reshape(-1, order="F"))).to("cuda")


def _divb_noalloc(lib, mf_host, bf0_host, n, nG=4):
    import torch
    mf_dev = _dev(mf_host)
    bf_dev = _dev(bf0_host) if bf0_host is not None else None
    out = torch.full((1,), -1.0, dtype=torch.float64, device="cuda")
    rc = lib.gam_divb_noalloc(C.c_void_p(mf_dev.data_ptr()), C.c_void_p(bf_dev.data_ptr()) if bf_dev is not None else None,
                              n[0], n[1], n[2], nG, C.c_void_p(out.data_ptr()))
    torch.cuda.synchronize()
    return rc, float(out.item())


def _face_diffs(f, n, nG=4):
    """Per active cell, the differences lower-minus-upper face value along i, j and k."""
    a = f[nG:nG + n[0] + 1, nG:nG + n[1] + 1, nG:nG + n[2] + 1, :]
    return (a[:-1, :-1, :-1, 0] - a[1:, :-1, :-1, 0], a[:-1, :-1, :-1, 1] - a[:-1, 1:, :-1, 1],
            a[:-1, :-1, :-1, 2] - a[:-1, :-1, 1:, 2])


def _divb_numpy(mf, bf0, n):
    """DivB's per-cell sum in its own order, dFi + dFj + dFk + dFi0 + dFj0 + dFk0, summed over the cells."""
    dFi, dFj, dFk = _face_diffs(mf, n)
    d = dFi + dFj + dFk
    if bf0 is not None:
        dFi0, dFj0, dFk0 = _face_diffs(bf0, n)
        d = d + dFi0 + dFj0 + dFk0
    return float(np.abs(d).sum())


def _close(got, ref, scale):
    return abs(got - ref) <= TOL * max(abs(ref), scale * 1e-16)


def test_divb_noalloc_matches_handle_and_oracle(gpu_lib, oracle_lib):
    from kaiju_b200 import gamera as gm
    lib = gm.load_library()
    cases = (("bw", (32, 16, 16), 4, {}), ("ot", (16, 16, 4), 3, {}),
             ("bw", (32, 16, 16), 3, dict(b0=("dipole", 0.05, (-1.0, 0.1, 0.2)))))
    results = []
    for kind, n, steps, kw in cases:
        o, g = oracle_and_gpu(kind, n, **kw)
        with g:
            g.run_steps(steps)
            device_to_oracle(g, o)
            ref_handle, ref_oracle = g.divb(), o.divb()
            mf = g.fetch("magflux")
            bf0 = g.fetch("bflux0") if kw.get("b0") else None
            rc, got = _divb_noalloc(lib, mf, bf0, n)
            assert rc == gm.GAM_OK
            scale = np.abs(mf).max() * np.prod(n)
            assert _close(got, ref_handle, scale), (kind, kw, got, ref_handle)
            assert _close(got, ref_oracle, scale), (kind, kw, got, ref_oracle)
            assert _close(got, _divb_numpy(mf, bf0, n), scale)
            if bf0 is not None:
                rc, got0 = _divb_noalloc(lib, mf, None, n)   # NULL bFlux0: magFlux alone
                assert rc == gm.GAM_OK
                assert _close(got0, _divb_numpy(mf, None, n), scale), (got0, _divb_numpy(mf, None, n))
            results.append(got)
        o.close()
    assert len(results) == 3


def test_divb_noalloc_rejects_oversize(gpu_lib):
    from kaiju_b200 import gamera as gm
    import torch
    lib = gm.load_library()
    buf = torch.zeros(16, dtype=torch.float64, device="cuda")
    rc = lib.gam_divb_noalloc(C.c_void_p(buf.data_ptr()), None, 512, 512, 512, 4, C.c_void_p(buf.data_ptr()))
    assert rc == gm.GAM_ERR_ARG
    assert lib.gam_divb_noalloc(None, None, 16, 16, 16, 4, C.c_void_p(buf.data_ptr())) == gm.GAM_ERR_ARG
