"""The allocation-free DivB entry point agrees with the handle-based one.

gam_divb_noalloc serves callers that cannot allocate device memory (device arrays owned by another
runtime, or code where an allocation would synchronise the device): it takes a device copy of
State%magFlux and a device output word and keeps its only scratch in a static device array. This test
calls it through the C ABI twice in a row, on two problems of different size (the second call runs over
scratch the first one left behind), and checks each total against gam_gpu_divb of the same state.
It runs last (file name) so a failure here does not hide the other GPU tests.
"""
import ctypes as C

import numpy as np
import pytest

from helpers import oracle_and_gpu

pytestmark = pytest.mark.gpu
TOL = 1e-10


def _divb_noalloc(lib, mf_host, n, nG=4):
    import torch
    mf_dev = torch.from_numpy(np.ascontiguousarray(mf_host.reshape(-1, order="F"))).to("cuda")
    out = torch.full((1,), -1.0, dtype=torch.float64, device="cuda")
    rc = lib.gam_divb_noalloc(C.c_void_p(mf_dev.data_ptr()), n[0], n[1], n[2], nG, C.c_void_p(out.data_ptr()))
    torch.cuda.synchronize()
    return rc, float(out.item())


def test_divb_noalloc_matches_handle(gpu_lib, oracle_lib):
    from kaiju_b200 import gamera as gm
    lib = gm.load_library()
    results = []
    for kind, n, steps in (("bw", (32, 16, 16), 4), ("ot", (16, 16, 4), 3)):
        o, g = oracle_and_gpu(kind, n)
        with g:
            g.run_steps(steps)
            ref = g.divb()
            rc, got = _divb_noalloc(lib, g.fetch("magflux"), n)
            assert rc == gm.GAM_OK
            scale = np.abs(g.fetch("magflux")).max() * np.prod(n)
            assert abs(got - ref) <= TOL * max(abs(ref), scale * 1e-16), (kind, got, ref)
            results.append(got)
    assert len(results) == 2


def test_divb_noalloc_rejects_oversize(gpu_lib):
    from kaiju_b200 import gamera as gm
    import torch
    lib = gm.load_library()
    buf = torch.zeros(16, dtype=torch.float64, device="cuda")
    rc = lib.gam_divb_noalloc(C.c_void_p(buf.data_ptr()), 512, 512, 512, 4, C.c_void_p(buf.data_ptr()))
    assert rc == gm.GAM_ERR_ARG
    assert lib.gam_divb_noalloc(None, 16, 16, 16, 4, C.c_void_p(buf.data_ptr())) == gm.GAM_ERR_ARG
