"""The C-ABI library loads and exports every entry point include/gamgpu.h declares (no GPU needed)."""
import ctypes as C
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "gamgpu.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(gam_\w+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    from kaiju_b200 import build as kb, gamera
    kb.build()
    return gamera.load_library()


def test_exports_every_declared_symbol(lib):
    syms = declared_symbols()
    assert len(syms) >= 14
    for s in syms:
        assert hasattr(lib, s), s


def test_python_signatures_cover_header():
    from kaiju_b200 import gamera
    assert set(declared_symbols()) == set(gamera.SIGNATURES)


def test_errstr_and_argument_checks(lib):
    from kaiju_b200 import gamera as gm
    assert gm.errstr(gm.GAM_ERR_NAN).startswith("NaN")
    h = C.c_void_p()
    m = gm.Model(32, 32, 4).to_c()
    # missing arrays: rejected before any CUDA call
    assert lib.gam_gpu_create(C.byref(h), C.byref(m), None, None, None, None, None, None, None, 0.0, 0.0) == gm.GAM_ERR_ARG
    m.doResistive = 1
    g = gm.GridC()
    assert lib.gam_gpu_create(C.byref(h), C.byref(m), C.byref(g), None, None, None, None, None, None, 0.0, 0.0) == gm.GAM_ERR_ARG
    # background requested without the background arrays: rejected before any CUDA call
    import numpy as np
    dummy = np.zeros(8, order="F")
    m = gm.Model(32, 32, 4, doBackground=True).to_c()
    g = gm.GridC()
    for n, _ in gm.GridC._fields_[:11]:
        setattr(g, n, gm._dp(dummy))
    dp = gm._dp(dummy)
    assert lib.gam_gpu_create(C.byref(h), C.byref(m), C.byref(g), dp, dp, dp, dp, dp, dp, 0.0, 0.0) == gm.GAM_ERR_ARG
    assert lib.gam_gpu_step(None, None, None, None) == gm.GAM_ERR_ARG
    assert lib.gam_gpu_fetch(None, b"gas", None, 0) == gm.GAM_ERR_ARG
    # tile switches and the closure's face-target entry points reject null handles before any CUDA call
    assert lib.gam_gpu_set_tile(None, gm.GAM_TILE_TMA, 1) == gm.GAM_ERR_ARG
    assert lib.gam_closure_accum_fine(None, None, 1.0, 1) == gm.GAM_ERR_ARG
    assert lib.gam_closure_set_loss(None, gm.GAM_CLOSURE_LOSS_FACE) == gm.GAM_ERR_ARG
    assert lib.gam_closure_face_stats(None, 0, None, None) == gm.GAM_ERR_ARG
    assert gm.errstr(gm.GAM_ERR_TIMEOUT)


def test_model_defaults_follow_initmodel():
    from kaiju_b200 import gamera as gm
    m = gm.Model(128, 128, 4)
    # CFL default: min(0.5/(pdmb+0.5), MaxCFL) with MaxCFL the single-precision literal 0.3
    assert m.cfl() == float(__import__("numpy").float32(0.3))
    assert gm.Model(64, 64, 1).do25D and not m.do25D
    c = m.to_c()
    assert c.cHogH == 0.25 and c.Ca == gm.HUGE and c.rmeth == gm.GAM_RM_8CENT


def test_corner_generators_match_oracle(oracle_lib):
    import numpy as np
    from kaiju_b200 import gamera as gm
    m = gm.Model(16, 8, 8)
    for grid, amp in (("uniform", 0.0), ("warp", 0.04)):
        o = oracle_lib.Oracle(16, 8, 8, ic="BW", grid=grid, warp_amp=amp, bounds=(-0.5, 0.5) * 3, bc=[1] * 6)
        ref = o.get("xyz")
        mine = gm.corners_uniform(m, (-0.5, 0.5) * 3) if grid == "uniform" else gm.corners_warped(m, (-0.5, 0.5) * 3, amp)
        np.testing.assert_allclose(mine, ref, rtol=0, atol=1e-15)
