"""Host-side front end of the B200 GAMERA step (ctypes over include/gamgpu.h).

Mirrors the reference's application object for this path: ``Model`` carries the Model_T knobs and
their defaults (src/gamera/init.F90:312-492), ``corners_*`` generate Grid_T corner arrays the way
genGridXML does (init.F90:572-798), and ``GameraGPU`` is the gamApp_T of the device path:
``step()`` is stepGamera (src/gamera/gamapp.F90:73-94), ``advance(dt)`` is gamAdvanceModel
(src/gamera/gamtypessub.F90:78-94). Arrays crossing the boundary use the reference's Fortran layout
(numpy arrays in order='F', ghosts included).

The compute path is libgamgpu.so (built in-tree by kaiju_b200/build.py); there is no CPU fallback --
loading fails loudly when the library or a GPU is missing.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
import os
from typing import Optional, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgamgpu.so")

GAM_OK, GAM_ERR_NAN, GAM_ERR_DT_COLLAPSE, GAM_ERR_CUDA, GAM_ERR_TIMEOUT, GAM_ERR_UNSUPPORTED, GAM_ERR_ARG = range(7)
GAM_FP64, GAM_FP32FLUX = 0, 1
GAM_BC_PERIODIC, GAM_BC_ZEROGRAD, GAM_BC_LFMPOLE, GAM_BC_LFMBW, GAM_BC_HALO, GAM_BC_ION, GAM_BC_WIND = range(7)
GAM_HALO_STATE, GAM_HALO_OSTATE, GAM_HALO_BXYZ = 1, 2, 4
GAM_RING_PLM, GAM_RING_PPM, GAM_RING_PCM = 0, 1, 2
GAM_RM_8CENT, GAM_RM_7UP = 0, 1
GAM_SYNC_STATE, GAM_SYNC_OSTATE = 1, 2
(GAM_IC_OT2D, GAM_IC_BW, GAM_IC_LFMBW, GAM_IC_KH, GAM_IC_ADV1D, GAM_IC_ADV2D, GAM_IC_LOOP2D, GAM_IC_ALFVEN,
 GAM_IC_MAGSPHERE) = range(9)
GAM_NMSPH = 23
GAM_SLICE_FAT = 1
GAM_B0_UNIFORM, GAM_B0_DIPOLE = 1, 2
GAM_TILE_FLUX_ROWS, GAM_TILE_FUSED_UPDATE, GAM_TILE_TMA, GAM_TILE_STAGE_WAIT = 1, 2, 3, 4
GAM_CLOSURE_LOSS_CELL, GAM_CLOSURE_LOSS_FACE = 0, 1
# closure network outputs per cell: 24 face-flux corrections (direction d, flux v at d*8+v), 3 edge EMF corrections
CLOSURE_OUT = 27
TINY, HUGE = 1.0e-12, 1.0e12


class GamError(RuntimeError):
    def __init__(self, code: int, what: str):
        self.code = code
        super().__init__(f"{what}: {errstr(code)} (code {code})")


class ModelC(C.Structure):
    _fields_ = [
        ("Nip", C.c_int), ("Njp", C.c_int), ("Nkp", C.c_int), ("nG", C.c_int),
        ("gamma", C.c_double), ("CFL", C.c_double), ("pdmb", C.c_double), ("Vd0", C.c_double),
        ("cHogH", C.c_double), ("cHogM", C.c_double), ("Ca", C.c_double), ("dFloor", C.c_double),
        ("pFloor", C.c_double), ("limDT0", C.c_double),
        ("t", C.c_double), ("tFin", C.c_double), ("dt", C.c_double), ("dt0", C.c_double),
        ("ts", C.c_int),
        ("doMHD", C.c_int), ("doBoris", C.c_int), ("do25D", C.c_int), ("doLFMLim", C.c_int),
        ("rmeth", C.c_int), ("fixedTimestep", C.c_int),
        ("doBackground", C.c_int), ("doGrav", C.c_int), ("doResistive", C.c_int), ("doRing", C.c_int),
        ("doMultiF", C.c_int), ("doAB3", C.c_int), ("nSpc", C.c_int), ("hasHooks", C.c_int),
        ("bc", C.c_int * 6),
        ("ringNumR", C.c_int), ("ringNch", C.c_int * 32), ("ringRecon", C.c_int), ("ringDoS", C.c_int),
        ("ringDoE", C.c_int), ("predFixLFM", C.c_int), ("bwD0", C.c_double), ("bwP0", C.c_double),
        ("dtActive", C.c_int),
    ]


class GridC(C.Structure):
    _fields_ = [(n, C.POINTER(C.c_double)) for n in
                ("xyzcc", "xfc", "di", "dj", "dk", "volume", "face", "edge", "Tf", "Te", "Teb",
                 "fcB0", "edgB0", "B0", "bFlux0", "dpB0", "xyz")]


class StatusC(C.Structure):
    _fields_ = [("t", C.c_double), ("dt", C.c_double), ("dt0", C.c_double), ("time", C.c_double),
                ("otime", C.c_double), ("ts", C.c_int), ("status", C.c_int), ("nanCells", C.c_int),
                ("precision", C.c_int), ("kernelLaunches", C.c_longlong)]


# every entry point declared in include/gamgpu.h with its ctypes signature
_DP = C.POINTER(C.c_double)
_FP = C.POINTER(C.c_float)
SIGNATURES = {
    "gam_gpu_create": (C.c_int, [C.POINTER(C.c_void_p), C.POINTER(ModelC), C.POINTER(GridC), _DP, _DP, _DP, _DP, _DP,
                                 _DP, C.c_double, C.c_double]),
    "gam_gpu_create_from_corners": (C.c_int, [C.POINTER(C.c_void_p), C.POINTER(ModelC), _DP, C.c_int]),
    "gam_gpu_slice_count": (C.c_longlong, [C.c_void_p, C.c_uint]),
    "gam_gpu_slice_begin": (C.c_int, [C.c_void_p, C.c_uint, _DP, C.c_longlong]),
    "gam_gpu_slice_wait": (C.c_int, [C.c_void_p]),
    "gam_gpu_slice": (C.c_int, [C.c_void_p, C.c_uint, _DP, C.c_longlong]),
    "gam_gpu_ensemble_create": (C.c_int, [C.POINTER(C.c_void_p), C.POINTER(C.c_void_p), C.c_int]),
    "gam_gpu_ensemble_run_steps": (C.c_int, [C.c_void_p, C.c_int]),
    "gam_gpu_ensemble_run_steps_timed": (C.c_int, [C.c_void_p, C.c_int, _DP]),
    "gam_gpu_ensemble_advance": (C.c_int, [C.c_void_p, C.c_double, C.c_int, C.c_int, C.POINTER(C.c_int)]),
    "gam_gpu_ensemble_destroy": (None, [C.c_void_p]),
    "gam_gpu_set_tile": (C.c_int, [C.c_void_p, C.c_int, C.c_int]),
    "gam_gpu_ensemble_set_queue": (C.c_int, [C.c_void_p, C.c_int]),
    "gam_gpu_ensemble_autotune": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "gam_gpu_create_from_corners_ic": (C.c_int, [C.POINTER(C.c_void_p), C.POINTER(ModelC), _DP, C.c_int, _DP,
                                                 C.c_int]),
    "gam_gpu_create_from_corners_b0": (C.c_int, [C.POINTER(C.c_void_p), C.POINTER(ModelC), _DP, C.c_int, C.c_int,
                                                 _DP]),
    "gam_gpu_step": (C.c_int, [C.c_void_p, _DP, C.POINTER(C.c_int), _DP]),
    "gam_gpu_advance": (C.c_int, [C.c_void_p, C.c_double]),
    "gam_gpu_run_steps": (C.c_int, [C.c_void_p, C.c_int]),
    "gam_gpu_run_steps_timed": (C.c_int, [C.c_void_p, C.c_int, _DP]),
    "gam_gpu_profile_phases": (C.c_int, [C.c_void_p, C.c_int, _DP, C.c_int]),
    "gam_gpu_sync_to_host": (C.c_int, [C.c_void_p, C.c_uint, _DP, _DP, _DP, _DP, _DP]),
    "gam_gpu_sync_to_device": (C.c_int, [C.c_void_p, C.c_uint, _DP, _DP, _DP, _DP, _DP, _DP, C.c_double,
                                         C.c_double]),
    "gam_gpu_get_status": (C.c_int, [C.c_void_p, C.POINTER(StatusC)]),
    "gam_gpu_set_scalars": (C.c_int, [C.c_void_p, C.c_double, C.c_double, C.c_double, C.c_int, C.c_double,
                                      C.c_double]),
    "gam_gpu_divb": (C.c_int, [C.c_void_p, _DP]),
    "gam_gpu_set_precision": (C.c_int, [C.c_void_p, C.c_int]),
    "gam_gpu_fetch": (C.c_int, [C.c_void_p, C.c_char_p, _DP, C.c_longlong]),
    "gam_gpu_destroy": (None, [C.c_void_p]),
    "gam_gpu_errstr": (C.c_char_p, [C.c_int]),
    "gam_divb_noalloc": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p]),
    "gam_tiles_create": (C.c_int, [C.POINTER(C.c_void_p), C.POINTER(C.c_void_p), C.c_int, C.c_int]),
    "gam_tiles_run_steps": (C.c_int, [C.c_void_p, C.c_int]),
    "gam_tiles_run_steps_timed": (C.c_int, [C.c_void_p, C.c_int, _DP]),
    "gam_tiles_destroy": (None, [C.c_void_p]),
    "gam_gpu_stream": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
    "gam_gpu_step_local": (C.c_int, [C.c_void_p, C.c_void_p]),
    "gam_gpu_step_bcs": (C.c_int, [C.c_void_p, C.c_void_p]),
    "gam_gpu_step_ghosts": (C.c_int, [C.c_void_p]),
    "gam_gpu_calcdt_local": (C.c_int, [C.c_void_p, C.c_void_p]),
    "gam_gpu_calcdt_finish": (C.c_int, [C.c_void_p, C.c_void_p]),
    "gam_gpu_halo_bytes": (C.c_int, [C.c_void_p, C.c_int, C.c_uint, C.POINTER(C.c_longlong),
                                     C.POINTER(C.c_longlong)]),
    "gam_gpu_halo_pack": (C.c_int, [C.c_void_p, C.c_int, C.c_uint, C.c_void_p]),
    "gam_gpu_halo_unpack": (C.c_int, [C.c_void_p, C.c_int, C.c_uint, C.c_void_p]),
    "gam_closure_create": (C.c_int, [C.POINTER(C.c_void_p), C.c_int, C.c_int, C.c_int, C.c_ulonglong]),
    "gam_closure_destroy": (None, [C.c_void_p]),
    "gam_closure_num_params": (C.c_longlong, [C.c_void_p]),
    "gam_closure_set_params": (C.c_int, [C.c_void_p, _FP, C.c_longlong]),
    "gam_closure_get_params": (C.c_int, [C.c_void_p, _FP, C.c_longlong]),
    "gam_closure_get_grads": (C.c_int, [C.c_void_p, _FP, C.c_longlong]),
    "gam_closure_forward_host": (C.c_int, [C.c_void_p, _FP, _FP]),
    "gam_closure_backward_host": (C.c_int, [C.c_void_p, _FP, _FP]),
    "gam_closure_set_norm": (C.c_int, [C.c_void_p, _FP, _FP, _FP, _FP]),
    "gam_closure_reserve": (C.c_int, [C.c_void_p, C.c_int]),
    "gam_closure_capture": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]),
    "gam_closure_train": (C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.c_int, C.c_float, _DP]),
    "gam_closure_eval": (C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.c_int, _DP, _DP]),
    "gam_closure_residual_rms": (C.c_int, [C.c_void_p, C.c_int, _DP]),
    "gam_closure_set_norm_emf": (C.c_int, [C.c_void_p, _FP, _FP]),
    "gam_closure_residual_rms_b": (C.c_int, [C.c_void_p, C.c_int, _DP]),
    "gam_closure_accum_fine": (C.c_int, [C.c_void_p, C.c_void_p, C.c_double, C.c_int]),
    "gam_closure_set_loss": (C.c_int, [C.c_void_p, C.c_int]),
    "gam_closure_face_stats": (C.c_int, [C.c_void_p, C.c_int, _DP, _DP]),
    "gam_gpu_set_closure": (C.c_int, [C.c_void_p, C.c_void_p]),
    "gam_gpu_set_magnetosphere": (C.c_int, [C.c_void_p, _DP, C.c_int]),
    "gam_gpu_closure_rejects": (C.c_int, [C.c_void_p, C.POINTER(C.c_int)]),
    "gam_gpu_restrict": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint]),
    "gam_gpu_init_dt": (C.c_int, [C.c_void_p]),
}

_lib = None


def load_library(path: str = LIB_PATH):
    """Load libgamgpu.so; raises if it is missing (no fallback path exists)."""
    global _lib
    if _lib is None:
        if not os.path.exists(path):
            raise RuntimeError(f"libgamgpu.so not built ({path}); run `python kaiju_b200/build.py`")
        L = C.CDLL(path)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def errstr(code: int) -> str:
    try:
        return load_library().gam_gpu_errstr(code).decode()
    except Exception:
        return str(code)


def _dp(a: Optional[np.ndarray]):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags["F_CONTIGUOUS"], "arrays must be float64, Fortran order"
    return a.ctypes.data_as(_DP)


@dataclasses.dataclass
class Model:
    """Model_T knobs used by the step, with the reference's defaults (init.F90:312-492)."""
    Nip: int
    Njp: int
    Nkp: int
    nG: int = 4
    gamma: float = 5.0 / 3.0
    pdmb: float = 0.75
    CFL: Optional[float] = None           # default min(0.5/(pdmb+0.5), MaxCFL); MaxCFL is the real(4) 0.3
    Vd0: float = 0.5
    doHogs: bool = True
    cHogH: float = 0.25
    cHogM: float = 0.25
    Ca: float = HUGE
    dFloor: float = TINY
    pFloor: float = TINY
    limDT0: float = 1.0e-3
    t: float = 0.0
    tFin: float = 1.0
    dt: float = 0.0
    dt0: float = 0.0
    ts: int = 0
    doMHD: bool = True
    doBoris: bool = False
    doLFMLim: bool = True
    rmeth: str = "8CENT"
    fixedTimestep: bool = False
    doBackground: bool = False            # background field B0 (grid arrays fcB0, edgB0, B0, bFlux0, dpB0)
    bc: Sequence[int] = (GAM_BC_PERIODIC,) * 6
    ring: Optional[dict] = None           # ring averaging about the LFM axis: dict(NumR=, Nch=[...], recon="PPM")
    predFixLFM: bool = False              # the LFM blast wave's predictor fix
    bwD0: float = 1.0                     # gas state of GAM_BC_LFMBW shells
    bwP0: float = 0.1
    dtActive: bool = False                # CalcDT over the active cells only

    @property
    def do25D(self) -> bool:
        return self.Nkp == 1

    def cfl(self) -> float:
        if self.CFL is not None:
            return self.CFL
        maxcfl = float(np.float32(0.3))
        return min(0.5 / (self.pdmb + 0.5), maxcfl)

    def to_c(self) -> ModelC:
        m = ModelC()
        m.Nip, m.Njp, m.Nkp, m.nG = self.Nip, self.Njp, self.Nkp, self.nG
        m.gamma, m.CFL, m.pdmb, m.Vd0 = self.gamma, self.cfl(), self.pdmb, self.Vd0
        m.cHogH = self.cHogH if self.doHogs else 0.0
        m.cHogM = self.cHogM if self.doHogs else 0.0
        m.Ca = self.Ca if self.doBoris else HUGE
        m.dFloor, m.pFloor, m.limDT0 = self.dFloor, self.pFloor, self.limDT0
        m.t, m.tFin, m.dt, m.dt0, m.ts = self.t, self.tFin, self.dt, self.dt0, self.ts
        m.doMHD, m.doBoris, m.do25D, m.doLFMLim = int(self.doMHD), int(self.doBoris), int(self.do25D), int(self.doLFMLim)
        m.rmeth = {"8CENT": GAM_RM_8CENT, "8C": GAM_RM_8CENT, "7UP": GAM_RM_7UP}[self.rmeth.upper()]
        m.fixedTimestep = int(self.fixedTimestep)
        m.doBackground = int(self.doBackground)
        for n in range(6):
            m.bc[n] = int(self.bc[n])
        if self.ring is not None:
            NumR, Nch = ring_config(self.Nkp, self.ring.get("NumR", 0), self.ring.get("Nch", ()))
            m.doRing = 1
            m.ringNumR = NumR
            for n, c in enumerate(Nch):
                m.ringNch[n] = c
            m.ringRecon = {"PLM": GAM_RING_PLM, "PPM": GAM_RING_PPM, "PCM": GAM_RING_PCM}[self.ring.get("recon", "PPM")]
            m.ringDoS = m.ringDoE = 1
        m.predFixLFM = int(self.predFixLFM)
        m.bwD0, m.bwP0 = self.bwD0, self.bwP0
        m.dtActive = int(self.dtActive)
        return m

    @property
    def shape(self):
        return (self.Nip + 2 * self.nG, self.Njp + 2 * self.nG, self.Nkp + 2 * self.nG)


# default rings per Np = Nkp (InitRings, ringutils.F90:126-200, the non-aggressive set)
_RING_DEFAULTS = {8: [4], 16: [8], 32: [8, 16], 64: [8, 16, 32, 32], 128: [8, 16, 32, 32, 64, 64, 64, 64],
                  256: [8, 16, 32, 32, 64, 64, 64, 64, 128, 128, 128, 128],
                  512: [8, 16, 32, 32, 64, 64, 64, 64, 128, 128, 128, 128, 256, 256, 256, 256]}


def ring_config(Np: int, NumR: int = 0, Nch=()):
    """Model%Ring%NumR and Nch as InitRings sets them: the table for Np, overridden by ring/Nr, ring/Nc<n>."""
    if Np not in _RING_DEFAULTS:
        raise ValueError(f"ring averaging needs Nkp in {sorted(_RING_DEFAULTS)}")
    NCr = _RING_DEFAULTS[Np]
    NumR = NumR or len(NCr)
    out = []
    for iR in range(1, NumR + 1):
        c = Nch[iR - 1] if iR <= len(Nch) and Nch[iR - 1] else NCr[min(iR, len(NCr)) - 1]
        if Np % c:
            raise ValueError("ring chunk count must divide Nkp")
        out.append(c)
    return NumR, out


def corners_lfm(model: Model, r_in: float, r_out: float, stretch: float, theta0: float) -> np.ndarray:
    """LFM-type spherical corners about the x axis: i -> r (geometric ratio `stretch` from r_in to r_out),
    j -> theta uniform on [theta0, pi - theta0], k -> phi uniform on [0, 2 pi); ghosts continue the formulas
    (theta beyond the axis reflects through it) and repeat exactly with period Nkp in k."""
    Ni, Nj, Nk = model.shape
    g = model.nG
    i = np.arange(-g + 1, model.Nip + g + 2) - 1          # i - is with is = 1
    j = np.arange(-g + 1, model.Njp + g + 2) - 1
    k = np.arange(-g + 1, model.Nkp + g + 2) - 1
    if stretch == 1.0:
        r = r_in + (r_out - r_in) * i / model.Nip
    else:
        dr0 = (r_out - r_in) * (stretch - 1.0) / (stretch ** model.Nip - 1.0)
        r = r_in + dr0 * (np.power(stretch, i.astype(float)) - 1.0) / (stretch - 1.0)
    th = theta0 + j * (np.pi - 2.0 * theta0) / model.Njp
    ph = np.mod(k, model.Nkp) * 2.0 * np.pi / model.Nkp
    R, TH, PH = np.meshgrid(r, th, ph, indexing="ij")
    xyz = np.zeros((Ni + 1, Nj + 1, Nk + 1, 3), order="F")
    xyz[..., 0] = R * np.cos(TH)
    xyz[..., 1] = R * np.sin(TH) * np.cos(PH)
    xyz[..., 2] = R * np.sin(TH) * np.sin(PH)
    return xyz


def corners_uniform(model: Model, bounds) -> np.ndarray:
    """Cartesian corners of genGridXML (init.F90:669-731): xyz(isg:ieg+1, jsg:jeg+1, ksg:keg+1, 3)."""
    Ni, Nj, Nk = model.shape
    xmin, xmax, ymin, ymax, zmin, zmax = bounds
    dx = (xmax - xmin) / model.Nip
    dy = (ymax - ymin) / model.Njp
    dz = (zmax - zmin) / model.Nkp
    g = model.nG
    i = np.arange(-g + 1, model.Nip + g + 2)     # Fortran i = isg..ieg+1 with is = 1
    j = np.arange(-g + 1, model.Njp + g + 2)
    k = np.arange(-g + 1, model.Nkp + g + 2)
    x = xmin + (i - 1) * dx
    y = ymin + (j - 1) * dy
    z = zmin + (k - 1) * dz
    xyz = np.zeros((Ni + 1, Nj + 1, Nk + 1, 3), order="F")
    xyz[..., 0] = x[:, None, None]
    xyz[..., 1] = y[None, :, None]
    xyz[..., 2] = z[None, None, :]
    return xyz


def corners_warped(model: Model, bounds, amp: float) -> np.ndarray:
    """Non-orthogonal corners x' = x + a sin(2 pi y) sin(2 pi z), cyclic in (x,y,z), applied to the
    uniform corners; the project-supplied grid of the 3D blast-wave problem."""
    xyz = corners_uniform(model, bounds)
    x, y, z = xyz[..., 0].copy(), xyz[..., 1].copy(), xyz[..., 2].copy()
    tp = 2.0 * np.pi
    xyz[..., 0] = x + amp * np.sin(tp * y) * np.sin(tp * z)
    xyz[..., 1] = y + amp * np.sin(tp * z) * np.sin(tp * x)
    xyz[..., 2] = z + amp * np.sin(tp * x) * np.sin(tp * y)
    return np.asfortranarray(xyz)


def array_shapes(model: Model):
    Ni, Nj, Nk = model.shape
    c = (Ni, Nj, Nk)
    f = (Ni + 1, Nj + 1, Nk + 1)
    return {
        "gas": c + (5,), "ogas": c + (5,), "hgas": c + (5,),
        "magflux": f + (3,), "omagflux": f + (3,), "hmagflux": f + (3,),
        "bxyz": c + (3,), "obxyz": c + (3,), "hbxyz": c + (3,), "efld": c + (3,),
        "gflx": c + (5, 3), "mflx": c + (3, 3), "vf": c + (3,), "dgash": c + (5,), "dgasm": c + (3,),
        "xyz": f + (3,), "xyzcc": c + (3,), "xfc": f + (3, 3), "di": c, "dj": c, "dk": c, "volume": c,
        "tf": f + (9, 3), "te": f + (9, 3), "teb": f + (4, 3), "face": f + (3,), "edge": f + (3,),
        "fcb0": c + (3, 3), "edgb0": c + (2, 3), "b0": c + (3,), "bflux0": c + (3,), "dpb0": c + (3,),
        "smoothe": c + (3,),
    }


BACKGROUND_NAMES = (("fcB0", "fcb0"), ("edgB0", "edgb0"), ("B0", "b0"), ("bFlux0", "bflux0"), ("dpB0", "dpb0"))


class GameraGPU:
    """One GAMERA problem resident on the current CUDA device."""

    def __init__(self, model: Model, handle: C.c_void_p):
        self.model = model
        self.h = handle
        self.shapes = array_shapes(model)

    # ---- construction
    @classmethod
    def from_arrays(cls, model: Model, grid: dict, gas, magflux, ogas, omagflux, time: float, otime: float,
                    bxyz=None, obxyz=None):
        """Drop-in path: the host ran Hatch; mirror its Grid_T/State_T arrays onto the device.
        bxyz/obxyz: State%Bxyz/oState%Bxyz as Hatch left them (None: recompute with bFlux2Fld)."""
        L = load_library()
        keep = {k: np.asfortranarray(v, dtype=np.float64) for k, v in grid.items()}
        g = GridC()
        for cname, key in (("xyzcc", "xyzcc"), ("xfc", "xfc"), ("di", "di"), ("dj", "dj"), ("dk", "dk"),
                           ("volume", "volume"), ("face", "face"), ("edge", "edge"), ("Tf", "tf"), ("Te", "te"),
                           ("Teb", "teb")):
            setattr(g, cname, _dp(keep[key]))
        if model.doBackground:
            for cname, key in BACKGROUND_NAMES:
                setattr(g, cname, _dp(keep[key]))
        if "xyz" in keep:
            g.xyz = _dp(keep["xyz"])
        arrs = [None if a is None else np.asfortranarray(a, dtype=np.float64)
                for a in (gas, magflux, bxyz, ogas, omagflux, obxyz)]
        h = C.c_void_p()
        m = model.to_c()
        rc = L.gam_gpu_create(C.byref(h), C.byref(m), C.byref(g), *[_dp(a) for a in arrs], time, otime)
        if rc:
            raise GamError(rc, "gam_gpu_create")
        return cls(model, h)

    @classmethod
    def from_corners(cls, model: Model, xyz: np.ndarray, ic: str, b0=None, ic_par=None):
        """Corners2Grid + initial condition (+ AddB0) + initial BCs/dt on the device.
        b0: None, ("uniform", bx, by, bz) or ("dipole", M0[, (cx, cy, cz)]); needs model.doBackground."""
        L = load_library()
        xyz = np.asfortranarray(xyz, dtype=np.float64)
        h = C.c_void_p()
        m = model.to_c()
        icn = {"OT2D": GAM_IC_OT2D, "BW": GAM_IC_BW, "LFMBW": GAM_IC_LFMBW, "KH": GAM_IC_KH, "ADV1D": GAM_IC_ADV1D,
               "ADV2D": GAM_IC_ADV2D, "LOOP2D": GAM_IC_LOOP2D, "ALFVEN": GAM_IC_ALFVEN,
               "MAGSPHERE": GAM_IC_MAGSPHERE}[ic]
        if icn == GAM_IC_ADV1D and ic_par is None:
            ic_par = np.zeros(0)
        if ic_par is not None:
            par = np.ascontiguousarray(ic_par, dtype=np.float64)
            rc = L.gam_gpu_create_from_corners_ic(C.byref(h), C.byref(m), _dp(xyz), icn, par.ctypes.data_as(_DP),
                                                  len(par))
        elif b0 is None:
            rc = L.gam_gpu_create_from_corners(C.byref(h), C.byref(m), _dp(xyz), icn)
        else:
            par = np.zeros(4)
            if b0[0] == "uniform":
                kind = GAM_B0_UNIFORM
                par[:3] = b0[1:4]
            elif b0[0] == "dipole":
                kind = GAM_B0_DIPOLE
                par[3] = b0[1]
                if len(b0) > 2:
                    par[:3] = b0[2]
            else:
                raise ValueError(b0)
            rc = L.gam_gpu_create_from_corners_b0(C.byref(h), C.byref(m), _dp(xyz), icn, kind,
                                                  par.ctypes.data_as(_DP))
        if rc:
            raise GamError(rc, "gam_gpu_create_from_corners")
        return cls(model, h)

    def close(self):
        if self.h:
            load_library().gam_gpu_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # ---- stepping
    def step(self):
        dt = C.c_double()
        ts = C.c_int()
        t = C.c_double()
        rc = load_library().gam_gpu_step(self.h, C.byref(dt), C.byref(ts), C.byref(t))
        if rc:
            raise GamError(rc, "gam_gpu_step")
        return dt.value, ts.value, t.value

    def advance(self, dt: float):
        rc = load_library().gam_gpu_advance(self.h, dt)
        if rc:
            raise GamError(rc, "gam_gpu_advance")

    def run_steps(self, n: int, check: bool = True) -> int:
        rc = load_library().gam_gpu_run_steps(self.h, n)
        if rc and check:
            raise GamError(rc, "gam_gpu_run_steps")
        return rc

    def run_steps_timed(self, n: int):
        """n graph-replayed steps timed with CUDA events on the library's stream; returns (ms, status)."""
        ms = C.c_double()
        rc = load_library().gam_gpu_run_steps_timed(self.h, n, C.byref(ms))
        if rc not in (GAM_OK, GAM_ERR_NAN, GAM_ERR_DT_COLLAPSE):
            raise GamError(rc, "gam_gpu_run_steps_timed")
        return ms.value, rc

    PHASES = ("predictor", "efield", "fluxes", "deltas", "update", "calcdt", "bcs")

    def profile_phases(self, nsteps: int = 2) -> dict:
        out = np.zeros(7)
        rc = load_library().gam_gpu_profile_phases(self.h, nsteps, _dp(np.asfortranarray(out)), 7)
        if rc not in (GAM_OK, GAM_ERR_NAN, GAM_ERR_DT_COLLAPSE):
            raise GamError(rc, "gam_gpu_profile_phases")
        return dict(zip(self.PHASES, out.tolist()))

    def set_precision(self, mode: int):
        rc = load_library().gam_gpu_set_precision(self.h, mode)
        if rc:
            raise GamError(rc, "gam_gpu_set_precision")

    # ---- data movement
    def fetch(self, name: str) -> np.ndarray:
        shp = self.shapes[name]
        out = np.zeros(shp, order="F")
        rc = load_library().gam_gpu_fetch(self.h, name.encode(), _dp(out), out.size)
        if rc:
            raise GamError(rc, f"gam_gpu_fetch({name})")
        return out

    def sync_to_host(self, gas=None, magflux=None, bxyz=None, ogas=None, omagflux=None):
        what = (GAM_SYNC_STATE if any(a is not None for a in (gas, magflux, bxyz)) else 0) | \
               (GAM_SYNC_OSTATE if any(a is not None for a in (ogas, omagflux)) else 0)
        rc = load_library().gam_gpu_sync_to_host(self.h, what, _dp(gas), _dp(magflux), _dp(bxyz), _dp(ogas),
                                                 _dp(omagflux))
        if rc:
            raise GamError(rc, "gam_gpu_sync_to_host")

    def sync_to_device(self, gas=None, magflux=None, ogas=None, omagflux=None, time=0.0, otime=0.0, bxyz=None,
                       obxyz=None):
        what = (GAM_SYNC_STATE if (gas is not None or magflux is not None) else 0) | \
               (GAM_SYNC_OSTATE if (ogas is not None or omagflux is not None) else 0)
        rc = load_library().gam_gpu_sync_to_device(self.h, what, _dp(gas), _dp(magflux), _dp(bxyz), _dp(ogas),
                                                   _dp(omagflux), _dp(obxyz), time, otime)
        if rc:
            raise GamError(rc, "gam_gpu_sync_to_device")

    def set_scalars(self, t, dt, dt0, ts, time, otime):
        rc = load_library().gam_gpu_set_scalars(self.h, t, dt, dt0, int(ts), time, otime)
        if rc:
            raise GamError(rc, "gam_gpu_set_scalars")

    def status(self) -> dict:
        s = StatusC()
        rc = load_library().gam_gpu_get_status(self.h, C.byref(s))
        if rc:
            raise GamError(rc, "gam_gpu_get_status")
        return dict(t=s.t, dt=s.dt, dt0=s.dt0, time=s.time, otime=s.otime, ts=s.ts, status=s.status,
                    nanCells=s.nanCells, precision=s.precision, kernelLaunches=s.kernelLaunches)

    SLICE_NAMES = ("D", "Vx", "Vy", "Vz", "P", "Cs", "Bx", "By", "Bz", "Pb", "Jx", "Jy", "Jz", "Ex", "Ey", "Ez",
                   "DivB", "DivdB")

    def slice(self, fat: bool = True, out: Optional[np.ndarray] = None) -> dict:
        """writeSlc's variables of the current State (active cells): name -> (Nip, Njp, Nkp) Fortran array."""
        L = load_library()
        flags = GAM_SLICE_FAT if fat else 0
        n = L.gam_gpu_slice_count(self.h, flags)
        buf = np.empty(n) if out is None else out
        rc = L.gam_gpu_slice(self.h, flags, buf.ctypes.data_as(_DP), buf.size)
        if rc:
            raise GamError(rc, "gam_gpu_slice")
        m = self.model
        nv = n // (m.Nip * m.Njp * m.Nkp)
        arr = buf[:n].reshape((m.Nip, m.Njp, m.Nkp, nv), order="F")
        return {self.SLICE_NAMES[v]: arr[..., v] for v in range(nv)}

    def set_tile(self, what: int, value: int):
        rc = load_library().gam_gpu_set_tile(self.h, what, value)
        if rc:
            raise GamError(rc, "gam_gpu_set_tile")

    def set_magnetosphere(self, par: np.ndarray):
        """The magnetosphere's hooks and gravity for a problem created from Hatch's arrays
        (gam_gpu_set_magnetosphere); par: kaiju_b200.magnetosphere.Magnetosphere().code_params()."""
        par = np.ascontiguousarray(par, dtype=np.float64)
        rc = load_library().gam_gpu_set_magnetosphere(self.h, par.ctypes.data_as(_DP), len(par))
        if rc:
            raise GamError(rc, "gam_gpu_set_magnetosphere")

    def set_closure(self, closure: Optional["Closure"]):
        rc = load_library().gam_gpu_set_closure(self.h, closure.c if closure is not None else None)
        if rc:
            raise GamError(rc, "gam_gpu_set_closure")
        self._closure = closure   # keep it alive while attached

    def closure_rejects(self) -> int:
        n = C.c_int()
        rc = load_library().gam_gpu_closure_rejects(self.h, C.byref(n))
        if rc:
            raise GamError(rc, "gam_gpu_closure_rejects")
        return n.value

    def restrict_from(self, fine: "GameraGPU", what: int = GAM_SYNC_STATE):
        rc = load_library().gam_gpu_restrict(fine.h, self.h, what)
        if rc:
            raise GamError(rc, "gam_gpu_restrict")

    def init_dt(self):
        rc = load_library().gam_gpu_init_dt(self.h)
        if rc:
            raise GamError(rc, "gam_gpu_init_dt")

    def divb(self) -> float:
        v = C.c_double()
        rc = load_library().gam_gpu_divb(self.h, C.byref(v))
        if rc:
            raise GamError(rc, "gam_gpu_divb")
        return v.value


class Ensemble:
    """Independent problems advanced together: one CUDA graph launch per batch step holds every member's
    step as a concurrent branch (gam_gpu_ensemble_*). The members stay owned by the caller."""

    def __init__(self, members: Sequence[GameraGPU]):
        L = load_library()
        self.members = list(members)
        arr = (C.c_void_p * len(self.members))(*[m.h.value if hasattr(m.h, "value") else m.h for m in self.members])
        self.e = C.c_void_p()
        rc = L.gam_gpu_ensemble_create(C.byref(self.e), arr, len(self.members))
        if rc:
            raise GamError(rc, "gam_gpu_ensemble_create")

    def run_steps(self, n: int) -> int:
        return load_library().gam_gpu_ensemble_run_steps(self.e, n)

    def run_steps_timed(self, n: int):
        ms = C.c_double()
        rc = load_library().gam_gpu_ensemble_run_steps_timed(self.e, n, C.byref(ms))
        return rc, ms.value

    def set_queue(self, on: bool = True):
        """One persistent flux launch over all members' tiles per batch step (gam_gpu_ensemble_set_queue)."""
        rc = load_library().gam_gpu_ensemble_set_queue(self.e, int(on))
        if rc:
            raise GamError(rc, "gam_gpu_ensemble_set_queue")

    def autotune(self, steps: int = 4):
        """Flux tile height per member shape, then per-member flux launches or the tile queue, by timing
        batch steps (the steps advance the run)."""
        rows = (C.c_int * len(self.members))()
        queue = C.c_int()
        rc = load_library().gam_gpu_ensemble_autotune(self.e, steps, rows, C.byref(queue))
        if rc:
            raise GamError(rc, "gam_gpu_ensemble_autotune")
        self.queue = bool(queue.value)
        return list(rows)

    def advance(self, t_end: float, chunk: int = 8, max_steps: int = 1 << 30):
        steps = C.c_int()
        rc = load_library().gam_gpu_ensemble_advance(self.e, t_end, chunk, max_steps, C.byref(steps))
        return rc, steps.value

    def close(self):
        if self.e:
            load_library().gam_gpu_ensemble_destroy(self.e)
            self.e = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class TileGroup:
    """Tiles of one problem split along k, stepped together in this process (gam_tiles_*): the tiles'
    halos are filled from their neighbours and every tile takes the tiles' minimum dt each step. The
    tiles stay owned by the caller and are stepped only through the group."""

    def __init__(self, tiles: Sequence[GameraGPU], periodic_k: bool = False):
        L = load_library()
        self.tiles = list(tiles)
        arr = (C.c_void_p * len(self.tiles))(*[t.h.value if hasattr(t.h, "value") else t.h for t in self.tiles])
        self.g = C.c_void_p()
        rc = L.gam_tiles_create(C.byref(self.g), arr, len(self.tiles), int(periodic_k))
        if rc:
            raise GamError(rc, "gam_tiles_create")

    def run_steps(self, n: int, check: bool = True) -> int:
        rc = load_library().gam_tiles_run_steps(self.g, n)
        if rc and check:
            raise GamError(rc, "gam_tiles_run_steps")
        return rc

    def run_steps_timed(self, n: int):
        ms = C.c_double()
        rc = load_library().gam_tiles_run_steps_timed(self.g, n, C.byref(ms))
        if rc:
            raise GamError(rc, "gam_tiles_run_steps_timed")
        return ms.value

    def close(self):
        if self.g:
            load_library().gam_tiles_destroy(self.g)
            self.g = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _fp(a: np.ndarray):
    assert a.dtype == np.float32 and (a.flags["F_CONTIGUOUS"] or a.ndim == 1), "float32, Fortran order"
    return a.ctypes.data_as(_FP)


class Closure:
    """The learned flux closure's network on the current device for grids of Nip x Njp x Nkp active cells
    (gam_closure_*)."""

    def __init__(self, Nip: int, Njp: int, Nkp: int, seed: int = 0):
        self.shape = (Nip, Njp, Nkp)
        self.c = C.c_void_p()
        rc = load_library().gam_closure_create(C.byref(self.c), Nip, Njp, Nkp, seed)
        if rc:
            raise GamError(rc, "gam_closure_create")
        self.nparams = load_library().gam_closure_num_params(self.c)

    def _call(self, name, *args):
        rc = getattr(load_library(), name)(self.c, *args)
        if rc:
            raise GamError(rc, name)

    def params(self) -> np.ndarray:
        p = np.zeros(self.nparams, dtype=np.float32)
        self._call("gam_closure_get_params", _fp(p), self.nparams)
        return p

    def set_params(self, p: np.ndarray):
        p = np.ascontiguousarray(p, dtype=np.float32)
        self._call("gam_closure_set_params", _fp(p), self.nparams)

    def grads(self) -> np.ndarray:
        g = np.zeros(self.nparams, dtype=np.float32)
        self._call("gam_closure_get_grads", _fp(g), self.nparams)
        return g

    def forward_host(self, x: np.ndarray) -> np.ndarray:
        """x: (Ni, Nj, Nk, 8) float32, ghosts included; returns (Nip, Njp, Nkp, CLOSURE_OUT)."""
        Nip, Njp, Nkp = self.shape
        x = np.asfortranarray(x, dtype=np.float32)
        out = np.zeros((Nip, Njp, Nkp, CLOSURE_OUT), dtype=np.float32, order="F")
        self._call("gam_closure_forward_host", _fp(x), _fp(out))
        return out

    def backward_host(self, x: np.ndarray, gout: np.ndarray) -> np.ndarray:
        x = np.asfortranarray(x, dtype=np.float32)
        gout = np.asfortranarray(gout, dtype=np.float32)
        self._call("gam_closure_backward_host", _fp(x), _fp(gout))
        return self.grads()

    def set_norm(self, in_mean, in_scale, flux_scale, res_scale):
        a = [np.ascontiguousarray(x, dtype=np.float32) for x in (in_mean, in_scale, flux_scale, res_scale)]
        assert [len(x) for x in a] == [8, 8, 8, 5]
        self._call("gam_closure_set_norm", *[_fp(x) for x in a])

    def set_norm_emf(self, emf_scale, res_scale_b):
        """EMF corrections: the EMF on an edge of direction e gains net output 24+e times emf_scale[e] times the
        edge length; the cell loss adds the face magnetic-flux residual of each direction over res_scale_b.
        emf_scale all zero (the default) leaves the EMFs and the loss as without them."""
        a = [np.ascontiguousarray(x, dtype=np.float32) for x in (emf_scale, res_scale_b)]
        assert [len(x) for x in a] == [3, 3]
        self._call("gam_closure_set_norm_emf", *[_fp(x) for x in a])

    def residual_rms_b(self, slot: int):
        """rms over the lower faces of the active cells of a sample's magnetic-flux residual per direction."""
        out = np.zeros(3)
        self._call("gam_closure_residual_rms_b", slot, out.ctypes.data_as(_DP))
        return out

    def reserve(self, n: int):
        self._call("gam_closure_reserve", n)

    def capture(self, slot: int, coarse: "GameraGPU", fine: "GameraGPU"):
        self._call("gam_closure_capture", slot, coarse.h, fine.h)

    def residual_rms(self, slot: int):
        out = np.zeros(6)
        self._call("gam_closure_residual_rms", slot, out.ctypes.data_as(_DP))
        return out[:5], out[5]

    def accum_fine(self, fine: "GameraGPU", weight: float, reset: bool = False):
        """Add weight x the fine problem's last-step fluxes, restricted to the coarse faces, to the next
        capture's face target (gam_closure_accum_fine)."""
        self._call("gam_closure_accum_fine", fine.h, float(weight), int(reset))

    def set_loss(self, mode: int):
        self._call("gam_closure_set_loss", int(mode))

    def face_stats(self, slot: int):
        """(rms of target / area per flux [8], relative mismatch of dt/V div(target) vs the residual [5])"""
        rms, rel = np.zeros(8), np.zeros(5)
        self._call("gam_closure_face_stats", slot, rms.ctypes.data_as(_DP), rel.ctypes.data_as(_DP))
        return rms, rel

    def train(self, slots, lr: float) -> float:
        arr = (C.c_int * len(slots))(*slots)
        loss = C.c_double()
        self._call("gam_closure_train", arr, len(slots), lr, C.byref(loss))
        return loss.value

    def eval(self, slots):
        arr = (C.c_int * len(slots))(*slots)
        a, b = C.c_double(), C.c_double()
        self._call("gam_closure_eval", arr, len(slots), C.byref(a), C.byref(b))
        return a.value, b.value

    def close(self):
        if self.c:
            load_library().gam_closure_destroy(self.c)
            self.c = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ------------------------------------------------------------------ Kelvin-Helmholtz ensemble problem
def kh_model(nx: int, fp32: bool = True, tFin: float = 2.0) -> Model:
    """One member of the Kelvin-Helmholtz ensemble: nx x nx/2 x 4 cells on [0,2] x [0,1] x [0, 8/nx]
    (square cells), periodic in x and z, zero-gradient in y."""
    return Model(nx, nx // 2, 4, CFL=0.3, tFin=tFin,
                 bc=(GAM_BC_PERIODIC, GAM_BC_PERIODIC, GAM_BC_ZEROGRAD, GAM_BC_ZEROGRAD, GAM_BC_PERIODIC,
                     GAM_BC_PERIODIC))


def kh_bounds(nx: int):
    return (0.0, 2.0, 0.0, 1.0, 0.0, 8.0 / nx)


def kh_ensemble_params(n: int = 96, seed: int = 0):
    """Member sizes and IC parameters drawn with numpy's default_rng(seed): nx uniform in {64,128,256,512},
    shear width a ~ U[0.01, 0.05], Bx ~ U[0, 0.2]; Vy noise amplitude 0.01, noise seed = member index."""
    rng = np.random.default_rng(seed)
    nx = rng.choice([64, 128, 256, 512], size=n)
    a = rng.uniform(0.01, 0.05, size=n)
    bx = rng.uniform(0.0, 0.2, size=n)
    return [dict(nx=int(nx[m]), a=float(a[m]), Bx=float(bx[m]), amp=0.01, seed=m) for m in range(n)]


def kh_member(par: dict, fp32: bool = True, tFin: float = 2.0) -> GameraGPU:
    m = kh_model(par["nx"], fp32, tFin)
    g = GameraGPU.from_corners(m, corners_uniform(m, kh_bounds(par["nx"])), "KH",
                               ic_par=(par["a"], par["Bx"], par["amp"], float(par["seed"])))
    if fp32:
        g.set_precision(GAM_FP32FLUX)
    return g
