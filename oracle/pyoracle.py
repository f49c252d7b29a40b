"""ctypes front end of the CPU oracle (oracle/gamera_oracle.cpp) -- test infrastructure only.

Only the tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` use this module,
to check the device results against; the product path never imports it.

Arrays come back in the reference's Fortran layout (column-major, ghosts included), reshaped to numpy
arrays indexed ``[i, j, k, var]`` with ``order='F'`` and zero-based offsets from ``isg``.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libgamora.so")

IC_OT2D, IC_BW, IC_LFMBW, IC_KH, IC_ADV1D, IC_ADV2D, IC_LOOP2D, IC_ALFVEN, IC_MAGSPHERE = range(9)
GRID_UNIFORM, GRID_WARP, GRID_LFM = 0, 1, 2
BC_PERIODIC, BC_ZEROGRAD, BC_LFMPOLE, BC_LFMBW, BC_HALO, BC_ION, BC_WIND = range(7)
# the reference's LFM blast-wave deck (tests/gamera/lfmbw.xml): prob x0, y0, z0, P0, pRat, D0, rC, B0
LFMBW_DECK = (-50.0, 30.0, 0.0, 0.1, 10.0, 1.0, 20.0, 1.0)
RM_8CENT, RM_7UP = 0, 1


class OrcParams(C.Structure):
    _fields_ = [
        ("Nip", C.c_int), ("Njp", C.c_int), ("Nkp", C.c_int),
        ("icType", C.c_int), ("gridType", C.c_int),
        ("xyzBds", C.c_double * 6), ("warpAmp", C.c_double),
        ("CFL", C.c_double), ("gamma", C.c_double), ("pdmb", C.c_double), ("Vd0", C.c_double),
        ("cHogH", C.c_double), ("cHogM", C.c_double), ("Ca", C.c_double), ("tFin", C.c_double),
        ("doMHD", C.c_int), ("doBoris", C.c_int), ("rmeth", C.c_int), ("doLFMLim", C.c_int),
        ("bc", C.c_int * 6), ("nThreads", C.c_int),
        ("b0Type", C.c_int), ("b0", C.c_double * 4),
        ("lfm", C.c_double * 4), ("dFloor", C.c_double), ("pFloor", C.c_double),
        ("doRing", C.c_int), ("ringNumR", C.c_int), ("ringNch", C.c_int * 32), ("ringRecon", C.c_int),
        ("dtActive", C.c_int), ("bw", C.c_double * 8), ("kh", C.c_double * 4), ("prob", C.c_double * 10),
        ("noSetup", C.c_int), ("msph", C.c_double * 24), ("xyzIn", C.POINTER(C.c_double)),
    ]


def build() -> str:
    """Compile the oracle with its Makefile (idempotent)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        L.orc_create.restype = C.c_void_p
        L.orc_create.argtypes = [C.POINTER(OrcParams)]
        L.orc_destroy.argtypes = [C.c_void_p]
        L.orc_step.argtypes = [C.c_void_p]
        L.orc_get_scalars.argtypes = [C.c_void_p, C.POINTER(C.c_double)]
        L.orc_set_scalars.argtypes = [C.c_void_p, C.POINTER(C.c_double)]
        L.orc_size.restype = C.c_long
        L.orc_size.argtypes = [C.c_void_p, C.c_char_p]
        L.orc_get.argtypes = [C.c_void_p, C.c_char_p, C.POINTER(C.c_double)]
        L.orc_set.argtypes = [C.c_void_p, C.c_char_p, C.POINTER(C.c_double)]
        L.orc_bflux2fld.argtypes = [C.c_void_p]
        L.orc_divb.restype = C.c_double
        L.orc_divb.argtypes = [C.c_void_p]
        L.orc_c2p.argtypes = [C.c_double, C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.orc_p2c.argtypes = [C.c_double, C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.orc_norm2.restype = C.c_double
        L.orc_norm2.argtypes = [C.POINTER(C.c_double), C.c_int]
        L.orc_face_integral_area.argtypes = [C.POINTER(C.c_double)] * 6
        L.orc_volume_integral.argtypes = [C.POINTER(C.c_double)] * 3
        L.orc_recon_lr.argtypes = [C.c_int, C.c_double] + [C.POINTER(C.c_double)] * 4
        L.orc_num_threads.restype = C.c_int
        L.orc_slice.restype = C.c_long
        L.orc_slice.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_double)]
        _lib = L
    return _lib


def dptr(a: np.ndarray):
    assert a.dtype == np.float64 and (a.flags["C_CONTIGUOUS"] or a.flags["F_CONTIGUOUS"])
    return a.ctypes.data_as(C.POINTER(C.c_double))


# Shapes (Fortran order, without lower bounds) of every array the oracle exposes
def array_shapes(Nip, Njp, Nkp, nG=4):
    Ni, Nj, Nk = Nip + 2 * nG, Njp + 2 * nG, Nkp + 2 * nG
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


class Oracle:
    """One GAMERA problem on the CPU oracle: Hatch-equivalent setup at construction, stepGamera per step()."""

    def __init__(self, Nip, Njp, Nkp, ic="OT2D", grid="uniform", bounds=None, warp_amp=0.0, CFL=0.3,
                 gamma=5.0 / 3.0, pdmb=0.75, Vd0=0.5, cHogH=0.25, cHogM=0.25, Ca=1.0e12, tFin=1.0e30,
                 doMHD=True, doBoris=False, rmeth="8CENT", doLFMLim=True, bc=None, threads=0, b0=None,
                 lfm=None, dFloor=0.0, pFloor=0.0, ring=None, dtActive=False, bw=LFMBW_DECK,
                 kh=(0.03, 0.1, 0.01, 0), prob=None, xyz=None, no_setup=False, msph=None):
        p = OrcParams()
        p.Nip, p.Njp, p.Nkp = Nip, Njp, Nkp
        p.icType = {"OT2D": IC_OT2D, "BW": IC_BW, "LFMBW": IC_LFMBW, "KH": IC_KH, "ADV1D": IC_ADV1D,
                    "ADV2D": IC_ADV2D, "LOOP2D": IC_LOOP2D, "ALFVEN": IC_ALFVEN, "MAGSPHERE": IC_MAGSPHERE}[ic]
        if msph is not None:   # the magnetosphere's 23 code-unit parameters (GAM_IC_MAGSPHERE order)
            for n, v in enumerate(msph):
                p.msph[n] = v
        if prob is not None:   # the problem's deck values (see CASE_DECKS)
            for n, v in enumerate(prob):
                p.prob[n] = v
        for n in range(4):   # Kelvin-Helmholtz {a, Bx, amp, seed}
            p.kh[n] = kh[n]
        p.gridType = {"uniform": GRID_UNIFORM, "warp": GRID_WARP, "lfm": GRID_LFM}[grid]
        if lfm is not None:   # (r_in, r_out, radial stretch ratio, theta0)
            for n in range(4):
                p.lfm[n] = lfm[n]
        p.dFloor, p.pFloor = dFloor, pFloor
        if ring is not None:  # dict(NumR=..., Nch=[...], recon="PPM"|"PLM"|"PCM")
            p.doRing = 1
            p.ringNumR = ring.get("NumR", 0)
            for n, c in enumerate(ring.get("Nch", [])):
                p.ringNch[n] = c
            p.ringRecon = {"PLM": 0, "PPM": 1, "PCM": 2}[ring.get("recon", "PPM")]
        p.dtActive = int(dtActive)
        p.noSetup = int(no_setup)   # allocate only: metrics, State, oState and scalars come from set()
        for n in range(8):
            p.bw[n] = bw[n]
        if xyz is not None:   # corners of a tile, (Ni+1, Nj+1, Nk+1, 3) Fortran order
            self._xyz = np.asfortranarray(xyz, dtype=np.float64)
            p.xyzIn = self._xyz.ctypes.data_as(C.POINTER(C.c_double))
        if bounds is None:
            bounds = (0.0, 1.0, 0.0, 1.0, 0.0, 1.0)
        for n in range(6):
            p.xyzBds[n] = bounds[n]
        p.warpAmp = warp_amp
        p.CFL, p.gamma, p.pdmb, p.Vd0 = CFL, gamma, pdmb, Vd0
        p.cHogH, p.cHogM, p.Ca, p.tFin = cHogH, cHogM, Ca, tFin
        p.doMHD, p.doBoris = int(doMHD), int(doBoris)
        p.rmeth = {"8CENT": RM_8CENT, "7UP": RM_7UP}[rmeth]
        p.doLFMLim = int(doLFMLim)
        if bc is None:
            bc = [BC_PERIODIC] * 6
        for n in range(6):
            p.bc[n] = bc[n]
        p.nThreads = threads
        # background field: None, ("uniform", bx, by, bz) or ("dipole", M0[, (cx, cy, cz)])
        p.b0Type = 0
        if b0 is not None:
            if b0[0] == "uniform":
                p.b0Type = 1
                p.b0[0], p.b0[1], p.b0[2] = b0[1], b0[2], b0[3]
            elif b0[0] == "dipole":
                p.b0Type = 2
                p.b0[3] = b0[1]
                if len(b0) > 2:
                    p.b0[0], p.b0[1], p.b0[2] = b0[2]
            else:
                raise ValueError(b0)
        self.params = p
        self.shape = (Nip, Njp, Nkp)
        self.h = lib().orc_create(C.byref(p))
        if not self.h:
            raise ValueError("oracle set-up rejected the problem (Nip must be >= 16 and a multiple of 8; ring "
                             "averaging needs Nkp in 8..512 a power of two and fewer rings than Njp)")
        self.shapes = array_shapes(Nip, Njp, Nkp)

    def close(self):
        if self.h:
            lib().orc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step(self, n=1):
        for _ in range(n):
            lib().orc_step(self.h)

    def get(self, name) -> np.ndarray:
        shp = self.shapes[name]
        a = np.zeros(int(np.prod(shp)), dtype=np.float64)
        rc = lib().orc_get(self.h, name.encode(), dptr(a))
        assert rc == 0, name
        return a.reshape(shp, order="F")

    def set(self, name, arr: np.ndarray):
        a = np.asfortranarray(arr, dtype=np.float64).reshape(-1, order="F").copy()
        assert a.size == int(np.prod(self.shapes[name])), name
        rc = lib().orc_set(self.h, name.encode(), dptr(a))
        assert rc == 0, name

    def scalars(self):
        out = np.zeros(7)
        lib().orc_get_scalars(self.h, dptr(out))
        return dict(t=out[0], dt=out[1], dt0=out[2], time=out[3], otime=out[4], ts=int(out[5]), status=int(out[6]))

    def set_scalars(self, t, dt, dt0, time, otime, ts):
        a = np.array([t, dt, dt0, time, otime, float(ts), 0.0])
        lib().orc_set_scalars(self.h, dptr(a))

    def bflux2fld(self):
        lib().orc_bflux2fld(self.h)

    def divb(self) -> float:
        return lib().orc_divb(self.h)

    SLICE_NAMES = ("D", "Vx", "Vy", "Vz", "P", "Cs", "Bx", "By", "Bz", "Pb", "Jx", "Jy", "Jz", "Ex", "Ey", "Ez",
                   "DivB", "DivdB")

    def slice(self, fat=True) -> dict:
        """writeSlc's variables of the current State, active cells, Fortran order: name -> (Nip,Njp,Nkp)."""
        Nip, Njp, Nkp = self.shape
        nv = 13 + (4 + (1 if self.params.b0Type else 0) if fat else 0)
        out = np.zeros(nv * Nip * Njp * Nkp)
        n = lib().orc_slice(self.h, int(fat), dptr(out))
        assert n == out.size
        out = out.reshape((Nip, Njp, Nkp, nv), order="F")
        return {self.SLICE_NAMES[v]: out[..., v] for v in range(nv)}


def c2p(con, gamma=5.0 / 3.0):
    con = np.ascontiguousarray(con, dtype=np.float64)
    out = np.zeros(5)
    lib().orc_c2p(gamma, dptr(con), dptr(out))
    return out


def p2c(prim, gamma=5.0 / 3.0):
    prim = np.ascontiguousarray(prim, dtype=np.float64)
    out = np.zeros(5)
    lib().orc_p2c(gamma, dptr(prim), dptr(out))
    return out
