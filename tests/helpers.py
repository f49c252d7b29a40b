"""Shared helpers: build matched oracle / device problems and compare arrays."""
import numpy as np

GRID_NAMES = ("xyzcc", "xfc", "di", "dj", "dk", "volume", "face", "edge", "tf", "te", "teb", "xyz")
BACKGROUND_NAMES = ("fcb0", "edgb0", "b0", "bflux0", "dpb0")


def rel_linf(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    den = np.max(np.abs(b))
    if den == 0.0:
        return float(np.max(np.abs(a)))
    return float(np.max(np.abs(a - b)) / den)


def per_var_rel(a, b):
    """Relative L-infinity per variable. Vector components share one scale (the largest component),
    so a component that is identically zero in exact arithmetic (Bz, Mz in 2D-like problems) is judged
    against the vector's size, not against its own round-off. Gas-like arrays (5 variables) are grouped
    as density | momentum (3) | energy."""
    if a.ndim == 3:
        return [rel_linf(a, b)]
    a2 = a.reshape(a.shape[:3] + (-1,), order="F")
    b2 = b.reshape(b.shape[:3] + (-1,), order="F")
    nv = a2.shape[3]
    if nv % 5 == 0:
        groups = []
        for base in range(0, nv, 5):
            groups += [[base], [base + 1, base + 2, base + 3], [base + 4]]
    elif nv % 3 == 0:
        groups = [[c, c + 1, c + 2] for c in range(0, nv, 3)]
    else:
        groups = [[v] for v in range(nv)]
    out = []
    for grp in groups:
        den = max(float(np.max(np.abs(b2[..., v]))) for v in grp)
        for v in grp:
            d = float(np.max(np.abs(a2[..., v] - b2[..., v])))
            out.append(d / den if den > 0 else d)
    return out


def problem(kind, n=(32, 32, 4), **kw):
    """Oracle keyword arguments and the matching Model settings for a named test problem."""
    from kaiju_b200 import gamera as gm
    Nip, Njp, Nkp = n
    if kind == "ot":
        okw = dict(ic="OT2D", grid="uniform", bounds=(0.0, 1.0, 0.0, 1.0, 0.0, 4.0 / 128.0 * (Nkp / 4.0)),
                   CFL=0.3, bc=[0] * 6)
        if Nkp == 1:
            okw["bounds"] = (0.0, 1.0, 0.0, 1.0, -0.5, 0.5)
    elif kind == "bw":
        okw = dict(ic="BW", grid="warp", warp_amp=0.04, bounds=(-0.5, 0.5, -0.5, 0.5, -0.5, 0.5),
                   CFL=0.3, bc=[1] * 6)
    elif kind == "lfmbw":
        # the reference's LFM blast-wave deck (tests/gamera/lfmbw.xml) on a spherical LFM-type grid
        okw = dict(ic="LFMBW", grid="lfm", lfm=(10.0, 100.0, 1.03, 0.05), CFL=0.3, pdmb=1.0, rmeth="7UP",
                   dFloor=1e-4, pFloor=1e-6, doBoris=True, Ca=10.0, bc=[3, 3, 2, 2, 0, 0],
                   ring=dict(NumR=4, Nch=[8, 16, 32, 32]), dtActive=True)
    else:
        raise ValueError(kind)
    okw.update(kw)
    mkw = dict(Nip=Nip, Njp=Njp, Nkp=Nkp, CFL=okw["CFL"], bc=tuple(okw["bc"]))
    for k in ("pdmb", "Vd0", "cHogH", "cHogM", "Ca", "doMHD", "doBoris", "rmeth", "doLFMLim", "tFin", "gamma"):
        if k in okw:
            mkw[k] = okw[k]
    if okw.get("b0") is not None:
        mkw["doBackground"] = True
    if okw.get("ring") is not None:
        mkw["ring"] = okw["ring"]
    if okw.get("ic") == "LFMBW":
        mkw["predFixLFM"] = True
        mkw["bwD0"], mkw["bwP0"] = 1.0, 0.1
    for k in ("dFloor", "pFloor"):
        if okw.get(k):
            mkw[k] = okw[k]
    if okw.get("dtActive"):
        mkw["dtActive"] = True
    if okw.get("doBoris"):
        mkw["Ca"] = okw["Ca"]
    mkw.setdefault("tFin", okw.get("tFin", 1.0e30))
    okw.setdefault("tFin", mkw["tFin"])
    return okw, gm.Model(**mkw)


def oracle_and_gpu(kind, n=(32, 32, 4), **kw):
    from oracle.pyoracle import Oracle
    from kaiju_b200 import gamera as gm
    okw, model = problem(kind, n, **kw)
    o = Oracle(*n, **okw)
    names = GRID_NAMES + (BACKGROUND_NAMES if model.doBackground else ())
    grid = {name: o.get(name) for name in names}
    sc = o.scalars()
    g = gm.GameraGPU.from_arrays(model, grid, o.get("gas"), o.get("magflux"), o.get("ogas"), o.get("omagflux"),
                                 sc["time"], sc["otime"], bxyz=o.get("bxyz"), obxyz=o.get("obxyz"))
    g.set_scalars(sc["t"], sc["dt"], sc["dt0"], sc["ts"], sc["time"], sc["otime"])
    return o, g


def resync(o, g):
    """Put the device on exactly the oracle's current state (State, oState and scalars)."""
    sc = o.scalars()
    g.sync_to_device(gas=o.get("gas"), magflux=o.get("magflux"), ogas=o.get("ogas"), omagflux=o.get("omagflux"),
                     time=sc["time"], otime=sc["otime"], bxyz=o.get("bxyz"), obxyz=o.get("obxyz"))
    g.set_scalars(sc["t"], sc["dt"], sc["dt0"], sc["ts"], sc["time"], sc["otime"])
