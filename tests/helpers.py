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
    elif kind == "msph":
        # the magnetosphere of the Earth deck with a constant solar wind (kaiju_b200/magnetosphere.py)
        from kaiju_b200 import magnetosphere as ms
        model = ms.magnetosphere_model(Nip, Njp, Nkp, tFin=kw.pop("tFin", 1.0e30))
        okw = dict(ic="MAGSPHERE", grid="lfm", lfm=ms.GRID, CFL=model.cfl(), pdmb=model.pdmb, rmeth="7UP",
                   dFloor=model.dFloor, pFloor=model.pFloor, doBoris=True, Ca=model.Ca, bc=[5, 6, 2, 2, 0, 0],
                   ring=dict(NumR=0, Nch=[]), dtActive=True, msph=tuple(ms.Magnetosphere().code_params()),
                   tFin=model.tFin)
        okw.update(kw)
        return okw, model
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


def mirror_to_gpu(o, model):
    """A device problem holding exactly the oracle's current Grid, State, oState and scalars."""
    from kaiju_b200 import gamera as gm
    names = GRID_NAMES + (BACKGROUND_NAMES if model.doBackground else ())
    grid = {name: o.get(name) for name in names}
    sc = o.scalars()
    g = gm.GameraGPU.from_arrays(model, grid, o.get("gas"), o.get("magflux"), o.get("ogas"), o.get("omagflux"),
                                 sc["time"], sc["otime"], bxyz=o.get("bxyz"), obxyz=o.get("obxyz"))
    g.set_scalars(sc["t"], sc["dt"], sc["dt0"], sc["ts"], sc["time"], sc["otime"])
    return g


def oracle_and_gpu(kind, n=(32, 32, 4), **kw):
    from oracle.pyoracle import Oracle
    okw, model = problem(kind, n, **kw)
    o = Oracle(*n, **okw)
    return o, mirror_to_gpu(o, model)


def resync(o, g):
    """Put the device on exactly the oracle's current state (State, oState and scalars)."""
    sc = o.scalars()
    g.sync_to_device(gas=o.get("gas"), magflux=o.get("magflux"), ogas=o.get("ogas"), omagflux=o.get("omagflux"),
                     time=sc["time"], otime=sc["otime"], bxyz=o.get("bxyz"), obxyz=o.get("obxyz"))
    g.set_scalars(sc["t"], sc["dt"], sc["dt0"], sc["ts"], sc["time"], sc["otime"])


# ---------------------------------------------------------------- the accuracy cases of testCases.pf
# Decks of the reference's tests/cases/*.xml with the defaults prob.F90 fills in. CFL is the initModel
# default min(0.5/(pdmb+0.5), MaxCFL) with MaxCFL the real(4) 0.3 (init.F90:343-353); every case is
# triply periodic (DefaultBCs, init.F90:541-554) and 2.5D (Nkp = 1, init.F90:612-616).
V0_DIAG = 1.41421356237
CASES = {
    # testAdv1D / testAdv1D_8CENT (testCases.pf:115-180): adv1d.xml, adv1d_8cent.xml; initADV1D sets gamma 1.4
    "adv1d": dict(n=(128, 1, 1), ic="ADV1D", bounds=(-1.0, 1.0, -0.5, 0.5, -0.5, 0.5), pdmb=4.0, rmeth="7UP",
                  doMHD=False, gamma=1.4, tFin=2.0, prob=()),
    "adv1d_8cent": dict(n=(128, 1, 1), ic="ADV1D", bounds=(-1.0, 1.0, -0.5, 0.5, -0.5, 0.5), pdmb=4.0,
                        rmeth="8CENT", doMHD=False, gamma=1.4, tFin=2.0, prob=()),
    # testAdv2D (:61-86): adv2d.xml; prob = {d0, P0, V0, alpha, R0, x0, y0}
    "adv2d": dict(n=(256, 256, 1), ic="ADV2D", bounds=(-0.5, 0.5, -0.5, 0.5, -0.5, 0.5), pdmb=4.0, tFin=1.0,
                  prob=(1.0, 1.0, V0_DIAG, 45.0, 0.3, 0.0, 0.0)),
    # testLoop2D (:33-58): loop2d.xml; prob = {d0, P0, V0, Vz0, alpha, A0, R0, x0, y0}
    "loop2d": dict(n=(256, 256, 1), ic="LOOP2D", bounds=(-0.5, 0.5, -0.5, 0.5, -0.5, 0.5), pdmb=4.0, tFin=1.0,
                   prob=(1.0, 1.0, V0_DIAG, 0.0, 45.0, 1.0e-3, 0.3, 0.0, 0.0)),
    # testAlfven (:89-112): alfven.xml; prob = {d0, P0, B_para, V_para, alp}
    "alfven": dict(n=(128, 256, 1), ic="ALFVEN", bounds=(0.0, 2.0, 0.0, 1.15470053838, -0.5, 0.5), pdmb=0.75,
                   tFin=1.0, prob=(1.0, 0.1, 1.0, 0.0, 1.0471975512)),
    # testOTSym (:183-225): ot2d.xml
    "otsym": dict(n=(128, 128, 1), ic="OT2D", bounds=(0.0, 1.0, 0.0, 1.0, -0.5, 0.5), pdmb=0.75, tFin=1.0,
                  prob=None),
}
# the loop condition of each test: testAdv1D/testOTSym step while t < tFin, the others while tFin - t > 1e-15
CASE_LOOP_LT = ("adv1d", "adv1d_8cent", "otsym")


def case_model(name):
    """(oracle keyword arguments, Model, icPar) of a reference accuracy case."""
    from kaiju_b200 import gamera as gm
    c = dict(CASES[name])
    n = c.pop("n")
    model = gm.Model(Nip=n[0], Njp=n[1], Nkp=n[2], pdmb=c["pdmb"], rmeth=c.get("rmeth", "8CENT"),
                     doMHD=c.get("doMHD", True), gamma=c.get("gamma", 5.0 / 3.0), tFin=c["tFin"],
                     bc=(gm.GAM_BC_PERIODIC,) * 6)
    okw = dict(ic=c["ic"], grid="uniform", bounds=c["bounds"], CFL=model.cfl(), gamma=model.gamma, pdmb=c["pdmb"],
               rmeth=model.rmeth, doMHD=model.doMHD, tFin=c["tFin"], bc=[0] * 6,
               prob=tuple(c["prob"]) if c["prob"] else None)
    return okw, model, c["prob"]


def case_running(name, t):
    tFin = CASES[name]["tFin"]
    return (t < tFin) if name in CASE_LOOP_LT else ((tFin - t) > 1e-15)


def case_properties(name, gas0, mf0, gas1, mf1, nG=4):
    """The quantities testCases.pf asserts on, from the initial and final State (Fortran-layout arrays)."""
    n = CASES[name]["n"]
    if name.startswith("adv1d"):   # L2err = norm2(sD - eD)/(1.0*Nip), active cells
        sD = gas0[nG:nG + n[0], nG:nG + n[1], nG:nG + n[2], 0]
        eD = gas1[nG:nG + n[0], nG:nG + n[1], nG:nG + n[2], 0]
        return {"L2": float(np.sqrt(np.sum((sD - eD) ** 2))) / float(np.float32(n[0])), "L2_max": 7.0e-3}
    if name == "otsym":            # point-reflection symmetry violation dG on the ks slice
        G = gas1[nG:nG + n[0], nG:nG + n[1], nG, :]
        Gp = G[::-1, ::-1, :].copy()
        Gp[..., 1:3] = -Gp[..., 1:3]
        dG = float(np.sum(np.sqrt(np.sum((G - Gp) ** 2, axis=-1)))) / float(np.float32(n[0] * n[1]))
        return {"dG": dG, "dG_max": 1.0e-11}
    if name == "adv2d":            # whole arrays, ghosts included, as the test sums them
        d0, d1 = gas0[..., 0], gas1[..., 0]
        return {"mass": float(abs(d1.sum() - d0.sum()) / d0.sum()), "mass_max": 1.0e-4,
                "L1": float(np.abs(d0 - d1).sum() / d0.sum()), "L1_max": 0.05}
    b0 = np.sqrt(np.sum(mf0 ** 2, axis=-1))   # NORM2(magFlux, 4) on every face index
    b1 = np.sqrt(np.sum(mf1 ** 2, axis=-1))
    lim = (0.005, 0.05) if name == "loop2d" else (0.001, 0.01)
    return {"total": float(abs(b1.sum() - b0.sum()) / b0.sum()), "total_max": lim[0],
            "L1": float(np.abs(b0 - b1).sum() / b0.sum()), "L1_max": lim[1]}


def case_field(name, gas, mf, nG=4, block=8):
    """Block sums (block x block active cells of the ks slice) of the field a case's test looks at:
    density for the hydro cases, |magFlux| of the I and J faces for the field cases, all five Gas
    variables for the OT symmetry case. A compact fingerprint of the final state for fixtures."""
    n = CASES[name]["n"]
    if name in ("loop2d", "alfven"):
        f = np.sqrt(np.sum(mf[nG:nG + n[0], nG:nG + n[1], nG, :2] ** 2, axis=-1))[..., None]
    elif name == "otsym":
        f = gas[nG:nG + n[0], nG:nG + n[1], nG, :]
    else:
        f = gas[nG:nG + n[0], nG:nG + n[1], nG, :1]
    bi, bj = min(block, n[0]), min(block, n[1])
    nb = (n[0] // bi, n[1] // bj)
    return f.reshape(nb[0], bi, nb[1], bj, f.shape[-1]).sum(axis=(1, 3))


def device_to_oracle(g, o):
    """Put the oracle on exactly the device's current state (State, oState and scalars)."""
    for name in ("gas", "magflux", "bxyz", "ogas", "omagflux", "obxyz"):
        o.set(name, g.fetch(name))
    s = g.status()
    o.set_scalars(s["t"], s["dt"], s["dt0"], s["time"], s["otime"], s["ts"])


def case_device(name, from_oracle=None):
    """The device problem of a reference accuracy case: built by the device's own set-up (corners, IC, BCs,
    dt), or mirrored from an oracle problem when one is given."""
    from kaiju_b200 import gamera as gm
    okw, model, prob = case_model(name)
    if from_oracle is not None:
        return mirror_to_gpu(from_oracle, model)
    xyz = gm.corners_uniform(model, CASES[name]["bounds"])
    return gm.GameraGPU.from_corners(model, xyz, CASES[name]["ic"], ic_par=None if prob is None else list(prob))
