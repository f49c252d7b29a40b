"""Device against the oracle on the benchmark configurations at their own sizes.

* Plain FP64 Orszag-Tang, periodic 128x128x4 on [0,1]^2 x [0,4/128], CFL 0.3, run to t = 0.5: the oracle
  runs the whole trajectory; every 50 steps the device is put on the oracle's state and one step of each
  is compared at relative L-infinity <= 1e-10 per variable. A second device problem runs the same
  trajectory free from the same initial state; it must take the same number of steps and end within
  C1_FREE_L1 (relative L1 per variable) of the oracle.
* The 3D blast wave on the warped 256^3 grid: the device builds the grid and the initial state itself and
  runs a few steps; slabs of 16 k-layers (the lower boundary, the blast centre, the upper boundary; full
  i/j extent, so all six zero-gradient boundaries are covered) of its grid and state are loaded into the
  oracle as k-tiles with halo faces (the oracle's k-tiling reproduces the undivided step bit for bit), and
  one step of each is compared on every active cell and face of the slab at <= 1e-10.
* The magnetosphere at its own size, 96x96x128 on the LFM-type grid from r = 2 to 30: the device's own
  set-up (grid, cut-dipole background, initial state) against the oracle's, then four steps through every
  hook from the oracle's state, each re-synchronised and compared at <= 1e-10 per variable.
* DivB against the oracle's DivB on the same state, with and without a background field.
"""
import numpy as np
import pytest

from helpers import (BACKGROUND_NAMES, GRID_NAMES, device_to_oracle, mirror_to_gpu, oracle_and_gpu, per_var_rel,
                     problem, resync)

pytestmark = pytest.mark.gpu
TOL = 1e-10
C1_FREE_L1 = 1e-8


def _rel_l1(a, b):
    """Relative L1 per variable group: density | momentum | energy for Gas, the three components together
    for magFlux (a component that is zero in exact arithmetic, Mz or the K flux of this 2D-like problem, is
    judged against its vector's size, not against its own round-off)."""
    a2 = a.reshape(a.shape[:3] + (-1,), order="F")
    b2 = b.reshape(b.shape[:3] + (-1,), order="F")
    groups = [[0], [1, 2, 3], [4]] if a2.shape[3] == 5 else [[0, 1, 2]]
    return [float(np.abs(a2[..., g] - b2[..., g]).sum() / max(np.abs(b2[..., g]).sum(), 1e-300)) for g in groups]


def test_c1_orszag_tang_to_half(gpu_lib, oracle_lib):
    n, t_end = (128, 128, 4), 0.5
    o, g = oracle_and_gpu("ot", n, tFin=t_end)
    _, model = problem("ot", n, tFin=t_end)
    free = mirror_to_gpu(o, model)
    with g, free:
        free_steps, t = 0, free.status()["t"]
        while t < t_end:
            _, _, t = free.step()
            free_steps += 1
        steps, checks = 0, 0
        while o.scalars()["t"] < t_end:
            if steps % 50 == 0:
                resync(o, g)
                o.step()
                dt, ts, _ = g.step()
                sc = o.scalars()
                assert ts == sc["ts"] and abs(dt - sc["dt"]) <= TOL * sc["dt"]
                for name in ("gas", "magflux", "bxyz"):
                    errs = per_var_rel(g.fetch(name), o.get(name))
                    assert max(errs) <= TOL, (steps, name, errs)
                checks += 1
            else:
                o.step()
            steps += 1
        assert steps == free_steps, (steps, free_steps)
        assert abs(free.status()["t"] - o.scalars()["t"]) <= 1e-12
        l1 = {name: _rel_l1(free.fetch(name), o.get(name)) for name in ("gas", "magflux")}
        print(f"C1: {steps} steps to t = {t_end}, {checks} re-synchronised steps <= {TOL}; free-running end-state "
              f"relative L1 gas {max(l1['gas']):.2e}, magFlux {max(l1['magflux']):.2e}")
        assert max(l1["gas"] + l1["magflux"]) <= C1_FREE_L1, l1
    o.close()


def _slab(a, k0, nk, faces):
    """k-layers of a Fortran-layout array for a k-tile of nk active layers starting at active layer k0."""
    return np.asfortranarray(a[:, :, k0:k0 + nk + 8 + (1 if faces else 0)])


FACE_ARRAYS = ("xyz", "xfc", "face", "edge", "tf", "te", "teb", "magflux", "omagflux")


@pytest.mark.parametrize("n,slabs", [((256, 256, 256), ((0, 16), (120, 16), (240, 16)))], ids=["256cubed"])
def test_c2_warped_blast_slabs_one_step(gpu_lib, oracle_lib, n, slabs):
    import psutil
    from kaiju_b200 import gamera as gm
    from oracle.pyoracle import Oracle
    if psutil.virtual_memory().available < 40 * 2 ** 30:
        pytest.skip("needs ~40 GiB of free host memory for the 256^3 arrays and the oracle slabs")
    okw, model = problem("bw", n)
    xyz = gm.corners_warped(model, okw["bounds"], okw["warp_amp"])
    with gm.GameraGPU.from_corners(model, xyz, "BW") as g:
        del xyz
        g.run_steps(3)
        st = g.status()
        pieces = {s: {} for s in slabs}
        for name in GRID_NAMES + ("gas", "magflux", "bxyz", "ogas", "omagflux", "obxyz"):
            full = g.fetch(name)
            for s in slabs:
                pieces[s][name] = _slab(full, s[0], s[1], name in FACE_ARRAYS)
            del full
        g.step()
        after = {name: g.fetch(name) for name in ("gas", "magflux")}
        for (k0, nk) in slabs:
            bc = [1, 1, 1, 1, 1 if k0 == 0 else 4, 1 if k0 + nk == n[2] else 4]   # zeroGrad or halo
            o = Oracle(n[0], n[1], nk, **dict(okw, bc=bc, no_setup=True))
            for name, arr in pieces[(k0, nk)].items():
                o.set(name, arr)
            o.set_scalars(st["t"], st["dt"], st["dt0"], st["time"], st["otime"], st["ts"])
            o.step()
            nG = 4
            dev_gas = after["gas"][nG:nG + n[0], nG:nG + n[1], k0 + nG:k0 + nG + nk]
            orc_gas = o.get("gas")[nG:nG + n[0], nG:nG + n[1], nG:nG + nk]
            # the faces of the slab's active cells: I faces is..ie+1, J faces js..je+1, K faces ks..ke+1 (the
            # I and J faces of the k layer above the slab are halo faces there, active only on the device)
            omf, em = o.get("magflux"), []
            for d in range(3):
                hi = [n[0] + (d == 0), n[1] + (d == 1), nk + (d == 2)]
                dev = after["magflux"][nG:nG + hi[0], nG:nG + hi[1], k0 + nG:k0 + nG + hi[2], d]
                orc = omf[nG:nG + hi[0], nG:nG + hi[1], nG:nG + hi[2], d]
                em.append(float(np.max(np.abs(dev - orc)) / np.max(np.abs(omf[nG:nG + hi[0], nG:nG + hi[1],
                                                                              nG:nG + hi[2], :]))))
            eg = per_var_rel(dev_gas, orc_gas)
            print(f"C2 slab k {k0}..{k0 + nk - 1}: gas {max(eg):.2e}, magFlux {max(em):.2e}")
            assert max(eg) <= TOL and max(em) <= TOL, (k0, eg, em)
            o.close()


def test_c3_magnetosphere_full_size(gpu_lib, oracle_lib):
    from kaiju_b200 import magnetosphere as ms
    from oracle.pyoracle import Oracle
    n = (96, 96, 128)
    okw, model = problem("msph", n)
    o = Oracle(*n, **okw)
    # the cell-centred field is an average of face fluxes over cell-centre areas: a derived quantity whose
    # rounding is a few ulps of the dipole's 3.1e4 nT at the inner boundary, against the field of the cell
    bounds = dict({name: 1e-12 for name in ("gas", "magflux") + BACKGROUND_NAMES}, bxyz=2e-11)
    with ms.magnetosphere_problem(n) as d:
        errs = {name: max(per_var_rel(d.fetch(name), o.get(name))) for name in bounds}
        print("C3 set-up: " + ", ".join(f"{k} {v:.2e}" for k, v in errs.items()))
        assert all(errs[k] <= bounds[k] for k in bounds), errs
        assert abs(d.status()["dt"] - o.scalars()["dt"]) <= 1e-12 * o.scalars()["dt"]
    g = mirror_to_gpu(o, model)
    with g:
        g.set_magnetosphere(ms.Magnetosphere().code_params())
        for s in range(4):
            o.step()
            g.step()
            errs = {name: max(per_var_rel(g.fetch(name), o.get(name))) for name in ("gas", "magflux", "bxyz")}
            print(f"C3 step {s + 1}: " + ", ".join(f"{k} {v:.2e}" for k, v in errs.items()))
            assert max(errs.values()) <= TOL, (s, errs)
            resync(o, g)
    o.close()


@pytest.mark.parametrize("kind,n,kw", [("bw", (32, 16, 16), {}), ("ot", (32, 32, 4), {}),
                                       ("bw", (32, 16, 16), dict(b0=("dipole", 0.05, (-1.0, 0.1, 0.2)))),
                                       ("lfmbw", (32, 24, 64), dict(b0=("dipole", 2000.0)))],
                         ids=["bw", "ot", "bw_dipole", "lfmbw_dipole"])
def test_divb_matches_oracle(gpu_lib, oracle_lib, kind, n, kw):
    o, g = oracle_and_gpu(kind, n, **kw)
    with g:
        g.run_steps(5)
        device_to_oracle(g, o)
        dev, orc = g.divb(), o.divb()
        mf = g.fetch("magflux")
        flux_scale = float(np.abs(mf).max()) * float(np.prod(n))
        print(f"DivB {kind} {kw}: device {dev:.6e}, oracle {orc:.6e}, flux scale {flux_scale:.3e}")
        assert abs(dev - orc) <= TOL * max(abs(orc), 1e-16 * flux_scale)
        assert dev <= 1e-10 * flux_scale   # div B at round-off
    o.close()
