"""Decaying MHD turbulence initial state on a periodic unit cube (the learned closure's training and
evaluation problem; no counterpart in the reference, whose user ICs live in src/gamera/prob.F90).

Seeded with numpy's default_rng(seed):
  * velocity: each component a real random-phase field with Fourier amplitudes |a(k)| ~ k^(-11/6) on the
    integer wavenumber shell 2 <= |k| <= 16, i.e. a shell spectrum E(k) ~ k^(-5/3); scaled to rms |v| = 0.5
    (rms Mach 0.5 at the sound speed 1 of rho = 1, P = 1/gamma);
  * magnetic field: B = (0, 0, 0.3) plus a field with the same spectrum and rms |dB| = 0.1, built from a
    random vector potential A (|a(k)| ~ k^(-17/6)) on the cell edges, each face flux being the circulation
    of A around the face, so the discrete divergence of every cell vanishes to round-off;
  * rho = 1, P = 1/gamma.
Arrays come out in the solver's Fortran layout with 4 ghost layers filled periodically.
"""
from __future__ import annotations

import numpy as np

NG = 4


def _shell_field(rng, n, kmin, kmax, slope):
    m = np.fft.fftfreq(n, d=1.0 / n)
    mz = np.fft.rfftfreq(n, d=1.0 / n)
    MX, MY, MZ = np.meshgrid(m, m, mz, indexing="ij")
    K = np.sqrt(MX * MX + MY * MY + MZ * MZ)
    shell = (K >= kmin) & (K <= kmax)
    amp = np.where(shell, np.maximum(K, 1.0) ** slope, 0.0)
    ph = rng.uniform(0.0, 2.0 * np.pi, size=K.shape)
    return np.fft.irfftn(amp * np.exp(1j * ph), s=(n, n, n), axes=(0, 1, 2))


def face_fluxes(Ax, Ay, Az, h):
    """Face fluxes (lower faces of each cell, periodic) from edge potentials: A_x[i,j,k] on the x-edge from
    corner (i,j,k), and likewise A_y, A_z; each flux is the circulation around its face."""
    r = np.roll
    Fx = (Ay + r(Az, -1, axis=1) - r(Ay, -1, axis=2) - Az) * h
    Fy = (Az + r(Ax, -1, axis=2) - r(Az, -1, axis=0) - Ax) * h
    Fz = (Ax + r(Ay, -1, axis=0) - r(Ax, -1, axis=1) - Ay) * h
    return Fx, Fy, Fz


def cell_divergence(Fx, Fy, Fz):
    r = np.roll
    return (r(Fx, -1, axis=0) - Fx) + (r(Fy, -1, axis=1) - Fy) + (r(Fz, -1, axis=2) - Fz)


def turbulence_fields(n: int, seed: int, gamma: float = 5.0 / 3.0, kmin: float = 2.0, kmax: float = 16.0,
                      mach: float = 0.5, b0: float = 0.3, brms: float = 0.1):
    """(gas (Ni,Nj,Nk,5), magflux (Ni+1,Nj+1,Nk+1,3)) in Fortran layout with ghosts, and the active
    velocity and face fluxes for inspection."""
    rng = np.random.default_rng(seed)
    h = 1.0 / n
    v = [_shell_field(rng, n, kmin, kmax, -11.0 / 6.0) for _ in range(3)]
    vr = np.sqrt(np.mean(v[0] ** 2 + v[1] ** 2 + v[2] ** 2))
    v = [c * (mach / vr) for c in v]   # sound speed sqrt(gamma * P / rho) = 1
    A = [_shell_field(rng, n, kmin, kmax, -17.0 / 6.0) for _ in range(3)]
    Fx, Fy, Fz = face_fluxes(*A, h)
    bx = 0.5 * (Fx + np.roll(Fx, -1, axis=0)) / h ** 2
    by = 0.5 * (Fy + np.roll(Fy, -1, axis=1)) / h ** 2
    bz = 0.5 * (Fz + np.roll(Fz, -1, axis=2)) / h ** 2
    s = brms / np.sqrt(np.mean(bx ** 2 + by ** 2 + bz ** 2))
    Fx, Fy, Fz = Fx * s, Fy * s, Fz * s
    Fz = Fz + b0 * h * h
    rho = np.ones((n, n, n))
    P = np.full((n, n, n), 1.0 / gamma)
    E = P / (gamma - 1.0) + 0.5 * rho * (v[0] ** 2 + v[1] ** 2 + v[2] ** 2)
    cells = np.stack([rho, rho * v[0], rho * v[1], rho * v[2], E], axis=-1)
    gas = np.asfortranarray(np.pad(cells, ((NG, NG), (NG, NG), (NG, NG), (0, 0)), mode="wrap"))
    faces = np.stack([Fx, Fy, Fz], axis=-1)
    magflux = np.asfortranarray(np.pad(faces, ((NG, NG + 1), (NG, NG + 1), (NG, NG + 1), (0, 0)), mode="wrap"))
    return gas, magflux, (v, (Fx, Fy, Fz))


def turbulence_model(n: int, fixed_dt: bool = False):
    from . import gamera as gm
    return gm.Model(n, n, n, CFL=0.3, tFin=1.0e30, fixedTimestep=fixed_dt,
                    bc=(gm.GAM_BC_PERIODIC,) * 6)


def turbulence_problem(n: int, seed: int, fixed_dt: bool = False):
    """A device problem holding the turbulence state of `seed` at t = 0 (State = oState, Hatch's dt)."""
    from . import gamera as gm
    model = turbulence_model(n, fixed_dt)
    xyz = gm.corners_uniform(model, (0.0, 1.0, 0.0, 1.0, 0.0, 1.0))
    g = gm.GameraGPU.from_corners(model, xyz, "OT2D")
    gas, magflux, _ = turbulence_fields(n, seed)
    g.sync_to_device(gas=gas, magflux=magflux, ogas=gas, omagflux=magflux, time=0.0, otime=0.0)
    g.init_dt()
    return g


def coarse_problem(n: int):
    """A device problem on the n^3 periodic unit cube with a fixed dt (set per step with set_scalars), the
    target of restrictions."""
    from . import gamera as gm
    model = turbulence_model(n, fixed_dt=True)
    xyz = gm.corners_uniform(model, (0.0, 1.0, 0.0, 1.0, 0.0, 1.0))
    return gm.GameraGPU.from_corners(model, xyz, "OT2D")
