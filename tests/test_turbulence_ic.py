"""The decaying-turbulence initial state (host generator): divergence-free to round-off, the stated rms
Mach number, mean field and spectrum, periodic ghosts."""
import numpy as np


def test_turbulence_ic_properties():
    from kaiju_b200 import turbulence as tu
    n = 48
    gas, magflux, (v, F) = tu.turbulence_fields(n, seed=3)
    # discrete divergence of every cell, against the flux scale
    div = tu.cell_divergence(*F)
    scale = max(np.abs(f).max() for f in F)
    assert np.abs(div).max() <= 1e-13 * scale
    # rms Mach 0.5 at sound speed 1
    assert abs(np.sqrt(np.mean(v[0] ** 2 + v[1] ** 2 + v[2] ** 2)) - 0.5) < 1e-12
    # mean field (0, 0, 0.3), rms of the rest 0.1
    h = 1.0 / n
    assert abs(F[2].mean() / h ** 2 - 0.3) < 1e-12
    assert abs(F[0].mean()) < 1e-12 * scale and abs(F[1].mean()) < 1e-12 * scale
    # ghosts: periodic copies; the face past the last cell repeats the first
    G = 4
    assert np.array_equal(gas[:G], gas[n:n + G]) and np.array_equal(gas[-G:], gas[G:2 * G])
    assert np.array_equal(magflux[G + n], magflux[G])
    assert gas.shape == (n + 8, n + 8, n + 8, 5) and magflux.shape == (n + 9, n + 9, n + 9, 3)


def test_velocity_spectrum_slope():
    from kaiju_b200 import turbulence as tu
    n = 64
    _, _, (v, _) = tu.turbulence_fields(n, seed=0)
    m = np.fft.fftfreq(n, d=1.0 / n)
    MX, MY, MZ = np.meshgrid(m, m, m, indexing="ij")
    K = np.rint(np.sqrt(MX ** 2 + MY ** 2 + MZ ** 2)).astype(int)
    e = sum(np.abs(np.fft.fftn(c)) ** 2 for c in v)
    ks = np.arange(3, 16)
    Ek = np.array([e[K == k].sum() for k in ks])
    slope = np.polyfit(np.log(ks), np.log(Ek), 1)[0]
    assert abs(slope - (-5.0 / 3.0)) < 0.25, slope
    assert e[K < 2].sum() < 1e-20 * e.sum() and e[K > 17].sum() < 1e-20 * e.sum()


def test_seeds_differ_and_repeat():
    from kaiju_b200 import turbulence as tu
    a, _, _ = tu.turbulence_fields(16, seed=1)
    b, _, _ = tu.turbulence_fields(16, seed=1)
    c, _, _ = tu.turbulence_fields(16, seed=2)
    assert np.array_equal(a, b) and not np.array_equal(a, c)
