"""The learned closure in the solver and its training pipeline on small grids: restriction keeps div B and
the totals, a step with the closure conserves mass and momentum to round-off and keeps div B, a rejected
correction (positivity) gives exactly the plain step, captured residuals match a host restriction, and
training on fine-run samples lowers the held-out loss below the no-correction loss."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
G = 4


def _totals(g):
    gas = g.fetch("gas")[G:-G, G:-G, G:-G]
    return np.array([gas[..., v].sum() for v in range(5)])


def _restrict_host(gas_f):
    a = gas_f[G:-G, G:-G, G:-G]
    n = a.shape[0] // 2
    return a.reshape(n, 2, n, 2, n, 2, 5).mean(axis=(1, 3, 5))


def test_restriction_keeps_divb_and_totals():
    from kaiju_b200 import gamera as gm, turbulence as tu
    fine = tu.turbulence_problem(32, seed=4)
    fine.run_steps(3)
    coarse = tu.coarse_problem(16)
    coarse.restrict_from(fine, gm.GAM_SYNC_STATE)
    tf, tc = _totals(fine), _totals(coarse)
    assert np.allclose(tc * 8.0, tf, rtol=1e-13, atol=1e-12)
    assert abs(coarse.divb()) < 1e-12
    assert np.allclose(coarse.fetch("gas")[G:-G, G:-G, G:-G], _restrict_host(fine.fetch("gas")), rtol=1e-13, atol=1e-14)
    fine.close(); coarse.close()


def _closure_for(n, scale=4.0, seed=1):
    from kaiju_b200 import gamera as gm
    c = gm.Closure(n, n, n, seed=seed)
    p = c.params()
    c.set_params(p * scale)
    c.set_norm(np.array([1, 0, 0, 0, 0.6, 0, 0, 0.3]), np.array([0.1, 0.3, 0.3, 0.3, 0.1, 0.1, 0.1, 0.1]),
               np.full(8, 1e-3), np.ones(5))
    return c


def test_closure_step_conserves_mass_momentum_and_divb():
    from kaiju_b200 import turbulence as tu
    g = tu.turbulence_problem(32, seed=5)
    c = _closure_for(32)
    g.set_closure(c)
    t0 = _totals(g)
    g.run_steps(4)
    t1 = _totals(g)
    assert g.closure_rejects() == 0
    assert abs(t1[0] - t0[0]) <= 1e-13 * abs(t0[0])
    mom = np.abs(g.fetch("gas")[G:-G, G:-G, G:-G, 1:4]).sum()
    assert np.all(np.abs(t1[1:4] - t0[1:4]) <= 1e-13 * mom)
    assert abs(g.divb()) < 1e-12
    # the closure changed the solution (it is not a no-op)
    h = tu.turbulence_problem(32, seed=5)
    h.run_steps(4)
    assert not np.array_equal(g.fetch("gas"), h.fetch("gas"))
    g.set_closure(None)
    g.close(); h.close(); c.close()


def test_emf_corrections_keep_divb_and_change_the_field():
    """The EMF outputs enter through E2Flux: the magnetic field changes against the step without them and
    div B stays at round-off; the gas update (mass and momentum totals) stays conservative."""
    from kaiju_b200 import turbulence as tu
    g = tu.turbulence_problem(32, seed=5)
    h = tu.turbulence_problem(32, seed=5)
    c = _closure_for(32)
    d = _closure_for(32)
    c.set_norm_emf(np.full(3, 1e-3), np.ones(3))
    g.set_closure(c)
    h.set_closure(d)
    t0 = _totals(g)
    g.run_steps(4)
    h.run_steps(4)
    t1 = _totals(g)
    assert g.closure_rejects() == 0
    assert abs(g.divb()) < 1e-12
    assert abs(t1[0] - t0[0]) <= 1e-13 * abs(t0[0])
    dmf = np.abs(g.fetch("magflux") - h.fetch("magflux")).max()
    assert dmf > 1e-9 * np.abs(h.fetch("magflux")).max(), dmf
    g.set_closure(None); h.set_closure(None)
    g.close(); h.close(); c.close(); d.close()


def test_rejected_correction_is_the_plain_step():
    from kaiju_b200 import turbulence as tu
    g = tu.turbulence_problem(32, seed=6)
    h = tu.turbulence_problem(32, seed=6)
    c = _closure_for(32)
    c.set_norm(np.array([1, 0, 0, 0, 0.6, 0, 0, 0.3]), np.array([0.1, 0.3, 0.3, 0.3, 0.1, 0.1, 0.1, 0.1]),
               np.full(8, 1e6), np.ones(5))   # corrections far too large: every step fails positivity
    c.set_norm_emf(np.full(3, 1e6), np.ones(3))   # the EMF corrections are dropped with the rest
    g.set_closure(c)
    g.run_steps(2)
    h.run_steps(2)
    assert g.closure_rejects() == 2
    assert np.array_equal(g.fetch("gas"), h.fetch("gas"))
    assert np.array_equal(g.fetch("magflux"), h.fetch("magflux"))
    g.set_closure(None)
    g.close(); h.close(); c.close()


def test_capture_residual_matches_host_restriction():
    from kaiju_b200 import gamera as gm, turbulence as tu, closure_train as ct
    n = 16
    c = gm.Closure(n, n, n, seed=0)
    c.reserve(1)
    fine = tu.turbulence_problem(2 * n, seed=7)
    coarse = tu.coarse_problem(n)
    coarse.restrict_from(fine, gm.GAM_SYNC_OSTATE)
    ta = fine.status()["time"]
    fine.step(); fine.step()
    tb = fine.status()["time"]
    coarse.restrict_from(fine, gm.GAM_SYNC_STATE)
    c.in_mean, c.in_std = ct.primitive_stats(coarse)
    c.set_norm(c.in_mean, c.in_std, np.ones(8), np.ones(5))
    fine.step(); fine.step()
    tc = fine.status()["time"]
    coarse.set_scalars(tb, tc - tb, 0.0, 1, tb, ta)
    c.capture(0, coarse, fine)
    st = coarse.status()
    assert abs(st["time"] - tc) <= 1e-15 * tc
    res = _restrict_host(fine.fetch("gas")) - coarse.fetch("gas")[G:-G, G:-G, G:-G]
    rms, dt = c.residual_rms(0)
    assert abs(dt - (tc - tb)) <= 1e-15 * dt
    ref = np.sqrt(np.mean(res.reshape(-1, 5) ** 2, axis=0))
    assert np.allclose(rms, ref, rtol=1e-4)   # the device keeps the residual in float
    c.close(); fine.close(); coarse.close()


def test_training_lowers_held_out_loss():
    from kaiju_b200 import gamera as gm, closure_train as ct
    n = 32
    c = gm.Closure(n, n, n, seed=0)
    c.reserve(16)
    tr = ct.collect(c, n, [0, 1], 6, warm=10, gap=2)
    ev = ct.collect(c, n, [64], 4, warm=10, gap=2, slot0=len(tr), set_input_norm=False)
    ct.set_output_norm(c, n, tr)
    before, none = c.eval(ev)
    hist = ct.train(c, tr, epochs=40, lr=2e-3)
    after, none2 = c.eval(ev)
    assert none2 == pytest.approx(none)
    assert hist[-1] < hist[0]
    assert after < 0.9 * none, (before, after, none)
    c.close()


def test_face_target_accounts_for_density_and_momentum_residual():
    """The face target (the two fine steps' fluxes, time-integrated and summed over each coarse face's fine
    sub-faces, over the coarse dt, minus the plain coarse step's flux) reproduces the cell residual of
    density and momentum through the divergence: their updates are flux divergences on both grids. Energy
    is not one (CellMaxwell keeps the pressure), so its mismatch is only reported."""
    from kaiju_b200 import gamera as gm, turbulence as tu, closure_train as ct
    n = 16
    c = gm.Closure(n, n, n, seed=0)
    c.reserve(1)
    fine = tu.turbulence_problem(2 * n, seed=7)
    coarse = tu.coarse_problem(n)
    coarse.restrict_from(fine, gm.GAM_SYNC_OSTATE)
    ta = fine.status()["time"]
    fine.step(); fine.step()
    tb = fine.status()["time"]
    coarse.restrict_from(fine, gm.GAM_SYNC_STATE)
    c.in_mean, c.in_std = ct.primitive_stats(coarse)
    c.set_norm(c.in_mean, c.in_std, np.ones(8), np.ones(5))
    t_prev = tb
    for q in range(2):
        fine.step()
        t_now = fine.status()["time"]
        c.accum_fine(fine, t_now - t_prev, reset=(q == 0))
        t_prev = t_now
    tc = fine.status()["time"]
    coarse.set_scalars(tb, tc - tb, 0.0, 1, tb, ta)
    c.capture(0, coarse, fine)
    rms, rel = c.face_stats(0)
    assert np.all(rms > 0) and np.all(np.isfinite(rel)), (rms, rel)
    assert rel[0] < 1e-3 and max(rel[1:4]) < 1e-3, rel   # float storage of the targets and residuals
    # the face loss with no correction is the mean square of the normalised targets; training lowers it
    c.set_loss(gm.GAM_CLOSURE_LOSS_FACE)
    c.set_norm(c.in_mean, c.in_std, rms, np.ones(5))
    _, none = c.eval([0])
    assert none == pytest.approx(1.0, rel=1e-3)
    first = c.train([0], 1e-3)
    for _ in range(20):
        last = c.train([0], 1e-3)
    assert last < first
    c.close(); fine.close(); coarse.close()
