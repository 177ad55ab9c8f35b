"""The oracle's FluidWorld::couple_points (phy-fluid/src/sph/world.rs:691-752), which the
device coupling is checked against, pinned on the CPU: the reference's own test
(sph/tests.rs:179-212), known answers that follow from the definition, and its
point-after-point semantics."""
import numpy as np

from helpers import assert_bits_equal, ref_test_params

DT = 0.0025


def _fluid(O, steps=15, vel=None):
    """sph/tests.rs:181-192: a resting block of fluid in the +-3 box, 15 steps."""
    p = ref_test_params(gravity=(0.0, -9.81, 0.0))
    w = O.OracleWorld(p)
    w.fill_box((-0.5, -0.5, -0.5), (0.5, 0.5, 0.5), 0.1, 0.05)
    if vel is not None:
        w.set(O.F_VEL, np.tile(np.asarray(vel, np.float64), (len(w), 1)))
    w.step(DT, steps)
    return w, p


def _momentum(O, w):
    return np.sum(w.get(O.F_VEL) * w.get(O.F_MASS)[:, None], axis=0)


def test_buoyancy_upward_and_reaction_downward(oracle_mod):
    """couple_points_buoyancy_upward (sph/tests.rs:179-212)."""
    O = oracle_mod
    w, p = _fluid(O)
    before = _momentum(O, w)
    f = w.couple_points([[0.0, 0.0, 0.0]], [[0.0, 0.0, 0.0]], [0.02], DT, 1.0, p.rest_density)
    assert f[0, 1] > 0.0
    assert (_momentum(O, w) - before)[1] < 0.0


def test_force_and_transfer_known_answers(oracle_mod):
    """With every fluid particle moving at u: v_f = u, f = -g rho0 m/rho_s + (u - v) drag m,
    and each neighbour's velocity changes by -f dt m_j / sum(m)."""
    O = oracle_mod
    u = np.array([0.25, 0.0, -0.5])
    w, p = _fluid(O, steps=0, vel=u)
    v0 = w.get(O.F_VEL)
    m = w.get(O.F_MASS)
    vp, mp, drag, rho_s = np.array([0.1, 0.2, 0.3]), 0.02, 1.5, 800.0
    f = w.couple_points([[0.05, 0.02, -0.03]], [vp], [mp], DT, drag, rho_s)[0]
    g = np.array(p.gravity)
    expect = -g * (p.rest_density * (mp / rho_s)) + (u - vp) * (drag * mp)
    np.testing.assert_allclose(f, expect, rtol=1e-13, atol=1e-15)
    dv = w.get(O.F_VEL) - v0
    moved = np.any(dv != 0.0, axis=1)
    nb = w.neighbors_of_point([0.05, 0.02, -0.03])
    assert set(np.flatnonzero(moved)) <= set(nb.tolist()) and moved.sum() > 0
    msum = m[nb].sum()
    np.testing.assert_allclose(dv[nb], np.outer(m[nb] / msum, -f * DT), rtol=1e-9, atol=1e-18)
    # The reference adds the impulse share to velocities unscaled by mass, so the fluid's
    # momentum changes by -f dt sum(m_j^2) / sum(m_j) (= -f dt m for equal masses).
    dp = np.sum(dv * m[:, None], axis=0)
    np.testing.assert_allclose(dp, -f * DT * np.sum(m[nb] ** 2) / msum, rtol=1e-9, atol=1e-18)


def test_points_outside_bounds_are_skipped(oracle_mod):
    O = oracle_mod
    w, p = _fluid(O, steps=3)
    v0 = w.get(O.F_VEL)
    prior = np.array([[7.0, 8.0, 9.0], [1.0, 2.0, 3.0]])
    f = w.couple_points([[3.5, 0.0, 0.0], [0.0, -3.0 - 1e-9, 0.0]], np.zeros((2, 3)), [0.02, 0.02], DT, 1.0,
                        1000.0, force=prior)
    assert_bits_equal(f, prior, "untouched forces")
    assert_bits_equal(w.get(O.F_VEL), v0, "untouched fluid")


def test_points_are_coupled_one_after_another(oracle_mod):
    """The second point samples the velocities the first one's reaction left; a point with
    no fluid in its 27 cells gets drag toward rest and moves no fluid."""
    O = oracle_mod
    pts = np.array([[0.0, 0.0, 0.0], [0.03, 0.0, 0.0], [2.0, 2.0, 2.0]])
    vel = np.array([[0.0, 0.5, 0.0], [0.2, 0.0, 0.0], [1.0, 0.0, 0.0]])
    mass = np.array([0.02, 0.05, 0.03])
    a, p = _fluid(O, steps=5)
    fa = a.couple_points(pts, vel, mass, DT, 2.0, 900.0)
    b, _ = _fluid(O, steps=5)
    fb = np.concatenate([b.couple_points(pts[k:k + 1], vel[k:k + 1], mass[k:k + 1], DT, 2.0, 900.0)
                         for k in range(3)])
    assert_bits_equal(fa, fb, "forces")
    assert_bits_equal(a.get(O.F_VEL), b.get(O.F_VEL), "fluid velocities")
    c, _ = _fluid(O, steps=5)
    f1 = c.couple_points(pts[1:2], vel[1:2], mass[1:2], DT, 2.0, 900.0)
    assert not np.array_equal(f1[0], fa[1]), "the second point must see the first one's reaction"
    g = np.array(p.gravity)
    assert_bits_equal(fa[2], -g * (p.rest_density * (mass[2] / 900.0)) + (np.zeros(3) - vel[2]) * (2.0 * mass[2]),
                      "empty neighbourhood")
