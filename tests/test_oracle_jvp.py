"""The oracle's forward-mode derivative (orc_jvp), which the product's adjoint is
checked against, pinned on the CPU against central differences of the oracle's own
f64 step on a small dam break (20 steps, walls and splashing included)."""
import numpy as np
import pytest

from helpers import ref_test_params
from physics_b200 import scenes

DT = 0.005
STEPS = 20


def _world(O, sc, v0, stiffness=250.0, visc=3.5):
    p = ref_test_params()
    p.bounds_min, p.bounds_max = sc.bounds_min, sc.bounds_max
    p.stiffness, p.visc_k = stiffness, [visc]
    w = O.OracleWorld(p, threads=O.max_threads())
    w.add_particles(sc.pos, np.full(sc.n, sc.mass), vel=v0)
    return w


def _loss(O, sc, v0, target, **kw):
    w = _world(O, sc, v0, **kw)
    w.step(DT, STEPS)
    return float(np.mean(np.sum((w.get(O.F_POS) - target) ** 2, axis=1)))


@pytest.fixture(scope="module")
def problem():
    sc = scenes.dam_break(6, 8, 6, box=1.6, dt=DT, steps=0)
    rng = np.random.default_rng(9)
    v0 = rng.normal(0.0, 0.1, (sc.n, 3))
    target = sc.pos + np.array([0.5, 0.0, 0.0])
    return sc, v0, target


def _jvp(O, sc, v0, target, dx, dv, dk=0.0, dc=0.0):
    w = _world(O, sc, v0)
    tx, _ = w.jvp(DT, STEPS, dx, dv, dk, dc)
    x = w.get(O.F_POS)
    return float(np.sum(2.0 * (x - target) / sc.n * tx))


def test_jvp_matches_central_differences_in_velocity_and_position(oracle_mod, problem):
    O = oracle_mod
    sc, v0, target = problem
    rng = np.random.default_rng(1)
    eps = 1e-5
    for which in ("vel", "pos"):
        d = rng.normal(size=v0.shape)
        d /= np.linalg.norm(d)
        if which == "vel":
            jvp = _jvp(O, sc, v0, target, np.zeros_like(v0), d)
            fd = (_loss(O, sc, v0 + eps * d, target) - _loss(O, sc, v0 - eps * d, target)) / (2 * eps)
        else:
            jvp = _jvp(O, sc, v0, target, d, np.zeros_like(v0))
            shifted = []
            for sgn in (1, -1):
                s2 = scenes.Scene(sc.name, sc.pos + sgn * eps * d, sc.vel, sc.mass, sc.bounds_min, sc.bounds_max,
                                  sc.dt, sc.steps)
                shifted.append(_loss(O, s2, v0, target))
            fd = (shifted[0] - shifted[1]) / (2 * eps)
        assert abs(jvp - fd) <= 1e-5 * abs(fd) + 1e-12, (which, jvp, fd)


def test_jvp_matches_central_differences_in_parameters(oracle_mod, problem):
    O = oracle_mod
    sc, v0, target = problem
    eps = 1e-4
    jc = _jvp(O, sc, v0, target, np.zeros_like(v0), np.zeros_like(v0), 0.0, 1.0)
    fd = (_loss(O, sc, v0, target, visc=3.5 + eps) - _loss(O, sc, v0, target, visc=3.5 - eps)) / (2 * eps)
    assert abs(jc - fd) <= 1e-5 * abs(fd), (jc, fd)
    # Stiffness: a relative step keeps rounding out of the quotient.
    jk = _jvp(O, sc, v0, target, np.zeros_like(v0), np.zeros_like(v0), 1.0, 0.0)
    h = 250.0 * 1e-4
    fd = (_loss(O, sc, v0, target, stiffness=250.0 + h) - _loss(O, sc, v0, target, stiffness=250.0 - h)) / (2 * h)
    assert abs(jk - fd) <= 1e-3 * abs(fd), (jk, fd)


def test_jvp_leaves_the_primal_unchanged(oracle_mod, problem):
    O = oracle_mod
    sc, v0, target = problem
    a = _world(O, sc, v0)
    a.step(DT, STEPS)
    b = _world(O, sc, v0)
    b.jvp(DT, STEPS, np.ones_like(v0), np.ones_like(v0), 1.0, 1.0)
    assert np.array_equal(a.get(O.F_POS).view(np.uint64), b.get(O.F_POS).view(np.uint64))
    assert np.array_equal(a.get(O.F_VEL).view(np.uint64), b.get(O.F_VEL).view(np.uint64))
