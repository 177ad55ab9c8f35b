"""Benchmark-size checks (1M and 4M particles).

At 1M the oracle still finishes a teacher-forced step in seconds, so the f64
plain step is compared bit for bit.  At 4M the checks are size-independent
properties: the sort is a permutation ordered by (cell, insertion index), the
f64 plain step repeats bit-exactly, and the compensated density stays within
1e-5 of the f64 plain density (itself bit-exact to the oracle)."""
import numpy as np
import pytest

from helpers import assert_bits_equal
from physics_b200 import scenes

pytestmark = [pytest.mark.gpu, pytest.mark.slow]


def _params(sc):
    from physics_b200 import SphParams
    p = SphParams.defaults()
    p.bounds_min, p.bounds_max = sc.bounds_min, sc.bounds_max
    return p


def test_plain_1m_teacher_forced_bit_exact(gpu, oracle_mod):
    O = oracle_mod
    sc = scenes.config("plain_1m")
    p = _params(sc)
    w = gpu.FluidWorld(p)
    w.add_particles(sc.pos, sc.mass)
    w.step(sc.dt, 20)  # develop the state on the GPU, then hand it to the oracle
    ow = O.OracleWorld(p, threads=O.max_threads())
    ow.add_particles(w.pos, w.mass, vel=w.vel)
    ow.step(sc.dt)
    w.step(sc.dt)
    for name, f in (("pos", O.F_POS), ("vel", O.F_VEL), ("rho", O.F_RHO), ("acc", O.F_ACC)):
        assert_bits_equal(getattr(w, name), ow.get(f), f"1M {name}")


def test_4m_comp_density_vs_plain_and_determinism(gpu):
    sc = scenes.config("comp_4m")
    p = _params(sc)
    plain = gpu.FluidWorld(p, "f64")
    plain.add_particles(sc.pos, sc.mass)
    plain.step(sc.dt, 10)
    pos, vel = plain.pos, plain.vel
    comp = gpu.FluidWorld(p, "comp")
    comp.add_particles(pos, sc.mass, vel=vel)
    plain.step(sc.dt)
    comp.step(sc.dt)
    rel = np.max(np.abs(comp.rho - plain.rho) / plain.rho)
    print("4M comp density max rel err vs f64 plain:", rel)
    assert rel <= 1e-5
    # plain repeats bit-exactly from the same state
    again = gpu.FluidWorld(p, "f64")
    again.add_particles(pos, sc.mass, vel=vel)
    again.step(sc.dt)
    assert_bits_equal(again.pos, plain.pos, "4M plain run-to-run")
    assert plain.len() == sc.n and np.isfinite(plain.pos).all()


def test_plain_1m_500_steps_free_running(gpu, oracle_mod):
    """The f64 plain-form configuration: 1,024,000 particles (80x160x80 at spacing h/2,
    bounds [0, 32]^3), dt 0.005, 500 free-running steps, through the column's collapse
    onto the floor (world.rs:183-397).
    * run to run: a second world repeats every bit of the checkpoints and the end state;
    * against the oracle, free-running: the first 10 steps bit for bit;
    * against the oracle, teacher-forced along the whole run: from the GPU state at
      steps 100, 250, 400 and 499 (the last in the collapsed regime) one oracle step
      equals the GPU's next state bit for bit.  Every step being bit-exact is what
      makes the free-running trajectory bit-exact; stepping the oracle itself through
      all 500 collapsing steps takes tens of CPU minutes, so the steps are sampled."""
    O = oracle_mod
    sc = scenes.config("plain_1m")
    p = _params(sc)
    probes = (100, 250, 400, 499)
    keep = set(probes) | {p_ + 1 for p_ in probes} | {10, sc.steps}

    def run():
        w = gpu.FluidWorld(p)
        w.add_particles(sc.pos, sc.mass)
        states, done = {}, 0
        for s in sorted(keep):
            w.step(sc.dt, s - done)
            done = s
            states[s] = (w.pos, w.vel)
        return states

    first = run()
    second = run()
    for s in sorted(keep):
        assert_bits_equal(second[s][0], first[s][0], f"run-to-run pos @{s}")
        assert_bits_equal(second[s][1], first[s][1], f"run-to-run vel @{s}")
    assert np.isfinite(first[sc.steps][0]).all()

    ow = O.OracleWorld(p, threads=O.max_threads())
    ow.add_particles(sc.pos, sc.mass)
    ow.step(sc.dt, 10)
    assert_bits_equal(first[10][0], ow.get(O.F_POS), "free-running pos @10")
    assert_bits_equal(first[10][1], ow.get(O.F_VEL), "free-running vel @10")
    mass = np.full(sc.n, sc.mass)
    for s in probes:
        tw = O.OracleWorld(p, threads=O.max_threads())
        tw.add_particles(first[s][0], mass, vel=first[s][1])
        tw.step(sc.dt)
        assert_bits_equal(first[s + 1][0], tw.get(O.F_POS), f"teacher-forced pos @{s}->{s + 1}")
        assert_bits_equal(first[s + 1][1], tw.get(O.F_VEL), f"teacher-forced vel @{s}->{s + 1}")
