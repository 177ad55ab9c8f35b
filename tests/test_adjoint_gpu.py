"""Adjoint of the f64 plain step (phy_fluid_step_backward) against the oracle's
forward-mode derivative and against central finite differences.

The loss is the differentiation form's: L = mean_i |x_i(T) - target_i|^2 with
target = initial lattice + (0.5, 0, 0) + N(0, 0.01^2), initial velocities
f32-drawn N(0, 0.1^2).  The oracle's JVP (oracle/sph_oracle.cpp, Jvp) pushes
tangents through the same piecewise-smooth map the adjoint reverses, so the
two agree to rounding; finite differences agree as far as no branch (wall,
neighbour set, max(0, .)) flips inside the +-eps interval."""
import numpy as np
import pytest

from physics_b200 import scenes

pytestmark = pytest.mark.gpu

DT = 0.005


def _problem(dims=(8, 12, 8), box=2.4, seed=5):
    sc = scenes.dam_break(*dims, box=box, dt=DT, steps=0)
    rng = np.random.default_rng(seed)
    v0 = (rng.standard_normal((sc.n, 3), dtype=np.float32) * np.float32(0.1)).astype(np.float64)
    target = sc.pos + np.array([0.5, 0.0, 0.0]) + rng.normal(0.0, 0.01, (sc.n, 3))
    return sc, v0, target


def _params(sc, stiffness=None, visc=None):
    from physics_b200 import SphParams
    p = SphParams.defaults()
    p.bounds_min, p.bounds_max = sc.bounds_min, sc.bounds_max
    if stiffness is not None:
        p.stiffness = stiffness
    if visc is not None:
        p.visc_k = [visc]
    return p


def _gpu_world(gpu, sc, v0, form="f64", **kw):
    w = gpu.FluidWorld(_params(sc, **kw), form)
    w.add_particles(sc.pos, np.full(sc.n, sc.mass), vel=v0)
    return w


def _loss_grad(x, target):
    n = x.shape[0]
    return float(np.mean(np.sum((x - target) ** 2, axis=1))), 2.0 * (x - target) / n


def _adjoint(gpu, sc, v0, target, steps, every, form="f64", **kw):
    w = _gpu_world(gpu, sc, v0, form, **kw)
    w.tape_begin(every)
    w.step(DT, steps)
    L, g = _loss_grad(w.pos, target)
    return w, L, w.step_backward(g, None)


def _loss(gpu, sc, v0, target, steps, form="f64", **kw):
    w = _gpu_world(gpu, sc, v0, form, **kw)
    w.step(DT, steps)
    return _loss_grad(w.pos, target)[0]


def _unit(rng, shape):
    d = rng.normal(size=shape)
    return d / np.linalg.norm(d)


def test_adjoint_matches_oracle_jvp(gpu, oracle_mod):
    O = oracle_mod
    sc, v0, target = _problem()
    steps = 24
    w, L, g = _adjoint(gpu, sc, v0, target, steps, every=5)
    xT = w.pos
    rng = np.random.default_rng(1)
    for k in range(3):
        dv = _unit(rng, v0.shape)
        dx = _unit(rng, v0.shape) if k == 2 else np.zeros_like(v0)
        ow = O.OracleWorld(_params(sc), threads=O.max_threads())
        ow.add_particles(sc.pos, np.full(sc.n, sc.mass), vel=v0)
        tx, _ = ow.jvp(DT, steps, dx, dv)
        assert np.array_equal(ow.get(O.F_POS).view(np.uint64), xT.view(np.uint64))  # same primal, bit for bit
        want = float(np.sum(2.0 * (xT - target) / sc.n * tx))
        got = float(np.sum(g["vel"] * dv) + np.sum(g["pos"] * dx))
        assert abs(got - want) <= 1e-9 * abs(want) + 1e-18, (k, got, want)
    for dk, dc, key in ((1.0, 0.0, "stiffness"), (0.0, 1.0, "visc_k0")):
        ow = O.OracleWorld(_params(sc), threads=O.max_threads())
        ow.add_particles(sc.pos, np.full(sc.n, sc.mass), vel=v0)
        tx, _ = ow.jvp(DT, steps, np.zeros_like(v0), np.zeros_like(v0), dk, dc)
        want = float(np.sum(2.0 * (xT - target) / sc.n * tx))
        assert abs(g[key] - want) <= 1e-8 * abs(want) + 1e-18, (key, g[key], want)


def test_adjoint_checkpoint_interval_changes_no_bit(gpu):
    sc, v0, target = _problem()
    outs = [_adjoint(gpu, sc, v0, target, 17, every)[2] for every in (1, 4, 17, 40)]
    for o in outs[1:]:
        assert np.array_equal(o["vel"].view(np.uint64), outs[0]["vel"].view(np.uint64))
        assert np.array_equal(o["pos"].view(np.uint64), outs[0]["pos"].view(np.uint64))
        assert o["stiffness"] == outs[0]["stiffness"] and o["visc_k0"] == outs[0]["visc_k0"]


def test_adjoint_central_differences(gpu):
    sc, v0, target = _problem()
    steps, eps = 24, 1e-4
    _, _, g = _adjoint(gpu, sc, v0, target, steps, every=6)
    rng = np.random.default_rng(2)
    for _ in range(4):
        d = _unit(rng, v0.shape)
        fd = (_loss(gpu, sc, v0 + eps * d, target, steps) - _loss(gpu, sc, v0 - eps * d, target, steps)) / (2 * eps)
        ad = float(np.sum(g["vel"] * d))
        assert abs(ad - fd) <= 1e-4 * abs(fd), (ad, fd)
    # visc_k[0] (3.5): eps = 1e-4 absolute.
    fd = (_loss(gpu, sc, v0, target, steps, visc=3.5 + eps) - _loss(gpu, sc, v0, target, steps, visc=3.5 - eps)) / (
        2 * eps)
    assert abs(g["visc_k0"] - fd) <= 1e-4 * abs(fd), (g["visc_k0"], fd)
    # stiffness (250): its derivative is small, so a relative step of 1e-4 keeps rounding out of the quotient.
    h = 250.0 * 1e-4
    fd = (_loss(gpu, sc, v0, target, steps, stiffness=250.0 + h) -
          _loss(gpu, sc, v0, target, steps, stiffness=250.0 - h)) / (2 * h)
    assert abs(g["stiffness"] - fd) <= 1e-3 * abs(fd), (g["stiffness"], fd)


def test_backward_keeps_state_and_tape(gpu):
    sc, v0, target = _problem()
    w = _gpu_world(gpu, sc, v0)
    w.tape_begin(4)
    w.step(DT, 9)
    assert w.tape_steps == 9
    before = (w.pos, w.vel, w.rho)
    L, gx = _loss_grad(w.pos, target)
    g1 = w.step_backward(gx, None)
    after = (w.pos, w.vel, w.rho)
    for a, b in zip(before, after):
        assert np.array_equal(a.view(np.uint64), b.view(np.uint64))
    g2 = w.step_backward(gx, None)  # the tape is kept
    assert np.array_equal(g1["vel"].view(np.uint64), g2["vel"].view(np.uint64))
    # Stepping on matches a world that never ran a backward sweep.
    ref = _gpu_world(gpu, sc, v0)
    ref.step(DT, 9)
    w.tape_clear()
    w.step(DT, 5)
    ref.step(DT, 5)
    assert np.array_equal(w.pos.view(np.uint64), ref.pos.view(np.uint64))


def test_tape_argument_errors(gpu):
    from physics_b200 import PhyError
    sc, v0, target = _problem()
    comp = gpu.FluidWorld(_params(sc), "comp")
    comp.set_tuning(comp_tile=0)  # the x-major compensated route has no adjoint
    comp.add_particles(sc.pos, np.full(sc.n, sc.mass))
    with pytest.raises(PhyError):
        comp.tape_begin(5)
    w = _gpu_world(gpu, sc, v0)
    with pytest.raises(PhyError):
        w.step_backward(np.zeros((sc.n, 3)))
    w.tape_begin(5)
    w.step(DT, 2)
    p = w.params
    p.stiffness = 300.0
    w.params = p
    with pytest.raises(PhyError):
        w.step(DT)


def test_gradient_64k_form(gpu):
    """The differentiation form: 64k-particle dam break, 100 steps at dt 0.005, a
    checkpoint every 10 steps; adjoint vs central differences on 4 directions."""
    sc, v0, target = _problem((32, 64, 32), 12.8, seed=64)
    steps, eps = 100, 1e-4
    _, L, g = _adjoint(gpu, sc, v0, target, steps, every=10)
    assert np.all(np.isfinite(g["vel"]))
    rng = np.random.default_rng(3)
    errs = []
    for _ in range(4):
        d = _unit(rng, v0.shape)
        fd = (_loss(gpu, sc, v0 + eps * d, target, steps) - _loss(gpu, sc, v0 - eps * d, target, steps)) / (2 * eps)
        errs.append(abs(float(np.sum(g["vel"] * d)) - fd) / abs(fd))
    print("64k relative errors vs central differences", errs)
    assert max(errs) <= 1e-4, errs


def test_gradient_64k_form_vs_oracle_jvp(gpu, oracle_mod):
    """The 64k differentiation form against the oracle's forward-mode derivative
    along one combined direction (initial velocities, stiffness and visc_k[0])."""
    O = oracle_mod
    sc, v0, target = _problem((32, 64, 32), 12.8, seed=64)
    steps = 100
    w, L, g = _adjoint(gpu, sc, v0, target, steps, every=10)
    xT = w.pos
    d = _unit(np.random.default_rng(4), v0.shape)
    ow = O.OracleWorld(_params(sc), threads=O.max_threads())
    ow.add_particles(sc.pos, np.full(sc.n, sc.mass), vel=v0)
    tx, _ = ow.jvp(DT, steps, np.zeros_like(v0), d, 1.0, 1.0)
    assert np.array_equal(ow.get(O.F_POS).view(np.uint64), xT.view(np.uint64))
    want = float(np.sum(2.0 * (xT - target) / sc.n * tx))
    got = float(np.sum(g["vel"] * d)) + g["stiffness"] + g["visc_k0"]
    print("64k adjoint vs oracle JVP", got, want, abs(got - want) / abs(want))
    assert abs(got - want) <= 1e-8 * abs(want), (got, want)


# ---- the compensated form ----------------------------------------------------------
#
# step_backward on a compensated world differentiates the step map along the
# compensated trajectory: every re-run step first takes an f64 plain recording step
# from the compensated state, then the compensated step, whose outputs replace the
# recorded ones, so the reverse sweep is the adjoint of the exact step map at the states
# the compensated forward visited.  Its gradient differs from the f64 trajectory's by
# the compensated form's own error (about 1e-6 relative per step).  Central differences
# of the compensated forward itself carry its f32 rounding: at eps = 1e-4 they scatter
# by about 1e-3 relative around any smooth gradient (the f64 adjoint's and the
# compensated adjoint's alike), so they are taken at eps = 1e-2 on the small problem,
# and the 64k form is checked against central differences of the smooth f64 map.

def test_comp_adjoint_vs_oracle_jvp_and_interval(gpu, oracle_mod):
    O = oracle_mod
    sc, v0, target = _problem()
    steps = 24
    w, L, g = _adjoint(gpu, sc, v0, target, steps, every=5, form="comp")
    assert np.all(np.isfinite(g["vel"]))
    rng = np.random.default_rng(1)
    for k in range(2):
        dv = _unit(rng, v0.shape)
        ow = O.OracleWorld(_params(sc), threads=O.max_threads())
        ow.add_particles(sc.pos, np.full(sc.n, sc.mass), vel=v0)
        tx, _ = ow.jvp(DT, steps, np.zeros_like(v0), dv, 1.0 if k else 0.0, 1.0 if k else 0.0)
        xo = ow.get(O.F_POS)
        want = float(np.sum(2.0 * (xo - target) / sc.n * tx))
        got = float(np.sum(g["vel"] * dv)) + (g["stiffness"] + g["visc_k0"] if k else 0.0)
        print("comp adjoint vs oracle JVP", got, want, abs(got - want) / abs(want))
        assert abs(got - want) <= 1e-3 * abs(want), (k, got, want)
    # The checkpoint interval changes no bit (the compensated forward repeats exactly).
    g2 = _adjoint(gpu, sc, v0, target, steps, every=7, form="comp")[2]
    assert np.array_equal(g2["vel"].view(np.uint64), g["vel"].view(np.uint64))


def test_comp_adjoint_central_differences_and_state(gpu):
    sc, v0, target = _problem()
    steps = 24
    w, _, g = _adjoint(gpu, sc, v0, target, steps, every=6, form="comp")
    ref = _gpu_world(gpu, sc, v0, "comp")
    ref.step(DT, steps)
    assert np.array_equal(w.pos.view(np.uint64), ref.pos.view(np.uint64)), "state kept by the sweep"
    rng = np.random.default_rng(2)
    errs = []
    for _ in range(4):
        d = _unit(rng, v0.shape)
        for form, eps in (("comp", 1e-2), ("f64", 1e-4)):
            fd = (_loss(gpu, sc, v0 + eps * d, target, steps, form) -
                  _loss(gpu, sc, v0 - eps * d, target, steps, form)) / (2 * eps)
            errs.append((form, abs(float(np.sum(g["vel"] * d)) - fd) / abs(fd)))
    print("comp adjoint vs central differences (compensated eps 1e-2, f64 eps 1e-4)", errs)
    assert max(e for _, e in errs) <= 1e-4, errs


def test_comp_gradient_64k_form(gpu):
    """The differentiation form on the compensated world (64k particles, 100 steps): the
    compensated adjoint against central differences of the f64 map on 4 directions and
    against the f64 adjoint; central differences of the compensated forward are no
    closer to the f64 adjoint than to the compensated one (their scatter is the
    forward's rounding, not the adjoint's)."""
    sc, v0, target = _problem((32, 64, 32), 12.8, seed=64)
    steps, eps = 100, 1e-4
    _, L, g = _adjoint(gpu, sc, v0, target, steps, every=10, form="comp")
    _, _, gf = _adjoint(gpu, sc, v0, target, steps, every=10)
    rel = float(np.linalg.norm(g["vel"] - gf["vel"]) / np.linalg.norm(gf["vel"]))
    rng = np.random.default_rng(3)
    errs, spread = [], []
    for _ in range(4):
        d = _unit(rng, v0.shape)
        fd = (_loss(gpu, sc, v0 + eps * d, target, steps) - _loss(gpu, sc, v0 - eps * d, target, steps)) / (2 * eps)
        errs.append(abs(float(np.sum(g["vel"] * d)) - fd) / abs(fd))
        fc = (_loss(gpu, sc, v0 + 1e-2 * d, target, steps, "comp") -
              _loss(gpu, sc, v0 - 1e-2 * d, target, steps, "comp")) / 2e-2
        spread.append((abs(float(np.sum(g["vel"] * d)) - fc), abs(float(np.sum(gf["vel"] * d)) - fc), abs(fc)))
    print("comp 64k: vs f64 central differences", errs, "vs f64 adjoint", rel,
          "compensated central differences (|comp adj - fd|, |f64 adj - fd|, |fd|)", spread)
    assert max(errs) <= 1e-4, errs
    assert rel <= 1e-5, rel
    for dc, df, f in spread:
        assert dc <= df + 1e-4 * f, spread
