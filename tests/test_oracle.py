"""CPU oracle checks: golden fixtures, the reference's own SPH property tests
(crates/phy-fluid/src/sph/tests.rs, crates/phy-demo/tests/*.rs) and analytic
known answers.  No GPU involved."""
import math

import numpy as np
import pytest

from helpers import assert_bits_equal, ref_test_params
from physics_b200 import SphParams, scenes


def world(oracle_mod, params=None, threads=1):
    return oracle_mod.OracleWorld(params or SphParams.defaults(), threads=threads)


# ---- golden fixtures (second restatement, tests/golden/gen_golden.py) -------------

def test_golden_quickstart(oracle_mod, golden):
    g = golden("quickstart")
    O = oracle_mod
    w = world(O)
    w.fill_box((-1, 1, -1), (1, 3, 1), 0.3, 0.1)
    assert len(w) == 343
    w.step(0.01)
    for k, f in (("pos", O.F_POS), ("vel", O.F_VEL), ("acc", O.F_ACC), ("rho", O.F_RHO), ("p", O.F_P),
                 ("mu_eff", O.F_MU_EFF), ("xsph", O.F_XSPH), ("mass", O.F_MASS)):
        assert_bits_equal(w.get(f), g[f"step1_{k}"], f"step1 {k}")
    done = 1
    for n in (50, 100, 200):
        w.step(0.01, n - done)
        done = n
        assert_bits_equal(w.get(O.F_POS), g[f"step{n}_pos"], f"step{n} pos")
        assert_bits_equal(w.get(O.F_VEL), g[f"step{n}_vel"], f"step{n} vel")
    assert_bits_equal(w.get(O.F_RHO), g["step200_rho"], "step200 rho")
    assert_bits_equal(w.get(O.F_ACC), g["step200_acc"], "step200 acc")


def test_golden_dam216(oracle_mod, golden):
    g = golden("dam216")
    O = oracle_mod
    p = SphParams.defaults()
    p.bounds_min, p.bounds_max = (0.0, 0.0, 0.0), (1.2, 1.2, 1.2)
    w = world(O, p)
    assert w.lattice_mass(0.1) == float(g["mass"])
    pos = scenes.dam_break_positions(6, 6, 6)
    assert_bits_equal(pos, g["init_pos"], "generator")
    w.add_particles(pos, float(g["mass"]))
    w.step(0.005)
    for k, f in (("pos", O.F_POS), ("vel", O.F_VEL), ("acc", O.F_ACC), ("rho", O.F_RHO), ("p", O.F_P),
                 ("mu_eff", O.F_MU_EFF), ("xsph", O.F_XSPH)):
        assert_bits_equal(w.get(f), g[f"step1_{k}"], f"step1 {k}")
    w.step(0.005, 29)
    for k, f in (("pos", O.F_POS), ("vel", O.F_VEL), ("acc", O.F_ACC), ("rho", O.F_RHO), ("p", O.F_P),
                 ("mu_eff", O.F_MU_EFF), ("xsph", O.F_XSPH)):
        assert_bits_equal(w.get(f), g[f"step30_{k}"], f"step30 {k}")


def test_golden_materials(oracle_mod, golden):
    g = golden("materials")
    O = oracle_mod
    p = ref_test_params(gravity=(0.0, 0.0, 0.0))
    p.visc_k, p.visc_n = [3.5, 10.0], [1.0, 1.0]
    w = world(O, p)
    w.add_particles([[0, 0, 0], [0, 0.06, 0]], 0.05, vel=[[-300, 0, 0], [300, 0, 0]], material=[0, 1])
    w.step(0.001)
    for k, f in (("pos", O.F_POS), ("vel", O.F_VEL), ("mu_eff", O.F_MU_EFF), ("acc", O.F_ACC), ("rho", O.F_RHO)):
        assert_bits_equal(w.get(f), g[f"twomat_{k}"], f"twomat {k}")
    for n in (0.5, 1.0, 1.5):
        p = ref_test_params(gravity=(0.0, 0.0, 0.0))
        p.visc_k, p.visc_n = [3.5], [n]
        w = world(O, p)
        pos = [((ix - 2.0) * 0.08, iy * 0.06, 0.0) for iy in range(2) for ix in range(5)]
        vel = [((-300.0 if iy == 0 else 300.0), 0.0, 0.0) for iy in range(2) for ix in range(5)]
        w.add_particles(pos, 0.05, vel=vel)
        w.step(0.001)
        tag = str(n).replace(".", "p")
        assert_bits_equal(w.get(O.F_MU_EFF), g[f"shear{tag}_mu_eff"], f"shear {n} mu")
        assert_bits_equal(w.get(O.F_POS), g[f"shear{tag}_pos"], f"shear {n} pos")


# ---- analytic known answers ------------------------------------------------------------

def test_kat_quickstart_mass_and_self_density(oracle_mod):
    """Spacing 0.3 > h: lattice_mass sums only the self term, so the first-step
    density of every particle is mass * poly6(0) = rest density (world.rs:148-169)."""
    O = oracle_mod
    w = world(O)
    w.fill_box((-1, 1, -1), (1, 3, 1), 0.3, 0.1)
    m = w.get(O.F_MASS)
    assert m[0] == 5.10633472583484
    h = 0.2
    poly6_0 = 315.0 / (64.0 * math.pi * h ** 9) * (h * h) ** 3
    w.step(0.01)
    rho = w.get(O.F_RHO)
    np.testing.assert_allclose(rho, 1000.0, rtol=1e-14)
    np.testing.assert_allclose(rho, m * poly6_0, rtol=1e-15)
    # no neighbours: acc = 0, so v = g dt and x = x0 + v dt exactly.
    v = w.get(O.F_VEL)
    assert np.all(v[:, 1] == -9.81 * 0.01) and np.all(v[:, [0, 2]] == 0.0)


def test_kat_two_particle_force(oracle_mod):
    """Two particles at r < h: symmetric pressure and viscosity evaluated by hand."""
    O = oracle_mod
    p = ref_test_params(gravity=(0.0, 0.0, 0.0))
    w = world(O, p)
    w.add_particles([[0.0, 0.0, 0.0], [0.05, 0.0, 0.0]], 2.0, vel=[[0.0, 0.0, 0.0], [1.0, 0.0, 0.0]])
    w.step(1e-3)
    h = 0.2
    r = 0.05
    c6 = 315.0 / (64.0 * math.pi * h ** 9)
    w0 = c6 * (h * h) ** 3
    wr = c6 * (h * h - r * r) ** 3
    rho = 2.0 * w0 + 2.0 * wr
    prs = 250.0 * (rho - 1000.0) if rho > 1000.0 else 0.0
    rho_o = w.get(O.F_RHO)
    np.testing.assert_allclose(rho_o, rho, rtol=1e-14)
    np.testing.assert_allclose(w.get(O.F_P), prs, rtol=1e-12, atol=1e-9)
    spiky = -45.0 / (math.pi * h ** 6) * (h - r) ** 2
    lap = 45.0 / (math.pi * h ** 6) * (h - r)
    coef = 4.0 * (2 * prs / rho ** 2)
    f_press0 = 1.0 * coef * spiky            # on particle 0, direction +x
    f_visc0 = 1.0 * (4.0 / rho * lap) * 3.5  # dv = +1
    acc0 = (f_press0 + f_visc0) / rho
    acc = w.get(O.F_ACC)
    np.testing.assert_allclose(acc[0, 0], acc0, rtol=1e-12)
    np.testing.assert_allclose(acc[1, 0], -acc0, rtol=1e-12)
    assert np.all(acc[:, 1:] == 0.0)


def test_kat_two_particle_xsph_and_power_law_viscosity(oracle_mod):
    """Two compressed particles at r < h with a shear-thinning material (visc_n = 0.5), by hand from
    compute_forces (world.rs:252-347): XSPH sum (v_j - v_i) m_j/rho_j W_poly6(r), the
    strain-rate proxy |v_j - v_i| / (r + 1e-4) m_j/rho_j, mu_eff = k max(shear,
    shear_min)^(n - 1), the equation of state, and the acceleration with its pressure term and
    its viscous term scaled by mu_eff."""
    O = oracle_mod
    p = ref_test_params(gravity=(0.0, 0.0, 0.0), visc_k=[3.5], visc_n=[0.5])
    w = world(O, p)
    w.add_particles([[0.0, 0.0, 0.0], [0.05, 0.0, 0.0]], 4.0, vel=[[0.0, 0.0, 0.0], [1.0, 0.0, 0.0]])
    w.step(1e-3)
    h, r, m = 0.2, 0.05, 4.0
    c6 = 315.0 / (64.0 * math.pi * h ** 9)
    wr = c6 * (h * h - r * r) ** 3
    rho = m * c6 * (h * h) ** 3 + m * wr
    np.testing.assert_allclose(w.get(O.F_RHO), rho, rtol=1e-14)
    prs = 250.0 * (rho - 1000.0) if rho > 1000.0 else 0.0
    assert prs > 0.0  # the pair is compressed: the pressure term is live
    np.testing.assert_allclose(w.get(O.F_P), [prs, prs], rtol=1e-12)
    xs = m / rho * wr  # dv = +1 on particle 0, -1 on particle 1
    xsph = w.get(O.F_XSPH)
    np.testing.assert_allclose(xsph[0], [xs, 0.0, 0.0], rtol=1e-13)
    np.testing.assert_allclose(xsph[1], [-xs, 0.0, 0.0], rtol=1e-13)
    shear = 1.0 / (r + 1e-4) * (m / rho)
    mu = 3.5 * max(shear, 0.01) ** (0.5 - 1.0)
    np.testing.assert_allclose(w.get(O.F_MU_EFF), [mu, mu], rtol=1e-13)
    spiky = -45.0 / (math.pi * h ** 6) * (h - r) ** 2
    lap = 45.0 / (math.pi * h ** 6) * (h - r)
    acc0 = (m * m * (2 * prs / rho ** 2) * spiky + (m * m / rho * lap) * mu) / rho
    acc = w.get(O.F_ACC)
    np.testing.assert_allclose(acc[:, 0], [acc0, -acc0], rtol=1e-12)
    assert np.all(acc[:, 1:] == 0.0)
    # With visc_n = 1 the same pair gives mu_eff = visc_k exactly (sph/tests.rs:406-427).
    p1 = ref_test_params(gravity=(0.0, 0.0, 0.0))
    w1 = world(O, p1)
    w1.add_particles([[0.0, 0.0, 0.0], [0.05, 0.0, 0.0]], 2.0, vel=[[0.0, 0.0, 0.0], [1.0, 0.0, 0.0]])
    w1.step(1e-3)
    assert np.all(w1.get(O.F_MU_EFF) == 3.5)


def test_kat_diagnostics_in_insertion_order(oracle_mod):
    """FluidSubsystem::total_momentum and kinetic_energy (subsystem.rs:149-163) by hand:
    p += v * m and e += (|v|^2 * m) / (1 + 1) over the particles in insertion order, with
    nalgebra's norm_squared as (x^2 + y^2) + z^2; bit for bit."""
    O = oracle_mod
    rng = np.random.default_rng(11)
    n = 257
    pos = rng.uniform(-2.5, 2.5, (n, 3))
    vel = rng.normal(0.0, 3.0, (n, 3))
    mass = rng.uniform(0.5, 2.0, n)
    w = world(O, ref_test_params())
    w.add_particles(pos, mass, vel=vel)
    px = py = pz = e = 0.0
    for i in range(n):
        vx, vy, vz = (float(c) for c in vel[i])
        m = float(mass[i])
        px, py, pz = px + vx * m, py + vy * m, pz + vz * m
        e = e + ((vx * vx + vy * vy) + vz * vz) * m / (1.0 + 1.0)
    assert_bits_equal(w.diagnostics(), np.array([px, py, pz, e]), "momentum and kinetic energy")


def _hand_step(pos, vel, mass, dt, h=0.2, rest=1000.0, stiff=250.0, visc=3.5, shear_min=0.01,
               g=(0.0, -9.81, 0.0), xsph_eps=0.5):
    """One FluidWorld<f64>::step written directly from grid.rs:25-56 (cell keys
    floor(x * (1/h)), cells listing their particles in insertion order, the 3x3x3 cells
    visited x-outer, z-inner), kernels.rs:21-66 (coefficients, poly6, spiky gradient,
    viscosity laplacian) and world.rs:204-363, each in its operation order; norm() is
    sqrt((x^2 + y^2) + z^2), the 3-vector case of nalgebra's dot product.  Material 0 with
    visc_n = 1, no walls met."""
    pi = math.pi
    h2 = h * h
    h3 = h2 * h
    h6 = h3 * h3
    h9 = h6 * h3
    c_poly6 = 315.0 / (64.0 * pi * h9)
    c_spiky = -45.0 / (pi * h6)
    c_lap = 45.0 / (pi * h6)

    def poly6(r):
        if r >= h:
            return 0.0
        d = h2 - r * r
        return c_poly6 * d * d * d

    def norm(a):
        return math.sqrt((a[0] * a[0] + a[1] * a[1]) + a[2] * a[2])

    def sub(a, b):
        return [a[0] - b[0], a[1] - b[1], a[2] - b[2]]

    n = len(pos)
    inv = 1.0 / h

    def key(p):
        return tuple(math.floor(c * inv) for c in p)

    cells = {}
    for i in range(n):
        cells.setdefault(key(pos[i]), []).append(i)

    def neighbours(i):
        ci, cj, ck = key(pos[i])
        for di in (-1, 0, 1):
            for dj in (-1, 0, 1):
                for dk in (-1, 0, 1):
                    yield from cells.get((ci + di, cj + dj, ck + dk), [])

    rho, prs = [], []
    for i in range(n):
        acc_rho = 0.0
        for j in neighbours(i):
            r = norm(sub(pos[i], pos[j]))
            if r < h:
                acc_rho += mass[j] * poly6(r)
        rho.append(acc_rho)
        over = acc_rho - rest
        prs.append(stiff * over if over > 0.0 else 0.0)
    acc, xsph, mu = [], [], []
    for i in range(n):
        fp, fv, xs, shear = [0.0] * 3, [0.0] * 3, [0.0] * 3, 0.0
        for j in neighbours(i):
            if j == i:
                continue
            d = sub(pos[j], pos[i])
            r = norm(d)
            if r >= h or r <= 0.0:
                continue
            grad = c_spiky * (h - r) * (h - r)
            coef = mass[i] * mass[j] * (prs[i] / (rho[i] * rho[i]) + prs[j] / (rho[j] * rho[j]))
            dv = sub(vel[j], vel[i])
            lap = c_lap * (h - r)
            wv = mass[i] * mass[j] / rho[j] * lap
            wx = mass[j] / rho[j] * poly6(r)
            for k in range(3):
                fp[k] += d[k] / r * (coef * grad)
                fv[k] += dv[k] * wv
                xs[k] += dv[k] * wx
            shear += norm(dv) / (r + 1e-4) * (mass[j] / rho[j])
        m_eff = visc * (shear if shear > shear_min else shear_min) ** (1.0 - 1.0)
        acc.append([(fp[k] + fv[k] * m_eff) / rho[i] if rho[i] > 0.0 else 0.0 for k in range(3)])
        xsph.append(xs)
        mu.append(m_eff)
    x, v = [list(r) for r in pos], [list(r) for r in vel]
    for i in range(n):
        for k in range(3):
            v[i][k] = v[i][k] + ((acc[i][k] + g[k]) + 0.0) * dt
            v[i][k] = v[i][k] + xsph[i][k] * xsph_eps
            x[i][k] = x[i][k] + v[i][k] * dt
    return rho, prs, acc, xsph, mu, x, v


def test_kat_one_cell_step_by_hand(oracle_mod):
    """A whole step of four compressed, moving particles in one grid cell, evaluated by hand
    from the reference's kernels and passes (_hand_step), equals the oracle bit for
    bit in every output: density, pressure, acceleration, XSPH, mu_eff, position, velocity."""
    O = oracle_mod
    pos = [[0.03, 0.04, 0.05], [0.09, 0.06, 0.08], [0.12, 0.15, 0.07], [0.05, 0.13, 0.16]]
    vel = [[0.5, -0.25, 0.0], [-0.75, 0.125, 0.5], [0.0, 1.0, -0.5], [0.25, 0.0, 0.375]]
    mass = [3.0, 3.5, 2.75, 4.0]
    dt = 0.002
    w = world(O, ref_test_params())
    w.add_particles(pos, np.array(mass), vel=vel)
    w.step(dt)
    rho, prs, acc, xsph, mu, x, v = _hand_step(pos, vel, mass, dt)
    assert all(p > 0.0 for p in prs)  # every particle compressed: the pressure terms are live
    _assert_step_outputs(O, w, (rho, prs, acc, xsph, mu, x, v))


def _assert_step_outputs(O, w, want):
    for name, field, values in zip(("rho", "p", "acc", "xsph", "mu_eff", "pos", "vel"),
                                   (O.F_RHO, O.F_P, O.F_ACC, O.F_XSPH, O.F_MU_EFF, O.F_POS, O.F_VEL), want):
        assert_bits_equal(w.get(field), np.array(values), name)


def test_kat_multi_cell_step_by_hand(oracle_mod):
    """The same hand evaluation over 80 random particles spread over a 5x5x5 block of grid
    cells, negative coordinates included (floor keys): the 27-cell visit order decides every
    sum's order, so bit equality pins the oracle's neighbour order as well as its arithmetic."""
    O = oracle_mod
    rng = np.random.default_rng(5)
    pos = rng.uniform(-0.35, 0.45, (80, 3))
    vel = rng.normal(0.0, 0.5, (80, 3))
    mass = rng.uniform(3.0, 6.0, 80)
    dt = 0.001
    w = world(O, ref_test_params())
    w.add_particles(pos, mass, vel=vel)
    w.step(dt)
    want = _hand_step(pos.tolist(), vel.tolist(), mass.tolist(), dt)
    assert sum(p > 0.0 for p in want[1]) > 40  # most particles are compressed
    assert len({tuple(np.floor(q / 0.2).astype(int)) for q in pos}) >= 27
    _assert_step_outputs(O, w, want)


def _hand_lattice_mass(s, h=0.2, rest=1000.0):
    """FluidWorld::lattice_mass (world.rs:148-169) restated: rest / sum of poly6 over the
    lattice points of spacing s within h, shells -n..n with n = ceil(h / s) + 1, visited
    i-outer, l-inner, r = s * sqrt(i^2 + j^2 + l^2)."""
    h2 = h * h
    h9 = (h2 * h) * (h2 * h) * (h2 * h)
    c6 = 315.0 / (64.0 * math.pi * h9)
    n_shell = math.ceil(h / s) + 1
    total = 0.0
    for i in range(-n_shell, n_shell + 1):
        for j in range(-n_shell, n_shell + 1):
            for l in range(-n_shell, n_shell + 1):
                r = s * math.sqrt(float(i * i + j * j + l * l))
                if r < h:
                    d = h2 - r * r
                    total += c6 * d * d * d
    return rest / total


def _hand_fill_box(mn, mx, spacing, margin):
    """FluidWorld::fill_box (world.rs:124-144) restated: the lattice from min + margin to
    max - margin by repeated addition of the spacing, x-outer, z-inner."""
    lo = [c + margin for c in mn]
    hi = [c - margin for c in mx]
    out = []
    x = lo[0]
    while x <= hi[0]:
        y = lo[1]
        while y <= hi[1]:
            z = lo[2]
            while z <= hi[2]:
                out.append([x, y, z])
                z += spacing
            y += spacing
        x += spacing
    return out


@pytest.mark.parametrize("mn,mx,spacing,margin", [((-1, 1, -1), (1, 3, 1), 0.3, 0.1),
                                                  ((0.0, 0.0, 0.0), (1.0, 0.7, 0.45), 0.1, 0.05),
                                                  ((-0.4, -0.2, 0.1), (0.3, 0.35, 0.9), 0.07, 0.0)])
def test_kat_fill_box_and_lattice_mass_by_hand(oracle_mod, mn, mx, spacing, margin):
    """fill_box's positions (accumulated coordinates, so the last point of a row can fall
    short of or land on hi) and lattice_mass, restated from world.rs:124-169, equal the
    oracle's bit for bit."""
    O = oracle_mod
    w = world(O)
    w.fill_box(mn, mx, spacing, margin)
    want = _hand_fill_box([float(c) for c in mn], [float(c) for c in mx], spacing, margin)
    assert len(w) == len(want) > 0
    assert_bits_equal(w.get(O.F_POS), np.array(want), "fill_box positions")
    m = _hand_lattice_mass(spacing)
    assert_bits_equal(w.get(O.F_MASS), np.full(len(want), m), "lattice mass")
    assert w.lattice_mass(spacing) == m


def test_kat_integrate_and_bounds_by_hand(oracle_mod):
    """integrate (world.rs:352-363) and enforce_bounds (world.rs:366-397) evaluated by hand in
    the reference's operation order on isolated particles (more than h apart: no pair term,
    so acc = xsph = 0): a = (acc + g) + body_acc; v += a dt; v += xsph eps; x += v dt;
    body_acc cleared; a coordinate past a wall is set to the wall and that velocity
    component becomes -v * damp.  Two steps, so the second sees body_acc cleared."""
    O = oracle_mod
    p = SphParams.defaults()
    p.bounds_min, p.bounds_max = (0.0, 0.0, 0.0), (1.0, 1.0, 1.0)
    g, damp, eps, dt = (0.0, -9.81, 0.0), 0.4, 0.5, 0.01
    pos = [[0.005, 0.5, 0.99], [0.5, 0.002, 0.5], [0.8, 0.8, 0.2]]
    vel = [[-1.0, 0.5, 2.0], [0.25, -0.5, 0.125], [0.1, 0.2, 0.3]]
    body = [[0.25, 1.5, -0.75], [0.0, 0.0, 0.0], [0.0, 0.0, 0.0]]
    w = world(O, p)
    w.add_particles(pos, 2.0, vel=vel)
    w.set(O.F_BODY_ACC, np.array(body))
    x = [list(r) for r in pos]
    v = [list(r) for r in vel]
    for step in range(2):
        w.step(dt)
        for i in range(3):
            for k in range(3):
                a = (0.0 + g[k]) + (body[i][k] if step == 0 else 0.0)
                v[i][k] = v[i][k] + a * dt
                v[i][k] = v[i][k] + 0.0 * eps
                x[i][k] = x[i][k] + v[i][k] * dt
                if x[i][k] < 0.0:
                    x[i][k], v[i][k] = 0.0, -v[i][k] * damp
                elif x[i][k] > 1.0:
                    x[i][k], v[i][k] = 1.0, -v[i][k] * damp
        assert np.all(w.get(O.F_ACC) == 0.0) and np.all(w.get(O.F_XSPH) == 0.0)
        assert np.all(w.get(O.F_BODY_ACC) == 0.0)
        assert_bits_equal(w.get(O.F_POS), np.array(x), f"positions after step {step + 1}")
        assert_bits_equal(w.get(O.F_VEL), np.array(v), f"velocities after step {step + 1}")
        if step == 0:
            # The first step meets the walls: x of particle 0 and y of particle 1 low, z of
            # particle 0 high; the second moves them back inside.
            assert x[0][0] == 0.0 and x[1][1] == 0.0 and x[0][2] == 1.0
            assert v[0][0] > 0.0 and v[1][1] > 0.0 and v[0][2] < 0.0


def test_kat_interior_lattice_density(oracle_mod):
    """An interior particle of an unjittered lattice has rho = rest density (world.rs:146-169)."""
    O = oracle_mod
    p = SphParams.defaults()
    p.gravity = (0.0, 0.0, 0.0)
    w = world(O, p)
    w.fill_box((-0.55, -0.55, -0.55), (0.55, 0.55, 0.55), 0.1, 0.0)
    w.step(1e-6)
    pos0 = w.get(O.F_POS)
    rho = w.get(O.F_RHO)
    centre = np.argmin(np.linalg.norm(pos0, axis=1))
    np.testing.assert_allclose(rho[centre], 1000.0, rtol=1e-12)


def test_cell_keys_floor_semantics(oracle_mod):
    """Grid::key_of is floor(x * (1/h)) per axis (grid.rs:25-33), negative included."""
    O = oracle_mod
    w = world(O)
    pts = np.array([[0.0, -0.0, 0.2], [-1e-12, 0.19999999999999998, -0.2], [4.99, -4.99, 0.3999999999]], np.float64)
    w.add_particles(pts, 1.0)
    keys = w.cell_keys()
    inv = 1.0 / 0.2
    expect = np.floor(pts * inv).astype(np.int64)
    assert np.array_equal(keys, expect)


def test_neighbor_visit_order(oracle_mod):
    """27 cells with di outer and dk inner, ascending insertion index in a cell (grid.rs:43-56)."""
    O = oracle_mod
    w = world(O)
    rng = np.random.default_rng(3)
    pts = rng.uniform(-0.5, 0.5, size=(300, 3))
    w.add_particles(pts, 1.0)
    keys = w.cell_keys()
    nb = w.neighbors(0)
    k0 = keys[0]
    expect = []
    for di in (-1, 0, 1):
        for dj in (-1, 0, 1):
            for dk in (-1, 0, 1):
                cell = k0 + np.array([di, dj, dk])
                expect.extend(np.flatnonzero(np.all(keys == cell, axis=1)).tolist())
    assert nb.tolist() == expect


# ---- the reference's property tests, on the oracle ------------------------------------

def test_fill_box_count_matches_grid(oracle_mod):
    """sph/tests.rs:18-29."""
    w = world(oracle_mod, ref_test_params())
    w.fill_box((-1, -1, -1), (1, 1, 1), 0.2, 0.05)
    assert 500 < len(w) < 2000


def test_density_converges_near_rest(oracle_mod):
    """sph/tests.rs:31-56."""
    w = world(oracle_mod, ref_test_params(gravity=(0.0, 0.0, 0.0)))
    w.fill_box((-0.5, -0.5, -0.5), (0.5, 0.5, 0.5), 0.1, 0.05)
    w.step(0.002, 15)
    avg = w.get(oracle_mod.F_RHO).mean()
    assert abs(avg - 1000.0) / 1000.0 < 0.25


def test_particle_count_conserved(oracle_mod):
    """sph/tests.rs:58-72."""
    w = world(oracle_mod, ref_test_params())
    w.fill_box((-1, -1, -1), (1, 1, 1), 0.1, 0.05)
    n0 = len(w)
    w.step(0.003, 50)
    assert len(w) == n0


def test_dam_break_stays_in_bounds(oracle_mod):
    """sph/tests.rs:74-95."""
    O = oracle_mod
    w = world(O, ref_test_params())
    w.fill_box((-1.5, -1.5, -0.5), (-0.5, 1.5, 0.5), 0.1, 0.05)
    for _ in range(12):
        w.step(0.0025, 10)
        pos = w.get(O.F_POS)
        assert np.isfinite(pos).all()
        assert (pos >= -3.0 - 1e-6).all() and (pos <= 3.0 + 1e-6).all()


def test_material_tag_distinguishes_viscosity(oracle_mod):
    """sph/tests.rs:406-427."""
    O = oracle_mod
    p = ref_test_params(gravity=(0.0, 0.0, 0.0))
    p.visc_k, p.visc_n = [3.5, 10.0], [1.0, 1.0]
    w = world(O, p)
    w.add_particles([[0, 0, 0], [0, 0.06, 0]], 0.05, vel=[[-300, 0, 0], [300, 0, 0]], material=[0, 1])
    w.step(0.001)
    mu = w.get(O.F_MU_EFF)
    assert abs(mu[0] - 3.5) < 1e-6 and abs(mu[1] - 10.0) < 1e-6


def test_non_newtonian_ordering(oracle_mod):
    """sph/tests.rs:392-404."""
    O = oracle_mod
    mus = []
    for n in (0.5, 1.0, 1.5):
        p = ref_test_params(gravity=(0.0, 0.0, 0.0))
        p.visc_k, p.visc_n = [3.5], [n]
        w = world(O, p)
        pos = [((ix - 2.0) * 0.08, iy * 0.06, 0.0) for iy in range(2) for ix in range(5)]
        vel = [((-300.0 if iy == 0 else 300.0), 0.0, 0.0) for iy in range(2) for ix in range(5)]
        w.add_particles(pos, 0.05, vel=vel)
        w.step(0.001)
        mus.append(w.get(O.F_MU_EFF)[0])
    assert mus[0] < mus[1] < mus[2]


def test_closed_system_invariants(oracle_mod):
    """phy-demo/tests/stability.rs:55-108 (800 particles, h = 2 spacing, no gravity),
    shortened from 1000 to 300 steps to keep the CPU suite fast."""
    O = oracle_mod
    half = 5.0
    spacing = (8.0 * half ** 3 / 800) ** (1.0 / 3.0)
    p = SphParams.defaults()
    p.h = spacing * 2.0
    p.gravity = (0.0, 0.0, 0.0)
    p.bounds_min, p.bounds_max = (-7.0, -1.0, -7.0), (7.0, 13.0, 7.0)
    w = world(O, p, threads=4)
    w.fill_box((-half, 1.0, -half), (half, 1.0 + 2 * half, half), spacing, 0.1)
    e0 = w.diagnostics()[3]
    w.step(0.01, 300)
    d = w.diagnostics()
    assert np.isfinite(w.get(O.F_POS)).all()
    assert abs(d[3] - e0) <= 1e-2
    assert np.linalg.norm(d[:3]) <= 1e-3


def test_thread_count_does_not_change_results(oracle_mod):
    """Write-disjoint per-particle maps (world.rs:201-203): rayon/OpenMP thread count is irrelevant."""
    O = oracle_mod
    pos = scenes.dam_break_positions(8, 10, 8)
    p = SphParams.defaults()
    p.bounds_min, p.bounds_max = (0.0, 0.0, 0.0), (1.6, 1.6, 1.6)
    outs = []
    for t in (1, 4):
        w = world(O, p, threads=t)
        w.add_particles(pos, scenes.lattice_mass(0.1))
        w.step(0.005, 10)
        outs.append(w.get(O.F_POS))
    assert_bits_equal(outs[0], outs[1], "threads 1 vs 4")


def test_live_h_change_keeps_captured_kernels(oracle_mod):
    """F7: kernels and grid keep the h of FluidWorld::new; the cutoff uses the live h."""
    O = oracle_mod
    pos = scenes.dam_break_positions(4, 4, 4)
    p = SphParams.defaults()
    p.bounds_min, p.bounds_max = (0.0, 0.0, 0.0), (0.8, 0.8, 0.8)
    a = world(O, p)
    a.add_particles(pos, 1.0)
    p2 = SphParams.defaults()
    p2.bounds_min, p2.bounds_max = p.bounds_min, p.bounds_max
    p2.h = 0.15
    a.set_params(p2)
    a.step(0.001)
    b = world(O, p2)  # constructed with h = 0.15: different kernels and cells
    b.add_particles(pos, 1.0)
    b.step(0.001)
    assert not np.array_equal(a.get(O.F_RHO), b.get(O.F_RHO))


def test_scene_generator_sizes():
    assert scenes.config("quickstart").n == 343
    assert scenes.dam_break_positions(80, 160, 80).shape == (1024000, 3)
    assert scenes.config("grad_64k").n == 65536
    assert scenes.lattice_mass(0.1) == 0.99031946198009
    u = scenes.uniform01(0xC0FFEE, 0, 1000)
    assert u.min() >= 0.0 and u.max() < 1.0


def test_dam_break_jitter_follows_its_recipe():
    """The scale configurations' lattice: points at ((i + 0.5) s, (j + 0.5) s, (k + 0.5) s),
    x-outer, each coordinate moved by U(-0.05 s, 0.05 s) from SplitMix64 draws in order
    (x, y, z per point), and the same block restated by the independent generator of the
    golden fixtures (tests/golden/gen_golden.py) bit for bit."""
    import importlib.util
    from pathlib import Path
    pos = scenes.dam_break_positions(6, 6, 6)
    s = scenes.SPACING
    i, j, k = np.meshgrid(np.arange(6), np.arange(6), np.arange(6), indexing="ij")
    base = np.stack([(i + 0.5) * s, (j + 0.5) * s, (k + 0.5) * s], axis=-1).reshape(-1, 3)
    assert np.abs(pos - base).max() <= 0.05 * s
    assert np.abs(pos - base).max() > 0.04 * s  # the jitter is there
    spec = importlib.util.spec_from_file_location(
        "gen_golden_for_jitter", Path(__file__).resolve().parent / "golden" / "gen_golden.py")
    gen = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(gen)
    assert_bits_equal(pos, np.array(gen.jittered_block(6, 6, 6)), "jittered block")


def test_batched_form_scenes_follow_their_configuration():
    """The batched form's 256 scenes: counts log-uniform in [2k, 200k] (rounded per axis, so
    within a few percent of the range), fill fraction U[0.2, 0.5] (rounding likewise), every
    particle inside its scene's box, about half the scenes below the geometric mean, and the
    same 12,067,610 particles on every call."""
    b = scenes.batch_scenes(256)
    n = np.array([x.n for x in b])
    assert int(n.sum()) == 12067610
    assert n.min() >= 0.95 * 2000 and n.max() <= 1.05 * 200000
    box = np.array([x.bounds_max for x in b])
    fill = n * scenes.SPACING ** 3 / box.prod(axis=1)
    assert fill.min() >= 0.19 and fill.max() <= 0.53
    for x in b:
        assert x.bounds_min == (0.0, 0.0, 0.0)
        assert (x.pos >= 0.0).all() and (x.pos <= np.array(x.bounds_max)).all()
    assert 0.4 <= float((n < np.sqrt(2000 * 200000)).mean()) <= 0.6
    again = scenes.batch_scenes(256)
    assert all(np.array_equal(x.pos, y.pos) and x.bounds_max == y.bounds_max for x, y in zip(b, again))


def test_splitmix_matches_sequential_definition():
    """Vectorised SplitMix64 equals the sequential Rng::next_u64 (replay.rs:40-46)."""
    mask = (1 << 64) - 1
    state = 12345
    ref = []
    for _ in range(8):
        state = (state + 0x9E3779B97F4A7C15) & mask
        z = state
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & mask
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & mask
        ref.append(z ^ (z >> 31))
    assert scenes.splitmix64(12345, 0, 8).tolist() == ref


def test_oracle_defaults_restatement_matches_library(oracle_mod):
    """The oracle's own SphParams::defaults() (params.rs:55-85), used where the product
    library must stay unloaded, equals the library's phy_sph_params_defaults field by field."""
    a, b = oracle_mod.RefParams.defaults(), SphParams.defaults()
    for name in ("rest_density", "stiffness", "viscosity", "visc_k", "visc_n", "shear_min", "mass", "h",
                 "gravity", "bounds_min", "bounds_max", "boundary_damp", "xsph_eps"):
        assert list(np.ravel(getattr(a, name))) == list(np.ravel(getattr(b, name))), name
