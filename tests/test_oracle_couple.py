"""The oracle's FluidWorld::couple_points (phy-fluid/src/sph/world.rs:691-752) and
couple_heat (world.rs:555-678), which the device coupling is checked against, pinned on the
CPU: the reference's own tests (sph/tests.rs:179-290), known answers that follow from the
definitions, and their particle-after-particle and point-after-point semantics."""
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


# ---- couple_heat (world.rs:555-678) -------------------------------------------------------

def _one_particle(O, pos, vel=(0.0, 0.0, 0.0), gravity=(0.0, -9.81, 0.0)):
    p = ref_test_params(gravity=gravity)
    w = O.OracleWorld(p)
    w.add_particles([pos], [0.05], vel=[vel])
    return w, p


def test_heat_warmer_fluid_rises(oracle_mod):
    """couple_heat_warmer_fluid_rises (sph/tests.rs:214-259): 16^3 field of unit cells at
    origin -8, warm (1) where iy - 8 > 0; the particle at y = 1 gets body_acc.y = 9.81 * 0.5."""
    O = oracle_mod
    w, p = _one_particle(O, (0.0, 1.0, 0.0))
    temp = np.zeros((16, 16, 16))
    temp[:, 9:, :] = 1.0  # (nz, ny, nx): rows iy with iy * 1 - 16 / 2 > 0
    src = w.couple_heat(temp, np.zeros_like(temp), (-8.0, -8.0, -8.0), 1.0, 0.01, 0.0, 0.5, 0.0)
    ba = w.get(O.F_BODY_ACC)[0]
    assert ba[1] == 9.81 * 0.5 and ba[0] == 0.0 and ba[2] == 0.0
    assert p.gravity[1] + ba[1] > -9.81
    assert not src.any()


def test_heat_injects_source_into_moving_region(oracle_mod):
    """couple_heat_injects_source_into_moving_region (sph/tests.rs:261-290): the source of
    the particle's cell grows by heat_gain * |v| * dt."""
    O = oracle_mod
    w, _ = _one_particle(O, (0.0, 0.0, 0.0), vel=(2.0, 0.0, 0.0), gravity=(0.0, 0.0, 0.0))
    temp = np.zeros((16, 16, 16))
    src = w.couple_heat(temp, np.zeros_like(temp), (0.0, 0.0, 0.0), 1.0, 0.01, 0.0, 0.0, 0.1)
    assert src[0, 0, 0] == 0.1 * 2.0 * 0.01 and np.count_nonzero(src) == 1


def test_heat_trilinear_and_sequential_sources(oracle_mod):
    """A field linear in the cell coordinates is sampled exactly (up to rounding); sources of
    particles sharing a cell are added one after another in insertion order; particles
    outside the bounds are skipped and those outside the field sample t_ref."""
    O = oracle_mod
    p = ref_test_params(gravity=(0.5, -9.81, 0.25))
    w = O.OracleWorld(p)
    rng = np.random.default_rng(4)
    pos = np.concatenate([rng.uniform(-0.9, 0.9, (40, 3)), [[0.11, 0.12, 0.13]] * 5, [[3.5, 0.0, 0.0]],
                          [[-2.5, 2.9, 0.0]]])
    vel = rng.normal(0.0, 1.0, pos.shape)
    w.add_particles(pos, np.full(len(pos), 0.02), vel=vel)
    nx, ny, nz, dx, origin = 7, 6, 5, 0.4, np.array([-1.2, -1.0, -1.1])
    iz, iy, ix = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    temp = 1.0 + 2.0 * ix + 3.0 * iy - 1.0 * iz
    src0 = rng.normal(0.0, 0.1, temp.shape)
    t_ref, beta, gain, dt = 0.5, 0.25, 0.3, 0.01
    src = w.couple_heat(temp, src0, origin, dx, dt, t_ref, beta, gain)
    ba = w.get(O.F_BODY_ACC)
    g = np.array(p.gravity)
    expect_src = src0.copy()
    for i in range(len(pos)):
        x = pos[i]
        inb = np.all(x >= -3.0) and np.all(x <= 3.0)
        top = origin + dx * np.array([nx - 1, ny - 1, nz - 1])
        inf = np.all(x >= origin) and np.all(x <= top)
        if not inb:
            assert not ba[i].any()
            continue
        if inf:
            c = (x - origin) / dx
            cell = np.floor(c).astype(int)
            lin = 1.0 + 2.0 * c[0] + 3.0 * c[1] - 1.0 * c[2]
            np.testing.assert_allclose(-ba[i] / (g * beta), lin - t_ref, rtol=1e-12)
            speed = np.sqrt((vel[i, 0] ** 2 + vel[i, 1] ** 2) + vel[i, 2] ** 2)
            expect_src[cell[2], cell[1], cell[0]] += gain * speed * dt
        else:
            assert not ba[i].any()
    assert_bits_equal(src, expect_src, "sources in insertion order")


# ---- couple_bodies (world.rs:414-503) -----------------------------------------------------

def test_static_body_blocks_fluid(oracle_mod):
    """static_body_blocks_fluid (sph/tests.rs:96-129)."""
    O = oracle_mod
    w = O.OracleWorld(ref_test_params())
    w.fill_box((-1.5, -1.5, -0.5), (1.5, -1.0, 0.5), 0.1, 0.05)
    box = {"shape": "box", "size": (1.0, 0.5, 1.0), "pos": (0.0, 0.0, 0.0), "inv_mass": 0.0}
    for _ in range(100):
        w.step(DT)
        w.couple_bodies([box], DT)
    x = w.get(O.F_POS)
    assert not np.any((np.abs(x[:, 0]) <= 1.0) & (np.abs(x[:, 1]) <= 0.5) & (np.abs(x[:, 2]) <= 1.0))


def test_dynamic_body_gets_buoyancy_upward(oracle_mod):
    """dynamic_body_gets_buoyancy_upward (sph/tests.rs:131-175): a sphere of a quarter of the
    fluid's density, submerged, rises."""
    O = oracle_mod
    p = ref_test_params(gravity=(0.0, -9.81, 0.0))
    w = O.OracleWorld(p, threads=O.max_threads())
    w.fill_box((-0.7, -0.7, -0.7), (0.7, 0.7, 0.7), 0.1, 0.05)
    w.step(DT, 15)
    vol = 4.0 / 3.0 * np.pi * 0.6 ** 3
    mass_b = p.rest_density * vol * 0.25
    pos, vel = np.zeros(3), np.zeros(3)
    g = np.array(p.gravity)
    for _ in range(120):
        vel = vel + g * DT
        pos = pos + vel * DT
        w.step(DT)
        vel = w.couple_bodies([{"shape": "sphere", "size": (0.6,), "pos": pos, "vel": vel, "inv_mass": 1.0 / mass_b}],
                              DT)[0]
    assert pos[1] > 0.0


def test_dynamic_contact_known_answer(oracle_mod):
    """One particle moving into a dynamic box: the body takes -j inv_mass with
    j = n * (-v_rel_n / (1/m + inv_mass)); the particle's own share is overwritten by the
    push-out (the reference keeps push_out's velocity); the particle lands on the support
    point and loses its inward normal velocity; buoyancy adds -g rho0 V_box dt inv_mass."""
    O = oracle_mod
    p = ref_test_params(gravity=(0.0, -9.81, 0.0))
    w = O.OracleWorld(p)
    m = 0.05
    w.add_particles([[0.3, 0.1, 0.0]], [m], vel=[[-1.0, 0.5, 0.0]])
    inv = 0.5
    box = {"shape": "box", "size": (0.5, 0.4, 0.3), "pos": (0.0, 0.0, 0.0), "vel": (0.2, 0.0, 0.0), "inv_mass": inv}
    vb = w.couple_bodies([box], DT)[0]
    local = np.array([0.3, 0.1, 0.0])
    n = local / np.sqrt((local[0] ** 2 + local[1] ** 2) + local[2] ** 2)
    v_rel_n = np.dot(np.array([-1.0, 0.5, 0.0]) - np.array([0.2, 0.0, 0.0]), n)
    j = n * (-(1.0 + 0.0) * v_rel_n / ((1.0 / m) + inv))
    v_after = np.array([0.2, 0.0, 0.0]) + (-j) * inv
    vol = 0.5 * 0.4 * 0.3 * 8.0
    expect_vb = v_after + (-np.array(p.gravity) * (p.rest_density * vol) * DT) * inv
    np.testing.assert_allclose(vb, expect_vb, rtol=1e-14, atol=1e-15)
    assert_bits_equal(w.get(O.F_POS)[0], np.array([0.5, 0.4, 0.3]), "support point")  # dir > 0 on x, y; z >= 0
    sd = np.array([0.5, 0.4, 0.3])
    nn = sd / np.linalg.norm(sd)
    v_rel = np.array([-1.0, 0.5, 0.0]) - v_after
    vn = np.dot(v_rel, nn)
    expect_v = np.array([-1.0, 0.5, 0.0]) - nn * vn if vn < 0 else np.array([-1.0, 0.5, 0.0])
    np.testing.assert_allclose(w.get(O.F_VEL)[0], expect_v, rtol=1e-13, atol=1e-15)


def test_rotated_static_box_pushes_out(oracle_mod):
    """A box of half extents (1, 0.2, 0.2) turned 90 degrees about z contains (0.05, 0.8, 0.03)
    (local (0.8, -0.05, 0.03)) and moves it to the turned support corner (1, -0.2, 0.2), i.e.
    (0.2, 1, 0.2) in the world."""
    O = oracle_mod
    w = O.OracleWorld(ref_test_params(gravity=(0.0, 0.0, 0.0)))
    w.add_particles([[0.05, 0.8, 0.03], [0.8, 0.0, 0.0]], [0.02, 0.02])
    s = np.sqrt(0.5)
    box = {"shape": "box", "size": (1.0, 0.2, 0.2), "pos": (0.0, 0.0, 0.0), "rot": (0.0, 0.0, s, s), "inv_mass": 0.0}
    w.couple_bodies([box], DT)
    x = w.get(O.F_POS)
    np.testing.assert_allclose(x[0], [0.2, 1.0, 0.2], atol=1e-15)
    assert_bits_equal(x[1], np.array([0.8, 0.0, 0.0]), "outside the turned box")


def test_compound_body_known_answers(oracle_mod):
    """Shape::Compound (phy-rigid shape.rs:176-192) in couple_bodies: two spheres of radius
    0.3 at body offsets (-0.5, 0, 0) and (0.5, 0, 0).  A particle inside the +x sphere is
    pushed to the farthest sub-shape support point along its direction from the body
    origin, (0.8, 0, 0) (shape.rs:238-254); a particle between the spheres is inside
    neither and stays; the body's buoyancy uses the summed sub-shape volume
    (world.rs:531-534)."""
    O = oracle_mod
    p = ref_test_params(gravity=(0.0, -9.81, 0.0))
    w = O.OracleWorld(p)
    w.add_particles(np.array([[0.5, 0.0, 0.0], [0.0, 0.0, 0.0]]), 0.02)
    r = 0.3
    body = {"shape": "compound", "pos": (0.0, 0.0, 0.0), "inv_mass": 0.5,
            "subs": [{"shape": "sphere", "size": (r,), "offset": (-0.5, 0.0, 0.0)},
                     {"shape": "sphere", "size": (r,), "offset": (0.5, 0.0, 0.0)}]}
    vb = w.couple_bodies([body], DT)[0]
    x = w.get(O.F_POS)
    assert_bits_equal(x[0], np.array([0.8, 0.0, 0.0]), "pushed to the +x sphere's support point")
    assert_bits_equal(x[1], np.array([0.0, 0.0, 0.0]), "outside both sub shapes")
    vol = 0.0
    for _ in range(2):
        vol = vol + 4.0 / 3.0 * np.pi * r * r * r
    buoy = -np.array(p.gravity) * (p.rest_density * vol)
    assert_bits_equal(vb, np.zeros(3) + (buoy * DT) * 0.5, "buoyancy of the summed volume (no contact at rest)")
    # Rotated sub shape: a box rotated 90 degrees about z inside the body swaps its x/y extents.
    w2 = O.OracleWorld(p)
    w2.add_particles(np.array([[0.0, 0.25, 0.0], [0.25, 0.0, 0.0]]), 0.02)
    q = (0.0, 0.0, np.sin(np.pi / 4), np.cos(np.pi / 4))
    box = {"shape": "compound", "pos": (0.0, 0.0, 0.0), "inv_mass": 0.0,
           "subs": [{"shape": "box", "size": (0.1, 0.3, 0.1), "rot": q}]}
    w2.couple_bodies([box], DT)
    x2 = w2.get(O.F_POS)
    assert not np.array_equal(x2[1], [0.25, 0.0, 0.0]), "inside the rotated box: pushed out"
    assert_bits_equal(x2[0], np.array([0.0, 0.25, 0.0]), "outside the rotated box: untouched")
