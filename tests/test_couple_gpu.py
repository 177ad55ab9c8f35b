"""The fluid's coupling on the device against the oracle's restatement, bit for bit:
FluidWorld::couple_points (phy_fluid_couple_points, phy-fluid/src/sph/world.rs:691-752:
forces on the points, fluid velocities that take the reactions, points in order, skipped
points untouched) and FluidWorld::couple_heat (phy_fluid_couple_heat, world.rs:555-678:
body accelerations from the trilinear temperature, sources added in insertion order), and
the steps that follow them."""
import numpy as np
import pytest

from helpers import assert_bits_equal, ref_test_params

pytestmark = pytest.mark.gpu

DT = 0.0025


def _pair(gpu, O, prec="f64", lo=-0.5, hi=0.5, spacing=0.1, steps=15):
    """A fluid block (sph/tests.rs:181-192 for the defaults) on the device and in the
    oracle; a compensated world's state is copied into the oracle (teacher forcing)."""
    p = ref_test_params(gravity=(0.0, -9.81, 0.0))
    w = gpu.FluidWorld(p, prec)
    w.fill_box((lo,) * 3, (hi,) * 3, spacing, spacing / 2)
    ow = O.OracleWorld(p)
    ow.fill_box((lo,) * 3, (hi,) * 3, spacing, spacing / 2)
    w.step(DT, steps)
    if prec == "f64":
        ow.step(DT, steps)
    else:
        ow.set(O.F_POS, w.pos)
        ow.set(O.F_VEL, w.vel)
    return w, ow, p


def _points(n_random=0, seed=3):
    pts = [[0.0, 0.0, 0.0], [0.03, 0.0, 0.0], [2.0, 2.0, 2.0], [3.5, 0.0, 0.0], [0.1, -0.3, 0.2],
           [-0.45, 0.4, 0.45], [0.0, -3.0 - 1e-9, 0.0]]
    rng = np.random.default_rng(seed)
    pts = np.concatenate([np.array(pts), rng.uniform(-0.6, 0.6, (n_random, 3))])
    vel = rng.normal(0.0, 0.3, pts.shape)
    mass = rng.uniform(0.005, 0.05, len(pts))
    prior = rng.normal(0.0, 1.0, pts.shape)
    return pts, vel, mass, prior


def _check(O, w, ow, pts, vel, mass, prior, drag=1.5, soft=900.0):
    fg = w.couple_points(pts, vel, mass, DT, drag, soft, force=prior)
    fo = ow.couple_points(pts, vel, mass, DT, drag, soft, force=prior)
    assert_bits_equal(fg, fo, "forces")
    assert_bits_equal(fg[[3, 6]], prior[[3, 6]], "points outside the bounds")
    assert_bits_equal(w.vel, ow.get(O.F_VEL), "fluid velocities")
    assert_bits_equal(w.pos, ow.get(O.F_POS), "fluid positions unchanged")


def test_couple_points_f64_bitwise_and_next_steps(gpu, oracle_mod):
    O = oracle_mod
    w, ow, _ = _pair(gpu, O)
    pts, vel, mass, prior = _points(n_random=120)
    _check(O, w, ow, pts, vel, mass, prior)
    w.step(DT, 5)
    ow.step(DT, 5)
    assert_bits_equal(w.pos, ow.get(O.F_POS), "positions after coupling and 5 steps")
    assert_bits_equal(w.vel, ow.get(O.F_VEL), "velocities after coupling and 5 steps")
    assert_bits_equal(w.rho, ow.get(O.F_RHO), "densities after coupling and 5 steps")


def test_couple_points_on_tiled_compensated_world(gpu, oracle_mod):
    """The coupling is f64 on any kernel form: on the staged-tile compensated world it
    equals the oracle's coupling of the same state, and the world keeps stepping."""
    O = oracle_mod
    w, ow, _ = _pair(gpu, O, prec="comp", steps=20)
    rho = w.rho.copy()
    pts, vel, mass, prior = _points(n_random=40, seed=5)
    _check(O, w, ow, pts, vel, mass, prior, drag=0.7, soft=1000.0)
    assert_bits_equal(w.rho, rho, "step outputs untouched")
    w.step(DT, 10)
    assert np.isfinite(w.pos).all()


@pytest.mark.parametrize("spacing,least", [(0.04, 1024), (0.03, 2048), (0.02, 4096)])
def test_couple_points_dense_neighbourhood(gpu, oracle_mod, spacing, least):
    """Points whose 27 cells hold more than the 512 candidates a warp stages at once (taken
    in chunks), and (spacing 0.02) more than the 4096 that get a candidate list (read
    through the cell table); the other points of the same call hold theirs in registers."""
    O = oracle_mod
    w, ow, _ = _pair(gpu, O, lo=-0.3, hi=0.3, spacing=spacing, steps=2)
    assert len(ow.neighbors_of_point([0.0, 0.0, 0.0])) > least
    pts, vel, mass, prior = _points(n_random=10, seed=7)
    _check(O, w, ow, pts, vel, mass, prior)


def test_couple_points_groups(gpu, oracle_mod):
    """Many points over a large block: runs of consecutive points with disjoint 27-cell
    neighbourhoods run at once, one warp each; interleaved with points next to the one
    before (same and adjacent cells), repeated points, and points outside the bounds,
    every force and fluid velocity matches the oracle's one-after-another walk."""
    O = oracle_mod
    w, ow, _ = _pair(gpu, O, lo=-2.0, hi=2.0, spacing=0.1, steps=2)
    rng = np.random.default_rng(11)
    pts = rng.uniform(-2.1, 2.1, (600, 3))
    pts[100:140] = pts[99] + rng.uniform(-0.45, 0.45, (40, 3))  # a cluster: overlapping runs
    pts[200:208] = pts[199]                                      # the same point 9 times
    pts[300:308:2] = [9.0, 0.0, 0.0]                             # outside, between others
    vel = rng.normal(0.0, 0.3, pts.shape)
    mass = rng.uniform(0.005, 0.05, len(pts))
    prior = rng.normal(0.0, 1.0, pts.shape)
    fg = w.couple_points(pts, vel, mass, DT, 1.2, 950.0, force=prior)
    fo = ow.couple_points(pts, vel, mass, DT, 1.2, 950.0, force=prior)
    assert_bits_equal(fg, fo, "forces")
    assert_bits_equal(w.vel, ow.get(O.F_VEL), "fluid velocities")


def test_couple_points_buoyancy_upward(gpu):
    """couple_points_buoyancy_upward (sph/tests.rs:179-212) on the device."""
    p = ref_test_params(gravity=(0.0, -9.81, 0.0))
    w = gpu.FluidWorld(p)
    w.fill_box((-0.5,) * 3, (0.5,) * 3, 0.1, 0.05)
    w.step(DT, 15)
    before = w.total_momentum()
    f = w.couple_points([[0.0, 0.0, 0.0]], [[0.0, 0.0, 0.0]], [0.02], DT, 1.0, p.rest_density)
    assert f[0, 1] > 0.0
    assert (w.total_momentum() - before)[1] < 0.0


def test_couple_points_rejected_configurations(gpu):
    p = ref_test_params()
    w = gpu.FluidWorld(p)
    w.fill_box((-0.5,) * 3, (0.5,) * 3, 0.1, 0.05)
    w.tape_begin(5)
    with pytest.raises(gpu.PhyError):
        w.couple_points([[0.0, 0.0, 0.0]], [[0.0, 0.0, 0.0]], [0.02], DT, 1.0, 1000.0)
    w.tape_clear()
    w.couple_points(np.zeros((0, 3)), np.zeros((0, 3)), np.zeros(0), DT, 1.0, 1000.0)  # no points: no-op
    b = gpu.FluidWorld(p, "comp")
    b.add_particles([[0.1, 0.1, 0.1], [0.2, 0.2, 0.2]], 0.02)
    b.set_scenes([1, 1], [(0, 0, 0)] * 2, [(1, 1, 1)] * 2)
    with pytest.raises(gpu.PhyError):
        b.couple_points([[0.5, 0.5, 0.5]], [[0.0, 0.0, 0.0]], [0.02], DT, 1.0, 1000.0)


# ---- couple_heat (world.rs:555-678) -------------------------------------------------------

def _heat_grid(dims, seed):
    rng = np.random.default_rng(seed)
    nx, ny, nz = dims
    return rng.uniform(-1.0, 2.0, (nz, ny, nx)), rng.normal(0.0, 0.1, (nz, ny, nx))


def _heat_check(O, w, ow, temp, src0, origin, cell, args):
    sg = w.couple_heat(temp, src0, origin, cell, *args)
    so = ow.couple_heat(temp, src0, origin, cell, *args)
    assert_bits_equal(sg, so, "sources")
    assert_bits_equal(w.body_acc, ow.get(O.F_BODY_ACC), "body accelerations")
    return sg


def test_couple_heat_f64_bitwise_and_next_steps(gpu, oracle_mod):
    """A grid that covers part of the fluid (particles outside it sample t_ref), two calls
    in a row (body accelerations accumulate), then steps that consume them."""
    O = oracle_mod
    w, ow, _ = _pair(gpu, O)
    temp, src0 = _heat_grid((12, 10, 9), 11)
    args = (0.01, 0.3, 0.2, 0.05)  # dt, t_ref, beta, heat_gain
    src = _heat_check(O, w, ow, temp, src0, (-0.7, -0.6, -0.4), 0.1, args)
    assert np.count_nonzero(src != src0) > 10
    _heat_check(O, w, ow, temp, src, (-0.2, -0.5, -0.3), 0.07, args)
    w.step(DT, 3)
    ow.step(DT, 3)
    assert_bits_equal(w.pos, ow.get(O.F_POS), "positions after coupling and 3 steps")
    assert_bits_equal(w.vel, ow.get(O.F_VEL), "velocities after coupling and 3 steps")
    assert not w.body_acc.any(), "integrate consumes the body accelerations"


def test_couple_heat_coarse_and_large_grids(gpu, oracle_mod):
    """Hundreds of particles per source cell (long in-order sums) and a grid of 2^17 cells
    (three radix passes), over a world of many sort blocks."""
    O = oracle_mod
    sc_dims = (24, 32, 24)
    from physics_b200 import scenes
    sc = scenes.dam_break(*sc_dims, box=4.0, dt=DT, steps=0)
    p = ref_test_params(gravity=(0.3, -9.81, -0.2))
    p.bounds_min, p.bounds_max = sc.bounds_min, sc.bounds_max
    w = gpu.FluidWorld(p)
    w.add_particles(sc.pos, sc.mass)
    ow = O.OracleWorld(p, threads=O.max_threads())
    ow.add_particles(sc.pos, np.full(sc.n, sc.mass))
    w.step(DT, 2)
    ow.step(DT, 2)
    args = (0.01, 0.0, 0.4, 0.2)
    temp, src0 = _heat_grid((5, 7, 4), 12)
    _heat_check(O, w, ow, temp, src0, (0.0, 0.0, 0.0), 0.6, args)
    temp, src0 = _heat_grid((64, 64, 32), 13)
    _heat_check(O, w, ow, temp, src0, (0.1, 0.05, 0.2), 0.05, args)


def test_couple_heat_reference_tests(gpu):
    """couple_heat_warmer_fluid_rises and couple_heat_injects_source_into_moving_region
    (sph/tests.rs:214-290) on the device."""
    p = ref_test_params(gravity=(0.0, -9.81, 0.0))
    w = gpu.FluidWorld(p)
    w.add_particles([[0.0, 1.0, 0.0]], 0.05)
    temp = np.zeros((16, 16, 16))
    temp[:, 9:, :] = 1.0
    src = w.couple_heat(temp, np.zeros_like(temp), (-8.0, -8.0, -8.0), 1.0, 0.01, 0.0, 0.5, 0.0)
    assert w.body_acc[0, 1] == 9.81 * 0.5 and p.gravity[1] + w.body_acc[0, 1] > -9.81
    assert not src.any()
    p = ref_test_params(gravity=(0.0, 0.0, 0.0))
    w = gpu.FluidWorld(p)
    w.add_particles([[0.0, 0.0, 0.0]], 0.05, vel=[[2.0, 0.0, 0.0]])
    src = w.couple_heat(np.zeros((16, 16, 16)), np.zeros((16, 16, 16)), (0.0, 0.0, 0.0), 1.0, 0.01, 0.0, 0.0, 0.1)
    assert src[0, 0, 0] == 0.1 * 2.0 * 0.01 and np.count_nonzero(src) == 1


# ---- couple_bodies (world.rs:414-503) -----------------------------------------------------

def _quat(axis, angle):
    a = np.asarray(axis, np.float64)
    a = a / np.linalg.norm(a)
    return tuple(np.sin(angle / 2) * a) + (np.cos(angle / 2),)


TETRA = {"verts": (np.array([[0.0, 0.0, 0.0], [1.0, 0.0, 0.0], [0.0, 1.0, 0.0], [0.0, 0.0, 1.0]]) - 0.25) * 0.5,
         "faces": [[0, 2, 1], [0, 1, 3], [0, 3, 2], [1, 2, 3]]}  # outward (b - a) x (c - a)


def _bodies(shift=0.0):
    return [
        {"shape": "sphere", "size": (0.22,), "pos": (0.15 + shift, 0.0, 0.05), "vel": (0.0, -0.4, 0.1),
         "inv_mass": 2.0},
        {"shape": "box", "size": (0.3, 0.12, 0.2), "pos": (-0.25, 0.2, 0.0), "rot": _quat((1, 2, 3), 0.7),
         "inv_mass": 0.0},
        {"shape": "capsule", "size": (0.15, 0.1), "pos": (0.0, -0.3, -0.25), "rot": _quat((0, 0, 1), 1.1),
         "vel": (0.3, 0.0, 0.0), "inv_mass": 5.0},
        {"shape": "convex", **TETRA, "pos": (0.3, 0.3, 0.3), "rot": _quat((1, -1, 0), 0.4), "inv_mass": 3.0},
        {"shape": "heightfield", "size": (3, 2, 0.5), "heights": [0.1, 0.3, -0.2, 0.4, 0.0, 0.2], "pos": (0, -0.5, 0),
         "inv_mass": 1.0},
        {"shape": "box", "size": (0.1, 0.1, 0.1), "pos": (2.0, 2.0, 2.0), "vel": (0.0, 0.0, -0.0), "inv_mass": 4.0},
    ]


def _bodies_check(O, w, ow, bodies):
    vg = w.couple_bodies(bodies, DT)
    vo = ow.couple_bodies(bodies, DT)
    assert_bits_equal(vg, vo, "body velocities")
    assert_bits_equal(w.pos, ow.get(O.F_POS), "fluid positions")
    assert_bits_equal(w.vel, ow.get(O.F_VEL), "fluid velocities")
    return vg


def test_couple_bodies_f64_bitwise_and_next_steps(gpu, oracle_mod):
    O = oracle_mod
    w, ow, _ = _pair(gpu, O)
    x0 = w.pos.copy()
    vg = _bodies_check(O, w, ow, _bodies())
    assert np.count_nonzero(np.any(w.pos != x0, axis=1)) > 20, "particles were pushed out"
    assert not np.array_equal(vg[0], [0.0, -0.4, 0.1])
    w.step(DT, 5)
    ow.step(DT, 5)
    assert_bits_equal(w.pos, ow.get(O.F_POS), "positions after coupling and 5 steps")
    assert_bits_equal(w.vel, ow.get(O.F_VEL), "velocities after coupling and 5 steps")


@pytest.mark.parametrize("layout", ["disjoint", "overlapping", "many"])
def test_couple_bodies_per_body_and_ordered_loops(gpu, oracle_mod, layout):
    """Disjoint bodies (every flagged particle in one body: each body's sequence on its own
    thread), two overlapping spheres and a particle in both (the ordered loops as
    written), and 40 bodies (more than the per-body path takes): bit for bit against the
    oracle's loops, body velocities included."""
    O = oracle_mod
    w, ow, _ = _pair(gpu, O, lo=-0.6, hi=0.6, spacing=0.06, steps=1)
    rng = np.random.default_rng({"disjoint": 1, "overlapping": 2, "many": 3}[layout])
    if layout == "disjoint":
        centres = [(x, y, z) for x in (-0.3, 0.3) for y in (-0.3, 0.3) for z in (-0.3, 0.3)]
        bodies = [{"shape": "sphere", "size": (0.12,), "pos": c, "vel": tuple(rng.normal(0, 0.3, 3)),
                   "inv_mass": float(rng.uniform(0.5, 5.0))} for c in centres]
        bodies[3] = {"shape": "box", "size": (0.1, 0.08, 0.12), "pos": centres[3], "rot": _quat((1, 1, 0), 0.5),
                     "inv_mass": 0.0}
    elif layout == "overlapping":
        bodies = [{"shape": "sphere", "size": (0.2,), "pos": (0.0, 0.0, 0.0), "vel": (0.0, -0.3, 0.0),
                   "inv_mass": 2.0},
                  {"shape": "sphere", "size": (0.2,), "pos": (0.15, 0.05, 0.0), "vel": (0.2, 0.0, 0.0),
                   "inv_mass": 3.0},
                  {"shape": "sphere", "size": (0.1,), "pos": (-0.4, 0.4, 0.4), "inv_mass": 1.0}]
    else:
        bodies = [{"shape": "sphere", "size": (0.05,), "pos": tuple(rng.uniform(-0.55, 0.55, 3)),
                   "vel": tuple(rng.normal(0, 0.2, 3)), "inv_mass": float(rng.uniform(0.5, 5.0))}
                  for _ in range(40)]
    vg = _bodies_check(O, w, ow, bodies)
    assert np.isfinite(vg).all()


def test_couple_bodies_repeated_with_moving_bodies(gpu, oracle_mod):
    """Bodies integrated by the caller between steps (sph/tests.rs:160-169 style): the
    coupled trajectory stays bit-identical."""
    O = oracle_mod
    w, ow, p = _pair(gpu, O, steps=5)
    bodies = _bodies()
    g = np.array(p.gravity)
    for _ in range(25):
        for b in bodies:
            if b["inv_mass"] > 0:
                b["vel"] = tuple(np.asarray(b.get("vel", (0.0, 0.0, 0.0))) + g * DT)
                b["pos"] = tuple(np.asarray(b["pos"]) + np.asarray(b["vel"]) * DT)
        w.step(DT)
        ow.step(DT)
        v = _bodies_check(O, w, ow, bodies)
        for b, vb in zip(bodies, v):
            b["vel"] = tuple(vb)


def test_couple_bodies_on_tiled_compensated_world(gpu, oracle_mod):
    O = oracle_mod
    w, ow, _ = _pair(gpu, O, prec="comp", steps=20)
    _bodies_check(O, w, ow, _bodies(shift=0.05))
    w.step(DT, 10)
    assert np.isfinite(w.pos).all()


def test_couple_bodies_reference_tests(gpu):
    """static_body_blocks_fluid and dynamic_body_gets_buoyancy_upward (sph/tests.rs:96-175)."""
    w = gpu.FluidWorld(ref_test_params())
    w.fill_box((-1.5, -1.5, -0.5), (1.5, -1.0, 0.5), 0.1, 0.05)
    box = {"shape": "box", "size": (1.0, 0.5, 1.0), "pos": (0.0, 0.0, 0.0), "inv_mass": 0.0}
    for _ in range(100):
        w.step(DT)
        w.couple_bodies([box], DT)
    x = w.pos
    assert not np.any((np.abs(x[:, 0]) <= 1.0) & (np.abs(x[:, 1]) <= 0.5) & (np.abs(x[:, 2]) <= 1.0))
    p = ref_test_params(gravity=(0.0, -9.81, 0.0))
    w = gpu.FluidWorld(p)
    w.fill_box((-0.7, -0.7, -0.7), (0.7, 0.7, 0.7), 0.1, 0.05)
    w.step(DT, 15)
    mass_b = p.rest_density * (4.0 / 3.0 * np.pi * 0.6 ** 3) * 0.25
    pos, vel = np.zeros(3), np.zeros(3)
    for _ in range(120):
        vel = vel + np.array(p.gravity) * DT
        pos = pos + vel * DT
        w.step(DT)
        vel = w.couple_bodies([{"shape": "sphere", "size": (0.6,), "pos": pos, "vel": vel, "inv_mass": 1.0 / mass_b}],
                              DT)[0]
    assert pos[1] > 0.0


def test_couple_bodies_rejects_invalid_input(gpu):
    import ctypes as C
    from physics_b200 import _lib as L
    w = gpu.FluidWorld(ref_test_params())
    w.fill_box((-0.5,) * 3, (0.5,) * 3, 0.1, 0.05)
    bad_face = {"shape": "convex", "verts": TETRA["verts"], "faces": [[0, 1, 4]], "pos": (0, 0, 0)}
    with pytest.raises(gpu.PhyError):
        w.couple_bodies([bad_face], DT)
    arr = (L.PhyCoupleBody * 1)()
    arr[0].shape = 5  # compound without sub shapes
    d = np.zeros(1)
    f = np.zeros(1, np.uint32)
    assert L.load().phy_fluid_couple_bodies(w._h, 0, C.cast(arr, C.c_void_p), 1, d.ctypes.data_as(L.DP), 0,
                                            f.ctypes.data_as(C.POINTER(C.c_uint32)), 0, DT, 0.0) == -1
    arr[0].shape = 6  # no such shape
    assert L.load().phy_fluid_couple_bodies(w._h, 0, C.cast(arr, C.c_void_p), 1, d.ctypes.data_as(L.DP), 0,
                                            f.ctypes.data_as(C.POINTER(C.c_uint32)), 0, DT, 0.0) == -1
    # A compound whose sub shape is itself a compound (nesting is not supported).
    rec = np.zeros(17)
    rec[0], rec[10], rec[12] = 5.0, 1.0, 1.0
    arr[0].shape, arr[0].data_first, arr[0].data_count = 5, 0, 1
    assert L.load().phy_fluid_couple_bodies(w._h, 0, C.cast(arr, C.c_void_p), 1, rec.ctypes.data_as(L.DP), 16,
                                            f.ctypes.data_as(C.POINTER(C.c_uint32)), 0, DT, 0.0) == -1
    assert "nest" in L.last_error()
    with pytest.raises(ValueError):
        w.couple_bodies([{"shape": "compound", "pos": (0, 0, 0), "subs": [{"shape": "compound", "subs": []}]}], DT)
    w.couple_bodies([], DT)  # no bodies: no-op


def _compounds(shift=0.0):
    """Compound bodies (Shape::Compound, shape.rs:176-192): sub shapes with their own
    offsets and rotations, one static, two dynamic, one holding a convex and a heightfield
    sub shape (their data ranges follow the sub-shape records)."""
    return [
        {"shape": "compound", "pos": (0.1 + shift, 0.05, 0.0), "rot": _quat((0, 1, 1), 0.5), "vel": (0.1, -0.3, 0.0),
         "inv_mass": 1.5,
         "subs": [{"shape": "sphere", "size": (0.15,), "offset": (0.2, 0.0, 0.0)},
                  {"shape": "box", "size": (0.1, 0.2, 0.08), "offset": (-0.15, 0.05, 0.0),
                   "rot": _quat((1, 0, 0), 0.9)},
                  {"shape": "capsule", "size": (0.12, 0.06), "offset": (0.0, -0.2, 0.1),
                   "rot": _quat((0, 0, 1), 1.3)}]},
        {"shape": "compound", "pos": (-0.3, -0.25, 0.2), "inv_mass": 0.0,
         "subs": [{"shape": "box", "size": (0.2, 0.05, 0.2)},
                  {"shape": "sphere", "size": (0.1,), "offset": (0, 0.1, 0)}]},
        {"shape": "compound", "pos": (0.25, 0.25, 0.25), "rot": _quat((1, -1, 0), 0.4), "inv_mass": 3.0,
         "subs": [{"shape": "convex", **TETRA, "offset": (0.05, 0.0, 0.0), "rot": _quat((0, 1, 0), 0.3)},
                  {"shape": "heightfield", "size": (2, 2, 0.3), "heights": [0.1, 0.2, -0.1, 0.05],
                   "offset": (0.0, -0.1, 0.0)}]},
    ]


def test_couple_bodies_compound_bitwise(gpu, oracle_mod):
    """Compound bodies: containment in any sub shape, push-out to the farthest sub-shape
    support point, buoyancy of the summed sub-shape volumes, bit for bit against the
    oracle, then 25 coupled steps with caller-integrated bodies."""
    O = oracle_mod
    w, ow, p = _pair(gpu, O)
    x0 = w.pos.copy()
    bodies = _compounds()
    vg = _bodies_check(O, w, ow, bodies)
    assert np.count_nonzero(np.any(w.pos != x0, axis=1)) > 20, "particles were pushed out"
    assert not np.array_equal(vg[0], [0.1, -0.3, 0.0])
    g = np.array(p.gravity)
    for b, vb in zip(bodies, vg):
        b["vel"] = tuple(vb)
    for _ in range(25):
        for b in bodies:
            if b["inv_mass"] > 0:
                b["vel"] = tuple(np.asarray(b.get("vel", (0.0, 0.0, 0.0))) + g * DT)
                b["pos"] = tuple(np.asarray(b["pos"]) + np.asarray(b["vel"]) * DT)
        w.step(DT)
        ow.step(DT)
        v = _bodies_check(O, w, ow, bodies + _bodies())
        for b, vb in zip(bodies, v):
            b["vel"] = tuple(vb)
