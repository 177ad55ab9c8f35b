"""f64-plain CUDA step vs the CPU oracle and the golden fixtures: bit-exact.

Everything goes through the C ABI of libphysph.so (physics_b200.fluid is a
ctypes mirror of the reference's FluidWorld API)."""
import numpy as np
import pytest

from helpers import assert_bits_equal, ref_test_params
from physics_b200 import scenes

pytestmark = pytest.mark.gpu

FIELDS = ("pos", "vel", "acc", "rho", "p", "mu_eff", "xsph")


def gpu_world(gpu, params, precision="f64"):
    return gpu.FluidWorld(params, precision)


def state(w):
    return {k: getattr(w, k).copy() for k in FIELDS}


def oracle_state(O, w):
    fm = {"pos": O.F_POS, "vel": O.F_VEL, "acc": O.F_ACC, "rho": O.F_RHO, "p": O.F_P, "mu_eff": O.F_MU_EFF,
          "xsph": O.F_XSPH}
    return {k: w.get(f) for k, f in fm.items()}


def assert_state_equal(a, b, what):
    for k in FIELDS:
        assert_bits_equal(a[k], b[k], f"{what} {k}")


def test_quickstart_golden_200_steps(gpu, golden):
    g = golden("quickstart")
    w = gpu_world(gpu, gpu.SphParams.defaults())
    w.fill_box((-1, 1, -1), (1, 3, 1), 0.3, 0.1)
    assert w.len() == 343
    w.step(0.01)
    for k in FIELDS + ("mass",):
        assert_bits_equal(getattr(w, k), g[f"step1_{k}"], f"step1 {k}")
    done = 1
    for n in (50, 100, 200):
        w.step(0.01, n - done)
        done = n
        assert_bits_equal(w.pos, g[f"step{n}_pos"], f"step{n} pos")
        assert_bits_equal(w.vel, g[f"step{n}_vel"], f"step{n} vel")
    assert_bits_equal(w.rho, g["step200_rho"], "step200 rho")
    assert_bits_equal(w.acc, g["step200_acc"], "step200 acc")


def test_dam216_golden(gpu, golden):
    g = golden("dam216")
    p = gpu.SphParams.defaults()
    p.bounds_min, p.bounds_max = (0.0, 0.0, 0.0), (1.2, 1.2, 1.2)
    w = gpu_world(gpu, p)
    assert w.lattice_mass(0.1) == float(g["mass"])
    w.add_particles(g["init_pos"], float(g["mass"]))
    w.step(0.005)
    for k in FIELDS:
        assert_bits_equal(getattr(w, k), g[f"step1_{k}"], f"step1 {k}")
    w.step(0.005, 29)
    for k in FIELDS:
        assert_bits_equal(getattr(w, k), g[f"step30_{k}"], f"step30 {k}")


def test_materials_golden(gpu, golden):
    g = golden("materials")
    p = ref_test_params(gravity=(0.0, 0.0, 0.0))
    p.visc_k, p.visc_n = [3.5, 10.0], [1.0, 1.0]
    w = gpu_world(gpu, p)
    w.add_particles([[0, 0, 0], [0, 0.06, 0]], 0.05, vel=[[-300, 0, 0], [300, 0, 0]], material=[0, 1])
    w.step(0.001)
    for k in ("pos", "vel", "mu_eff", "acc", "rho"):
        assert_bits_equal(getattr(w, k), g[f"twomat_{k}"], f"twomat {k}")
    assert abs(w.effective_viscosity(0) - 3.5) < 1e-6 and abs(w.effective_viscosity(1) - 10.0) < 1e-6
    for n in (0.5, 1.0, 1.5):
        p = ref_test_params(gravity=(0.0, 0.0, 0.0))
        p.visc_k, p.visc_n = [3.5], [n]
        w = gpu_world(gpu, p)
        pos = [((ix - 2.0) * 0.08, iy * 0.06, 0.0) for iy in range(2) for ix in range(5)]
        vel = [((-300.0 if iy == 0 else 300.0), 0.0, 0.0) for iy in range(2) for ix in range(5)]
        w.add_particles(pos, 0.05, vel=vel)
        w.step(0.001)
        tag = str(n).replace(".", "p")
        if n == 1.0:
            assert_bits_equal(w.mu_eff, g[f"shear{tag}_mu_eff"], "shear n=1 mu")
            assert_bits_equal(w.pos, g[f"shear{tag}_pos"], "shear n=1 pos")
        else:
            # powf with n != 1: CUDA pow (<= 2 ulp) vs the C library's pow.
            np.testing.assert_allclose(w.mu_eff, g[f"shear{tag}_mu_eff"], rtol=1e-14)
            np.testing.assert_allclose(w.pos, g[f"shear{tag}_pos"], rtol=1e-12, atol=1e-14)


def _dam(nx, ny, nz):
    sc = scenes.dam_break(nx, ny, nz, box=2.0 * max(nx, ny, nz) * 0.1, dt=0.005, steps=0)
    p = scenes_params(sc)
    return sc, p


def scenes_params(sc):
    from physics_b200 import SphParams
    p = SphParams.defaults()
    p.bounds_min, p.bounds_max = sc.bounds_min, sc.bounds_max
    return p


@pytest.mark.parametrize("dims,steps", [((16, 24, 16), 100), ((5, 7, 3), 60), ((1, 1, 1), 5), ((2, 1, 1), 5)])
def test_free_running_bit_exact_vs_oracle(gpu, oracle_mod, dims, steps):
    sc, p = _dam(*dims)
    O = oracle_mod
    ow = O.OracleWorld(p, threads=O.max_threads())
    ow.add_particles(sc.pos, sc.mass)
    w = gpu_world(gpu, p)
    w.add_particles(sc.pos, sc.mass)
    chunks = [1, steps // 2 - 1, steps - steps // 2]
    for c in chunks:
        if c <= 0:
            continue
        ow.step(sc.dt, c)
        w.step(sc.dt, c)
        assert_state_equal(state(w), oracle_state(O, ow), f"{dims}")


def test_teacher_forced_mid_run_state(gpu, oracle_mod):
    """Upload a developed (splashing) oracle state, take one step on both, compare."""
    O = oracle_mod
    sc, p = _dam(12, 16, 12)
    ow = O.OracleWorld(p, threads=O.max_threads())
    ow.add_particles(sc.pos, sc.mass)
    ow.step(0.005, 150)
    w = gpu_world(gpu, p)
    w.add_particles(ow.get(O.F_POS), ow.get(O.F_MASS), vel=ow.get(O.F_VEL))
    ow.step(0.005)
    w.step(0.005)
    assert_state_equal(state(w), oracle_state(O, ow), "teacher-forced")


def test_run_to_run_bit_exact(gpu):
    sc, p = _dam(20, 30, 20)
    outs = []
    for _ in range(2):
        w = gpu_world(gpu, p)
        w.add_particles(sc.pos, sc.mass)
        w.step(0.005, 40)
        outs.append(state(w))
    assert_state_equal(outs[0], outs[1], "run-to-run")


def test_empty_world_step_is_noop(gpu):
    w = gpu_world(gpu, gpu.SphParams.defaults())
    w.step(0.01, 3)
    assert w.len() == 0 and w.is_empty()
    assert w.pos.shape == (0, 3)


def test_live_h_change_matches_oracle(gpu, oracle_mod):
    """F7: kernels/grid keep the construction h; the cutoff follows params.h."""
    O = oracle_mod
    sc, p = _dam(6, 6, 6)
    ow = O.OracleWorld(p)
    ow.add_particles(sc.pos, sc.mass)
    w = gpu_world(gpu, p)
    w.add_particles(sc.pos, sc.mass)
    p2 = scenes_params(sc)
    p2.h = 0.17
    ow.set_params(p2)
    w.params = p2
    ow.step(0.005, 3)
    w.step(0.005, 3)
    assert_state_equal(state(w), oracle_state(O, ow), "live h")
    p3 = scenes_params(sc)
    p3.h = 0.26  # larger than the captured h: still only 27 cells of the captured size
    ow.set_params(p3)
    w.params = p3
    ow.step(0.005, 2)
    w.step(0.005, 2)
    assert_state_equal(state(w), oracle_state(O, ow), "live h up")


def test_host_mutation_between_steps(gpu, oracle_mod):
    """Writes to particles between steps (sph/tests.rs:222-225 style): velocity, body_acc,
    mass, material and params all take effect on the next step."""
    O = oracle_mod
    sc, p = _dam(8, 8, 8)
    p.visc_k, p.visc_n = [3.5, 7.0, 1.0], [1.0, 1.0, 1.0]
    ow = O.OracleWorld(p)
    ow.add_particles(sc.pos, sc.mass)
    w = gpu_world(gpu, p)
    w.add_particles(sc.pos, sc.mass)
    ow.step(0.005, 5)
    w.step(0.005, 5)
    rng = np.random.default_rng(7)
    n = w.len()
    vel = ow.get(O.F_VEL) + rng.normal(0, 0.1, (n, 3))
    ba = rng.normal(0, 1.0, (n, 3))
    mat = rng.integers(0, 5, n).astype(np.float64)  # 3 and 4 fall back to material 0
    ow.set(O.F_VEL, vel)
    w.vel = vel
    ow.set(O.F_BODY_ACC, ba)
    w.body_acc = ba
    ow.set(O.F_MATERIAL, mat)
    w.material = mat
    p.gravity = (0.5, -3.0, 0.0)
    ow.set_params(p)
    w.params = p
    ow.step(0.005)
    w.step(0.005)
    assert_state_equal(state(w), oracle_state(O, ow), "after host writes")
    assert np.all(w.body_acc == 0.0)  # integrate clears body_acc (world.rs:361)
    ow.step(0.005, 4)
    w.step(0.005, 4)
    assert_state_equal(state(w), oracle_state(O, ow), "continued")


def test_particles_outside_bounds_are_clamped(gpu, oracle_mod):
    """Initial positions outside bounds and negative coordinates (the grid box grows to hold them)."""
    O = oracle_mod
    p = ref_test_params()
    rng = np.random.default_rng(11)
    pos = rng.uniform(-4.5, 4.5, (400, 3))
    pos[:50] = rng.uniform(-0.3, 0.3, (50, 3))  # a dense clump
    vel = rng.normal(0, 2.0, (400, 3))
    ow = O.OracleWorld(p)
    ow.add_particles(pos, 0.5, vel=vel)
    w = gpu_world(gpu, p)
    w.add_particles(pos, 0.5, vel=vel)
    for _ in range(3):
        ow.step(0.004, 4)
        w.step(0.004, 4)
        assert_state_equal(state(w), oracle_state(O, ow), "outside bounds")
    assert (w.pos >= -3.0).all() and (w.pos <= 3.0).all()


def test_append_after_steps(gpu, oracle_mod):
    """add_particle after stepping keeps insertion order (world.rs:171-174)."""
    O = oracle_mod
    sc, p = _dam(5, 5, 5)
    ow = O.OracleWorld(p)
    ow.add_particles(sc.pos, sc.mass)
    w = gpu_world(gpu, p)
    w.add_particles(sc.pos, sc.mass)
    ow.step(0.005, 3)
    w.step(0.005, 3)
    extra = sc.pos[:7] + 0.013
    ow.add_particles(extra, sc.mass, vel=np.ones_like(extra), material=[0] * 7)
    w.add_particles(extra, sc.mass, vel=np.ones_like(extra), material=[0] * 7)
    ow.step(0.005, 3)
    w.step(0.005, 3)
    assert_state_equal(state(w), oracle_state(O, ow), "append")


def test_nonfinite_particle_matches_reference_semantics(gpu, oracle_mod):
    """A NaN particle sits in cell key 0 on its NaN axes (grid.rs:29-31, to_i64 None -> 0):
    it is skipped by the density sums but poisons neighbours' forces, exactly as the
    reference does; step_checked reports NonFinite (2)."""
    O = oracle_mod
    p = ref_test_params(gravity=(0.0, 0.0, 0.0))
    rng = np.random.default_rng(5)
    pos = rng.uniform(-0.3, 0.3, (200, 3))
    pos[17] = (np.nan, 0.05, 0.05)
    ow = O.OracleWorld(p)
    ow.add_particles(pos, 0.2)
    w = gpu_world(gpu, p)
    w.add_particles(pos, 0.2)
    ow.step(0.001)
    w.step(0.001)
    a, b = state(w), oracle_state(O, ow)
    for k in FIELDS:
        x, y = np.asarray(a[k]), np.asarray(b[k])
        assert np.array_equal(np.isnan(x), np.isnan(y)), k
        m = ~np.isnan(x)
        assert_bits_equal(x[m], y[m], f"nan case {k}")
    world = gpu.World()
    sub = world.add_fluid(p)
    sub.world.add_particles(pos, 0.2)
    assert world.step_checked(0.001) == 2
