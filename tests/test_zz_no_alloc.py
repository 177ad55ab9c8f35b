"""phy_fluid_density_noalloc: the density pass for callers that cannot allocate
device memory at the moment they need it (an engine that owns all device
memory, an allocator policy that forbids foreign cudaMalloc, a loop that must
not enter the driver's allocator).  It must match the density and pressure
that FluidWorld::step computes through the regular entry points, bit for bit
(the f64 plain tolerance), on two calls in a row that share its fixed scratch
array.  This file sorts last so that a run stopping at the first failure has
already run every other test."""
import ctypes as C

import numpy as np
import pytest

from helpers import assert_bits_equal
from physics_b200 import _lib as L
from physics_b200 import scenes

pytestmark = pytest.mark.gpu


def _ptr(t):
    return C.c_void_p(t.data_ptr())


def _step_density(gpu, p, pos, mass, dt=0.005):
    """rho and p that FluidWorld::step computes from the positions it starts from."""
    w = gpu.FluidWorld(p, "f64")
    w.add_particles(pos, mass)
    w.step(dt)
    return w.rho, w.p


def _noalloc(gpu, p, pos, mass, stream_ptr):
    """Calls the entry point on device copies of pos/mass; returns (rc, rho, p) with
    the outputs preset to NaN so that an unwritten value shows."""
    import torch
    lib = L.load()
    dev = torch.device("cuda", 0)
    n = pos.shape[0]
    d_pos = torch.tensor(pos, dtype=torch.float64, device=dev).contiguous()
    d_mass = torch.tensor(mass, dtype=torch.float64, device=dev)
    d_rho = torch.full((n,), float("nan"), dtype=torch.float64, device=dev)
    d_p = torch.full((n,), float("nan"), dtype=torch.float64, device=dev)
    torch.cuda.synchronize(dev)
    c = p.to_c()
    rc = lib.phy_fluid_density_noalloc(C.byref(c), n, _ptr(d_pos), _ptr(d_mass), _ptr(d_rho), _ptr(d_p),
                                       stream_ptr)
    torch.cuda.synchronize(dev)
    return rc, d_rho.cpu().numpy(), d_p.cpu().numpy()


def test_density_without_allocation_matches_step(gpu):
    import torch

    lib = L.load()
    sc = scenes.dam_break(14, 20, 14, box=4.0, dt=0.005, steps=0)
    rng = np.random.default_rng(9)
    pos = sc.pos + rng.uniform(-0.02, 0.02, sc.pos.shape)
    mass = np.full(sc.n, sc.mass) * rng.uniform(0.9, 1.1, sc.n)
    p = gpu.SphParams.defaults()
    p.bounds_min, p.bounds_max = sc.bounds_min, sc.bounds_max

    # The regular entry points: FluidWorld::step computes rho and p of the
    # positions it starts from.
    ref_rho, ref_p = _step_density(gpu, p, pos, mass, sc.dt)

    dev = torch.device("cuda", 0)
    d_pos = torch.tensor(pos, dtype=torch.float64, device=dev).contiguous()
    d_mass = torch.tensor(mass, dtype=torch.float64, device=dev)
    d_rho = torch.empty(sc.n, dtype=torch.float64, device=dev)
    d_p = torch.empty(sc.n, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)
    c = p.to_c()
    for _ in range(2):
        d_rho.fill_(float("nan"))
        d_p.fill_(float("nan"))
        torch.cuda.synchronize(dev)
        rc = lib.phy_fluid_density_noalloc(C.byref(c), sc.n, _ptr(d_pos), _ptr(d_mass), _ptr(d_rho), _ptr(d_p),
                                           C.c_void_p(stream.cuda_stream))
        assert rc == 0, L.last_error()
        assert_bits_equal(d_rho.cpu().numpy(), ref_rho, "rho")
        assert_bits_equal(d_p.cpu().numpy(), ref_p, "p")


def test_density_without_allocation_on_the_default_stream(gpu):
    """A NULL stream is the legacy default stream; the call returns after it finished.
    A larger scene is followed by a smaller one, so the second call also checks that
    the shared scratch starts from cleared counts."""
    p = gpu.SphParams.defaults()
    for dims in ((12, 16, 12), (6, 9, 5)):
        sc = scenes.dam_break(*dims, box=3.2, dt=0.005, steps=0)
        p.bounds_min, p.bounds_max = sc.bounds_min, sc.bounds_max
        mass = np.full(sc.n, sc.mass)
        ref_rho, ref_p = _step_density(gpu, p, sc.pos, mass)
        rc, rho, pr = _noalloc(gpu, p, sc.pos, mass, None)
        assert rc == 0, L.last_error()
        assert_bits_equal(rho, ref_rho, "rho (default stream)")
        assert_bits_equal(pr, ref_p, "p (default stream)")


def test_density_without_allocation_nan_particle(gpu):
    """A NaN coordinate maps to cell key 0 on that axis (grid.rs:29-31); the NaN particle
    takes no density term (r = NaN is never < h) and adds none to its neighbours, as in
    FluidWorld::step, bit for bit."""
    p = gpu.SphParams.defaults()
    p.bounds_min, p.bounds_max = (-1.0, -1.0, -1.0), (1.0, 1.0, 1.0)
    rng = np.random.default_rng(5)
    pos = rng.uniform(-0.3, 0.3, (300, 3))
    pos[17] = (np.nan, 0.05, 0.05)
    pos[101] = (0.1, np.nan, np.nan)
    mass = np.full(pos.shape[0], 0.2)
    ref_rho, ref_p = _step_density(gpu, p, pos, mass, 0.001)
    rc, rho, pr = _noalloc(gpu, p, pos, mass, None)
    assert rc == 0, L.last_error()
    assert_bits_equal(rho, ref_rho, "rho (NaN particle)")
    assert_bits_equal(pr, ref_p, "p (NaN particle)")
    assert rho[17] == 0.0 and rho[101] == 0.0


def test_density_without_allocation_rejects_oversize(gpu):
    lib = L.load()
    c = gpu.SphParams.defaults().to_c()
    rc = lib.phy_fluid_density_noalloc(C.byref(c), L.NOALLOC_MAX_PARTICLES + 1, C.c_void_p(8), C.c_void_p(8),
                                       C.c_void_p(8), C.c_void_p(8), None)
    assert rc == -1 and "scratch capacity" in L.last_error()


@pytest.mark.parametrize("far", [100.0, 1.0e18])
def test_density_without_allocation_rejects_wide_box(gpu, far):
    """Few particles whose padded cell-key box exceeds PHY_NOALLOC_MAX_CELLS: -1 and the
    'grid cells' message, before any kernel touches the scratch.  At 1e18 the keys lie
    near opposite ends of the int64 range (their difference overflows int64)."""
    p = gpu.SphParams.defaults()
    pos = np.array([[-far, 0.0, 0.0], [0.0, 0.0, 0.0], [far, far, 0.0]])
    mass = np.full(3, 0.02)
    rc, rho, _ = _noalloc(gpu, p, pos, mass, None)
    assert rc == -1 and "grid cells" in L.last_error(), L.last_error()
    assert np.isnan(rho).all()
    # The entry point still works after a rejected call.
    sc = scenes.dam_break(6, 8, 6, box=3.2, dt=0.005, steps=0)
    p.bounds_min, p.bounds_max = sc.bounds_min, sc.bounds_max
    m = np.full(sc.n, sc.mass)
    ref_rho, _ = _step_density(gpu, p, sc.pos, m)
    rc, rho, _ = _noalloc(gpu, p, sc.pos, m, None)
    assert rc == 0, L.last_error()
    assert_bits_equal(rho, ref_rho, "rho after a rejected call")
