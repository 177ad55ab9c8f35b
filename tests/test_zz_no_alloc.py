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
    w = gpu.FluidWorld(p, "f64")
    w.add_particles(pos, mass)
    w.step(sc.dt)
    ref_rho, ref_p = w.rho, w.p

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


def test_density_without_allocation_rejects_oversize(gpu):
    lib = L.load()
    c = gpu.SphParams.defaults().to_c()
    rc = lib.phy_fluid_density_noalloc(C.byref(c), L.NOALLOC_MAX_PARTICLES + 1, C.c_void_p(8), C.c_void_p(8),
                                       C.c_void_p(8), C.c_void_p(8), None)
    assert rc == -1 and "scratch capacity" in L.last_error()
