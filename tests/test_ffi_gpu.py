"""The reference's phy-ffi tests (crates/phy-ffi/src/lib.rs:901-1016) run on the
CUDA build through the raw C ABI, plus checkpoint and World-level behaviour."""
import ctypes as C
import math

import numpy as np
import pytest

from helpers import assert_bits_equal
from physics_b200 import _lib as L

pytestmark = pytest.mark.gpu


def dp(a):
    return a.ctypes.data_as(L.DP)


def test_ffi_fluid_lifecycle_and_readback(gpu):
    lib = L.load()
    w = lib.phy_world_create_fluid()
    assert w
    assert lib.phy_world_sub_count(w) >= 1
    n = lib.phy_world_fluid_count(w)
    assert n > 0
    t0 = lib.phy_world_time(w)
    for _ in range(200):
        assert lib.phy_world_step(w, 0.005) == 0
    t1 = lib.phy_world_time(w)
    assert abs(t1 - t0 - 1.0) < 1e-6
    buf = np.empty(3 * n, np.float64)
    assert lib.phy_world_get_fluid_positions(w, dp(buf), buf.size) == n
    assert np.isfinite(buf).all()
    # truncation: a short buffer receives len/3 particles
    short = np.empty(3 * 5 + 2, np.float64)
    assert lib.phy_world_get_fluid_positions(w, dp(short), short.size) == 5
    assert_bits_equal(short[:15], buf[:15], "truncated readback")
    lib.phy_world_destroy(w)


def test_create_fluid_scene_matches_oracle(gpu, oracle_mod):
    """build_fluid_world (lib.rs:113-126) stepped 50 x 0.005 equals the oracle bit for bit."""
    O = oracle_mod
    lib = L.load()
    w = lib.phy_world_create_fluid()
    for _ in range(50):
        assert lib.phy_world_step(w, 0.005) == 0
    n = lib.phy_world_fluid_count(w)
    pos = np.empty(3 * n, np.float64)
    vel = np.empty(3 * n, np.float64)
    lib.phy_world_get_fluid_positions(w, dp(pos), pos.size)
    lib.phy_world_get_fluid_velocities(w, dp(vel), vel.size)
    lib.phy_world_destroy(w)
    ow = O.OracleWorld(gpu.SphParams.defaults(), threads=O.max_threads())
    ow.fill_box((-4.0, -4.0, -1.0), (0.0, 4.0, 1.0), 0.18, 0.05)
    assert len(ow) == n
    ow.step(0.005, 50)
    assert_bits_equal(pos.reshape(-1, 3), ow.get(O.F_POS), "create_fluid pos")
    assert_bits_equal(vel.reshape(-1, 3), ow.get(O.F_VEL), "create_fluid vel")


def test_ffi_checked_step_reports_health(gpu):
    lib = L.load()
    w = lib.phy_world_create_fluid()
    for _ in range(200):
        assert lib.phy_world_step_checked(w, 0.005) == 0
    assert lib.phy_world_step_checked(None, 0.01) == -1
    lib.phy_world_destroy(w)


def test_ffi_f32_channel_matches_f64(gpu):
    lib = L.load()
    w = lib.phy_world_create_fluid()
    for _ in range(120):
        assert lib.phy_world_step_f32(w, 0.005) == 0
    n = lib.phy_world_fluid_count(w)
    b64 = np.empty(3 * n, np.float64)
    b32 = np.empty(3 * n, np.float32)
    assert lib.phy_world_get_fluid_positions(w, dp(b64), b64.size) == n
    assert lib.phy_world_get_fluid_positions_f32(w, b32.ctypes.data_as(L.FP), b32.size) == n
    assert np.array_equal(b32, b64.astype(np.float32))
    v64 = np.empty(3 * n, np.float64)
    v32 = np.empty(3 * n, np.float32)
    lib.phy_world_get_fluid_velocities(w, dp(v64), v64.size)
    lib.phy_world_get_fluid_velocities_f32(w, v32.ctypes.data_as(L.FP), v32.size)
    assert np.array_equal(v32, v64.astype(np.float32))
    # A short buffer takes whole particles only, in insertion order (lib.rs:399-460).
    half = np.full(3 * (n // 2) + 2, -1.0, np.float32)
    assert lib.phy_world_get_fluid_positions_f32(w, half.ctypes.data_as(L.FP), half.size) == n // 2
    assert np.array_equal(half[:3 * (n // 2)], b32[:3 * (n // 2)]) and (half[3 * (n // 2):] == -1.0).all()
    lib.phy_world_destroy(w)


def test_save_load_roundtrip_bit_exact(gpu, tmp_path):
    """phy_world_save / phy_world_load (lib.rs:517-542): the archive is lossless and the
    reloaded world continues on the same trajectory."""
    lib = L.load()
    w = lib.phy_world_create_fluid()
    for _ in range(30):
        lib.phy_world_step(w, 0.005)
    path = str(tmp_path / "world.json").encode()
    assert lib.phy_world_save(w, path) == 0
    w2 = lib.phy_world_load(path)
    assert w2
    assert lib.phy_world_sub_count(w2) == lib.phy_world_sub_count(w)
    assert lib.phy_world_time(w2) == lib.phy_world_time(w)
    n = lib.phy_world_fluid_count(w)
    for _ in range(20):
        lib.phy_world_step(w, 0.005)
        lib.phy_world_step(w2, 0.005)
    a = np.empty(3 * n, np.float64)
    b = np.empty(3 * n, np.float64)
    lib.phy_world_get_fluid_positions(w, dp(a), a.size)
    lib.phy_world_get_fluid_positions(w2, dp(b), b.size)
    assert_bits_equal(a, b, "continued after reload")
    text = open(path, "rb").read().decode()
    assert text.startswith('{"version":1,"time":{"__f64":') and '"Fluid":{"world":{"params":' in text
    lib.phy_world_destroy(w)
    lib.phy_world_destroy(w2)


def test_world_multiple_fluid_subsystems(gpu):
    """Two fluid subsystems in one World: readbacks concatenate in subsystem order."""
    p = gpu.SphParams.defaults()
    world = gpu.World()
    a = world.add_fluid(p)
    b = world.add_fluid(p, "comp")
    a.world.fill_box((-1, -1, -1), (0, 0, 0), 0.1, 0.05)
    b.world.fill_box((1, 1, 1), (2, 2, 2), 0.1, 0.05)
    for _ in range(5):
        world.step(0.005)
    assert world.fluid_count() == a.world.len() + b.world.len()
    allpos = world.fluid_positions()
    assert_bits_equal(allpos[: a.world.len()], a.world.pos, "sub 0")
    assert_bits_equal(allpos[a.world.len():], b.world.pos, "sub 1")
    assert math.isclose(world.time(), 0.025)
    sub = world.get(0)
    sub.drag = 2.5
    assert sub.drag == 2.5 and sub.friction == 0.1


def test_readback_into_pinned_buffer_and_across_subsystems(gpu):
    """phy_world_get_fluid_positions/velocities copy straight into the caller's buffer
    (lib.rs:399-460): the same bits whether the buffer is pageable or registered with
    phy_fluid_pin_host, and truncation at len/3 particles that stops inside the second
    subsystem keeps the first subsystem whole and the second's leading particles."""
    lib = L.load()
    p = gpu.SphParams.defaults()
    world = gpu.World()
    a = world.add_fluid(p)
    b = world.add_fluid(p, "comp")
    a.world.fill_box((-1, -1, -1), (0, 0, 0), 0.1, 0.05)
    b.world.fill_box((1, 1, 1), (2, 2, 2), 0.1, 0.05)
    for _ in range(3):
        world.step(0.005)
    na, nb = a.world.len(), b.world.len()
    ref_pos = np.concatenate([a.world.pos, b.world.pos]).reshape(-1)
    ref_vel = np.concatenate([a.world.vel, b.world.vel]).reshape(-1)
    h = world.handle
    pinned = np.empty(3 * (na + nb), np.float64)
    assert lib.phy_fluid_pin_host(pinned.ctypes.data, pinned.nbytes) == 0, L.last_error()
    try:
        for fn, ref in ((lib.phy_world_get_fluid_positions, ref_pos), (lib.phy_world_get_fluid_velocities, ref_vel)):
            pinned[:] = np.nan
            assert fn(h, dp(pinned), pinned.size) == na + nb
            assert_bits_equal(pinned, ref, "pinned readback")
            k = na + 7
            short = np.full(3 * k + 1, -1.0)
            assert fn(h, dp(short), short.size) == k
            assert_bits_equal(short[: 3 * k], ref[: 3 * k], "truncated across subsystems")
            assert short[-1] == -1.0  # nothing written past len/3 particles
            pinned[:] = np.nan
            assert fn(h, dp(pinned), 3 * k) == k
            assert_bits_equal(pinned[: 3 * k], ref[: 3 * k], "truncated pinned readback")
            assert np.isnan(pinned[3 * k:]).all()
    finally:
        assert lib.phy_fluid_unpin_host(pinned.ctypes.data) == 0, L.last_error()
    assert lib.phy_fluid_unpin_host(pinned.ctypes.data) == -1  # no longer registered


def test_diagnostics_match_oracle(gpu, oracle_mod):
    O = oracle_mod
    p = gpu.SphParams.defaults()
    w = gpu.FluidWorld(p)
    w.fill_box((-1, -1, -1), (0, 0.5, 0), 0.1, 0.05)
    ow = O.OracleWorld(p)
    ow.fill_box((-1, -1, -1), (0, 0.5, 0), 0.1, 0.05)
    w.step(0.005, 20)
    ow.step(0.005, 20)
    d = ow.diagnostics()
    assert_bits_equal(w.total_momentum(), d[:3], "momentum")
    assert w.kinetic_energy() == d[3]


def test_invalid_arguments_fail_cleanly(gpu):
    lib = L.load()
    p = gpu.SphParams.defaults()
    w = gpu.FluidWorld(p)
    w.fill_box((0, 0, 0), (0.3, 0.3, 0.3), 0.1, 0.0)
    small = np.empty(2, np.float64)
    assert lib.phy_fluid_get_field(w._h, 0, L.FIELD_POS, dp(small), 2) == -1
    assert "too small" in L.last_error()
    assert lib.phy_fluid_get_field(w._h, 0, 42, dp(small), 2) == -1
    assert lib.phy_fluid_len(w._h, 7) == -1
    bad = L.PhySphParams()
    lib.phy_sph_params_defaults(C.byref(bad))
    bad.n_visc_k = 0
    assert not lib.phy_fluid_world_create(C.byref(bad), 0)
    assert not lib.phy_fluid_world_create(C.byref(bad), 9)
    # bounds spanning more than 2^27 cells of size h are rejected, not silently clamped
    huge = gpu.SphParams.defaults()
    huge.bounds_min, huge.bounds_max = (-1e6, -1e6, -1e6), (1e6, 1e6, 1e6)
    hw = gpu.FluidWorld(huge)
    with pytest.raises(gpu.PhyError):
        hw.add_particles([[0.0, 0.0, 0.0]], 1.0)
        hw.step(0.01)
