"""Spatial decomposition of one scene into x-slabs (physics_b200.decomp), checked on the
CPU with the oracle as each slab's world: slabs in one process and two gloo ranks that
exchange halos and migrating particles point to point both give the same bits as the
whole scene stepped in one world."""
import os
import socket

import numpy as np
import pytest

from helpers import assert_bits_equal
from physics_b200 import decomp, scenes

DT = 0.005
STEPS = 30


class OracleSlabWorld:
    """The oracle behind the steppers' world interface."""

    def __init__(self, O, params):
        self.O = O
        self.w = O.OracleWorld(params)

    def add(self, pos, vel, mass, material):
        if len(mass):
            self.w.add_particles(pos, mass, vel=vel, material=material)

    def step(self, dt):
        self.w.step(dt)

    def read(self):
        O = self.O
        f = {"pos": O.F_POS, "vel": O.F_VEL, "rho": O.F_RHO, "p": O.F_P, "acc": O.F_ACC, "mu_eff": O.F_MU_EFF,
             "xsph": O.F_XSPH}
        return {k: self.w.get(v) for k, v in f.items()}


def _scene(seed=5):
    sc = scenes.dam_break(10, 16, 10, box=3.2, dt=DT, steps=0)
    from physics_b200 import SphParams
    p = SphParams.defaults()
    p.bounds_min, p.bounds_max = sc.bounds_min, sc.bounds_max
    vel = np.random.default_rng(seed).normal(0.0, 0.5, sc.pos.shape)  # particles cross slab edges
    mat = (np.arange(sc.n) % 3 == 0).astype(np.uint32)
    return sc, p, vel, mat


def _whole(make_world, sc, vel, mat, steps):
    w = make_world()
    w.add(sc.pos, vel, np.full(sc.n, sc.mass), mat)
    for _ in range(steps):
        w.step(DT)
    return w.read()


@pytest.mark.parametrize("nslabs", [1, 2, 3, 5])
def test_slabs_in_one_process_equal_the_whole_world(oracle_mod, nslabs):
    O = oracle_mod
    sc, p, vel, mat = _scene()
    p.visc_k, p.visc_n = [3.5, 7.0], [1.0, 1.0]
    st = decomp.SlabStepper(lambda: OracleSlabWorld(O, p), p.h, nslabs, sc.pos, sc.mass, vel=vel, material=mat)
    st.step(DT, STEPS)
    ref = _whole(lambda: OracleSlabWorld(O, p), sc, vel, mat, STEPS)
    for f in decomp.FIELDS:
        assert_bits_equal(st.state[f], ref[f], f"{f}, {nslabs} slabs")
    if nslabs > 1:
        k = decomp.key_x(st.state["pos"], p.h)
        owned = [int(decomp.slab_mask(k, st.edges[r], st.edges[r + 1]).sum()) for r in range(nslabs)]
        assert min(owned) > 0 and sum(owned) == sc.n


def test_one_cell_halo_is_not_enough(oracle_mod, monkeypatch):
    """With a 1-cell halo the halo particles' densities miss their own outer neighbours, and
    the owned particles next to a slab edge take wrong pressure forces: the check above
    would see it."""
    O = oracle_mod
    sc, p, vel, mat = _scene()
    monkeypatch.setattr(decomp, "HALO", 1)
    st = decomp.SlabStepper(lambda: OracleSlabWorld(O, p), p.h, 3, sc.pos, sc.mass, vel=vel, material=mat)
    st.step(DT, 3)
    ref = _whole(lambda: OracleSlabWorld(O, p), sc, vel, mat, 3)
    assert not np.array_equal(st.state["acc"], ref["acc"])


def test_more_slabs_than_columns_and_a_nan_particle(oracle_mod):
    """Twelve slabs over a block five cell columns wide (most slabs own nothing), and a
    particle whose x is NaN (its cell key is 0 on that axis, as Grid::key_of gives it):
    still the whole world's bits."""
    O = oracle_mod
    sc, p, vel, mat = _scene(seed=8)
    pos = sc.pos.copy()
    pos[17, 0] = np.nan
    st = decomp.SlabStepper(lambda: OracleSlabWorld(O, p), p.h, 12, pos, sc.mass, vel=vel, material=mat)
    st.step(DT, 5)
    from types import SimpleNamespace
    ref = _whole(lambda: OracleSlabWorld(O, p), SimpleNamespace(n=sc.n, mass=sc.mass, pos=pos), vel, mat, 5)
    for f in decomp.FIELDS:
        assert_bits_equal(st.state[f], ref[f], f"{f}, 12 slabs with a NaN particle")


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world_size, port, q):
    import torch.distributed as dist
    from oracle import oracle as O
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world_size)
    try:
        O.build()
        sc, p, vel, mat = _scene()
        mine = np.flatnonzero(np.arange(sc.n) % world_size == rank)  # any start; the first step re-slabs
        st = decomp.RankSlabStepper(lambda: OracleSlabWorld(O, p), p.h, mine, sc.pos[mine], sc.mass,
                                    vel=vel[mine], material=mat[mine])
        st.step(DT, 15)
        ids, state = st.gather_state()
        q.put((rank, len(st.ids), ids, state if rank == 0 else None))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_equal_the_whole_world(oracle_mod):
    import multiprocessing as mp
    O = oracle_mod
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for pr in procs:
        pr.start()
    out = sorted([q.get(timeout=300) for _ in procs], key=lambda t: t[0])
    for pr in procs:
        pr.join(timeout=60)
        assert pr.exitcode == 0
    sc, p, vel, mat = _scene()
    assert out[0][1] > 0 and out[1][1] > 0 and out[0][1] + out[1][1] == sc.n
    ids, state = out[0][2], out[0][3]
    assert np.array_equal(ids, np.arange(sc.n))
    ref = _whole(lambda: OracleSlabWorld(O, p), sc, vel, mat, 15)
    for f in decomp.FIELDS:
        assert_bits_equal(state[f], ref[f], f"{f}, two ranks")


@pytest.mark.gpu
def test_device_slabs_equal_the_whole_device_world(gpu):
    """The same decomposition over device f64 worlds (one per slab, in one process): the
    slabs give the whole device world's bits."""
    sc, p, vel, mat = _scene()
    make = lambda: decomp.DeviceWorld(p, "f64")  # noqa: E731
    st = decomp.SlabStepper(make, p.h, 3, sc.pos, sc.mass, vel=vel, material=mat)
    st.step(DT, 10)
    ref = _whole(make, sc, vel, mat, 10)
    for f in decomp.FIELDS:
        assert_bits_equal(st.state[f], ref[f], f"{f}, device slabs")


class OracleResidentWorld:
    """The oracle behind the resident steppers' tensor interface (host tensors)."""

    def __init__(self, O, params):
        self.O, self.params = O, params

    def load(self, pos, vel, mass, material):
        self.w = self.O.OracleWorld(self.params)
        if mass.shape[0]:
            self.w.add_particles(pos.numpy(), mass.numpy(), vel=vel.numpy(), material=material.numpy())

    def step(self, dt):
        self.w.step(dt)

    def read(self):
        import torch
        return {k: torch.from_numpy(np.ascontiguousarray(v)) for k, v in OracleSlabWorld.read(self).items()}


def _resident_rank_main(rank, world_size, port, q):
    import torch.distributed as dist
    from oracle import oracle as O
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world_size)
    try:
        O.build()
        sc, p, vel, mat = _scene()
        mine = np.flatnonzero(np.arange(sc.n) % world_size == rank)
        st = decomp.ResidentSlabStepper(lambda: OracleResidentWorld(O, p), p.h, mine, sc.pos[mine], sc.mass,
                                        vel=vel[mine], material=mat[mine])
        st.step(DT, 15)
        ids, state = st.gather_state()
        q.put((rank, int(st.ids.shape[0]), ids, state if rank == 0 else None))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world_size", [2, 3])
def test_resident_ranks_equal_the_whole_world(oracle_mod, world_size):
    """The device-resident form's exchange (typed records, grouped point-to-point,
    persistent slab worlds reloaded in place) on gloo ranks over host tensors: the whole
    world's bits."""
    import multiprocessing as mp
    O = oracle_mod
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_resident_rank_main, args=(r, world_size, port, q)) for r in range(world_size)]
    for pr in procs:
        pr.start()
    out = sorted([q.get(timeout=300) for _ in procs], key=lambda t: t[0])
    for pr in procs:
        pr.join(timeout=60)
        assert pr.exitcode == 0
    sc, p, vel, mat = _scene()
    assert all(o[1] > 0 for o in out) and sum(o[1] for o in out) == sc.n
    ids, state = out[0][2], out[0][3]
    assert np.array_equal(ids, np.arange(sc.n))
    ref = _whole(lambda: OracleSlabWorld(O, p), sc, vel, mat, 15)
    for f in decomp.FIELDS:
        assert_bits_equal(state[f], ref[f], f"{f}, {world_size} resident ranks")


@pytest.mark.gpu
def test_resident_device_slabs_equal_the_whole_device_world(gpu):
    """Persistent device worlds, one per slab, reloaded in place from device tensors each
    step (phy_fluid_set_particles_device / phy_fluid_get_field_device; the state never
    leaves the GPU): the whole device world's bits, particles migrating between slabs."""
    sc, p, vel, mat = _scene()
    st = decomp.ResidentSlabs(lambda: decomp.ResidentDeviceWorld(p, "f64"), p.h, 3, sc.pos, sc.mass, vel=vel,
                              material=mat)
    st.step(DT, 12)
    ref = _whole(lambda: decomp.DeviceWorld(p, "f64"), sc, vel, mat, 12)
    for f in decomp.FIELDS:
        assert_bits_equal(st.state[f].cpu().numpy(), ref[f], f"{f}, resident device slabs")
