"""Partition of the batched form's scenes across GPUs (one process per GPU, no
collective in the step).  Checked on CPU: the greedy bin packing itself, two gloo
ranks that each take their part and together cover every scene once, and two gloo
ranks that each step their part (every scene on the oracle) and together give the
same bits as one process stepping every scene."""
import os
import socket

import numpy as np
import pytest

from physics_b200 import scenes


@pytest.mark.parametrize("nparts", [1, 2, 3, 8])
def test_partition_covers_and_balances(nparts):
    counts = [b.n for b in scenes.batch_scenes(256)]
    parts = scenes.partition_scenes(counts, nparts)
    assert len(parts) == nparts
    flat = sorted(i for p in parts for i in p)
    assert flat == list(range(len(counts)))
    loads = [sum(counts[i] for i in p) for p in parts]
    assert max(loads) - sum(counts) / nparts <= max(counts)
    assert parts == scenes.partition_scenes(counts, nparts)  # deterministic


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world_size, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world_size)
    try:
        counts = [b.n for b in scenes.batch_scenes(64, 2000, 20000)]
        mine = scenes.partition_scenes(counts, world_size)[rank]
        gathered = [None] * world_size
        dist.all_gather_object(gathered, mine)
        # Max over ranks of a per-rank load, as the bench takes the max of per-rank times.
        import torch
        t = torch.tensor([float(sum(counts[i] for i in mine))])
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        q.put((rank, gathered, float(t.item()), sum(counts)))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_disjoint_complete_parts():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    out.sort()
    g0, g1 = out[0][1], out[1][1]
    assert g0 == g1
    a, b = set(g0[0]), set(g0[1])
    assert not (a & b) and len(a | b) == 64
    mx, total = out[0][2], out[0][3]
    assert total / 2 <= mx < total


BATCH_DT = 0.005
STEPS = 4


def _step_scenes(batch, idx):
    """The listed scenes, each stepped alone on the oracle (a batched world gives every
    scene the bits of that scene alone): final positions and velocities per scene."""
    from oracle import oracle as O
    mass = scenes.lattice_mass(scenes.SPACING)
    out = {}
    for i in idx:
        b = batch[i]
        p = O.RefParams.defaults()
        p.bounds_min, p.bounds_max = b.bounds_min, b.bounds_max
        w = O.OracleWorld(p)
        w.add_particles(b.pos, np.full(b.n, mass))
        w.step(BATCH_DT, STEPS)
        out[i] = np.concatenate([w.get(O.F_POS).ravel(), w.get(O.F_VEL).ravel()])
    return out


def _small_batch():
    return scenes.batch_scenes(6, 150, 600)


def _stepping_rank_main(rank, world_size, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world_size)
    try:
        batch = _small_batch()
        mine = scenes.partition_scenes([b.n for b in batch], world_size)[rank]
        gathered = [None] * world_size
        dist.all_gather_object(gathered, {i: v.tobytes() for i, v in _step_scenes(batch, mine).items()})
        q.put((rank, gathered))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_step_their_scenes_like_one_process(oracle_mod):
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_stepping_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    out.sort(key=lambda t: t[0])
    assert out[0][1] == out[1][1]
    merged = {}
    for part in out[0][1]:
        assert not (set(part) & set(merged))
        merged.update(part)
    batch = _small_batch()
    assert sorted(merged) == list(range(len(batch)))
    alone = _step_scenes(batch, range(len(batch)))
    for i, v in alone.items():
        assert merged[i] == v.tobytes(), f"scene {i}"
