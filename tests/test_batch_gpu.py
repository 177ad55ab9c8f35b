"""Batched scenes (phy_fluid_set_scenes), CUDA-graph stepping and the autotuner.

The batched form runs many independent scenes through one sort and one
persistent launch per pass.  Its gate is identity: every scene of a batch is
bit-identical to the same scene stepped alone in its own world of the same
form and kernel configuration, and the launch knobs (graph capture, CTAs per
SM, work queue, sort block) change no bit of any result.  The single-scene
compensated form is checked against the f64 oracle in test_parity_comp.py;
one batched scene is checked against the oracle here as well."""
import numpy as np
import pytest

from physics_b200 import scenes

pytestmark = pytest.mark.gpu

DT = 0.005
FIELDS = ("pos", "vel", "rho", "p", "acc")


def _params(lo, hi):
    from physics_b200 import SphParams
    p = SphParams.defaults()
    p.bounds_min, p.bounds_max = tuple(lo), tuple(hi)
    return p


def _batch_world(gpu, batch, **tuning):
    mass = scenes.lattice_mass(scenes.SPACING)
    w = gpu.FluidWorld(_params(batch[0].bounds_min, batch[0].bounds_max), "comp")
    pos = np.concatenate([b.pos for b in batch])
    w.add_particles(pos, np.full(pos.shape[0], mass))
    w.set_scenes([b.n for b in batch], [b.bounds_min for b in batch], [b.bounds_max for b in batch])
    if tuning:
        w.set_tuning(**tuning)
    return w


def _alone(gpu, b, steps, tile=4):
    w = gpu.FluidWorld(_params(b.bounds_min, b.bounds_max), "comp")
    w.set_tuning(comp_tile=tile)
    w.add_particles(b.pos, np.full(b.n, scenes.lattice_mass(scenes.SPACING)))
    w.step(DT, steps)
    return {f: getattr(w, f) for f in FIELDS}


def _state(w):
    return {f: getattr(w, f) for f in FIELDS}


def _assert_same(a, b, what):
    for f in FIELDS:
        assert np.array_equal(a[f].view(np.uint64), b[f].view(np.uint64)), f"{what}: {f} differs"


def _split(state, batch):
    out, o = [], 0
    for b in batch:
        out.append({f: v[o:o + b.n] for f, v in state.items()})
        o += b.n
    return out


@pytest.mark.parametrize("tile", [4, 2])
def test_batch_scenes_bit_identical_to_alone(gpu, tile):
    batch = scenes.batch_scenes(6, 300, 3000)
    w = _batch_world(gpu, batch, comp_tile=tile)
    assert w.scene_count == 6
    w.step(DT, 12)
    for k, (b, got) in enumerate(zip(batch, _split(_state(w), batch))):
        _assert_same(got, _alone(gpu, b, 12, tile), f"scene {k}")


def test_batch_graph_and_launch_knobs_change_no_bit(gpu):
    batch = scenes.batch_scenes(5, 500, 4000, seed=7)
    ref = _batch_world(gpu, batch)
    ref.step(DT, 12)
    want = _state(ref)
    for knobs in ({"graph_chunk": 4}, {"graph_chunk": 3}, {"queue": 1},
                  {"ctas_per_sm": 1, "sort_block": 128}, {"queue": 1, "ctas_per_sm": 2, "graph_chunk": 6}):
        w = _batch_world(gpu, batch, **knobs)
        w.step(DT, 5)  # chunked runs plus an uncaptured remainder
        w.step(DT, 7)
        _assert_same(_state(w), want, str(knobs))


def test_single_world_graph_matches_eager(gpu):
    sc = scenes.dam_break(16, 24, 16, box=4.8, dt=DT, steps=0)
    outs = []
    for chunk in (0, 4):
        w = gpu.FluidWorld(_params(sc.bounds_min, sc.bounds_max), "comp")
        w.add_particles(sc.pos, np.full(sc.n, sc.mass))
        w.set_tuning(graph_chunk=chunk)
        w.step(DT, 10)
        outs.append(_state(w))
    _assert_same(outs[0], outs[1], "graph vs eager")


def test_batched_scene_vs_oracle_teacher_forced(gpu, oracle_mod):
    O = oracle_mod
    batch = scenes.batch_scenes(3, 800, 2500, seed=11)
    w = _batch_world(gpu, batch)
    w.step(DT, 30)  # a developed state
    pos, vel = w.pos, w.vel
    w.step(DT)
    o = 0
    for b in batch:
        ow = O.OracleWorld(_params(b.bounds_min, b.bounds_max), threads=O.max_threads())
        ow.add_particles(pos[o:o + b.n], np.full(b.n, scenes.lattice_mass(scenes.SPACING)), vel=vel[o:o + b.n])
        ow.step(DT)
        rho_o = ow.get(O.F_RHO)
        err = float(np.max(np.abs(w.rho[o:o + b.n] - rho_o) / rho_o))
        assert err <= 1e-5, err
        o += b.n


@pytest.mark.parametrize("horizon", [0, 6])
def test_autotune_restores_state_and_keeps_fastest(gpu, horizon):
    """The autotuner over the launch knobs and 4 or 2 cells per tile edge, from the current
    state (horizon 0) or also from the states 3 and 6 steps ahead (its six fastest
    candidates): the world returns to its state, keeps the fastest candidate among those
    timed on every sample, and steps on exactly like a world that never tuned (with the
    chosen tile edge, the one knob that changes the summation order)."""
    batch = scenes.batch_scenes(4, 1000, 5000, seed=3)
    w = _batch_world(gpu, batch, graph_chunk=2)
    w.step(DT, 3)
    before = _state(w)
    trials = w.autotune(DT, 4, horizon=horizon)
    assert len(trials) >= 8 and {t["comp_tile"] for t in trials} == {2, 4}
    _assert_same(_state(w), before, "state after autotune")
    full = 3 if horizon else 1
    finalists = [t for t in trials if t["samples"] == full]
    assert len(finalists) == (6 if horizon else len(trials))
    best = min(finalists, key=lambda t: t["ms_per_step"])
    tun = w.tuning()
    assert (tun["ctas_per_sm"], tun["queue"], tun["sort_block"], tun["comp_tile"]) == (
        best["ctas_per_sm"], best["queue"], best["sort_block"], best["comp_tile"])
    # Stepping on from the restored state matches a world that never tuned (its first
    # three steps at the default tile edge, like the tuned world's).
    ref = _batch_world(gpu, batch, graph_chunk=2)
    ref.step(DT, 3)
    ref.set_tuning(comp_tile=tun["comp_tile"])
    w.step(DT, 4)
    ref.step(DT, 4)
    _assert_same(_state(w), _state(ref), "after tuning")


def test_batch_standard_scenes_subset_identical(gpu):
    """The standard 256-scene batch (about 12M particles): three scenes of the
    batch bit-identical to the same scenes alone after a few steps."""
    batch = scenes.batch_scenes()
    w = _batch_world(gpu, batch, graph_chunk=2)
    w.step(DT, 4)
    state = _state(w)
    offs = np.concatenate([[0], np.cumsum([b.n for b in batch])])
    for k in (0, 101, 255):
        got = {f: v[offs[k]:offs[k + 1]] for f, v in state.items()}
        _assert_same(got, _alone(gpu, batch[k], 4), f"scene {k}")


def test_batch_argument_errors(gpu):
    from physics_b200 import PhyError
    batch = scenes.batch_scenes(2, 300, 600)
    w = _batch_world(gpu, batch)
    with pytest.raises(PhyError):
        w.add_particles(np.zeros((1, 3)), np.ones(1))
    with pytest.raises(PhyError):
        w.set_scenes([1, 2], [(0, 0, 0)] * 2, [(1, 1, 1)] * 2)  # counts do not add up
    with pytest.raises(PhyError):
        w.set_tuning(comp_tile=0)
    w.clear_scenes()
    assert w.scene_count == 0
    plain = gpu.FluidWorld(_params((0, 0, 0), (2, 2, 2)), "f64")
    plain.add_particles(batch[0].pos, np.ones(batch[0].n))
    with pytest.raises(PhyError):
        plain.set_scenes([batch[0].n], [(0, 0, 0)], [(2, 2, 2)])
