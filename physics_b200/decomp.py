"""Spatial decomposition of one scene into x-slabs of grid cells, bit-identical to stepping
the whole scene in one world (no counterpart in the reference, which steps one world).

A step of FluidWorld<f64> (phy-fluid/src/sph/world.rs:183-397) gives particle i a density
from the particles of the 27 cells around its own (grid.rs:43-56) and a force from those
particles' densities, so its new state depends on particles at most two cells away along
each axis.  Slab r owns the particles whose cell key x lies in [lo_r, hi_r); its world holds
them plus every particle with a key in [lo_r - 2, lo_r) or [hi_r, hi_r + 2) (the halo),
inserted in ascending global insertion index.  Inside a cell the grid visits particles in
insertion order, so every sum of an owned particle runs over the same terms in the same
order as in the whole world, and the owned particles' results are the same bits; the halo's
results are dropped.  Ownership is recomputed from the new positions before every step
(particles migrate between slabs), with slab edges that balance the particle counts.

`SlabStepper` runs the slabs in one process (each slab's world may live on its own device);
`RankSlabStepper` gives each rank of a torch.distributed group one slab and exchanges the
halo and the migrating particles as typed records in grouped point-to-point messages.  A world is
made by a factory returning an adapter with add(pos, vel, mass, material), step(dt) and
read() -> {field: array in insertion order}; `DeviceWorld` adapts FluidWorld.
"""
from __future__ import annotations

import numpy as np

HALO = 2  # cells of halo on each side of a slab
FIELDS = ("pos", "vel", "rho", "p", "acc", "mu_eff", "xsph")


def key_x(pos: np.ndarray, h0: float) -> np.ndarray:
    """Grid::key_of along x (grid.rs:25-33): floor(x * (1/h0)) as i64, 0 when not
    representable (non-finite or out of range)."""
    f = np.floor(pos[:, 0] * (1.0 / h0))
    ok = np.isfinite(f) & (f > -9.223372036854775808e18) & (f < 9.223372036854775808e18)
    out = np.zeros(len(f), np.int64)
    out[ok] = f[ok].astype(np.int64)
    return out


I64_MIN, I64_MAX = -(1 << 63), (1 << 63) - 1


def slab_edges_from_counts(uniq: np.ndarray, counts: np.ndarray, nslabs: int) -> list:
    """nslabs + 1 key edges (Python ints; the first and last span the whole int64 range)
    splitting keys, given as distinct values with their counts, into slabs of about equal
    particle counts: edge r is the key at rank r * total / nslabs of the sorted keys.
    Deterministic and strictly increasing."""
    order = np.argsort(uniq, kind="stable")
    uniq, counts = np.asarray(uniq)[order], np.asarray(counts, np.int64)[order]
    cum = np.cumsum(counts)
    total = int(cum[-1]) if len(cum) else 0
    edges = [I64_MIN]
    for r in range(1, nslabs):
        e = int(uniq[int(np.searchsorted(cum, (r * total) // nslabs, side="right"))]) if total else 0
        edges.append(max(e, edges[-1] + 1))
    edges.append(I64_MAX)
    return edges


def slab_edges(keys: np.ndarray, nslabs: int) -> list:
    """slab_edges_from_counts of a key array."""
    uniq, counts = np.unique(keys, return_counts=True)
    return slab_edges_from_counts(uniq, counts, nslabs)


def slab_mask(keys: np.ndarray, lo: int, hi: int, halo: int = 0) -> np.ndarray:
    """keys in [lo - halo, hi + halo), the bounds clamped to the int64 range."""
    return (keys >= max(lo - halo, I64_MIN)) & (keys < min(hi + halo, I64_MAX))


class DeviceWorld:
    """Adapter of a device FluidWorld (physics_b200.FluidWorld) for the steppers."""

    def __init__(self, params, precision: str = "f64"):
        from .fluid import FluidWorld
        self.w = FluidWorld(params, precision)

    def add(self, pos, vel, mass, material):
        if len(mass):
            self.w.add_particles(pos, mass, vel=vel, material=material)

    def step(self, dt: float):
        self.w.step(dt)

    def read(self) -> dict:
        return {f: getattr(self.w, f) for f in FIELDS}


def _step_slab(make_world, state: dict, local: np.ndarray, own_in_local: np.ndarray, dt: float) -> dict:
    """Steps the particles `local` (ascending insertion index) in a fresh world and returns
    the fields of those flagged by own_in_local."""
    w = make_world()
    w.add(state["pos"][local], state["vel"][local], state["mass"][local], state["material"][local])
    w.step(dt)
    out = w.read()
    return {f: np.asarray(out[f])[own_in_local] for f in FIELDS}


class SlabStepper:
    """All slabs in one process; the state is kept in insertion order."""

    def __init__(self, make_world, h0: float, nslabs: int, pos, mass, vel=None, material=None):
        n = len(pos)
        self.make_world, self.h0, self.nslabs = make_world, h0, nslabs
        self.state = {
            "pos": np.array(pos, np.float64).reshape(n, 3),
            "vel": np.zeros((n, 3)) if vel is None else np.array(vel, np.float64).reshape(n, 3),
            "mass": np.broadcast_to(np.asarray(mass, np.float64), (n,)).copy(),
            "material": np.zeros(n, np.uint32) if material is None else np.asarray(material, np.uint32).copy(),
        }
        for f in FIELDS[2:]:
            self.state[f] = np.zeros((n, 3) if f in ("acc", "xsph") else n)
        self.edges = None

    def step(self, dt: float, n: int = 1):
        for _ in range(n):
            s = self.state
            k = key_x(s["pos"], self.h0)
            self.edges = e = slab_edges(k, self.nslabs)
            new = {f: s[f].copy() for f in FIELDS}
            for r in range(self.nslabs):
                own = slab_mask(k, e[r], e[r + 1])
                if not own.any():
                    continue
                local = np.flatnonzero(slab_mask(k, e[r], e[r + 1], HALO))
                res = _step_slab(self.make_world, s, local, own[local], dt)
                ids = local[own[local]]
                for f in FIELDS:
                    new[f][ids] = res[f]
            s.update(new)


class RankSlabStepper:
    """One slab per rank of the default torch.distributed group.  Each rank keeps the
    particles it owns (with their insertion indices); before a step the ranks agree on the
    slab edges from the gathered key counts, then every rank sends each other rank the
    particles that rank owns or needs as halo.

    Every message is a typed tensor of fixed layout (no pickles): per particle an int64
    record (insertion index, cell key x) and an f64 record (pos, vel, mass, material).
    Counts travel first through all_gather; the records then move in one grouped
    batch_isend_irecv, so no rank's send waits behind another rank's receive (a plain
    isend/irecv sequence can deadlock under NCCL once messages exceed its buffers).  With
    NCCL the buffers live on the rank's current device; with gloo on the host."""

    def __init__(self, make_world, h0: float, ids, pos, mass, vel=None, material=None):
        import torch.distributed as dist
        self.dist = dist
        self.rank, self.size = dist.get_rank(), dist.get_world_size()
        n = len(ids)
        self.make_world, self.h0 = make_world, h0
        self.ids = np.asarray(ids, np.int64)
        self.state = {
            "pos": np.array(pos, np.float64).reshape(n, 3),
            "vel": np.zeros((n, 3)) if vel is None else np.array(vel, np.float64).reshape(n, 3),
            "mass": np.broadcast_to(np.asarray(mass, np.float64), (n,)).copy(),
            "material": np.zeros(n, np.uint32) if material is None else np.asarray(material, np.uint32).copy(),
        }
        for f in FIELDS[2:]:
            self.state[f] = np.zeros((n, 3) if f in ("acc", "xsph") else n)

    def _device(self):
        import torch
        if self.dist.get_backend() == "nccl":
            return torch.device("cuda", torch.cuda.current_device())
        return torch.device("cpu")

    def _allgather_rows(self, arr: np.ndarray) -> list:
        """all_gather of a 2-D array whose row count differs by rank (same dtype and
        width everywhere): the counts first, then the rows padded to the largest count."""
        import torch
        dev = self._device()
        t = torch.from_numpy(np.ascontiguousarray(arr)).to(dev)
        cnt = torch.tensor([t.shape[0]], dtype=torch.int64, device=dev)
        cnts = [torch.zeros_like(cnt) for _ in range(self.size)]
        self.dist.all_gather(cnts, cnt)
        cnts = [int(c.item()) for c in cnts]
        width = t.shape[1]
        pad = torch.zeros((max(cnts), width), dtype=t.dtype, device=dev)
        pad[: t.shape[0]] = t
        outs = [torch.empty_like(pad) for _ in range(self.size)]
        self.dist.all_gather(outs, pad)
        return [o[:c].cpu().numpy() for o, c in zip(outs, cnts)]

    def step(self, dt: float, n: int = 1):
        for _ in range(n):
            s = self.state
            k = key_x(s["pos"], self.h0)
            # Slab edges from all ranks' distinct keys and counts (one entry per cell column;
            # every rank computes the same edges).
            u, c = np.unique(k, return_counts=True)
            parts = self._allgather_rows(np.stack([u, c.astype(np.int64)], axis=1))
            allk = np.concatenate([q[:, 0] for q in parts])
            uniq, inv = np.unique(allk, return_inverse=True)
            counts = np.zeros(len(uniq), np.int64)
            np.add.at(counts, inv, np.concatenate([q[:, 1] for q in parts]))
            e = slab_edges_from_counts(uniq, counts, self.size)
            # Outgoing: for each rank, the particles it owns or needs as halo.
            packets = []
            for r in range(self.size):
                sel = slab_mask(k, e[r], e[r + 1], HALO)
                packets.append(_pack(self.ids[sel], k[sel], s, sel))
            inbox = self._exchange(packets)
            ids = np.concatenate([p[0][:, 0] for p in inbox])
            keys = np.concatenate([p[0][:, 1] for p in inbox])
            rec = np.concatenate([p[1] for p in inbox])
            order = np.argsort(ids, kind="stable")  # ascending insertion index
            ids, keys, rec = ids[order], keys[order], rec[order]
            merged = _unpack(rec)
            own = slab_mask(keys, e[self.rank], e[self.rank + 1])
            if own.any():
                res = _step_slab(self.make_world, merged, np.arange(len(ids)), own, dt)
            else:
                res = {f: np.zeros((0, 3) if f in ("pos", "vel", "acc", "xsph") else 0) for f in FIELDS}
            self.ids = ids[own]
            self.state = {"mass": merged["mass"][own], "material": merged["material"][own], **res}

    def _exchange(self, packets):
        """packets[r] = (int64 [m, 2], f64 [m, 8]) goes to rank r; returns the packets
        received from every rank in rank order (this rank's own packet included)."""
        import torch
        dev = self._device()
        # Every rank learns every (sender, receiver) count.
        mine = torch.tensor([p[0].shape[0] for p in packets], dtype=torch.int64, device=dev)
        table = [torch.zeros_like(mine) for _ in range(self.size)]
        self.dist.all_gather(table, mine)
        incoming = [int(table[r][self.rank].item()) for r in range(self.size)]
        ops, recv = [], {}
        for r in range(self.size):
            if r == self.rank:
                continue
            if packets[r][0].shape[0]:
                for a in packets[r]:
                    ops.append(self.dist.P2POp(self.dist.isend, torch.from_numpy(np.ascontiguousarray(a)).to(dev), r))
            if incoming[r]:
                recv[r] = (torch.empty((incoming[r], 2), dtype=torch.int64, device=dev),
                           torch.empty((incoming[r], _REC), dtype=torch.float64, device=dev))
                for t in recv[r]:
                    ops.append(self.dist.P2POp(self.dist.irecv, t, r))
        if ops:
            for q in self.dist.batch_isend_irecv(ops):
                q.wait()
        out = []
        for r in range(self.size):
            if r == self.rank:
                out.append(packets[r])
            elif r in recv:
                out.append((recv[r][0].cpu().numpy(), recv[r][1].cpu().numpy()))
            else:
                out.append((np.zeros((0, 2), np.int64), np.zeros((0, _REC))))
        return out

    def gather_state(self):
        """The whole state in insertion order (on every rank)."""
        s = self.state
        n = len(self.ids)
        cols = [self.ids.astype(np.float64)[:, None]]
        for f in FIELDS:
            cols.append(np.asarray(s[f], np.float64).reshape(n, -1))
        cols += [np.asarray(s["mass"], np.float64)[:, None], np.asarray(s["material"], np.float64)[:, None]]
        parts = self._allgather_rows(np.concatenate(cols, axis=1))
        allrows = np.concatenate(parts)
        ids = allrows[:, 0].astype(np.int64)
        order = np.argsort(ids, kind="stable")
        allrows = allrows[order]
        out, c = {}, 1
        for f in FIELDS:
            w = 3 if f in ("pos", "vel", "acc", "xsph") else 1
            out[f] = allrows[:, c:c + w] if w == 3 else allrows[:, c].copy()
            c += w
        out["mass"] = allrows[:, c].copy()
        out["material"] = allrows[:, c + 1].astype(np.uint32)
        return ids[order], out


_REC = 8  # f64 record: pos 3, vel 3, mass, material (a u32, exact in f64)


def _pack(ids, keys, s, sel):
    """The fixed-layout records of the particles `sel` of state s."""
    head = np.stack([ids, keys], axis=1).astype(np.int64)
    rec = np.concatenate([s["pos"][sel], s["vel"][sel], s["mass"][sel][:, None],
                          s["material"][sel].astype(np.float64)[:, None]], axis=1)
    return head, np.ascontiguousarray(rec, np.float64)


def _unpack(rec):
    return {"pos": rec[:, 0:3].copy(), "vel": rec[:, 3:6].copy(), "mass": rec[:, 6].copy(),
            "material": rec[:, 7].astype(np.uint32)}


# ---- Device-resident form -------------------------------------------------------------
#
# The state stays in torch tensors on the slab's device (the rank's GPU under NCCL,
# the host under gloo), each slab keeps one persistent world that is reloaded in
# place every step (FluidWorld.set_particles_device: no host copy, no allocation
# while the slab's size fits), and the halo and migrant records travel between
# ranks as typed device tensors in grouped point-to-point messages.  The ownership
# and ordering rules are those above, so the owned results are again the whole
# world's bits.

def key_x_t(pos, h0: float):
    """key_x on a torch tensor of positions (same f64 operations: x * (1/h0), floor,
    0 outside the int64 range or for non-finite values)."""
    import torch
    f = torch.floor(pos[:, 0] * (1.0 / h0))
    ok = torch.isfinite(f) & (f > -9.223372036854775808e18) & (f < 9.223372036854775808e18)
    return torch.where(ok, f, torch.zeros_like(f)).to(torch.int64)


def slab_mask_t(keys, lo: int, hi: int, halo: int = 0):
    return (keys >= max(lo - halo, I64_MIN)) & (keys < min(hi + halo, I64_MAX))


class ResidentDeviceWorld:
    """A persistent device FluidWorld reloaded in place each step from device tensors."""

    def __init__(self, params, precision: str = "f64"):
        from . import _lib as L
        from .fluid import FluidWorld
        self.w = FluidWorld(params, precision)
        self.ids = {"pos": L.FIELD_POS, "vel": L.FIELD_VEL, "rho": L.FIELD_RHO, "p": L.FIELD_P, "acc": L.FIELD_ACC,
                    "mu_eff": L.FIELD_MU_EFF, "xsph": L.FIELD_XSPH}

    def load(self, pos, vel, mass, material):
        import torch
        self.w.set_particles_device(pos.contiguous(), mass.contiguous(), vel=vel.contiguous(),
                                    material=material.to(torch.int32).contiguous())

    def step(self, dt: float):
        self.w.step(dt)

    def read(self) -> dict:
        import torch
        n = len(self.w)
        out = {}
        for f, fid in self.ids.items():
            t = torch.empty((n, 3) if f in ("pos", "vel", "acc", "xsph") else (n,), dtype=torch.float64,
                            device=torch.device("cuda", torch.cuda.current_device()))
            if n:
                self.w.get_device(fid, t)
            out[f] = t
        return out


def _state_t(pos, vel, mass, material, device):
    import torch
    n = pos.shape[0]
    st = {
        "pos": torch.as_tensor(pos, dtype=torch.float64, device=device).reshape(n, 3).contiguous(),
        "vel": (torch.zeros((n, 3), dtype=torch.float64, device=device) if vel is None
                else torch.as_tensor(vel, dtype=torch.float64, device=device).reshape(n, 3).contiguous()),
        "mass": torch.as_tensor(np.broadcast_to(np.asarray(mass, np.float64), (n,)).copy(), device=device),
        "material": (torch.zeros(n, dtype=torch.int64, device=device) if material is None
                     else torch.as_tensor(np.asarray(material, np.int64), device=device)),
    }
    for f in FIELDS[2:]:
        st[f] = torch.zeros((n, 3) if f in ("acc", "xsph") else (n,), dtype=torch.float64, device=device)
    return st


class ResidentSlabs:
    """All slabs in one process on one device, each with its persistent world; the state
    is kept in insertion order in device tensors."""

    def __init__(self, make_world, h0: float, nslabs: int, pos, mass, vel=None, material=None, device="cuda"):
        self.h0, self.nslabs = h0, nslabs
        self.state = _state_t(np.asarray(pos, np.float64), vel, mass, material, device)
        self.worlds = [make_world() for _ in range(nslabs)]
        self.edges = None

    def step(self, dt: float, n: int = 1):
        import torch
        for _ in range(n):
            s = self.state
            k = key_x_t(s["pos"], self.h0)
            uniq, counts = torch.unique(k, return_counts=True)
            self.edges = e = slab_edges_from_counts(uniq.cpu().numpy(), counts.cpu().numpy(), self.nslabs)
            new = {f: s[f].clone() for f in FIELDS}
            for r in range(self.nslabs):
                own = slab_mask_t(k, e[r], e[r + 1])
                if not bool(own.any()):
                    continue
                local = torch.nonzero(slab_mask_t(k, e[r], e[r + 1], HALO)).squeeze(1)  # ascending index
                w = self.worlds[r]
                w.load(s["pos"][local], s["vel"][local], s["mass"][local], s["material"][local])
                w.step(dt)
                res = w.read()
                keep = own[local]
                ids = local[keep]
                for f in FIELDS:
                    new[f][ids] = res[f][keep]
            s.update(new)


class ResidentSlabStepper:
    """One slab per rank of the default torch.distributed group, state resident on the
    rank's device (CUDA under NCCL, the host under gloo) with one persistent world.  Each
    step: the ranks agree on slab edges from all-gathered (key, count) rows; every rank
    sends each other rank the particles that rank owns or needs as halo as two typed
    records (int64 [insertion index, key], f64 [pos, vel, mass, material]) in one grouped
    batch_isend_irecv; the received rows are ordered by insertion index, loaded into the
    slab's world, stepped, and the owned rows kept."""

    def __init__(self, make_world, h0: float, ids, pos, mass, vel=None, material=None):
        import torch
        import torch.distributed as dist
        self.dist = dist
        self.rank, self.size = dist.get_rank(), dist.get_world_size()
        self.dev = (torch.device("cuda", torch.cuda.current_device()) if dist.get_backend() == "nccl"
                    else torch.device("cpu"))
        self.h0 = h0
        self.ids = torch.as_tensor(np.asarray(ids, np.int64), device=self.dev)
        self.state = _state_t(np.asarray(pos, np.float64), vel, mass, material, self.dev)
        self.world = make_world()

    def _allgather_rows(self, t) -> list:
        import torch
        cnt = torch.tensor([t.shape[0]], dtype=torch.int64, device=self.dev)
        cnts = [torch.zeros_like(cnt) for _ in range(self.size)]
        self.dist.all_gather(cnts, cnt)
        cnts = [int(c.item()) for c in cnts]
        pad = torch.zeros((max(cnts), t.shape[1]), dtype=t.dtype, device=self.dev)
        pad[: t.shape[0]] = t
        outs = [torch.empty_like(pad) for _ in range(self.size)]
        self.dist.all_gather(outs, pad)
        return [o[:c] for o, c in zip(outs, cnts)]

    def step(self, dt: float, n: int = 1):
        import torch
        for _ in range(n):
            s = self.state
            k = key_x_t(s["pos"], self.h0)
            u, c = torch.unique(k, return_counts=True)
            rows = torch.cat(self._allgather_rows(torch.stack([u, c.to(torch.int64)], dim=1)))
            uniq, inv = torch.unique(rows[:, 0], return_inverse=True)
            counts = torch.zeros(uniq.shape[0], dtype=torch.int64, device=self.dev).index_add_(0, inv, rows[:, 1])
            e = slab_edges_from_counts(uniq.cpu().numpy(), counts.cpu().numpy(), self.size)
            rec = torch.cat([s["pos"], s["vel"], s["mass"][:, None], s["material"].to(torch.float64)[:, None]], 1)
            head = torch.stack([self.ids, k], dim=1)
            packets = []
            for r in range(self.size):
                sel = slab_mask_t(k, e[r], e[r + 1], HALO)
                packets.append((head[sel].contiguous(), rec[sel].contiguous()))
            inbox = self._exchange(packets)
            head_in = torch.cat([p[0] for p in inbox])
            rec_in = torch.cat([p[1] for p in inbox])
            order = torch.sort(head_in[:, 0], stable=True).indices  # ascending insertion index
            head_in, rec_in = head_in[order], rec_in[order]
            own = slab_mask_t(head_in[:, 1], e[self.rank], e[self.rank + 1])
            res = None
            if bool(own.any()):
                self.world.load(rec_in[:, 0:3], rec_in[:, 3:6], rec_in[:, 6], rec_in[:, 7].to(torch.int64))
                self.world.step(dt)
                res = self.world.read()
            self.ids = head_in[own, 0].contiguous()
            self.state = {"mass": rec_in[own, 6].contiguous(), "material": rec_in[own, 7].to(torch.int64)}
            for f in FIELDS:
                shape = (0, 3) if f in ("pos", "vel", "acc", "xsph") else (0,)
                self.state[f] = (res[f][own].to(self.dev).contiguous() if res is not None
                                 else torch.zeros(shape, dtype=torch.float64, device=self.dev))

    def _exchange(self, packets):
        import torch
        mine = torch.tensor([p[0].shape[0] for p in packets], dtype=torch.int64, device=self.dev)
        table = [torch.zeros_like(mine) for _ in range(self.size)]
        self.dist.all_gather(table, mine)
        incoming = [int(table[r][self.rank].item()) for r in range(self.size)]
        ops, recv = [], {}
        for r in range(self.size):
            if r == self.rank:
                continue
            if packets[r][0].shape[0]:
                ops += [self.dist.P2POp(self.dist.isend, packets[r][0], r),
                        self.dist.P2POp(self.dist.isend, packets[r][1], r)]
            if incoming[r]:
                recv[r] = (torch.empty((incoming[r], 2), dtype=torch.int64, device=self.dev),
                           torch.empty((incoming[r], _REC), dtype=torch.float64, device=self.dev))
                ops += [self.dist.P2POp(self.dist.irecv, t, r) for t in recv[r]]
        if ops:
            for q in self.dist.batch_isend_irecv(ops):
                q.wait()
        empty = (torch.zeros((0, 2), dtype=torch.int64, device=self.dev),
                 torch.zeros((0, _REC), dtype=torch.float64, device=self.dev))
        return [packets[r] if r == self.rank else recv.get(r, empty) for r in range(self.size)]

    def gather_state(self):
        """The whole state in insertion order, as numpy arrays (on every rank)."""
        import torch
        n = self.ids.shape[0]
        cols = [self.ids.to(torch.float64)[:, None]]
        for f in FIELDS:
            cols.append(self.state[f].reshape(n, -1).to(torch.float64))
        cols += [self.state["mass"][:, None], self.state["material"].to(torch.float64)[:, None]]
        allrows = torch.cat(self._allgather_rows(torch.cat(cols, 1))).cpu().numpy()
        order = np.argsort(allrows[:, 0].astype(np.int64), kind="stable")
        allrows = allrows[order]
        out, col = {}, 1
        for f in FIELDS:
            w = 3 if f in ("pos", "vel", "acc", "xsph") else 1
            out[f] = allrows[:, col:col + w] if w == 3 else allrows[:, col].copy()
            col += w
        out["mass"] = allrows[:, col].copy()
        out["material"] = allrows[:, col + 1].astype(np.uint32)
        return allrows[:, 0].astype(np.int64), out
