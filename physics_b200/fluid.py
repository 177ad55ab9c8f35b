"""Python mirror of the reference's fluid API over the C ABI of libphysph.so.

Names, argument meaning and error behaviour follow crates/phy-fluid
(`SphParams<T>` src/sph/params.rs:12-86, `FluidWorld<T>` src/sph/world.rs:
21-197, `FluidSubsystem<T>` src/subsystem.rs:26-164) and phy-core's `World<T>`
(crates/phy-core/src/world.rs:78-294).  All mechanics run in the CUDA library;
this module only marshals arguments.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

from . import _lib as L

_PREC = {"f64": L.PRECISION_F64_PLAIN, "plain": L.PRECISION_F64_PLAIN,
         "f32c": L.PRECISION_F32_COMP, "comp": L.PRECISION_F32_COMP}


def _precision(p) -> int:
    if isinstance(p, int):
        return p
    return _PREC[p]


def _pack_shape_data(b: dict, data: list, faces: list) -> tuple:
    """Appends the shape data of body or sub-shape dict `b` to the shared data / faces
    lists (PhyCoupleBody layout, include/phy_fluid.h) and returns (data_first,
    data_count, face_first, face_count): convex vertices and index faces, heightfield
    heights, or a compound's 16-double sub-shape records (shape, size[3], offset[3],
    quaternion i j k w, data_first, data_count, face_first, face_count, 0)."""
    kind = b["shape"]
    if kind == "convex":
        d0, f0 = len(data), len(faces) // 3
        data.extend(np.asarray(b["verts"], np.float64).reshape(-1).tolist())
        faces.extend(np.asarray(b["faces"], np.uint32).reshape(-1).tolist())
        return d0, len(b["verts"]), f0, len(b["faces"])
    if kind == "heightfield":
        d0 = len(data)
        data.extend(float(h) for h in b["heights"])
        return d0, len(b["heights"]), 0, 0
    if kind == "compound":
        subs = b["subs"]
        d0 = len(data)
        data.extend([0.0] * (16 * len(subs)))
        for q, sub in enumerate(subs):
            if sub["shape"] == "compound":
                raise ValueError("nested compound shapes are not supported")
            size = list(sub.get("size", ())) + [0.0] * 3
            rec = [float(L.SHAPES[sub["shape"]])] + [float(v) for v in size[:3]]
            rec += [float(v) for v in sub.get("offset", (0.0, 0.0, 0.0))]
            rec += [float(v) for v in sub.get("rot", (0.0, 0.0, 0.0, 1.0))]
            rec += [float(v) for v in _pack_shape_data(sub, data, faces)] + [0.0]
            data[d0 + 16 * q: d0 + 16 * (q + 1)] = rec
        return d0, len(subs), 0, 0
    return 0, 0, 0, 0


def _dp(a: np.ndarray):
    return a.ctypes.data_as(L.DP)


@dataclass
class SphParams:
    """SphParams<f64> (crates/phy-fluid/src/sph/params.rs:12-86)."""
    rest_density: float = 1000.0
    stiffness: float = 250.0
    viscosity: float = 3.5
    visc_k: list = field(default_factory=lambda: [3.5])
    visc_n: list = field(default_factory=lambda: [1.0])
    shear_min: float = 0.01
    mass: float = 0.02
    h: float = 0.2
    gravity: tuple = (0.0, -9.81, 0.0)
    bounds_min: tuple = (-5.0, -5.0, -5.0)
    bounds_max: tuple = (5.0, 5.0, 5.0)
    boundary_damp: float = 0.4
    xsph_eps: float = 0.5

    @staticmethod
    def defaults() -> "SphParams":
        """SphParams::defaults() (params.rs:55-85), read from the library."""
        c = L.PhySphParams()
        L.load().phy_sph_params_defaults(C.byref(c))
        return SphParams.from_c(c)

    def to_c(self) -> L.PhySphParams:
        if not (1 <= len(self.visc_k) <= L.MAX_MATERIALS) or len(self.visc_n) > L.MAX_MATERIALS:
            raise ValueError("visc_k must hold 1..16 entries and visc_n at most 16")
        c = L.PhySphParams()
        for name in ("rest_density", "stiffness", "viscosity", "shear_min", "mass", "h", "boundary_damp",
                     "xsph_eps"):
            setattr(c, name, float(getattr(self, name)))
        for name in ("gravity", "bounds_min", "bounds_max"):
            v = getattr(self, name)
            arr = getattr(c, name)
            for k in range(3):
                arr[k] = float(v[k])
        c.n_visc_k = len(self.visc_k)
        c.n_visc_n = len(self.visc_n)
        for k, v in enumerate(self.visc_k):
            c.visc_k[k] = float(v)
        for k, v in enumerate(self.visc_n):
            c.visc_n[k] = float(v)
        return c

    @staticmethod
    def from_c(c: L.PhySphParams) -> "SphParams":
        return SphParams(
            rest_density=c.rest_density, stiffness=c.stiffness, viscosity=c.viscosity,
            visc_k=[c.visc_k[k] for k in range(c.n_visc_k)], visc_n=[c.visc_n[k] for k in range(c.n_visc_n)],
            shear_min=c.shear_min, mass=c.mass, h=c.h, gravity=tuple(c.gravity), bounds_min=tuple(c.bounds_min),
            bounds_max=tuple(c.bounds_max), boundary_damp=c.boundary_damp, xsph_eps=c.xsph_eps)


class World:
    """World<f64> holding fluid subsystems (phy-core/src/world.rs:78-294)."""

    def __init__(self, handle: Optional[int] = None):
        self._lib = L.load()
        self._h = handle
        self._subs: list = []
        if handle is not None:
            for k in range(int(self._lib.phy_world_sub_count(handle))):
                self._subs.append(FluidSubsystem(FluidWorld._view(self, k)))

    @property
    def handle(self):
        return self._h

    def add_fluid(self, params: SphParams, precision="f64") -> "FluidSubsystem":
        """World::add_subsystem(Box::new(FluidSubsystem::new(FluidWorld::new(params))))."""
        c = params.to_c()
        if self._h is None:
            h = self._lib.phy_fluid_world_create(C.byref(c), _precision(precision))
            if not h:
                raise L.PhyError("phy_fluid_world_create")
            self._h = h
            idx = 0
        else:
            idx = self._lib.phy_fluid_add_subsystem(self._h, C.byref(c), _precision(precision))
            if idx < 0:
                raise L.PhyError("phy_fluid_add_subsystem")
        sub = FluidSubsystem(FluidWorld._view(self, idx))
        self._subs.append(sub)
        return sub

    def subsystem_count(self) -> int:
        return int(self._lib.phy_world_sub_count(self._h)) if self._h else 0

    def get(self, i: int) -> "FluidSubsystem":
        return self._subs[i]

    def step(self, dt: float) -> None:
        """World::step (world.rs:265-267)."""
        if self._h is None:
            return
        L.check(self._lib.phy_world_step(self._h, dt), "phy_world_step")

    def step_checked(self, dt: float) -> int:
        """World::step_checked (world.rs:291-293): 0, or 2 NonFinite / 5 grid box."""
        if self._h is None:
            return 0
        rc = self._lib.phy_world_step_checked(self._h, dt)
        if rc < 0:
            raise L.PhyError("phy_world_step_checked", rc)
        return rc

    def time(self) -> float:
        return float(self._lib.phy_world_time(self._h)) if self._h else 0.0

    def fluid_count(self) -> int:
        return int(self._lib.phy_world_fluid_count(self._h)) if self._h else 0

    def fluid_positions(self) -> np.ndarray:
        n = self.fluid_count()
        buf = np.empty(3 * n, np.float64)
        got = self._lib.phy_world_get_fluid_positions(self._h, _dp(buf), buf.size)
        return buf[: 3 * got].reshape(-1, 3)

    def fluid_velocities(self) -> np.ndarray:
        n = self.fluid_count()
        buf = np.empty(3 * n, np.float64)
        got = self._lib.phy_world_get_fluid_velocities(self._h, _dp(buf), buf.size)
        return buf[: 3 * got].reshape(-1, 3)

    def set_stream(self, stream_ptr: int) -> None:
        L.check(self._lib.phy_fluid_set_stream(self._h, C.c_void_p(stream_ptr)), "phy_fluid_set_stream")

    def synchronize(self) -> None:
        L.check(self._lib.phy_fluid_synchronize(self._h), "phy_fluid_synchronize")

    def save(self, path: str) -> None:
        L.check(self._lib.phy_world_save(self._h, str(path).encode()), "phy_world_save")

    @staticmethod
    def load(path: str) -> "World":
        h = L.load().phy_world_load(str(path).encode())
        if not h:
            raise L.PhyError("phy_world_load")
        return World(h)

    def close(self) -> None:
        if self._h:
            self._lib.phy_world_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class FluidWorld:
    """FluidWorld<f64> (crates/phy-fluid/src/sph/world.rs:21-197).

    `params` is live: assigning it (or calling set_params) changes the
    parameters used by the next step, while the smoothing length of the
    kernel coefficients and grid stays the one given at construction
    (world.rs:94-102).  Particle fields are numpy arrays in insertion order.
    """

    def __init__(self, params: SphParams, precision="f64"):
        w = World()
        sub = w.add_fluid(params, precision)
        self._world = w
        self._sub = sub.world._sub

    @classmethod
    def _view(cls, world: World, sub: int) -> "FluidWorld":
        obj = cls.__new__(cls)
        obj._world = world
        obj._sub = sub
        return obj

    @property
    def _lib(self):
        return self._world._lib

    @property
    def _h(self):
        return self._world.handle

    # ---- params -------------------------------------------------------------
    @property
    def params(self) -> SphParams:
        c = L.PhySphParams()
        L.check(self._lib.phy_fluid_get_params(self._h, self._sub, C.byref(c)), "phy_fluid_get_params")
        return SphParams.from_c(c)

    @params.setter
    def params(self, p: SphParams) -> None:
        c = p.to_c()
        L.check(self._lib.phy_fluid_set_params(self._h, self._sub, C.byref(c)), "phy_fluid_set_params")

    # ---- particles ------------------------------------------------------------
    def __len__(self) -> int:
        return self.len()

    def len(self) -> int:
        n = self._lib.phy_fluid_len(self._h, self._sub)
        if n < 0:
            raise L.PhyError("phy_fluid_len")
        return int(n)

    def is_empty(self) -> bool:
        return self.len() == 0

    def fill_box(self, mn: Sequence[float], mx: Sequence[float], spacing: float, margin: float) -> None:
        a = np.asarray(mn, np.float64)
        b = np.asarray(mx, np.float64)
        L.check(self._lib.phy_fluid_fill_box(self._h, self._sub, _dp(a), _dp(b), spacing, margin),
                "phy_fluid_fill_box")

    def lattice_mass(self, spacing: float) -> float:
        return float(self._lib.phy_fluid_lattice_mass(self._h, self._sub, spacing))

    def add_particles(self, pos, mass, vel=None, material=None) -> None:
        pos = np.ascontiguousarray(pos, np.float64).reshape(-1)
        n = pos.size // 3
        mass = np.ascontiguousarray(np.broadcast_to(np.asarray(mass, np.float64), (n,)))
        vp = None
        if vel is not None:
            vel = np.ascontiguousarray(vel, np.float64).reshape(-1)
            vp = _dp(vel)
        mp = None
        if material is not None:
            material = np.ascontiguousarray(np.broadcast_to(np.asarray(material, np.uint32), (n,)))
            mp = material.ctypes.data_as(C.POINTER(C.c_uint32))
        L.check(self._lib.phy_fluid_add_particles(self._h, self._sub, n, _dp(pos), vp, _dp(mass), mp),
                "phy_fluid_add_particles")

    def add_particle(self, pos, mass, vel=(0.0, 0.0, 0.0), material=0) -> None:
        """FluidWorld::add_particle(Particle::with_material(pos, mass, material))."""
        self.add_particles(np.asarray(pos, np.float64), [mass], np.asarray(vel, np.float64), [material])

    def get(self, fld: int, out: Optional[np.ndarray] = None) -> np.ndarray:
        n = self.len()
        nc = L.FIELD_COMPONENTS[fld]
        if out is None:
            out = np.empty(n * nc, np.float64)
        L.check(self._lib.phy_fluid_get_field(self._h, self._sub, fld, _dp(out), out.size), "phy_fluid_get_field")
        return out.reshape(n, nc) if nc == 3 else out

    def set_particles_device(self, pos, mass, vel=None, material=None) -> None:
        """Replaces the particle set with device tensors (phy_fluid_set_particles_device):
        pos / vel (n, 3) float64, mass (n,) float64, material (n,) int32/uint32, all
        contiguous on this world's device; no host copy."""
        n = int(mass.shape[0])
        for t, want in ((pos, 3 * n), (vel, 3 * n), (mass, n), (material, n)):
            if t is not None and (not t.is_cuda or not t.is_contiguous() or t.numel() != want):
                raise ValueError("set_particles_device: contiguous CUDA tensors of matching sizes")
        ptr = (lambda t: C.c_void_p(t.data_ptr()) if t is not None else None)
        L.check(self._lib.phy_fluid_set_particles_device(self._h, self._sub, n, ptr(pos), ptr(vel), ptr(mass),
                                                         ptr(material)), "phy_fluid_set_particles_device")

    def get_device(self, fld: int, out) -> None:
        """Writes field `fld` in insertion order into the contiguous float64 CUDA tensor
        `out` (phy_fluid_get_field_device); no host copy."""
        if not out.is_cuda or not out.is_contiguous():
            raise ValueError("get_device: a contiguous CUDA tensor")
        L.check(self._lib.phy_fluid_get_field_device(self._h, self._sub, fld, C.c_void_p(out.data_ptr()),
                                                     out.numel()), "phy_fluid_get_field_device")

    def set(self, fld: int, values) -> None:
        a = np.ascontiguousarray(values, np.float64).reshape(-1)
        L.check(self._lib.phy_fluid_set_field(self._h, self._sub, fld, _dp(a), a.size), "phy_fluid_set_field")

    pos = property(lambda s: s.get(L.FIELD_POS), lambda s, v: s.set(L.FIELD_POS, v))
    vel = property(lambda s: s.get(L.FIELD_VEL), lambda s, v: s.set(L.FIELD_VEL, v))
    acc = property(lambda s: s.get(L.FIELD_ACC), lambda s, v: s.set(L.FIELD_ACC, v))
    body_acc = property(lambda s: s.get(L.FIELD_BODY_ACC), lambda s, v: s.set(L.FIELD_BODY_ACC, v))
    rho = property(lambda s: s.get(L.FIELD_RHO), lambda s, v: s.set(L.FIELD_RHO, v))
    p = property(lambda s: s.get(L.FIELD_P), lambda s, v: s.set(L.FIELD_P, v))
    mass = property(lambda s: s.get(L.FIELD_MASS), lambda s, v: s.set(L.FIELD_MASS, v))
    mu_eff = property(lambda s: s.get(L.FIELD_MU_EFF), lambda s, v: s.set(L.FIELD_MU_EFF, v))
    xsph = property(lambda s: s.get(L.FIELD_XSPH), lambda s, v: s.set(L.FIELD_XSPH, v))
    material = property(lambda s: s.get(L.FIELD_MATERIAL).astype(np.int64),
                        lambda s, v: s.set(L.FIELD_MATERIAL, np.asarray(v, np.float64)))

    def effective_viscosity(self, i: int) -> float:
        """FluidWorld::effective_viscosity (world.rs:176-180)."""
        return float(self.mu_eff[i])

    # ---- stepping ---------------------------------------------------------------
    def step(self, dt: float, n: int = 1) -> None:
        """FluidWorld::step (world.rs:183-192), n times."""
        L.check(self._lib.phy_fluid_step(self._h, self._sub, dt, n), "phy_fluid_step")

    def synchronize(self) -> None:
        self._world.synchronize()

    def set_stream(self, stream_ptr: int) -> None:
        self._world.set_stream(stream_ptr)

    def set_counting(self, on: bool) -> None:
        L.check(self._lib.phy_fluid_set_counting(self._h, self._sub, 1 if on else 0), "phy_fluid_set_counting")

    def step_counters(self) -> dict:
        out = (C.c_uint64 * 4)()
        L.check(self._lib.phy_fluid_step_counters(self._h, self._sub, out), "phy_fluid_step_counters")
        return {"candidates": out[0], "pairs": out[1], "particles": out[2], "cells": out[3]}

    def dense_mask_info(self) -> dict:
        """The dense-cell mask buffer (phy_fluid_dense_mask_info): entries allocated, the
        entries the last step's dense-cell tasks reserved, and whether the last step found a
        task's kept masks outside the buffer."""
        out = (C.c_uint64 * 3)()
        L.check(self._lib.phy_fluid_dense_mask_info(self._h, self._sub, out), "phy_fluid_dense_mask_info")
        return {"capacity": out[0], "demand": out[1], "bad_table": bool(out[2])}

    def set_tuning(self, **knobs: int) -> None:
        """Kernel configuration (phy_fluid_set_tuning): comp_tile, halo_cap, ctas_per_sm, queue,
        sort_block, graph_chunk, dense_mean, dense_masks.  Results of the f64 form never
        change; the launch knobs (ctas_per_sm, queue, sort_block, graph_chunk, dense_masks)
        change no result of either form."""
        for name, value in knobs.items():
            if name not in L.TUNE_PARAMS:
                raise ValueError(f"unknown tuning parameter {name!r}")
            if value is None:
                continue
            L.check(self._lib.phy_fluid_set_tuning(self._h, self._sub, L.TUNE_PARAMS[name], int(value)),
                    "phy_fluid_set_tuning")

    def tuning(self) -> dict:
        """Current value of every tuning parameter (phy_fluid_get_tuning)."""
        out = {}
        v = C.c_int64()
        for name, code in L.TUNE_PARAMS.items():
            L.check(self._lib.phy_fluid_get_tuning(self._h, self._sub, code, C.byref(v)), "phy_fluid_get_tuning")
            out[name] = int(v.value)
        return out

    def autotune(self, dt: float, steps: int = 10, horizon: int = 0) -> list:
        """The library's autotuner (phy_fluid_autotune_horizon): every knob combination (launch
        knobs and, for tiled worlds, 4 or 2 cells per tile edge) timed over `steps` steps from
        the same state; with horizon > 0 the fastest also from the states horizon/2 and
        horizon steps ahead, ranked by the mean.  The state is restored and the fastest kept.
        Returns the trials as dicts in the order run."""
        cap = 256
        out = (L.PhyTuneTrial * cap)()
        n = C.c_uint32()
        L.check(self._lib.phy_fluid_autotune_horizon(self._h, self._sub, dt, steps, horizon, out, cap, C.byref(n)),
                "phy_fluid_autotune_horizon")
        return [{"ctas_per_sm": t.ctas_per_sm, "queue": t.queue, "sort_block": t.sort_block,
                 "comp_tile": t.comp_tile, "ms_per_step": t.ms_per_step, "samples": t.samples}
                for t in out[:min(n.value, cap)]]

    # ---- adjoint (f64 plain form) ----------------------------------------------------
    def tape_begin(self, checkpoint_every: int = 10) -> None:
        """Starts recording steps for step_backward (phy_fluid_tape_begin)."""
        L.check(self._lib.phy_fluid_tape_begin(self._h, self._sub, checkpoint_every), "phy_fluid_tape_begin")

    def tape_clear(self) -> None:
        L.check(self._lib.phy_fluid_tape_clear(self._h, self._sub), "phy_fluid_tape_clear")

    @property
    def tape_steps(self) -> int:
        return int(self._lib.phy_fluid_tape_steps(self._h, self._sub))

    def step_backward(self, grad_pos=None, grad_vel=None) -> dict:
        """Reverse sweep over the recorded steps (phy_fluid_step_backward).  grad_pos, grad_vel:
        dL/dpos_T, dL/dvel_T as (N, 3) arrays (None = zero).  Returns dL/dpos_0, dL/dvel_0 and the
        parameter gradients {"stiffness", "visc_k0"}."""
        n = len(self)
        gp = None if grad_pos is None else np.ascontiguousarray(grad_pos, np.float64).reshape(-1)
        gv = None if grad_vel is None else np.ascontiguousarray(grad_vel, np.float64).reshape(-1)
        for g in (gp, gv):
            if g is not None and g.size != 3 * n:
                raise ValueError("gradients must hold 3 values per particle")
        op = np.empty((n, 3), np.float64)
        ov = np.empty((n, 3), np.float64)
        par = np.empty(2, np.float64)
        L.check(self._lib.phy_fluid_step_backward(self._h, self._sub, None if gp is None else _dp(gp),
                                                  None if gv is None else _dp(gv), _dp(op), _dp(ov), _dp(par)),
                "phy_fluid_step_backward")
        return {"pos": op, "vel": ov, "stiffness": float(par[0]), "visc_k0": float(par[1])}

    # ---- batched scenes -----------------------------------------------------------
    def set_scenes(self, counts, bounds_min, bounds_max) -> None:
        """Partitions the particles (insertion order) into consecutive scenes with their own
        bounds (phy_fluid_set_scenes); one step then advances every scene."""
        counts = np.ascontiguousarray(counts, np.uint64)
        lo = np.ascontiguousarray(bounds_min, np.float64).reshape(-1, 3)
        hi = np.ascontiguousarray(bounds_max, np.float64).reshape(-1, 3)
        if lo.shape[0] != counts.size or hi.shape[0] != counts.size:
            raise ValueError("one bounds pair per scene")
        L.check(self._lib.phy_fluid_set_scenes(self._h, self._sub, counts.size,
                                               counts.ctypes.data_as(C.POINTER(C.c_uint64)), _dp(lo), _dp(hi)),
                "phy_fluid_set_scenes")

    def clear_scenes(self) -> None:
        L.check(self._lib.phy_fluid_clear_scenes(self._h, self._sub), "phy_fluid_clear_scenes")

    @property
    def scene_count(self) -> int:
        return int(self._lib.phy_fluid_scene_count(self._h, self._sub))

    def set_timing(self, on: bool) -> None:
        L.check(self._lib.phy_fluid_set_timing(self._h, self._sub, 1 if on else 0), "phy_fluid_set_timing")

    def phase_times(self, reset: bool = True) -> dict:
        """Accumulated per-phase device milliseconds while timing is on."""
        out = np.empty(5, np.float64)
        L.check(self._lib.phy_fluid_phase_times(self._h, self._sub, _dp(out), 1 if reset else 0),
                "phy_fluid_phase_times")
        return {"sort": out[0], "prep": out[1], "density": out[2], "force": out[3], "steps": int(out[4])}

    # ---- coupling (world.rs:691-752) ------------------------------------------------
    def couple_points(self, pos, vel, mass, dt: float, drag: float, soft_density: float, force=None) -> np.ndarray:
        """FluidWorld::couple_points on the device: returns the (n, 3) forces on the points;
        rows of points outside the bounds keep the values of `force` (zeros when None).
        The fluid velocities take the reactions."""
        pos = np.ascontiguousarray(pos, np.float64).reshape(-1)
        vel = np.ascontiguousarray(vel, np.float64).reshape(-1)
        mass = np.ascontiguousarray(mass, np.float64).reshape(-1)
        if pos.size != 3 * mass.size or vel.size != pos.size:
            raise ValueError("couple_points: pos and vel need 3 values per mass")
        out = np.zeros(pos.size, np.float64) if force is None else np.array(force, np.float64).reshape(-1)
        L.check(self._lib.phy_fluid_couple_points(self._h, self._sub, mass.size, _dp(pos), _dp(vel), _dp(mass),
                                                  _dp(out), dt, drag, soft_density), "phy_fluid_couple_points")
        return out.reshape(-1, 3)

    def couple_heat(self, temp, src, origin, cell: float, dt: float, t_ref: float, beta: float,
                    heat_gain: float) -> np.ndarray:
        """FluidWorld::couple_heat on the device: temp is the (nz, ny, nx) grid of temperatures
        (x fastest in memory); returns the updated copy of src.  The particles' body
        accelerations take the buoyancy terms."""
        temp = np.ascontiguousarray(temp, np.float64)
        if temp.ndim != 3:
            raise ValueError("couple_heat: temp must be a (nz, ny, nx) array")
        out = np.array(src, np.float64, copy=True, order="C").reshape(temp.shape)
        dims = (C.c_uint64 * 3)(temp.shape[2], temp.shape[1], temp.shape[0])
        o = np.ascontiguousarray(origin, np.float64).reshape(3)
        L.check(self._lib.phy_fluid_couple_heat(self._h, self._sub, dims, _dp(o), cell, _dp(temp), _dp(out), dt, t_ref,
                                                beta, heat_gain), "phy_fluid_couple_heat")
        return out

    def couple_bodies(self, bodies, dt: float, friction: float = 0.0) -> np.ndarray:
        """FluidWorld::couple_bodies on the device over body dicts: `shape` (sphere, capsule,
        box, convex, heightfield, compound), `size` (sphere (r,), capsule (half_height, r), box
        half extents, heightfield (nx, nz, cell)), `pos`, `rot` (unit quaternion i, j, k, w;
        default identity), `vel`, `inv_mass` (0 = static), `verts` + `faces` (convex),
        `heights` (heightfield), or `subs` (compound: a list of shape dicts with their own
        `offset` and `rot` relative to the body; no nested compounds).  Returns the bodies'
        updated velocities (n, 3); the fluid particles inside a body are pushed out."""
        arr = (L.PhyCoupleBody * max(len(bodies), 1))()
        data, faces = [], []
        for k, b in enumerate(bodies):
            o = arr[k]
            o.shape = L.SHAPES[b["shape"]]
            size = list(b.get("size", ())) + [0.0] * 3
            vel = b.get("vel", (0.0, 0.0, 0.0))
            for a in range(3):
                o.size[a], o.pos[a], o.vel[a] = size[a], b["pos"][a], vel[a]
            for a, q in enumerate(b.get("rot", (0.0, 0.0, 0.0, 1.0))):
                o.rot[a] = q
            o.inv_mass = b.get("inv_mass", 0.0)
            o.data_first, o.data_count, o.face_first, o.face_count = _pack_shape_data(b, data, faces)
        d = np.array(data + [0.0], np.float64)
        f = np.array(faces + [0], np.uint32)
        L.check(self._lib.phy_fluid_couple_bodies(self._h, self._sub, C.cast(arr, C.c_void_p), len(bodies), _dp(d),
                                                  len(data), f.ctypes.data_as(C.POINTER(C.c_uint32)), len(faces), dt,
                                                  friction), "phy_fluid_couple_bodies")
        return np.array([list(o.vel) for o in arr[:len(bodies)]], np.float64).reshape(-1, 3)

    # ---- diagnostics (FluidSubsystem, subsystem.rs:149-163) ------------------------
    def _diag(self) -> np.ndarray:
        out = np.empty(4, np.float64)
        L.check(self._lib.phy_fluid_diagnostics(self._h, self._sub, _dp(out)), "phy_fluid_diagnostics")
        return out

    def total_momentum(self) -> np.ndarray:
        return self._diag()[:3]

    def kinetic_energy(self) -> float:
        return float(self._diag()[3])


class FluidSubsystem:
    """FluidSubsystem<f64> (crates/phy-fluid/src/subsystem.rs:26-164)."""

    _COUPLING = ("thermal_expansion", "heat_gain", "t_ref", "drag", "friction")

    def __init__(self, world: FluidWorld):
        self.world = world

    def _coupling(self) -> np.ndarray:
        out = np.empty(5, np.float64)
        L.check(self.world._lib.phy_fluid_get_coupling(self.world._h, self.world._sub, _dp(out)),
                "phy_fluid_get_coupling")
        return out

    def __getattr__(self, name):
        if name in FluidSubsystem._COUPLING:
            return float(self._coupling()[FluidSubsystem._COUPLING.index(name)])
        raise AttributeError(name)

    def __setattr__(self, name, value):
        if name in FluidSubsystem._COUPLING:
            c = self._coupling()
            c[FluidSubsystem._COUPLING.index(name)] = float(value)
            L.check(self.world._lib.phy_fluid_set_coupling(self.world._h, self.world._sub, _dp(c)),
                    "phy_fluid_set_coupling")
        else:
            object.__setattr__(self, name, value)

    def name(self) -> str:
        return "fluid"

    def total_momentum(self) -> np.ndarray:
        return self.world.total_momentum()

    def kinetic_energy(self) -> float:
        return self.world.kinetic_energy()
