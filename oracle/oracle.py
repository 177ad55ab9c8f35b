"""TEST INFRASTRUCTURE ONLY — ctypes wrapper of the CPU oracle (liboracle.so).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
module, always as the checker or the timed CPU baseline, never on the product
path.  Parity against reference-generated outputs is unpinned (the Rust
reference cannot be built here; see sph_oracle.cpp).
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "liboracle.so"

F_POS, F_VEL, F_ACC, F_BODY_ACC, F_RHO, F_P, F_MASS, F_MU_EFF, F_XSPH, F_MATERIAL = range(10)
_VEC = {F_POS, F_VEL, F_ACC, F_BODY_ACC, F_XSPH}


class OrcParams(C.Structure):
    _fields_ = [
        ("rest_density", C.c_double), ("stiffness", C.c_double), ("viscosity", C.c_double),
        ("shear_min", C.c_double), ("mass", C.c_double), ("h", C.c_double),
        ("gravity", C.c_double * 3), ("bounds_min", C.c_double * 3), ("bounds_max", C.c_double * 3),
        ("boundary_damp", C.c_double), ("xsph_eps", C.c_double),
        ("n_visc_k", C.c_uint32), ("n_visc_n", C.c_uint32),
        ("visc_k", C.c_double * 16), ("visc_n", C.c_double * 16),
    ]


class RefParams:
    """SphParams<f64>::defaults() restated for the oracle alone
    (crates/phy-fluid/src/sph/params.rs:55-85), so that a CPU-only run of the
    reference's step (the bench's reference arm) needs nothing from the
    product library."""

    def __init__(self):
        self.rest_density = 1000.0
        self.stiffness = 250.0
        self.viscosity = 3.5
        self.visc_k = [3.5]
        self.visc_n = [1.0]
        self.shear_min = 0.01
        self.mass = 0.02
        self.h = 0.2
        self.gravity = (0.0, -9.81, 0.0)
        self.bounds_min = (-5.0, -5.0, -5.0)
        self.bounds_max = (5.0, 5.0, 5.0)
        self.boundary_damp = 0.4
        self.xsph_eps = 0.5

    @staticmethod
    def defaults() -> "RefParams":
        return RefParams()


_lib = None
DP = C.POINTER(C.c_double)
SRC = Path(__file__).resolve().parent / "sph_oracle.cpp"


def build(force: bool = False) -> Path:
    """Compiles liboracle.so with the flags of oracle/Makefile (no FMA contraction)."""
    if not force and LIB_PATH.exists() and LIB_PATH.stat().st_mtime >= SRC.stat().st_mtime:
        return LIB_PATH
    import subprocess
    r = subprocess.run(["make", "-C", os.fspath(LIB_PATH.parent), "liboracle.so"], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + r.stdout + r.stderr)
    return LIB_PATH


def load():
    global _lib
    if _lib is None:
        build()
        lib = C.CDLL(os.fspath(LIB_PATH))
        sig = {
            "orc_new": (C.c_void_p, [C.POINTER(OrcParams)]),
            "orc_free": (None, [C.c_void_p]),
            "orc_len": (C.c_uint64, [C.c_void_p]),
            "orc_set_threads": (None, [C.c_void_p, C.c_int]),
            "orc_max_threads": (C.c_int, []),
            "orc_set_params": (None, [C.c_void_p, C.POINTER(OrcParams)]),
            "orc_get_params": (None, [C.c_void_p, C.POINTER(OrcParams)]),
            "orc_fill_box": (None, [C.c_void_p, DP, DP, C.c_double, C.c_double]),
            "orc_lattice_mass": (C.c_double, [C.c_void_p, C.c_double]),
            "orc_add": (None, [C.c_void_p, C.c_uint64, DP, DP, DP, C.POINTER(C.c_uint64)]),
            "orc_get": (C.c_int, [C.c_void_p, C.c_int, DP]),
            "orc_set": (C.c_int, [C.c_void_p, C.c_int, DP]),
            "orc_step": (None, [C.c_void_p, C.c_double]),
            "orc_step_n": (None, [C.c_void_p, C.c_double, C.c_int]),
            "orc_cell_keys": (None, [C.c_void_p, C.POINTER(C.c_int64)]),
            "orc_neighbors": (C.c_uint64, [C.c_void_p, C.c_uint64, C.POINTER(C.c_uint64), C.c_uint64]),
            "orc_diagnostics": (None, [C.c_void_p, DP]),
            "orc_counters": (None, [C.c_void_p, C.POINTER(C.c_uint64), C.c_int]),
            "orc_jvp": (None, [C.c_void_p, C.c_double, C.c_int, DP, DP, C.c_double, C.c_double]),
            "orc_point_neighbors": (C.c_uint64, [C.c_void_p, DP, C.POINTER(C.c_uint64), C.c_uint64]),
            "orc_couple_heat": (None, [C.c_void_p, C.POINTER(C.c_uint64), DP, C.c_double, DP, DP, C.c_double,
                                        C.c_double, C.c_double, C.c_double]),
            "orc_couple_bodies": (None, [C.c_void_p, C.c_void_p, C.c_uint32, DP, C.POINTER(C.c_uint32), C.c_double]),
            "orc_couple_points": (None, [C.c_void_p, C.c_uint64, DP, DP, DP, DP, C.c_double, C.c_double,
                                          C.c_double]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


def params_struct(p) -> OrcParams:
    """OrcParams from any object with SphParams' attribute names."""
    c = OrcParams()
    for name in ("rest_density", "stiffness", "viscosity", "shear_min", "mass", "h", "boundary_damp",
                 "xsph_eps"):
        setattr(c, name, float(getattr(p, name)))
    for name in ("gravity", "bounds_min", "bounds_max"):
        arr = getattr(c, name)
        v = getattr(p, name)
        for k in range(3):
            arr[k] = float(v[k])
    c.n_visc_k = len(p.visc_k)
    c.n_visc_n = len(p.visc_n)
    for k, v in enumerate(p.visc_k):
        c.visc_k[k] = float(v)
    for k, v in enumerate(p.visc_n):
        c.visc_n[k] = float(v)
    return c


class OracleWorld:
    """CPU restatement of FluidWorld<f64> (crates/phy-fluid/src/sph/world.rs)."""

    def __init__(self, params, threads: int = 1):
        self._lib = load()
        c = params_struct(params)
        self._w = self._lib.orc_new(C.byref(c))
        self._lib.orc_set_threads(self._w, threads)

    def __del__(self):
        try:
            self._lib.orc_free(self._w)
        except Exception:
            pass

    def set_threads(self, n: int) -> None:
        self._lib.orc_set_threads(self._w, n)

    def set_params(self, params) -> None:
        c = params_struct(params)
        self._lib.orc_set_params(self._w, C.byref(c))

    def __len__(self) -> int:
        return int(self._lib.orc_len(self._w))

    def fill_box(self, mn, mx, spacing, margin) -> None:
        a = np.asarray(mn, np.float64)
        b = np.asarray(mx, np.float64)
        self._lib.orc_fill_box(self._w, a.ctypes.data_as(DP), b.ctypes.data_as(DP), spacing, margin)

    def lattice_mass(self, s: float) -> float:
        return float(self._lib.orc_lattice_mass(self._w, s))

    def add_particles(self, pos, mass, vel=None, material=None) -> None:
        pos = np.ascontiguousarray(pos, np.float64).reshape(-1)
        n = pos.size // 3
        mass = np.ascontiguousarray(np.broadcast_to(np.asarray(mass, np.float64), (n,)))
        vp = None
        if vel is not None:
            vel = np.ascontiguousarray(vel, np.float64).reshape(-1)
            vp = vel.ctypes.data_as(DP)
        mp = None
        if material is not None:
            material = np.ascontiguousarray(np.broadcast_to(np.asarray(material, np.uint64), (n,)))
            mp = material.ctypes.data_as(C.POINTER(C.c_uint64))
        self._lib.orc_add(self._w, n, pos.ctypes.data_as(DP), vp, mass.ctypes.data_as(DP), mp)

    def get(self, field: int) -> np.ndarray:
        n = len(self)
        out = np.empty(3 * n if field in _VEC else n, np.float64)
        if self._lib.orc_get(self._w, field, out.ctypes.data_as(DP)) != 0:
            raise ValueError(field)
        return out.reshape(n, 3) if field in _VEC else out

    def set(self, field: int, values) -> None:
        a = np.ascontiguousarray(values, np.float64).reshape(-1)
        if self._lib.orc_set(self._w, field, a.ctypes.data_as(DP)) != 0:
            raise ValueError(field)

    def step(self, dt: float, n: int = 1) -> None:
        self._lib.orc_step_n(self._w, dt, n)

    def jvp(self, dt: float, n: int, tx, tv, dk: float = 0.0, dc: float = 0.0) -> tuple:
        """n steps with forward-mode tangents (orc_jvp): tx, tv are the (N, 3) tangents of the
        positions and velocities, dk and dc those of stiffness and visc_k[0].  Advances the world
        and returns the tangents of the final positions and velocities."""
        x = np.array(tx, np.float64, copy=True).reshape(-1)
        v = np.array(tv, np.float64, copy=True).reshape(-1)
        self._lib.orc_jvp(self._w, dt, n, x.ctypes.data_as(DP), v.ctypes.data_as(DP), dk, dc)
        return x.reshape(-1, 3), v.reshape(-1, 3)

    def cell_keys(self) -> np.ndarray:
        out = np.empty(3 * len(self), np.int64)
        self._lib.orc_cell_keys(self._w, out.ctypes.data_as(C.POINTER(C.c_int64)))
        return out.reshape(-1, 3)

    def neighbors(self, i: int, cap: int = 4096) -> np.ndarray:
        out = np.empty(cap, np.uint64)
        n = self._lib.orc_neighbors(self._w, i, out.ctypes.data_as(C.POINTER(C.c_uint64)), cap)
        return out[: min(n, cap)].copy()

    def diagnostics(self) -> np.ndarray:
        out = np.empty(4, np.float64)
        self._lib.orc_diagnostics(self._w, out.ctypes.data_as(DP))
        return out

    def neighbors_of_point(self, p3, cap: int = 65536) -> np.ndarray:
        """Indices for_each_neighbor visits for point p3 (grid of the current positions)."""
        q = np.ascontiguousarray(p3, np.float64).reshape(3)
        out = np.empty(cap, np.uint64)
        n = self._lib.orc_point_neighbors(self._w, q.ctypes.data_as(DP), out.ctypes.data_as(C.POINTER(C.c_uint64)),
                                          cap)
        return out[: min(n, cap)].astype(np.int64)

    def couple_heat(self, temp, src, origin, cell: float, dt: float, t_ref: float, beta: float,
                    heat_gain: float) -> np.ndarray:
        """FluidWorld::couple_heat (world.rs:555-678): temp is the (nz, ny, nx) grid of
        temperatures (x fastest in memory); returns the updated copy of src.  The particles'
        body accelerations take the buoyancy terms."""
        temp = np.ascontiguousarray(temp, np.float64)
        out = np.array(src, np.float64, copy=True, order="C")
        dims = (C.c_uint64 * 3)(temp.shape[2], temp.shape[1], temp.shape[0])
        o = np.ascontiguousarray(origin, np.float64).reshape(3)
        self._lib.orc_couple_heat(self._w, dims, o.ctypes.data_as(DP), cell, temp.ctypes.data_as(DP),
                                  out.ctypes.data_as(DP), dt, t_ref, beta, heat_gain)
        return out

    def couple_bodies(self, bodies, dt: float) -> np.ndarray:
        """FluidWorld::couple_bodies (world.rs:414-503) over body dicts (see pack_bodies);
        returns the bodies' updated velocities (n, 3)."""
        arr, data, faces = pack_bodies(bodies, OrcBody)
        self._lib.orc_couple_bodies(self._w, C.cast(arr, C.c_void_p), len(bodies), data.ctypes.data_as(DP),
                                    faces.ctypes.data_as(C.POINTER(C.c_uint32)), dt)
        return np.array([list(b.vel) for b in arr], np.float64).reshape(-1, 3)

    def couple_points(self, pos, vel, mass, dt: float, drag: float, soft_density: float, force=None):
        """FluidWorld::couple_points (world.rs:691-752): returns the (n, 3) forces; rows of
        points outside the bounds keep the values of `force` (zeros when None)."""
        pos = np.ascontiguousarray(pos, np.float64).reshape(-1)
        vel = np.ascontiguousarray(vel, np.float64).reshape(-1)
        mass = np.ascontiguousarray(mass, np.float64).reshape(-1)
        out = np.zeros(pos.size, np.float64) if force is None else np.array(force, np.float64).reshape(-1)
        self._lib.orc_couple_points(self._w, mass.size, pos.ctypes.data_as(DP), vel.ctypes.data_as(DP),
                                    mass.ctypes.data_as(DP), out.ctypes.data_as(DP), dt, drag, soft_density)
        return out.reshape(-1, 3)

    def counters(self, reset: bool = True) -> tuple:
        out = (C.c_uint64 * 2)()
        self._lib.orc_counters(self._w, out, 1 if reset else 0)
        return int(out[0]), int(out[1])


class OrcBody(C.Structure):
    """Same layout as PhyCoupleBody (include/phy_fluid.h)."""
    _fields_ = [("shape", C.c_int32), ("data_first", C.c_uint32), ("data_count", C.c_uint32),
                ("face_first", C.c_uint32), ("face_count", C.c_uint32), ("reserved", C.c_uint32),
                ("size", C.c_double * 3), ("pos", C.c_double * 3), ("rot", C.c_double * 4), ("vel", C.c_double * 3),
                ("inv_mass", C.c_double)]


SHAPES = {"sphere": 0, "capsule": 1, "box": 2, "convex": 3, "heightfield": 4, "compound": 5}


def pack_bodies(bodies, struct):
    """Body dicts -> (struct array, data doubles, face indices).  A dict holds `shape`
    (a SHAPES name), `size` (sphere (r,), capsule (half_height, r), box half extents,
    heightfield (nx, nz, cell)), `pos`, `rot` (unit quaternion i, j, k, w; default identity),
    `vel`, `inv_mass`, and `verts` + `faces` (convex), `heights` (heightfield) or `subs`
    (compound: shape dicts with `offset` and `rot` relative to the body)."""
    arr = (struct * max(len(bodies), 1))()
    data, faces = [], []
    for k, b in enumerate(bodies):
        o = arr[k]
        o.shape = SHAPES[b["shape"]]
        size = list(b.get("size", ())) + [0.0] * 3
        for a in range(3):
            o.size[a] = size[a]
            o.pos[a] = b["pos"][a]
            o.vel[a] = b.get("vel", (0.0, 0.0, 0.0))[a]
        rot = b.get("rot", (0.0, 0.0, 0.0, 1.0))
        for a in range(4):
            o.rot[a] = rot[a]
        o.inv_mass = b.get("inv_mass", 0.0)
        o.data_first, o.data_count, o.face_first, o.face_count = _shape_data(b, data, faces)
    return arr, np.array(data + [0.0], np.float64), np.array(faces + [0], np.uint32)


def _shape_data(b, data, faces):
    """Appends a shape's convex vertices and faces, heightfield heights, or compound
    sub-shape records (16 doubles each: shape, size[3], offset[3], quaternion, data_first,
    data_count, face_first, face_count, 0) to data / faces; returns (data_first,
    data_count, face_first, face_count)."""
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
        d0 = len(data)
        data.extend([0.0] * (16 * len(b["subs"])))
        for q, sub in enumerate(b["subs"]):
            size = list(sub.get("size", ())) + [0.0] * 3
            rec = [float(SHAPES[sub["shape"]])] + [float(v) for v in size[:3]]
            rec += [float(v) for v in sub.get("offset", (0.0, 0.0, 0.0))]
            rec += [float(v) for v in sub.get("rot", (0.0, 0.0, 0.0, 1.0))]
            rec += [float(v) for v in _shape_data(sub, data, faces)] + [0.0]
            data[d0 + 16 * q: d0 + 16 * (q + 1)] = rec
        return d0, len(b["subs"]), 0, 0
    return 0, 0, 0, 0


def max_threads() -> int:
    return int(load().orc_max_threads())
