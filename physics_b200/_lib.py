"""ctypes declarations of libphysph.so (include/phy_ffi.h, include/phy_fluid.h).

The library is the product; this module only loads it.  There is no fallback:
if the shared library cannot be loaded the import fails with the reason.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "lib" / "libphysph.so"

MAX_MATERIALS = 16

PRECISION_F64_PLAIN = 0
PRECISION_F32_COMP = 1

TUNE_COMP_TILE = 0
TUNE_HALO_CAP = 1
TUNE_CTAS_PER_SM = 2
TUNE_QUEUE = 3
TUNE_SORT_BLOCK = 4
TUNE_GRAPH_CHUNK = 5
TUNE_DENSE_MEAN = 6
TUNE_DENSE_MASKS = 7
TUNE_PARAMS = {"comp_tile": TUNE_COMP_TILE, "halo_cap": TUNE_HALO_CAP, "ctas_per_sm": TUNE_CTAS_PER_SM,
               "queue": TUNE_QUEUE, "sort_block": TUNE_SORT_BLOCK, "graph_chunk": TUNE_GRAPH_CHUNK,
               "dense_mean": TUNE_DENSE_MEAN, "dense_masks": TUNE_DENSE_MASKS}

NOALLOC_MAX_PARTICLES = 65536
NOALLOC_MAX_CELLS = 262144

FIELD_POS = 0
FIELD_VEL = 1
FIELD_ACC = 2
FIELD_BODY_ACC = 3
FIELD_RHO = 4
FIELD_P = 5
FIELD_MASS = 6
FIELD_MU_EFF = 7
FIELD_XSPH = 8
FIELD_MATERIAL = 9
FIELD_COMPONENTS = {FIELD_POS: 3, FIELD_VEL: 3, FIELD_ACC: 3, FIELD_BODY_ACC: 3, FIELD_RHO: 1, FIELD_P: 1,
                    FIELD_MASS: 1, FIELD_MU_EFF: 1, FIELD_XSPH: 3, FIELD_MATERIAL: 1}


class PhyTuneTrial(C.Structure):
    _fields_ = [("ctas_per_sm", C.c_int32), ("queue", C.c_int32), ("sort_block", C.c_int32),
                ("comp_tile", C.c_int32), ("ms_per_step", C.c_double), ("samples", C.c_int32),
                ("reserved", C.c_int32)]


class PhyCoupleBody(C.Structure):
    """PhyCoupleBody of include/phy_fluid.h (a rigid body for phy_fluid_couple_bodies)."""
    _fields_ = [("shape", C.c_int32), ("data_first", C.c_uint32), ("data_count", C.c_uint32),
                ("face_first", C.c_uint32), ("face_count", C.c_uint32), ("reserved", C.c_uint32),
                ("size", C.c_double * 3), ("pos", C.c_double * 3), ("rot", C.c_double * 4), ("vel", C.c_double * 3),
                ("inv_mass", C.c_double)]


SHAPES = {"sphere": 0, "capsule": 1, "box": 2, "convex": 3, "heightfield": 4, "compound": 5}


class PhySphParams(C.Structure):
    _fields_ = [
        ("rest_density", C.c_double),
        ("stiffness", C.c_double),
        ("viscosity", C.c_double),
        ("shear_min", C.c_double),
        ("mass", C.c_double),
        ("h", C.c_double),
        ("gravity", C.c_double * 3),
        ("bounds_min", C.c_double * 3),
        ("bounds_max", C.c_double * 3),
        ("boundary_damp", C.c_double),
        ("xsph_eps", C.c_double),
        ("n_visc_k", C.c_uint32),
        ("n_visc_n", C.c_uint32),
        ("visc_k", C.c_double * MAX_MATERIALS),
        ("visc_n", C.c_double * MAX_MATERIALS),
    ]


H = C.c_void_p  # PhyWorldHandle*
DP = C.POINTER(C.c_double)
FP = C.POINTER(C.c_float)

# name: (restype, argtypes) — every symbol declared in include/*.h.
SIGNATURES = {
    "phy_ffi_abi_version": (C.c_uint32, []),
    "phy_world_create_fluid": (H, []),
    "phy_world_create_rigid": (H, []),
    "phy_world_create_rigid_empty": (H, []),
    "phy_world_create_granular": (H, []),
    "phy_world_create_coupled": (H, []),
    "phy_world_create_soft_empty": (H, []),
    "phy_world_create_field_empty": (H, []),
    "phy_world_create_optics_empty": (H, []),
    "phy_world_create_solid_empty": (H, []),
    "phy_world_step": (C.c_int32, [H, C.c_double]),
    "phy_world_step_checked": (C.c_int32, [H, C.c_double]),
    "phy_world_time": (C.c_double, [H]),
    "phy_world_sub_count": (C.c_size_t, [H]),
    "phy_world_fluid_count": (C.c_size_t, [H]),
    "phy_world_get_fluid_positions": (C.c_size_t, [H, DP, C.c_size_t]),
    "phy_world_get_fluid_velocities": (C.c_size_t, [H, DP, C.c_size_t]),
    "phy_world_rigid_count": (C.c_size_t, [H]),
    "phy_world_get_rigid_transforms": (C.c_size_t, [H, DP, C.c_size_t]),
    "phy_world_save": (C.c_int32, [H, C.c_char_p]),
    "phy_world_load": (H, [C.c_char_p]),
    "phy_world_destroy": (None, [H]),
    "phy_world_step_f32": (C.c_int32, [H, C.c_float]),
    "phy_world_get_fluid_positions_f32": (C.c_size_t, [H, FP, C.c_size_t]),
    "phy_world_get_fluid_velocities_f32": (C.c_size_t, [H, FP, C.c_size_t]),
    "phy_world_get_rigid_transforms_f32": (C.c_size_t, [H, FP, C.c_size_t]),
    "phy_world_rigid_add_body": (C.c_int64, [H, C.c_int32, C.c_double, DP, DP]),
    "phy_world_rigid_apply_force": (C.c_int32, [H, C.c_int64, DP, C.c_double, C.c_int32]),
    "phy_world_rigid_apply_torque": (C.c_int32, [H, C.c_int64, DP, C.c_double, C.c_int32]),
    "phy_world_rigid_get_velocity": (C.c_int32, [H, C.c_int64, DP]),
    "phy_world_rigid_get_angular_velocity": (C.c_int32, [H, C.c_int64, DP]),
    "phy_sph_params_defaults": (None, [C.POINTER(PhySphParams)]),
    "phy_fluid_world_create": (H, [C.POINTER(PhySphParams), C.c_int32]),
    "phy_fluid_add_subsystem": (C.c_int32, [H, C.POINTER(PhySphParams), C.c_int32]),
    "phy_fluid_fill_box": (C.c_int32, [H, C.c_uint32, DP, DP, C.c_double, C.c_double]),
    "phy_fluid_lattice_mass": (C.c_double, [H, C.c_uint32, C.c_double]),
    "phy_fluid_add_particles": (C.c_int32, [H, C.c_uint32, C.c_uint64, DP, DP, DP, C.POINTER(C.c_uint32)]),
    "phy_fluid_len": (C.c_int64, [H, C.c_uint32]),
    "phy_fluid_get_field": (C.c_int32, [H, C.c_uint32, C.c_int32, DP, C.c_uint64]),
    "phy_fluid_set_field": (C.c_int32, [H, C.c_uint32, C.c_int32, DP, C.c_uint64]),
    "phy_fluid_get_params": (C.c_int32, [H, C.c_uint32, C.POINTER(PhySphParams)]),
    "phy_fluid_set_params": (C.c_int32, [H, C.c_uint32, C.POINTER(PhySphParams)]),
    "phy_fluid_step": (C.c_int32, [H, C.c_uint32, C.c_double, C.c_uint32]),
    "phy_fluid_diagnostics": (C.c_int32, [H, C.c_uint32, DP]),
    "phy_fluid_couple_heat": (C.c_int32, [H, C.c_uint32, C.POINTER(C.c_uint64), DP, C.c_double, DP, DP, C.c_double,
                                          C.c_double, C.c_double, C.c_double]),
    "phy_fluid_couple_bodies": (C.c_int32, [H, C.c_uint32, C.c_void_p, C.c_uint32, DP, C.c_uint64,
                                            C.POINTER(C.c_uint32), C.c_uint64, C.c_double, C.c_double]),
    "phy_fluid_couple_points": (C.c_int32, [H, C.c_uint32, C.c_uint64, DP, DP, DP, DP, C.c_double, C.c_double,
                                            C.c_double]),
    "phy_fluid_get_coupling": (C.c_int32, [H, C.c_uint32, DP]),
    "phy_fluid_set_coupling": (C.c_int32, [H, C.c_uint32, DP]),
    "phy_fluid_set_stream": (C.c_int32, [H, C.c_void_p]),
    "phy_fluid_synchronize": (C.c_int32, [H]),
    "phy_fluid_set_particles_device": (C.c_int32, [H, C.c_uint32, C.c_uint64, C.c_void_p, C.c_void_p, C.c_void_p,
                                                   C.c_void_p]),
    "phy_fluid_get_field_device": (C.c_int32, [H, C.c_uint32, C.c_int32, C.c_void_p, C.c_uint64]),
    "phy_fluid_pin_host": (C.c_int32, [C.c_void_p, C.c_uint64]),
    "phy_fluid_unpin_host": (C.c_int32, [C.c_void_p]),
    "phy_fluid_set_counting": (C.c_int32, [H, C.c_uint32, C.c_int32]),
    "phy_fluid_step_counters": (C.c_int32, [H, C.c_uint32, C.POINTER(C.c_uint64)]),
    "phy_fluid_dense_mask_info": (C.c_int32, [H, C.c_uint32, C.POINTER(C.c_uint64)]),
    "phy_fluid_set_timing": (C.c_int32, [H, C.c_uint32, C.c_int32]),
    "phy_fluid_phase_times": (C.c_int32, [H, C.c_uint32, DP, C.c_int32]),
    "phy_fluid_set_tuning": (C.c_int32, [H, C.c_uint32, C.c_int32, C.c_int64]),
    "phy_fluid_get_tuning": (C.c_int32, [H, C.c_uint32, C.c_int32, C.POINTER(C.c_int64)]),
    "phy_fluid_set_scenes": (C.c_int32, [H, C.c_uint32, C.c_uint32, C.POINTER(C.c_uint64), DP, DP]),
    "phy_fluid_clear_scenes": (C.c_int32, [H, C.c_uint32]),
    "phy_fluid_scene_count": (C.c_uint32, [H, C.c_uint32]),
    "phy_fluid_tape_begin": (C.c_int32, [H, C.c_uint32, C.c_uint32]),
    "phy_fluid_tape_clear": (C.c_int32, [H, C.c_uint32]),
    "phy_fluid_tape_steps": (C.c_uint32, [H, C.c_uint32]),
    "phy_fluid_step_backward": (C.c_int32, [H, C.c_uint32, DP, DP, DP, DP, DP]),
    "phy_fluid_autotune": (C.c_int32, [H, C.c_uint32, C.c_double, C.c_uint32, C.POINTER(PhyTuneTrial),
                                       C.c_uint32, C.POINTER(C.c_uint32)]),
    "phy_fluid_autotune_horizon": (C.c_int32, [H, C.c_uint32, C.c_double, C.c_uint32, C.c_uint32,
                                               C.POINTER(PhyTuneTrial), C.c_uint32, C.POINTER(C.c_uint32)]),
    "phy_fluid_density_noalloc": (C.c_int32, [C.POINTER(PhySphParams), C.c_uint64, C.c_void_p, C.c_void_p,
                                              C.c_void_p, C.c_void_p, C.c_void_p]),
    "phy_fluid_last_error": (C.c_char_p, []),
}

_lib = None


def load() -> C.CDLL:
    """Loads libphysph.so once and declares every entry point."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python -c 'import __graft_entry__ as g; g.build()'` "
            "or `python physics_b200/csrc/build.py` (needs nvcc)")
    lib = C.CDLL(os.fspath(LIB_PATH))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def last_error() -> str:
    msg = load().phy_fluid_last_error()
    return msg.decode() if msg else ""


class PhyError(RuntimeError):
    """A phy_* call returned its failure value."""

    def __init__(self, what: str, code=None):
        detail = last_error()
        super().__init__(f"{what} failed" + (f" (rc={code})" if code is not None else "") +
                         (f": {detail}" if detail else ""))
        self.code = code


def check(rc: int, what: str) -> int:
    if rc != 0:
        raise PhyError(what, rc)
    return rc
