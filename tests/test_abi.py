"""The C ABI of libphysph.so without a GPU: the library loads, exports every
symbol declared in include/*.h, and the calls that touch no device memory
behave like the reference's phy-ffi (crates/phy-ffi/src/lib.rs:954-1015)."""
import ctypes as C
import math
import re
from pathlib import Path

import numpy as np

from physics_b200 import _lib as L

INCLUDE = Path(__file__).resolve().parent.parent / "include"


def declared_functions():
    names = set()
    for h in INCLUDE.glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        for m in re.finditer(r"\b(phy_[a-z0-9_]+)\s*\(", text):
            names.add(m.group(1))
    return names


def test_header_symbols_are_exported():
    lib = L.load()
    names = declared_functions()
    assert len(names) >= 50
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing


def test_bindings_cover_header():
    assert declared_functions() == set(L.SIGNATURES)


def test_abi_version():
    assert L.load().phy_ffi_abi_version() == 3
    text = (INCLUDE / "phy_ffi.h").read_text()
    assert "#define PHY_FFI_ABI_VERSION 3" in text


def test_null_pointer_is_safe():
    """ffi_null_pointer_is_safe / ffi_f32_null_pointer_is_safe (lib.rs:954-1015)."""
    lib = L.load()
    assert lib.phy_world_step(None, 0.01) == -1
    assert lib.phy_world_step_checked(None, 0.01) == -1
    assert lib.phy_world_step_f32(None, 0.01) == -1
    assert math.isnan(lib.phy_world_time(None))
    assert lib.phy_world_fluid_count(None) == 0
    assert lib.phy_world_sub_count(None) == 0
    assert lib.phy_world_get_fluid_positions(None, None, 0) == 0
    assert lib.phy_world_get_fluid_positions_f32(None, None, 0) == 0
    assert lib.phy_world_get_rigid_transforms_f32(None, None, 0) == 0
    assert lib.phy_world_save(None, b"/tmp/x.json") == -1
    assert not lib.phy_world_load(None)
    lib.phy_world_destroy(None)
    assert lib.phy_fluid_len(None, 0) == -1
    assert lib.phy_fluid_step(None, 0, 0.01, 1) == -1
    one = np.zeros(3)
    assert lib.phy_fluid_couple_points(None, 0, 1, one.ctypes.data_as(L.DP), one.ctypes.data_as(L.DP),
                                       one.ctypes.data_as(L.DP), one.ctypes.data_as(L.DP), 0.01, 1.0, 1000.0) == -1
    assert lib.phy_fluid_couple_points(None, 0, 1, None, None, None, None, 0.01, 1.0, 1000.0) == -1
    dims = (C.c_uint64 * 3)(1, 1, 1)
    assert lib.phy_fluid_couple_heat(None, 0, dims, one.ctypes.data_as(L.DP), 1.0, one.ctypes.data_as(L.DP),
                                     one.ctypes.data_as(L.DP), 0.01, 0.0, 0.0, 0.0) == -1
    assert lib.phy_fluid_couple_heat(None, 0, None, None, 1.0, None, None, 0.01, 0.0, 0.0, 0.0) == -1
    assert lib.phy_fluid_couple_bodies(None, 0, None, 1, None, 0, None, 0, 0.01, 0.0) == -1
    assert lib.phy_fluid_pin_host(None, 64) == -1
    assert lib.phy_fluid_pin_host(one.ctypes.data, 0) == -1
    assert lib.phy_fluid_unpin_host(None) == -1
    assert lib.phy_fluid_last_error()  # a message was recorded


def test_non_fluid_factories_return_null():
    lib = L.load()
    for name in ("rigid", "rigid_empty", "granular", "coupled", "soft_empty", "field_empty", "optics_empty",
                 "solid_empty"):
        assert not getattr(lib, f"phy_world_create_{name}")()
    assert lib.phy_world_rigid_add_body(None, 0, 1.0, None, None) == -1


def test_params_defaults_match_reference():
    """SphParams::defaults() (params.rs:55-85)."""
    c = L.PhySphParams()
    L.load().phy_sph_params_defaults(C.byref(c))
    assert (c.rest_density, c.stiffness, c.viscosity, c.shear_min, c.mass, c.h) == (1000.0, 250.0, 3.5, 0.01,
                                                                                     0.02, 0.2)
    assert tuple(c.gravity) == (0.0, -9.81, 0.0)
    assert tuple(c.bounds_min) == (-5.0, -5.0, -5.0) and tuple(c.bounds_max) == (5.0, 5.0, 5.0)
    assert (c.boundary_damp, c.xsph_eps) == (0.4, 0.5)
    assert (c.n_visc_k, c.n_visc_n, c.visc_k[0], c.visc_n[0]) == (1, 1, 3.5, 1.0)


def test_params_struct_layout():
    assert C.sizeof(L.PhySphParams) == 8 * 17 + 8 + 2 * 8 * 16


def test_struct_layouts_match_the_header(tmp_path):
    """The ctypes mirrors of PhySphParams and PhyCoupleBody have the C header's sizes and
    field offsets (compiled here with the system C compiler)."""
    import shutil
    import subprocess
    import pytest
    cc = shutil.which("gcc") or shutil.which("cc")
    if not cc:
        pytest.skip("no C compiler")
    checks = {"PhySphParams": L.PhySphParams, "PhyCoupleBody": L.PhyCoupleBody}
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "phy_fluid.h"', "int main(void) {"]
    for name, st in checks.items():
        lines.append(f'  printf("{name} size %zu\\n", sizeof({name}));')
        for f, _ in st._fields_:
            lines.append(f'  printf("{name} {f} %zu\\n", offsetof({name}, {f}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run([cc, "-I", str(INCLUDE), str(src), "-o", str(exe)], check=True)
    got = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    want = []
    for name, st in checks.items():
        want.append(f"{name} size {C.sizeof(st)}")
        want += [f"{name} {f} {getattr(st, f).offset}" for f, _ in st._fields_]
    assert [g for g in got if g] == want
