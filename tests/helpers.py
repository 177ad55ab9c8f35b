"""Shared helpers of the test suite."""
import numpy as np


def ref_test_params(**over):
    """sph/tests.rs:11-16: defaults with bounds +-3."""
    from physics_b200 import SphParams
    p = SphParams.defaults()
    p.bounds_min = (-3.0, -3.0, -3.0)
    p.bounds_max = (3.0, 3.0, 3.0)
    for k, v in over.items():
        setattr(p, k, v)
    return p


def bits_equal(a, b) -> bool:
    a = np.ascontiguousarray(a, np.float64)
    b = np.ascontiguousarray(b, np.float64)
    return a.shape == b.shape and np.array_equal(a.view(np.uint64), b.view(np.uint64))


def assert_bits_equal(a, b, what=""):
    a = np.ascontiguousarray(a, np.float64)
    b = np.ascontiguousarray(b, np.float64)
    assert a.shape == b.shape, f"{what}: shape {a.shape} != {b.shape}"
    diff = a.view(np.uint64) != b.view(np.uint64)
    if diff.any():
        idx = np.argwhere(diff)[:5]
        detail = ", ".join(f"{tuple(i)}: {a[tuple(i)]!r} vs {b[tuple(i)]!r}" for i in idx)
        raise AssertionError(f"{what}: {int(diff.sum())} values differ bitwise (first: {detail})")
