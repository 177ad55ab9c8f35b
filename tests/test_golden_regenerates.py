"""The committed golden fixtures are what their generator writes: tests/golden/gen_golden.py
(the pure-Python restatement of the reference's step) is re-run into a temporary folder and
every array must equal the committed one byte for byte, so the fixtures the oracle and the
device tests are checked against cannot drift from the script that defines them."""
import importlib.util
from pathlib import Path

import numpy as np
import pytest

GOLDEN = Path(__file__).resolve().parent / "golden"


def _generator(tmp_path):
    spec = importlib.util.spec_from_file_location("gen_golden_under_test", GOLDEN / "gen_golden.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    mod.HERE = tmp_path  # the cases write their .npz files into HERE
    return mod


def _bytes(x):
    x = np.ascontiguousarray(np.atleast_1d(x))
    return x.dtype.str, x.shape, x.tobytes()


@pytest.mark.parametrize("case,fixture", [("case_quickstart", "quickstart.npz"), ("case_dam216", "dam216.npz"),
                                          ("case_materials", "materials.npz")])
def test_fixture_regenerates_byte_for_byte(tmp_path, case, fixture):
    getattr(_generator(tmp_path), case)()
    fresh = dict(np.load(tmp_path / fixture))
    committed = dict(np.load(GOLDEN / fixture))
    assert sorted(fresh) == sorted(committed)
    for key in committed:
        assert _bytes(fresh[key]) == _bytes(committed[key]), f"{fixture}: {key}"
