"""FemState JSON checkpoints: byte-identical round trip of pmsim's own files (no GPU needed)."""
import glob
import os

import numpy as np
import pytest

from pmsim_b200 import state_io

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FILES = sorted(glob.glob(os.path.join(GOLDEN, "femstate_*.json")))


@pytest.mark.parametrize("path", FILES, ids=[os.path.basename(f) for f in FILES])
def test_pmsim_state_files_round_trip_byte_for_byte(path):
    text = open(path).read().strip()
    st = state_io.loads(text)
    assert state_io.dumps(st) == text


@pytest.mark.parametrize("x,expected", [(1.0, "1.0"), (0.0123, "0.0123"), (2.6020852139652106e-16, "2.6020852139652106e-16"),
                                        (7.379999999999999, "7.379999999999999"), (1e21, "1e21"), (1e-5, "0.00001"),
                                        (1.5e-7, "1.5e-7"), (-3.25, "-3.25"), (123456789012345680.0, "1.2345678901234568e17"),
                                        (0.0, "0.0")])
def test_float_notation(x, expected):
    assert state_io.format_float(x) == expected
    assert float(state_io.format_float(x)) == x


def test_random_values_round_trip_exactly():
    rng = np.random.default_rng(0)
    for v in np.concatenate([rng.normal(0, 1, 200), 10.0 ** rng.uniform(-30, 30, 200)]):
        assert float(state_io.format_float(v)) == v
