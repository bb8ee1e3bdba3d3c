"""The oracle reproduces the committed golden fixtures (tests/golden/*.npz) bit for bit."""
import os
import sys

import numpy as np
import pytest

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
sys.path.insert(0, HERE)
import make_golden  # noqa: E402

CASES = make_golden.golden_cases()


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_reproduces_golden(oracle, name):
    builder, steps, ifr, nsub = CASES[name]
    ref = np.load(os.path.join(HERE, name + ".npz"))
    c, f, di, pr = make_golden.run(builder, steps, ifr, nsub)
    assert float(ref["dt"]) == c.dt
    assert np.array_equal(ref["f"], f)
    assert np.array_equal(ref["di"], di)
    assert np.array_equal(ref["prims"], pr)
