"""The oracle against the committed golden fixtures (tests/golden/, made by
tests/golden/make_golden.py)."""
import os

import numpy as np
import pytest

from conftest import ROOT, rel

GOLD = os.path.join(ROOT, "tests", "golden")


@pytest.mark.parametrize("name", ["channel_16x12x8", "stretched_16x12x10"])
def test_oracle_reproduces_golden(name):
    import sys
    sys.path.insert(0, GOLD)
    from make_golden import CASES, run_case
    kw, steps = CASES[name]
    gold = np.load(os.path.join(GOLD, name + ".npz"))
    _, st, proj, out = run_case(kw, steps)
    assert np.array_equal(st[0], gold["U0"])
    for a, key in zip(proj, ("Up", "Vp", "Wp", "Pp")):
        assert rel(a, gold[key]) < 1e-13, key
    for a, key in zip(out, ("U", "V", "W", "P")):
        assert rel(a, gold[key]) < 1e-12, key
