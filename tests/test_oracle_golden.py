"""The oracle reproduces the committed golden fixtures (tests/golden), so a
change to the oracle that moves its numbers is caught."""
import os
import sys

import numpy as np

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))

import make_golden  # noqa: E402


def test_oracle_reproduces_golden_fixtures():
    ref = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "golden.npz"))
    got = make_golden.make()
    assert set(got) == set(ref.files)
    for k in ref.files:
        a, b = got[k], ref[k]
        scale = max(float(np.abs(b).max()), 1e-300)
        assert float(np.abs(a - b).max()) <= 1e-12 * scale, k
