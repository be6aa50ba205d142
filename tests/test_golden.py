"""The oracle reproduces its committed golden fixtures (tests/golden/make_golden.py)."""
import os

import numpy as np

from golden.make_golden import compute

HERE = os.path.dirname(os.path.abspath(__file__))


def test_oracle_matches_golden(rg, orc):
    g = np.load(os.path.join(HERE, "golden", "oracle_golden.npz"))
    now = compute(rg, orc)
    np.testing.assert_array_equal(now["lds"], g["lds"])
    np.testing.assert_array_equal(now["prng"], g["prng"])
    np.testing.assert_array_equal(now["prim"], g["prim"])
    np.testing.assert_allclose(now["tuv"], g["tuv"], rtol=1e-6)
    np.testing.assert_allclose(now["img_sum"], g["img_sum"], rtol=1e-5, atol=1e-6)
