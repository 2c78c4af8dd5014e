"""The oracle reproduces the committed golden fixtures (tests/golden/,
made by tests/golden/make_golden.py) exactly: a regression pin of the
restated algorithm."""
import ctypes as C
import os

import numpy as np
import pytest

from oracle import oracle as O
from tests.golden import make_golden as G

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.mark.parametrize("name", sorted(G.CASES))
def test_oracle_reproduces_fixture(name):
    z = np.load(os.path.join(HERE, f"{name}.npz"))
    x, f = G.make(name)
    np.testing.assert_array_equal(x, z["xPoints"])
    np.testing.assert_allclose(f, z["randField"], rtol=0, atol=1e-13 * max(1.0, np.abs(z["randField"]).max()))


def test_rnglib_stream_fixture():
    z = np.load(os.path.join(HERE, "rnglib_stream.npz"))
    for s in (0, 1, 99):
        r = O.rng(s)
        got = np.array([O.lib().rfo_rng_i4_uni(C.byref(r)) for _ in range(1000)])
        np.testing.assert_array_equal(got, z[f"seed{s}"])
