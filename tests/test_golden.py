"""The oracle reproduces its committed golden vectors (tests/golden/)."""
import os

import numpy as np

from tests.golden.make_golden import digest, make

HERE = os.path.dirname(os.path.abspath(__file__))


def test_oracle_matches_golden_vectors():
    gold = np.load(os.path.join(HERE, "golden", "tiny_oracle.npz"))
    now = make()
    for k in gold.files:
        assert np.array_equal(gold[k], now[k]), k
    assert digest(np.zeros(1)) == digest(np.zeros(1))
