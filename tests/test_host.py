"""CPU tests of the product's host-side protocol code against the oracle."""
import numpy as np
import pytest

import oracle
from pyro_cmc_b200.anneal import generate_T_profile


@pytest.mark.parametrize("args", [(10.0, 0.05, [1.0, 0.1, 0.05], 100), (10.062, 0.02, [0.5, 0.1, 0.02], 200),
                                  (2.0, 0.01, [1.5, 1.0, 0.7, 0.5, 0.3, 0.1, 0.05, 0.01], 400),
                                  (1.0, 0.5, [0.7, 2.0], 5), (3.0, 0.1, [0.1], 1)])
def test_T_profile_matches_oracle(args):
    T, idx = generate_T_profile(*args)
    To, io = oracle.T_profile(*args)
    np.testing.assert_array_equal(np.array(T), To)
    assert list(idx) == list(io)
