"""The oracle's C generator (used where the product library must not be
loaded, e.g. the reference's CPU arm of the benchmark) builds exactly the
fields of the product's seeded workloads."""
import numpy as np
import pytest

import cpsz_b200
from cpsz_b200 import workloads as W
from tests._util import assert_bits_equal


@pytest.mark.parametrize("seed,r1,r2,n_flows,sigma", [(1, 1, 1, 1, 40.0), (5, 120, 90, 3, 40.0),
                                                      (7, 333, 517, 25, 60.0), (9, 64, 2000, 0, 10.0),
                                                      (11, 1000, 1000, 40, 60.0)])
def test_oracle_field_2d_equals_product(oracle, seed, r1, r2, n_flows, sigma):
    a = W.field_2d(seed, r1, r2, n_flows, sigma)
    b = oracle.field_2d(seed, r1, r2, n_flows, sigma)
    for x, y in zip(a, b):
        assert_bits_equal(x, y)


@pytest.mark.parametrize("seed,r,n_flows,sigma", [(2, (20, 30, 17), 4, 6.0), (3, (48, 40, 44), 12, 20.0)])
def test_oracle_field_3d_equals_product(oracle, seed, r, n_flows, sigma):
    a = W.field_3d(seed, *r, n_flows, sigma)
    b = oracle.field_3d(seed, *r, n_flows, sigma)
    for x, y in zip(a, b):
        assert_bits_equal(x, y)


def test_oracle_batch_layout_equals_product(oracle):
    assert oracle.batch_layout(3, 256, 128, 4096) == W.batch_layout(3, 256, 128, 4096)
    assert oracle.batch_layout(17, 40, 2, 9) == W.batch_layout(17, 40, 2, 9)
