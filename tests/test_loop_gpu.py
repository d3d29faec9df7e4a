"""Flush-and-repeat with sliding views on the engine (the reference's test/python/tests/
test_loop.py cases, as restated on the oracle in tests/test_oracle_reference_cases.py), against
NumPy's loops: exact, since the values are small integers."""
import numpy as np
import pytest

from tests import programs as P

pytestmark = pytest.mark.gpu


def test_loop_sliding_views_triangular_numbers(gpu_rt):
    got, want = P.loop_triangular_numbers(gpu_rt)
    np.testing.assert_array_equal(got, want)


def test_loop_one_and_two_dimensional_sliding_views(gpu_rt):
    got, want = P.loop_diagonal(gpu_rt)
    np.testing.assert_array_equal(got, want)
