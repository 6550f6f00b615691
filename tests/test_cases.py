"""Synthetic workload generators (CPU)."""
import numpy as np

from prandtl_b200 import cases


def test_sweep_generator_matches_spec():
    cs = cases.sweep_cases(256, seed=3)
    assert len(cs) == 256
    assert all(8 <= n <= 64 and 2 <= N <= 5 and 1.0 <= e <= 5.0 for n, N, e in cs)
    assert {N for _, N, _ in cs} == {2, 3, 4, 5}
    assert cs == cases.sweep_cases(256, seed=3)  # deterministic


def test_counter_rng_is_deterministic_and_uniform():
    a = cases.uniform01(0, np.arange(100000))
    assert np.array_equal(a, cases.uniform01(0, np.arange(100000)))
    assert 0.0 <= a.min() and a.max() < 1.0
    assert abs(a.mean() - 0.5) < 0.01
