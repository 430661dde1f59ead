"""Pins the oracle's MT19937 restatement (common_mt19937ar.f90) to published answers."""
import numpy as np

from oracle import mt19937 as mt


def test_known_answer_10000th_output():
    # init_genrand(5489): the 10000th genrand_int32 output is 4123659995
    # (the value the C++ standard requires of std::mt19937).
    g = mt.MT19937Batch([5489])
    for _ in range(9999):
        g.int32()
    assert int(g.int32()[0]) == 4123659995


def test_first_output_default_seed():
    g = mt.MT19937Batch([5489])
    assert int(g.int32()[0]) == 3499211612


def test_res53_matches_numpy_legacy_randomstate():
    # numpy's RandomState(int) seeds with init_genrand and random_sample uses
    # the same 53-bit construction as genrand_res53 (independent code).
    seeds = [1, 42, 5489, 123456789, 2**31 - 1]
    ours = mt.com_rand_seed(700, seeds)
    for s, row in zip(seeds, ours):
        ref = np.random.RandomState(s).random_sample(700)
        assert np.array_equal(row, ref)


def test_vectorised_streams_are_independent():
    a = mt.com_rand_seed(5, [7, 8])
    b = mt.com_rand_seed(5, [8])
    assert np.array_equal(a[1], b[0])
    assert not np.array_equal(a[0], a[1])
