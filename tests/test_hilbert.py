"""Compact Hilbert keys: oracle invariants and the product's key function.

The reference defines the cell order by compact_p_to_h (src/hilbert.f90:241-271,
Hamilton's compact Hilbert index).  These CPU tests pin the oracle against
properties every Hilbert index must have and then require the product's key
function (the one the LUT and the device fallback use) to agree with the
oracle on every cell, including positions outside the box, which the
reference hashes rather than rejects.
"""
import itertools

import numpy as np
import pytest

MS = [(1, 1, 1), (2, 2, 2), (3, 3, 3), (4, 4, 4), (3, 3, 4), (1, 5, 3), (2, 3, 1), (5, 2, 4), (7, 5, 5)]


def all_points(M):
    return itertools.product(*(range(1 << m) for m in M))


@pytest.mark.parametrize("m", [1, 2, 3, 4])
def test_compact_equals_hilbert_for_equal_bits(oracle, m):
    M = (m, m, m)
    for p in all_points(M):
        assert oracle.compact_p_to_h(p, M) == oracle.p_to_h(p, m)


@pytest.mark.parametrize("M", MS)
def test_compact_index_is_a_bijection_with_round_trip(oracle, M):
    S = 1 << sum(M)
    seen = np.zeros(S, bool)
    for p in all_points(M):
        h = oracle.compact_p_to_h(p, M)
        assert 0 <= h < S
        assert not seen[h]
        seen[h] = True
        assert tuple(oracle.compact_h_to_p(h, M)) == p
    assert seen.all()


@pytest.mark.parametrize("M", [(1, 1, 1), (2, 2, 2), (3, 3, 3), (4, 4, 4), (5, 5, 5)])
def test_consecutive_keys_are_face_neighbours(oracle, M):
    # a Hilbert curve on a cube visits face neighbours in turn (the compact
    # index of an unequal box is not continuous, so only cubes are checked)
    S = 1 << sum(M)
    prev = oracle.compact_h_to_p(0, M)
    for h in range(1, S):
        cur = oracle.compact_h_to_p(h, M)
        assert np.abs(cur - prev).sum() == 1, (h, prev, cur)
        prev = cur


@pytest.mark.parametrize("M", MS)
def test_product_key_function_matches_oracle(oracle, rm, M):
    for p in all_points(M):
        assert rm.compact_p_to_h(p, M) == oracle.compact_p_to_h(p, M)
    S = 1 << sum(M)
    for h in range(S):
        assert tuple(rm.compact_h_to_p(h, M)) == tuple(oracle.compact_h_to_p(h, M))


def test_product_key_function_out_of_box_matches_oracle(oracle, rm):
    rng = np.random.default_rng(5)
    for M in [(3, 3, 4), (5, 5, 5), (7, 7, 7)]:
        for _ in range(2000):
            p = rng.integers(-300, 300, size=3)
            assert rm.compact_p_to_h(p, M) == oracle.compact_p_to_h(p, M)
