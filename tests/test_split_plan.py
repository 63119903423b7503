"""Host logic of split products (no GPU): which unbalanced products the
default plan cuts into chunks of the long operand, and with which chunk
transform length (gpu_mpn_mul_split_plan).  The decisions on the shapes
measured on the B200 are pinned; random shapes check the rule's invariants.
"""
import numpy as np
import pytest

import flint_b200 as FB


@pytest.mark.parametrize("an,bn,want", [
    (1 << 24, 1 << 20, 22),          # 0.66 of the single transform's time
    (1 << 22, 3000, 20),             # 0.71
    (3000, 1 << 22, 20),             # operand order does not matter
    ((1 << 23) + (1 << 20), 1, 21),  # 0.60
    (5_000_000, 300_000, 21),        # 0.77
    (1 << 23, 700_000, 22),          # 0.70
    (1 << 24, 1 << 22, 23),          # 0.90
    (1 << 23, 1, 0),                 # eight 2^20-point chunks measured 1.06: single transform
    (3 << 20, 1 << 16, 0),           # measured 1.10: single transform
    (1 << 21, 1 << 17, 0),
    (1 << 24, 1 << 24, 0),           # balanced
    (1 << 24, 1 << 23, 0),
    (1000, 3, 0),                    # small products are never split
])
def test_measured_shapes(an, bn, want):
    assert FB.mpn_mul_split_plan(an, bn) == want


def test_invariants_on_random_shapes():
    rng = np.random.default_rng(7)
    for _ in range(400):
        an = int(2 ** rng.uniform(10, 25))
        bn = int(2 ** rng.uniform(0, np.log2(an)))
        if an + bn - 1 > 1 << 25:
            continue
        lc = FB.mpn_mul_split_plan(an, bn)
        logM = FB.mpn_mul_plan(an, bn)[1]
        if lc:
            assert 20 <= lc < logM
            assert (1 << lc) >= 2 * min(an, bn)          # chunks at least twice the short operand
            assert max(an, bn) > 2 * min(an, bn)          # only unbalanced products
        assert FB.mpn_mul_split_plan(bn, an) == lc


def test_errors_match_the_plan():
    with pytest.raises(FB.GpuFftSmallError):
        FB.mpn_mul_split_plan(0, 5)
    with pytest.raises(FB.GpuFftSmallError) as e:
        FB.mpn_mul_split_plan(1 << 25, (1 << 25) + 1)   # too balanced to split
    assert e.value.code == FB.ETOOBIG
    with pytest.raises(FB.GpuFftSmallError) as e:
        FB.mpn_mul_split_plan(1 << 30, 5)                # beyond 2^30 coefficients
    assert e.value.code == FB.ETOOBIG


@pytest.mark.parametrize("an,bn,want", [
    ((1 << 25) + (1 << 20), 1000, 21),
    ((1 << 26) + 12345, 4096, 22),
    (1 << 26, 1 << 20, 23),
    (1 << 28, 1 << 22, 25),
    (1 << 26, 1 << 24, 25),           # short operand of 2^24 limbs: chunks of 2^25 points
])
def test_products_beyond_the_longest_transform_split(an, bn, want):
    with pytest.raises(FB.GpuFftSmallError):
        FB.mpn_mul_plan(an, bn)                          # no single transform holds them
    assert FB.mpn_mul_split_plan(an, bn) == want


def test_transform_points_truncated_lengths():
    """Whole products between 2^(m-1) and 3 2^(m-2) coefficients (m >= 20)
    run 3 2^(m-2)-point transforms; elsewhere the power of two stays."""
    import flint_b200 as FB
    assert FB.mpn_mul_transform_points(1 << 23, 1 << 23) == 1 << 24        # L = 2^24 - 1: a power of two
    assert FB.mpn_mul_transform_points((1 << 23) + (1 << 20), (1 << 23) + (1 << 20)) == 3 << 23
    assert FB.mpn_mul_transform_points(3 << 22, 3 << 22) == 3 << 23
    assert FB.mpn_mul_transform_points((3 << 22) + 1, 3 << 22) == 3 << 23   # L = 3 2^23 exactly
    assert FB.mpn_mul_transform_points((3 << 22) + 1, (3 << 22) + 1) == 1 << 25
    assert FB.mpn_mul_transform_points(1 << 24, 1 << 24) == 1 << 25
    # below 2^19 coefficients the columns are too short for the radix-3 kernels
    assert FB.mpn_mul_transform_points(150000, 150000) == 1 << 19
    assert FB.mpn_mul_transform_points((1 << 18) + 100, (1 << 18) + 7) == 3 << 18
    # squarings take the same lengths
    assert FB.mpn_mul_transform_points(3000000, 3000000, square=True) == 3 << 21
