"""The oracle's radix-partition choice and partition hash against the
reference's own tests of them (exec/radix_join_test.go): RadixBitsFor's
table of estimates (:93-118), the mixed hash spreading sequential keys with
gaps over 64 partitions where masking the raw low bits leaves partitions
empty (:120-154), and the unpartitioned mask giving partition 0 for every
key (:156-162)."""
from __future__ import annotations

import pytest

from oracle import refcpu as R

MIN_BUILD_ROWS, TARGET_ROWS, MIN_BITS, MAX_BITS = 65536, 8192, 4, 6  # exec/parallel_join.go:28-33


@pytest.mark.parametrize("est,bits", [
    (0, 0), (1, 0), (MIN_BUILD_ROWS - 1, 0), (MIN_BUILD_ROWS, MIN_BITS), (16 * TARGET_ROWS, MIN_BITS),
    (16 * TARGET_ROWS + 1, MIN_BITS + 1), (300_000, MAX_BITS), (1_500_000, MAX_BITS), (1 << 40, MAX_BITS),
])
def test_radix_bits_for(est, bits):
    assert R.radix_bits_for(est) == bits


def test_radix_hash_spreads_sequential_keys():
    nkeys, nparts, step = 1 << 16, 64, 8
    counts = [0] * nparts
    raw = [0] * nparts
    for i in range(nkeys):
        counts[R.radix_part(i * step, nparts - 1)] += 1
        raw[(i * step) & (nparts - 1)] += 1
    want = nkeys // nparts
    assert all(want // 2 <= c <= want * 2 for c in counts), counts
    assert raw.count(0) > 0  # the premise: the unmixed low bits leave partitions empty


def test_unpartitioned_mask_is_partition_zero():
    for key in (-(1 << 63), -1, 0, 1, 1 << 40, (1 << 63) - 1):
        assert R.radix_part(key, 0) == 0
