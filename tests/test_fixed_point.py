"""The core force sums of the step kernel (md_nucleation_b200/csrc/advance.cu,
acc_add / core_reduce): every 64-bit fixed-point term u is split into its
low 16 bits, the next 16 bits and the high 32 bits; each part is summed in a
32-bit unsigned accumulator (32-bit shared-memory atomics, wrapping modulo
2^32), and the reduction folds the three sums back into one 64-bit value.

Restated here in integer arithmetic: the fold equals the 64-bit sum of the
terms exactly, for any signs and magnitudes up to the saturation limit
(2^21 kcal/mol/A at 2^40 per unit), as long as an accumulator takes at most
65,536 terms (the engine caps the near list at 64,511 molecules, leaving
room for pair tiles and bonded terms).  At 65,538 maximal low parts the
16-bit sum would no longer fit 32 bits, which is why the cap exists.  Like
the 64-bit sums themselves, the fold is exact modulo 2^64: a true sum
outside the int64 range wraps in both.
"""
import random

import pytest

M32 = (1 << 32) - 1
M64 = (1 << 64) - 1
SAT = (1 << 21) * (1 << 40)  # saturated term, kcal/mol/A at the 2^-40 scale


def split(v):
    u = v & M64
    return u & 0xFFFF, (u >> 16) & 0xFFFF, (u >> 32) & M32


def wrap64(v):
    """A sum as the 64-bit accumulators hold it (two's complement)."""
    v &= M64
    return v - (1 << 64) if v >> 63 else v


def chunked_sum(terms):
    a0 = a1 = a2 = 0
    for v in terms:
        c0, c1, c2 = split(v)
        a0 = (a0 + c0) & M32
        a1 = (a1 + c1) & M32
        a2 = (a2 + c2) & M32
    s = (a0 + (a1 << 16) + (a2 << 32)) & M64
    return s - (1 << 64) if s >> 63 else s


@pytest.mark.parametrize("seed", range(5))
def test_fold_equals_the_64_bit_sum(seed):
    rng = random.Random(seed)
    for n in (1, 2, 31, 1000, 4096):
        terms = [rng.randint(-SAT, SAT) for _ in range(n)]
        assert chunked_sum(terms) == wrap64(sum(terms))
        small = [rng.randint(-(1 << 44), 1 << 44) for _ in range(n)]
        assert chunked_sum(small) == sum(small)


def test_order_does_not_matter():
    rng = random.Random(7)
    terms = [rng.randint(-SAT, SAT) for _ in range(3000)]
    want = chunked_sum(terms)
    for _ in range(5):
        rng.shuffle(terms)
        assert chunked_sum(terms) == want


def test_bound_of_65536_terms():
    # the worst low parts: every term ends in 0xFFFF, in both 16-bit chunks
    worst = 0x0000_0000_FFFF_FFFF
    terms = [worst] * 65536
    assert chunked_sum(terms) == sum(terms)
    # 65,537 still fit (65,537 * 65,535 = 2^32 - 1); 65,538 overflow the
    # 32-bit low accumulator
    assert sum(split(v)[0] for v in terms + [worst]) == M32
    assert sum(split(v)[0] for v in terms + [worst, worst]) > M32
    # negative terms have all-ones low parts too (two's complement)
    neg = [-1] * 65536
    assert chunked_sum(neg) == -65536


def test_saturated_terms_of_both_signs():
    terms = [SAT, -SAT] * 5000 + [SAT]
    assert chunked_sum(terms) == SAT
