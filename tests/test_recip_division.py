"""The alias build's division by a topic normaliser, restated on the CPU.

The device turns a Poisson draw x into q = floor(x * 2^32 / S[k]) without a
64-bit division per cell: topic_recip_kernel stores inv = floor((2^64 - 1) / S)
once per Phi step, and alias_word takes the high 64 bits of (x << 32) * inv and
corrects the estimate at most twice while the remainder is at least S
(csrc/kernels.cu).  The reference divides in float (src/cu/polyaurn.cu:115-122);
the exact quotient is this library's fixed-point Phi, which the GPU parity
tests compare cell by cell.  Here the same integer steps run in Python
integers against the true quotient, including the extreme normalisers and
draws, so the two-correction bound is checked where it is tight.
"""
import numpy as np

M64 = (1 << 64) - 1


def recip(s: int) -> int:
    return M64 // s if s else 0


def quotient_from_recip(x: int, s: int, inv: int) -> tuple[int, int]:
    """The device's steps; returns (quotient, corrections used)."""
    num = x << 32
    q = (num * inv) >> 64  # __umul64hi
    r = num - q * s
    used = 0
    if r >= s:
        q += 1
        r -= s
        used += 1
    if r >= s:
        q += 1
        used += 1
    return q, used


def _check(x: int, s: int) -> int:
    q, used = quotient_from_recip(x, s, recip(s))
    assert q == (x << 32) // s, (x, s)
    return used


def test_extremes():
    xs = [1, 2, 3, 7, 255, 65535, (1 << 31) - 1, 1 << 31, (1 << 32) - 2, (1 << 32) - 1]
    ss = [1, 2, 3, 5, 7, (1 << 32) - 1, 1 << 32, (1 << 32) + 1, (1 << 40) + 12345, (1 << 63) - 1, 1 << 63, M64]
    for s in ss:
        for x in xs:
            if x <= s:  # a cell's draw is part of its topic's normaliser
                _check(x, s)


def test_random_normalisers_and_draws():
    rng = np.random.default_rng(7)
    worst = 0
    for _ in range(20000):
        s = int(rng.integers(1, 1 << int(rng.integers(1, 64)), dtype=np.uint64)) or 1
        x = int(rng.integers(1, min(s, (1 << 32) - 1) + 1, dtype=np.uint64))
        worst = max(worst, _check(x, s))
    assert worst <= 2


def test_quotient_clamp_matches_plain_division():
    """x == S gives 2^32, which both paths clamp to 2^32 - 1."""
    for s in (1, 3, 1 << 20, (1 << 32) - 1):
        q, _ = quotient_from_recip(s, s, recip(s))
        assert q == 1 << 32
        assert min(q, (1 << 32) - 1) == min((s << 32) // s, (1 << 32) - 1)
