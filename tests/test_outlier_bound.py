"""The rank-pass skip of the outlier zeroing, checked as a rule on the CPU.

The CUDA kernels (outlier_column in afr_kernels.cuh) skip the O(S^2) median
of a column when one of two lower bounds of the median already shows that no
element exceeds the zeroing threshold 1e4 * max(median |R|, 1e-9 mean|U|,
1e-300) (core/fr_operators/troubled_cell.py:346-408).  This restates that
decision in numpy and checks, on many random and adversarial columns (ties,
zeros, wide ranges, infinities), that a skipped column never has an element the
reference's rule would zero."""
import numpy as np
import pytest


def skip_decision(R, Umean):
    """The kernel's test for one column R (length S) with mean |U| Umean."""
    S = len(R)
    need = S - (S // 2 if S & 1 else S // 2 - 1)
    x = np.abs(R)
    if np.isnan(x).any():
        return False
    lo, hi = x.min(), x.max()
    fl = 1e-9 * Umean
    if hi <= 1e4 * max(max(lo, fl), 1e-300):
        return True
    p = hi * 1e-4
    for _ in range(4):
        if 1e4 * p >= hi:
            break
        p = np.nextafter(p, np.inf)
    if 1e4 * p < hi:
        return False
    return int(np.sum(x >= p)) >= need


def zeroes_something(R, Umean):
    med = np.median(np.abs(R))
    ref = max(max(med, 1e-9 * Umean), 1e-300)
    return bool(np.any(np.abs(R) > 1e4 * ref))


@pytest.mark.parametrize("S", [8, 27, 64])
def test_skipped_columns_have_nothing_to_zero(S):
    rng = np.random.default_rng(S)
    n_skip = 0
    for trial in range(4000):
        kind = trial % 5
        if kind == 0:
            R = rng.standard_normal(S) * 10.0 ** rng.uniform(-12, 12)
        elif kind == 1:  # a few large entries over a small background
            R = rng.standard_normal(S) * 1e-3
            R[rng.integers(0, S, rng.integers(1, S // 2 + 2))] *= 10.0 ** rng.uniform(2, 9)
        elif kind == 2:  # ties and exact zeros
            R = rng.choice([0.0, 1.0, -1.0, 1e-5, 1e5], size=S)
        elif kind == 3:  # log-uniform magnitudes over many decades
            R = np.sign(rng.standard_normal(S)) * 10.0 ** rng.uniform(-20, 20, S)
        else:  # near the threshold: half the column at 1, the rest near 1e4 * 1
            R = np.ones(S)
            R[: S // 2] = 1e4 * (1 + rng.uniform(-1e-12, 1e-12, S // 2))
            rng.shuffle(R)
        Umean = float(10.0 ** rng.uniform(-3, 6))
        if skip_decision(R, Umean):
            n_skip += 1
            assert not zeroes_something(R, Umean), (S, trial, R)
    assert n_skip > 1000  # the rule does skip most ordinary columns


def test_columns_with_infinities_follow_the_rule():
    R = np.array([np.inf] * 14 + [1.0] * 13)
    assert skip_decision(R, 1.0) and not zeroes_something(R, 1.0)
    R = np.array([np.inf] * 2 + [1.0] * 25)
    assert not skip_decision(R, 1.0) and zeroes_something(R, 1.0)
