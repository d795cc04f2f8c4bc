"""CPU: the sieve launches of a table build (host logic of the library, no GPU).

After the first wave of segments (full mode), odd-mode launches sieve the odd values
of their segments and take every even value 2m from the Mobius bits of m, written by
an earlier launch.  The plan must therefore cover the segments once, in order, and
every half floor(v/2) of a value v of an odd-mode launch must lie in a segment before
that launch's first one.  Odd mode needs the dense cutoff on a 64-value word.
"""
import random

import pytest

import dr_b200


def _segments(u_total, u_dense, S):
    dense = (u_dense + S - 1) // S
    return dense, dense + (u_total - u_dense + S - 1) // S


def _segment_of(v, dense, u_dense, S):
    return (v - 1) // S if v <= u_dense else dense + (v - 1 - u_dense) // S


def _end_of(seg, dense, u_dense, u_total, S):
    base = seg * S if seg < dense else u_dense + (seg - dense) * S
    return min(base + S, u_dense if seg < dense else u_total)


def _check(u_total, u_dense, lg, wave):
    S = 1 << lg
    plan = dr_b200.sieve_plan(u_total, u_dense, lg, wave)
    dense, nseg = _segments(u_total, u_dense, S)
    assert plan[0][0] == 0 and plan[-1][1] == nseg
    for (b0, b1, _), (c0, _, _) in zip(plan, plan[1:]):
        assert b1 == c0 and b0 < b1
    assert not plan[0][2]
    odd_ok = u_dense % 64 == 0 and nseg > min(nseg, wave)
    assert any(odd for _, _, odd in plan) == odd_ok
    for b0, b1, odd in plan:
        if odd:
            # the largest half of the launch's values lies below b0
            assert _segment_of(_end_of(b1 - 1, dense, u_dense, u_total, S) // 2, dense, u_dense, S) < b0
    return plan


def test_plan_cases():
    cases = [(1, 0, 12, 148), (4096, 0, 12, 1), (10**6, 64 * 5000, 12, 148), (2000003, 300032, 12, 296),
             (2000003, 300001, 12, 148), (300000007, 40000000, 18, 148), (17762693632, 1110168576, 18, 148),
             (250000000000, 4000000000, 18, 148), (262144, 262144, 12, 3), (10**7, 0, 13, 7)]
    for c in cases:
        _check(*c)
    # the M(10^16) table of the B200 policy: one full wave, then ranges that roughly double
    plan = _check(17762693632, 1110168576, 18, 148)
    assert len(plan) == 10
    sizes = [b1 - b0 for b0, b1, _ in plan[1:-1]]
    assert all(b >= a for a, b in zip(sizes, sizes[1:]))


def test_plan_random():
    rng = random.Random(20261204)
    for _ in range(300):
        lg = rng.choice([12, 13, 14, 17, 18])
        S = 1 << lg
        u_total = rng.randrange(1, 400 * S)
        u_dense = rng.choice([0, u_total, rng.randrange(0, u_total + 1), 64 * rng.randrange(0, u_total // 64 + 1)])
        _check(u_total, u_dense, lg, rng.choice([1, 2, 7, 148, 296]))


def test_plan_rejects_bad_arguments():
    with pytest.raises(dr_b200.DRError):
        dr_b200.sieve_plan(100, 200, 12, 1)
    with pytest.raises(dr_b200.DRError):
        dr_b200.sieve_plan(100, 0, 19, 1)
