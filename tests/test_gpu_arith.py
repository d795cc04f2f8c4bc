"""GPU: the device's exact quotient and S2 summands.

Every S1 lookup and S2 term of the engine goes through these two routines, so
they are checked exhaustively on edge classes: y near 2^53 (where the
reference switches from double to integer division, mertens_dr.hpp:80-86),
2^63 - 1, 10^18, divisors near sqrt(y), y/u, 2^31, 2^32 and above.
"""
import random

import pytest

import dr_b200

pytestmark = pytest.mark.gpu


def _edge_pairs():
    ys = [0, 1, 2, 3, 11, 12, 13, 2**31 - 1, 2**31, 2**32 - 1, 2**32, 2**32 + 1, 2**40 + 7,
          2**53 - 1, 2**53, 2**53 + 1, 2**53 + 2, 10**16, 10**16 + 1, 10**17, 10**18 - 1, 10**18, 10**18 + 1,
          2**62, 2**63 - 1, 2**63, 2**64 - 1]
    pairs = []
    for y in ys:
        r = int(y**0.5)
        ds = [1, 2, 3, 5, 6, 7, 12, 97, 65535, 65536, 2**31 - 1, 2**31, 2**32 - 1, 2**32, 2**32 + 1, 2**40 + 3,
              max(1, r - 1), max(1, r), r + 1, max(1, y // 8000000000), y // 8000000000 + 1,
              max(1, y // 400000000000), max(1, y) if y else 1]
        for d in ds:
            if d >= 1:
                pairs.append((y, d))
    return pairs


def test_udiv_edges(engine):
    pairs = _edge_pairs()
    ys, ds = zip(*pairs)
    q = engine.debug_udiv(ys, ds)
    for (y, d), got in zip(pairs, q):
        assert got == y // d, (y, d, got)


def test_udiv_random(engine):
    rng = random.Random(20261203)
    ys, ds = [], []
    for _ in range(200000):
        bits = rng.choice([20, 32, 40, 53, 54, 60, 63, 64])
        y = rng.getrandbits(bits)
        dbits = rng.choice([1, 8, 16, 24, 31, 32, 33, 40])
        d = max(1, rng.getrandbits(dbits))
        ys.append(y)
        ds.append(d)
    q = engine.debug_udiv(ys, ds)
    bad = [(y, d, g) for y, d, g in zip(ys, ds, q) if g != y // d]
    assert not bad, bad[:5]


def test_udiv_s1_shapes(engine):
    # consecutive n near sqrt(y)/cx and near y/u for y = X/k at X = 10^16, 10^18
    ys, ds = [], []
    for X in (10**16, 10**18, 2**63 - 1):
        for k in (1, 5, 7, 11, 1001, 99991):
            y = X // k
            r = int((y / 1.35) ** 0.5)
            for n in list(range(r - 300, r + 300)) + list(range(y // 8000000000 + 1, y // 8000000000 + 300)):
                if n >= 1:
                    ys.append(y)
                    ds.append(n)
    q = engine.debug_udiv(ys, ds)
    assert all(g == y // d for y, d, g in zip(ys, ds, q))


def _rcp_domain_pairs():
    """(y, d) with d < 2^32 and y/d < 2^50: random, and y = q*d + {-1, 0, 1, d-1}
    for q and d at the edges of the domain, where the double estimate of y/d is
    least accurate relative to the integer boundaries."""
    rng = random.Random(20261204)
    pairs = []
    for _ in range(150000):
        d = max(1, rng.getrandbits(rng.choice([1, 6, 12, 20, 26, 30, 31, 32])))
        q = rng.getrandbits(rng.choice([1, 10, 20, 33, 40, 45, 48, 49, 50]))
        y = q * d + rng.randrange(d)
        if y < 2**64 and (y >> 50) < d:
            pairs.append((y, d))
    for d in (1, 2, 3, 5, 6, 7, 2**20 - 1, 2**31 - 1, 2**31, 2**32 - 5, 2**32 - 1, 3037000493, 4000000000):
        for q in (1, 2, 2**40 + 1, 2**49 - 1, 2**49, 2**50 - 2, 2**50 - 1, 10**15, 10**12 + 39):
            for r in (-1, 0, 1, d - 1):
                y = q * d + r
                if 0 <= y < 2**64 and (y >> 50) < d:
                    pairs.append((y, d))
    return pairs


def test_udiv_rcp_matches_floor(engine):
    pairs = _rcp_domain_pairs()
    ys, ds = zip(*pairs)
    q = engine.debug_udiv(ys, ds, rcp=True)
    bad = [(y, d, g) for (y, d), g in zip(pairs, q) if g != y // d]
    assert not bad, bad[:5]


def test_udiv_rcp_domain_flag(engine):
    ys = [2**63, 2**62, 5, 2**50 * 7]
    ds = [3, 2**32, 0, 7]
    assert engine.debug_udiv(ys, ds, rcp=True) == [2**64 - 1] * 4


def test_pieces_match_oracle(engine, oracle):
    rng = random.Random(5)
    qs = list(range(0, 300)) + [rng.getrandbits(b) for b in (20, 40, 53, 60, 62) for _ in range(200)]
    qs += [2**53 - 1, 2**53, 2**53 + 1, 10**18, 2**63 - 1]
    pieces, vals = [], []
    for p in range(1, 13):
        for q in qs:
            pieces.append(p)
            vals.append(q)
    got = engine.debug_piece(pieces, vals)
    for p, q, g in zip(pieces, vals, got):
        assert g == oracle.piece(p, q), (p, q, g)


def _fast_domain_pairs():
    """(y, d) with d <= y, d < 2^31 and y/d < 2^31 (the 32-bit route of the fast
    S1/S2 paths): random, and y = q*d + {-1, 0, 1, d-1} at the domain's edges, where
    the remainder's low 32 bits and the estimate's rounding are tightest."""
    rng = random.Random(20261205)
    pairs = []
    for _ in range(150000):
        d = max(1, rng.getrandbits(rng.choice([1, 6, 12, 20, 26, 30, 31])))
        q = rng.getrandbits(rng.choice([1, 10, 20, 26, 29, 30, 31]))
        y = q * d + rng.randrange(d)
        if d <= y and (y >> 31) < d:
            pairs.append((y, d))
    for d in (1, 2, 3, 5, 6, 7, 12, 2**16 + 1, 2**20 - 1, 2**30 + 3, 2**31 - 2, 2**31 - 1):
        for q in (1, 2, 11, 12, 13, 2**20 + 1, 2**30, 2**31 - 2, 2**31 - 1):
            for r in (-1, 0, 1, d - 1):
                y = q * d + r
                if d <= y and (y >> 31) < d:
                    pairs.append((y, d))
    return pairs


def test_udiv32_matches_floor(engine):
    pairs = _fast_domain_pairs()
    ys, ds = zip(*pairs)
    q = engine.debug_udiv(ys, ds, rcp="32")
    bad = [(y, d, g) for (y, d), g in zip(pairs, q) if g != y // d]
    assert not bad, bad[:5]


def test_udiv32_domain_flag(engine):
    ys = [2**31 * 5, 7, 2**40, 3, 0, 4]
    ds = [5, 2**31, 3, 0, 1, 5]
    assert engine.debug_udiv(ys, ds, rcp="32") == [2**64 - 1] * 6


def test_pieces32_match_oracle(engine, oracle):
    rng = random.Random(6)
    qs = list(range(0, 300)) + [rng.getrandbits(b) for b in (12, 20, 28, 30, 31) for _ in range(300)]
    qs += [2**31 - 12, 2**31 - 2, 2**31 - 1]
    pieces, vals = [], []
    for p in range(1, 13):
        for q in qs:
            pieces.append(p)
            vals.append(q)
    got = engine.debug_piece(pieces, vals, fast=True)
    for p, q, g in zip(pieces, vals, got):
        assert g == oracle.piece(p, q), (p, q, g)
    assert engine.debug_piece([1, 8], [2**31, 2**40], fast=True) == [-(2**63)] * 2


def test_measure_peaks_plausible():
    # the ceilings bench.py divides by: positive, finite and in the range a B200's
    # units allow (148 SMs at up to ~2 GHz); the conflict-free atomic pattern is the
    # faster one
    pk = dr_b200.measure_peaks(0)
    assert 1e11 < pk["smem_atomic_per_s"] < 1e14, pk
    assert 1e10 < pk["smem_atomic_stride_per_s"] <= 1.1 * pk["smem_atomic_per_s"], pk
    assert 1e12 < pk["imad_per_s"] < 1e14, pk
    assert 1e11 < pk["dfma_per_s"] < 1e14, pk
