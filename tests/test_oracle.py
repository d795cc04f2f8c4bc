"""CPU: pin the oracle (oracle/dr_oracle.c) before trusting it.

* against the reference's published known answers (tests/golden/kat.json),
* against the reference engine compiled from its own sources (oracle/_ref),
  when that build is present: M(X), C/S1/S2 checksums, tables, S2 intervals,
  byte finalisation and parameter heuristics,
* against the golden fixtures produced by that build.
Follows the reference's own test strategy (test_dr.cpp, test_sieve.cpp).
"""
import numpy as np
import pytest

from conftest import load_golden

M64 = (1 << 64) - 1


def test_oracle_kat(oracle):
    for c in load_golden("kat.json")["cases"]:
        if c["X"] <= 10**13:
            assert oracle.mertens(c["X"]) == c["M"], c


def test_oracle_direct_small(oracle):
    # independent Eratosthenes prefix vs the DR path at small X (test_sieve.cpp:12-42)
    for X in [1, 2, 3, 4, 5, 7, 31, 256, 257, 262145, 1000033, 4000037]:
        assert oracle.mertens_direct(X) == oracle.mertens(X)


def test_oracle_table_vs_direct(oracle):
    # get_M / get_mu of the streamed table vs a direct sieve (test_sieve.cpp:79-96)
    n = 300000
    direct = np.zeros(n + 1, dtype=np.int64)
    mu = np.ones(n + 1, dtype=np.int64)
    mu[0] = 0
    comp = np.zeros(n + 1, dtype=bool)
    for p in range(2, n + 1):
        if comp[p]:
            continue
        comp[p::p] = True
        mu[p::p] *= -1
        if p * p <= n:
            mu[p * p::p * p] = 0
    direct = np.cumsum(mu)
    for total, dense in [(n, 0), (n, 7), (n, 64), (n, 13861), (n, n), (17325, 17324), (131073, 131072)]:
        M, mut, _ = oracle.table(total, dense, total)
        assert np.array_equal(M, direct[: total + 1]), (total, dense)
        assert np.array_equal(mut.astype(np.int64), mu[: total + 1]), (total, dense)


def test_oracle_checksums_golden(oracle):
    for c in load_golden("checksums.json")["cases"]:
        if c["X"] > 10**13:
            continue
        r = oracle.run(c["X"], c["u_total"], c["u_dense"], c["cx"], c["mu_limit"])
        assert (r["M"], r["C"], r["S1"], r["S2"]) == (c["M"], c["C"], c["S1"], c["S2"]), c


def test_oracle_tables_golden(oracle):
    for c in load_golden("tables.json")["cases"]:
        if c["u_total"] > 5 * 10**7:
            continue
        _, _, sums = oracle.table(c["u_total"], c["u_dense"], c["mu_limit"])
        assert list(sums) == c["sums"], c


def test_oracle_params_match_reference(oracle, reference):
    for X in [10**5, 5 * 10**7, 5 * 10**7 + 1, 10**9, 123456789012, 10**13, 10**15, 10**16, 3 * 10**16,
              10**17, 10**18, 2**62]:
        assert oracle.L.dro_choose_cx(X) == reference.L.ref_choose_cx(X)
        assert oracle.L.dro_choose_sieve_limit(X) == reference.L.ref_choose_sieve_limit(X)
        assert oracle.L.dro_choose_compressed_limit(X) == reference.L.ref_choose_compressed_limit(X)
    for n in [0, 1, 2, 3, 4, 15, 16, 17, 2**53, 10**16, 3037000499**2 - 1, 3037000499**2, 2**63 - 1]:
        assert oracle.L.dro_isqrt(n) == reference.L.ref_isqrt(n)


def test_oracle_vs_reference_mertens(oracle, reference):
    for X in [54321, 987654, 12345678, 99975680, 987654321, 5 * 10**9, 123456789012]:
        assert oracle.mertens(X) == reference.compute_mertens(X)


def test_oracle_vs_reference_checksums(oracle, reference):
    # identical parameters on both sides, including non-default ones
    rng = np.random.default_rng(7)
    for _ in range(6):
        X = int(10 ** rng.uniform(8, 12))
        p = oracle.default_params(X, True)
        cx = float(rng.uniform(0.5, 2.0))
        A = int(cx * X**0.5) + 1000  # endpoints must lie in the dense tier and the mu table
        ud = int(rng.integers(min(A, p.u_total), p.u_total + 1))
        ml = min(p.u_total, max(A, X // p.u_total + 1000))
        a = oracle.run(X, p.u_total, ud, cx, ml)
        b = reference.checksums(X, p.u_total, ud, cx, ml)
        assert (a["M"], a["C"], a["S1"], a["S2"]) == (b["M"], b["C"], b["S1"], b["S2"]), (X, cx, ud)


def test_oracle_tables_vs_reference(oracle, reference):
    for total, dense in [(0, 0), (1, 0), (3, 1), (65, 63), (257, 255), (13861, 1000), (17326, 17325),
                         (262147, 131071), (1000033, 1024)]:
        Mr, mur, sr, _ = reference.table(total, dense, total)
        Mo, muo, so = oracle.table(total, dense, total)
        assert np.array_equal(Mr, Mo), (total, dense)
        assert np.array_equal(mur[: len(muo)], muo), (total, dense)
        assert tuple(sr) == tuple(so), (total, dense)


def test_oracle_s2_pieces_vs_reference(oracle, reference):
    # every piece at y around 2^53 and above, against the reference's run_s2_fast
    # over the same mu (test_sieve.cpp:98-116)
    _, mu, _ = oracle.table(1 << 20, 1 << 20, 1 << 20)
    mu = np.ascontiguousarray(mu, dtype=np.int8)
    import ctypes

    mp = mu.ctypes.data_as(ctypes.POINTER(ctypes.c_int8))
    for y in [37, 65535, 999999937, 2**53 - 1, 2**53, 2**53 + 1, 10**16, 10**17, 10**18 - 1]:
        for first in [1, 2, 5, 6, 7, 11, 12, 13, 97, 99991]:
            for count in [0, 1, 2, 5, 6, 7, 23, 24, 25, 57]:
                last = first + count - 1
                for piece in range(1, 13):
                    a = oracle.s2_interval(piece, first, last, y, mu)
                    b = reference.L.ref_s2_interval(piece, first, last, y, mp)
                    assert a == b, (y, first, count, piece)
    for piece in range(1, 13):
        for q in list(range(0, 200)) + [2**53 + 5, 10**18 + 7, 2**62 + 11]:
            assert oracle.piece(piece, q) == reference.L.ref_piece(piece, q)


def test_oracle_finalize_vs_reference(oracle, reference):
    import ctypes

    for first in [3, 31, 32, 33, 127, 128, 129, (1 << 31) - 31, (1 << 31) + 1, (1 << 33) + 1]:
        vals = np.array([(i * 37 + 11) & 0xFF for i in range(64)], dtype=np.uint8)
        ref = vals.copy()
        reference.L.ref_finalize_bytes(ref.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)), len(ref), first, 1)
        mine = np.array([oracle.L.dro_finalize_byte(int(v), first + i) & 0xFF for i, v in enumerate(vals)],
                        dtype=np.uint8)
        assert np.array_equal(ref, mine), first


# The reference's own cross-validation points (test_dr.cpp:74-76) and its known answers
CROSS = [54321, 987654, 12345678, 987654321, 5000000000, 123456789012, 1000000000000]
_DIRICHLET = {}


def _dirichlet(oracle, x):
    if x not in _DIRICHLET:
        _DIRICHLET[x] = oracle.mertens_dirichlet(x)
    return _DIRICHLET[x]


def test_independent_method_vs_known_answers(oracle):
    """The second method (sum_{d<=x} M(x/d) = 1, dirichlet_dp.c) reproduces the
    reference's published known answers and equals the direct sieve on small x."""
    for c in load_golden("kat.json")["cases"]:
        if c["X"] <= 10**12:
            assert _dirichlet(oracle, c["X"]) == c["M"], c
    for x in list(range(0, 300)) + [999, 1000, 1001, 65536, 99975680]:
        assert oracle.mertens_dirichlet(x) == oracle.mertens_direct(x), x


def test_independent_method_vs_deleglise_rivat(oracle):
    """Cross-validation as in test_dr.cpp:69-89: the Deleglise-Rivat restatement and
    the independent method agree at the reference's cross-check points."""
    for x in CROSS:
        assert oracle.mertens(x) == _dirichlet(oracle, x), x


def test_independent_method_vs_reference(reference, oracle):
    for x in CROSS:
        assert reference.compute_mertens(x) == _dirichlet(oracle, x), x
