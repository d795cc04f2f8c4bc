"""GPU: Mobius / Mertens tables built on the device vs the oracle.

Sizes follow the reference's streamed-table test (test_sieve.cpp:79-96):
around 64/256-value words and chunks, the stencil period 13860, the odd
stencil 17325 and 128 Ki block edges, with arbitrary dense cutoffs.  Small
segments (4096 values) put many segment boundaries inside those patterns.
"""
import numpy as np
import pytest

import dr_b200
from conftest import load_golden

pytestmark = pytest.mark.gpu

TOTALS = [1, 2, 3, 63, 64, 65, 127, 128, 129, 255, 256, 257, 13859, 13860, 13861, 17324, 17325, 17326,
          131071, 131072, 131073, 262147, 1000033]
DENSES = [0, 1, 7, 63, 64, 65, 255, 256, 257, 1000, 131071]


def _check_table(engine, oracle, total, dense, mu_limit, seg_log2):
    tun = dr_b200.Params(segment_log2=seg_log2)
    engine.table_build(total, dense, mu_limit, tun)
    M, mu = engine.table_read(0, total + 1)
    Mo, muo, so = oracle.table(total, dense, mu_limit)
    assert np.array_equal(M, Mo), (total, dense, seg_log2, np.nonzero(M != Mo)[0][:5])
    assert np.array_equal(mu[: mu_limit + 1], muo), (total, dense)
    assert not mu[mu_limit + 1:].any()
    wm = engine.table_read_wheel(0, mu_limit + 1)
    n = np.arange(mu_limit + 1)
    cop = (n % 2 == 1) & (n % 3 != 0)
    assert np.array_equal(wm[cop], muo[cop]), (total, dense)
    assert not wm[~cop].any()
    assert engine.table_checksums() == tuple(so), (total, dense)


@pytest.mark.parametrize("total", TOTALS)
def test_tables_vs_oracle(engine, oracle, total):
    for dense in DENSES + [total]:
        if dense > total:
            continue
        for seg_log2 in (12, 17):
            _check_table(engine, oracle, total, dense, total, seg_log2)


def test_table_mu_limit_below_dense(engine, oracle):
    for total, dense, ml in [(1000033, 500000, 20000), (262147, 1024, 262147), (1000033, 0, 999)]:
        _check_table(engine, oracle, total, dense, ml, 13)


def test_tables_golden(engine):
    for c in load_golden("tables.json")["cases"]:
        for seg_log2 in (12, 16, 17):
            engine.table_build(c["u_total"], c["u_dense"], c["mu_limit"], dr_b200.Params(segment_log2=seg_log2))
            assert list(engine.table_checksums()) == c["sums"], (c, seg_log2)


def test_large_table_vs_oracle(engine, oracle):
    # ~2^28 values: thousands of segments, both tiers, many primes per segment
    total, dense = 300000007, 40000003
    engine.table_build(total, dense, 5000000)
    s = engine.table_checksums()
    _, _, so = oracle.table(total, dense, 5000000)
    assert s == tuple(so)
    M, _ = engine.table_read(total - 5000, 5001)
    Mo, _, _ = oracle.table(total, total, 10)
    assert np.array_equal(M, Mo[total - 5000:])


def test_block_shapes(engine, oracle):
    total, dense = 2000003, 300001
    _, _, so = oracle.table(total, dense, total)
    for block in (256, 512, 1024):
        for seg_log2 in (12, 14, 16, 17, 18):  # 2^18: full mode in two passes per segment
            engine.table_build(total, dense, total, dr_b200.Params(segment_log2=seg_log2, block_threads=block))
            assert engine.table_checksums() == tuple(so), (block, seg_log2)


def test_odd_mode_tables(engine, oracle):
    # Dense cutoffs on 64-value words: after the first wave of segments every segment
    # is sieved on its odd values and takes its even ones from their halves, in
    # launches whose halves lie in earlier launches (many launches at 4096 values).
    for total, dense in [(1000033, 0), (1000033, 64 * 5000), (2000003, 300032), (4000037, 3999936)]:
        for seg_log2 in (12, 13, 17, 18):
            _check_table(engine, oracle, total, dense, total, seg_log2)
        # a small mu limit: segments above it finalise inside the plane assembly
        for seg_log2 in (12, 18):
            _check_table(engine, oracle, total, dense, 999, seg_log2)
    _, _, so = oracle.table(2000003, 300032, 2000003)
    for block in (256, 512):
        for seg_log2 in (12, 18):  # at 2^18 and 256 threads the items exceed 32 per warp: read from memory
            engine.table_build(2000003, 300032, 2000003, dr_b200.Params(segment_log2=seg_log2, block_threads=block))
            assert engine.table_checksums() == tuple(so), (block, seg_log2)


def test_odd_mode_large_table(engine, oracle):
    total, dense = 300000007, 40000000
    _, _, so = oracle.table(total, dense, 5000000)
    for seg_log2 in (12, 17, 18):
        engine.table_build(total, dense, 5000000, dr_b200.Params(segment_log2=seg_log2))
        assert engine.table_checksums() == tuple(so), seg_log2
    M, _ = engine.table_read(total - 5000, 5001)
    Mo, _, _ = oracle.table(total, total, 10)
    assert np.array_equal(M, Mo[total - 5000:])
