"""GPU: the streamed table (dr_ctx_set_resident_limit) against the whole table.

With a resident limit, a single query keeps M only up to u_res in device memory; the
compressed tier above is sieved band by band and, after each band, the S1 lookups whose
quotient falls in it are summed (the idea of mertens_dr_windowed.hpp:218-374, which
streams M windows over [1, u] instead of storing them).  Every lookup is the same term of
the same sum, so M(X), the C/S1/S2 checksums and the op counts equal those of the whole
table at the same parameters -- for every resident limit, band length and segment length,
including bands of one segment, a last band that ends inside a segment, and bands sieved
in odd mode (their halves n/2 in the resident table: 3e9 resident of M(10^15)'s 5.4e9)
beside bands sieved in full mode.
"""
import pytest

import dr_b200

pytestmark = pytest.mark.gpu


@pytest.fixture
def streaming(engine):
    yield engine
    engine.set_resident_limit(0)


def _run(e, X, p, u_resident=0, band=0):
    e.set_resident_limit(u_resident, band)
    r = e.mertens(X, p)
    s = r.stats
    return (r.M, s.C, s.S1, s.S2, s.s1_ops, s.s2_ops, s.terms, s.s1_comp_ops)


def test_streamed_matches_whole_table(streaming):
    # (X, policy, segment_log2, [(u_resident, band_values), ...], known M or None)
    cases = [
        (10**12, dr_b200.POLICY_COMPRESSED, 14, [(20000000, 1 << 16), (30000000, 0), (14000000, 5000000)], 62366),
        (10**13 + 7, dr_b200.POLICY_COMPRESSED, 16, [(10**8, 3 * 10**7), (5 * 10**7, 1)], None),
        (10**15, dr_b200.POLICY_COMPRESSED, 18, [(10**9, 1 << 30), (6 * 10**8, 2 * 10**9), (3 * 10**9, 10**9)],
         -3216373),
        (10**15, dr_b200.POLICY_GPU, 17, [(2 * 10**9, 10**9)], -3216373),
    ]
    for X, policy, lg, splits, known in cases:
        p = dr_b200.default_params(X, policy)
        p.segment_log2 = lg
        assert p.u_total - p.u_dense > 4 << lg, (X, p)  # a compressed tier to stream
        whole = _run(streaming, X, p)
        if known is not None:
            assert whole[0] == known
        for ures, band in splits:
            assert ures < p.u_total
            assert _run(streaming, X, p, ures, band) == whole, (X, lg, ures, band)


def test_streamed_m1e16(streaming):
    """M(10^16) under the B200 policy (u = 2.27e10) with 6e9 values resident and bands
    of 5e9: the reference's known answer and the whole table's checksums."""
    X = 10**16
    p = dr_b200.default_params(X, dr_b200.POLICY_GPU)
    whole = _run(streaming, X, p)
    got = _run(streaming, X, p, 6 * 10**9, 5 * 10**9)
    assert whole[0] == got[0] == -3195437
    assert got == whole


def test_streamed_needs_x_above_table(streaming):
    """A streamed table answers no X <= u_total (the whole table would): refused."""
    X = 10**9
    p = dr_b200.default_params(X, dr_b200.POLICY_COMPRESSED)
    q = dr_b200.Params(u_total=X + 1000, u_dense=10**6, cx=p.cx, mu_limit=p.mu_limit)
    streaming.set_resident_limit(10**6 + (1 << 20))
    with pytest.raises(dr_b200.DRError):
        streaming.mertens(X, q)
    # without the limit nothing streams and the same call is answered from the table
    streaming.set_resident_limit(0)
    assert streaming.mertens(X, q).M == -222
