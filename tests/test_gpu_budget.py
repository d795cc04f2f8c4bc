"""GPU: a context's device buffers only grow, so after calls of other shapes it can hold
more than the next call leaves room for under its budget.  Such a call releases the
buffers kept from earlier calls (each call rebuilds its table) and runs once more."""
import pytest

import dr_b200

pytestmark = pytest.mark.gpu

M_1E15 = -3216373  # test_dr.cpp:26-47


def test_budget_retry_releases_earlier_buffers(engine):
    X = 10**15
    a = dr_b200.default_params(X, dr_b200.POLICY_GPU)  # mostly compressed tier
    b = dr_b200.Params(u_total=1500000000, u_dense=1500000000, cx=a.cx, mu_limit=a.mu_limit)  # all dense
    assert dr_b200.check_params(X, b) == 0
    na, nb = dr_b200.query_bytes(X, a), dr_b200.query_bytes(X, b)
    budget = int(max(na, nb) * 1.1)
    assert na + nb > budget  # alternating the two cannot keep both sets of buffers
    try:
        engine.set_hbm_budget(budget)
        for p in (a, b, a, b):
            r = engine.mertens(X, p)
            assert r.M == M_1E15, p
            assert (r.stats.C - r.stats.S1 - r.stats.S2) % (1 << 64) == M_1E15 % (1 << 64)
    finally:
        engine.set_hbm_budget(0)
    # a call that does not fit the budget even alone still fails cleanly (the budget
    # caps growth: a, after b, must grow the compressed tier's buffers)
    try:
        engine.set_hbm_budget(min(na, nb) // 4)
        with pytest.raises(dr_b200.DRError) as ei:
            engine.mertens(X, a)
        assert ei.value.code == dr_b200.DR_ERR_NOMEM
    finally:
        engine.set_hbm_budget(0)
    assert engine.mertens(X, a).M == M_1E15
