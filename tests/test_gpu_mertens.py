"""GPU: M(X) and the C/S1/S2 checksums vs the reference and the oracle.

* known answers 1 .. 10^17 (test_dr.cpp:26-47, test_cuda.cu:38-60, README.md:188),
* the reference's own C/S1/S2 checksums at its default parameters, dense and
  streamed, up to 10^16 (tests/golden/checksums.json from oracle/_ref),
* random X with randomised parameters against the oracle (any valid
  parameters give the same M(X); the checksums must match at equal ones),
* boundary inputs: tiny X, X = u, X = u + 1, the dense/compressed quotient
  boundary X = 99,975,680 (test_sieve.cpp:206-209),
* M(10^18) under three parameter sets, M(2^63 - 1) under two.
"""
import math
import random

import pytest

import dr_b200
from conftest import load_golden

pytestmark = pytest.mark.gpu


def _p(c):
    return dr_b200.Params(u_total=c["u_total"], u_dense=c["u_dense"], cx=c["cx"], mu_limit=c["mu_limit"])


def test_known_answers(engine):
    for c in load_golden("kat.json")["cases"]:
        assert engine.compute_mertens(c["X"]) == c["M"], c


def test_known_answers_compressed_policy(engine):
    for c in load_golden("kat.json")["cases"]:
        if c["X"] >= 10**5:
            assert engine.compute_compressed(c["X"]) == c["M"], c


def test_reference_checksums(engine):
    for c in load_golden("checksums.json")["cases"]:
        r = engine.mertens(c["X"], _p(c))
        s = r.stats
        assert (r.M, s.C, s.S1, s.S2, s.terms) == (c["M"], c["C"], c["S1"], c["S2"], c["terms"]), c


def test_random_params_vs_oracle(engine, oracle):
    rng = random.Random(20261203)
    for _ in range(40):
        X = int(10 ** rng.uniform(6, 11.5))
        p = dr_b200.default_params(X, dr_b200.POLICY_COMPRESSED)
        cx = rng.uniform(0.3, 3.0)
        A = int(cx * X**0.5)
        u = max(p.u_total, A + 2000, int(X**0.5) * 3)
        u = rng.randint(max(A + 2, 3 * int(X**0.5)), max(A + 2, 3 * int(X**0.5)) * 4)
        ud = rng.randint(0, u)
        ml = rng.randint(min(u, max(A, X // u) + 1), u)
        q = dr_b200.Params(u_total=u, u_dense=ud, cx=cx, mu_limit=ml, segment_log2=rng.choice([12, 14, 16, 17]))
        r = engine.mertens(X, q)
        o = oracle.run(X, u, ud, cx, ml)
        assert (r.M, r.stats.C, r.stats.S1, r.stats.S2) == (o["M"], o["C"], o["S1"], o["S2"]), (X, q)


def test_random_params_large_x(engine):
    """Any valid parameters give the same M(X): M(10^15) under seeded random splits over
    the whole valid range -- cx 0.4 .. 3, u from its lower limit up to 2e10, the dense tier
    anywhere from 0 to all of u (beyond 2^32 values where u allows), mu_limit anywhere
    between its lower limit and u, segments 2^15 .. 2^18 -- each with C - S1 - S2 = M."""
    X, want = 10**15, -3216373
    rng = random.Random(20261204)
    done = 0
    while done < 16:
        cx = rng.uniform(0.4, 3.0)
        A = int(cx * math.isqrt(X))
        lo = max(A + 2, 3 * math.isqrt(X))
        u = int(math.exp(rng.uniform(math.log(lo), math.log(2e10))))
        ud = rng.choice([0, u, rng.randint(0, u), min(u, 5000000000)])
        ml = rng.randint(min(u, max(A, X // u) + 1), u)
        p = dr_b200.Params(u_total=u, u_dense=ud, cx=cx, mu_limit=ml, segment_log2=rng.choice([15, 16, 17, 18]))
        if dr_b200.check_params(X, p) != 0 or dr_b200.query_bytes(X, p) > (48 << 30):
            continue
        r = engine.mertens(X, p)
        assert r.M == want, p
        assert (r.stats.C - r.stats.S1 - r.stats.S2) % (1 << 64) == want % (1 << 64), p
        done += 1


def test_small_and_boundary_inputs(engine, oracle):
    for X in list(range(0, 200)) + [1000, 10**5, 10**5 + 1, 5 * 10**7, 5 * 10**7 + 1, 99975680]:
        want = oracle.mertens(X) if X > 0 else 0
        assert engine.compute_mertens(X) == want, X
        if X > 100000:
            assert engine.compute_compressed(X) == want, X
    # X at and just above the table limit
    for X in (10**9, 10**10):
        p = dr_b200.default_params(X, dr_b200.POLICY_COMPRESSED)
        for u in (p.u_total, X - 1, X, X + 1):
            u = min(u, X + 1)
            q = dr_b200.Params(u_total=u, u_dense=min(u, p.u_dense), cx=p.cx, mu_limit=min(u, p.mu_limit))
            if dr_b200.check_params(X, q) != 0:
                continue
            assert engine.mertens(X, q).M == oracle.mertens(X)


def test_dense_config_1e12(engine):
    # config: plain dense M(10^12), MERTENS_USE_CHMT=0 parameters
    p = dr_b200.default_params(10**12, dr_b200.POLICY_DENSE)
    assert p.u_total == p.u_dense == 14381928
    r = engine.mertens(10**12, p)
    assert r.M == 62366


def test_bad_params_raise(engine):
    p = dr_b200.default_params(10**12)
    bad = dr_b200.Params(**{**p.as_dict(), "mu_limit": 5})
    with pytest.raises(dr_b200.DRError) as ei:
        engine.mertens(10**12, bad)
    assert ei.value.code == dr_b200.DR_ERR_PARAMS
    # the context stays usable after a rejected call
    assert engine.compute_mertens(10**9) == -222


def test_gpu_policy_known_answers(engine):
    # the B200 policy (larger u, cx = 1.3) gives the same exact values
    for c in load_golden("kat.json")["cases"]:
        p = dr_b200.default_params(c["X"], dr_b200.POLICY_GPU)
        assert dr_b200.check_params(c["X"], p) == 0
        assert engine.mertens(c["X"], p).M == c["M"], c


def _m1e18(engine, p):
    # pinned only by the reference engine's own run (tests/golden/m1e18.json)
    g = load_golden("m1e18.json")
    assert dr_b200.check_params(g["X"], p) == 0
    r = engine.mertens(g["X"], p)
    assert r.M == g["M"], p
    assert (r.stats.C - r.stats.S1 - r.stats.S2) % (1 << 64) == g["M"] % (1 << 64)
    return r


def test_m1e18(engine):
    # the B200 policy: u = 2.5e11 values, 94 GB of device data
    _m1e18(engine, dr_b200.default_params(10**18, dr_b200.POLICY_GPU))


def test_m1e18_reference_default_params(engine):
    """M(10^18) with the reference's own default parameters (compute_compressed,
    mertens_dr.hpp:1442-1461): u = 8e9 (its cap), u_dense = 1,350,001,152, cx = 1.35."""
    p = dr_b200.default_params(10**18, dr_b200.POLICY_REFERENCE)
    assert (p.u_total, p.u_dense, p.cx) == (8000000000, 1350001152, 1.35)
    r = _m1e18(engine, p)
    assert r.stats.terms > 0


def test_m1e18_learned_tuner_params(engine):
    """M(10^18) with the learned tuner's proposal (the committed weights; X = 10^18
    lies beyond the training domain, so the proposal is carried along the X^(2/3)
    law from its edge) -- no fallback to the reference heuristic."""
    import json
    import os

    import numpy as np

    path = os.path.join(os.path.dirname(dr_b200.__file__), "tuner_weights.json")
    with open(path) as f:
        w = np.array(json.load(f)["weights"], dtype=np.float32)
    mlp = dr_b200.MLP(engine)
    try:
        mlp.set_weights(w)
        _, hbm = dr_b200.device_info(0)
        p, fb = mlp.propose(10**18, int(hbm * 0.9), 148, 1)
    finally:
        mlp.close()
    assert not fb
    _m1e18(engine, p)


def test_int64_max_two_parameter_sets(engine):
    """M(2^63 - 1), the largest X of the int64 interface, under two parameter sets
    (u = 2.5e11, cx = 1.25, 120 GB of device data; u = 2e11, cx = 1.5): the splits
    give different C, S1 and S2 (different tables, split points and term lists) and
    must give the same M, each with C - S1 - S2 = M (mod 2^64).  No independently
    computed M is known at this X (the reference's CPU engine would take days); the
    pinned 580197744 is this engine's value, agreed by both splits."""
    X = (1 << 63) - 1
    got = []
    for cx, u in ((1.25, 250000000000), (1.5, 200000000000)):
        p = dr_b200.default_params(X, dr_b200.POLICY_GPU)
        p.cx, p.u_total = cx, u
        p.mu_limit = int(cx * math.isqrt(X)) + 2000
        assert dr_b200.check_params(X, p) == 0
        r = engine.mertens(X, p)
        assert (r.stats.C - r.stats.S1 - r.stats.S2) % (1 << 64) == r.M % (1 << 64)
        got.append((r.M, r.stats.C, r.stats.S1, r.stats.S2))
    assert got[0][0] == got[1][0] == 580197744
    assert got[0][1:] != got[1][1:]


def test_dense_tier_above_2_32(engine):
    """A dense int16 tier beyond 2^32 values (up to the int16 prefix's 7.6e9): S1 lookups
    with quotients in (2^32, u_dense] read the dense tier through the 64-bit route.  How
    the table is split into tiers changes no sum, so C, S1 and S2 equal those of the
    B200 policy's 4e9-value dense tier."""
    X = 10**17
    p = dr_b200.default_params(X, dr_b200.POLICY_GPU)
    assert p.u_dense <= (1 << 32) < 5000000000 < p.u_total
    q = dr_b200.Params(**{**p.as_dict(), "u_dense": 5000000000})
    r0, r1 = engine.mertens(X, p), engine.mertens(X, q)
    assert r0.M == r1.M == -21830254
    assert (r0.stats.C, r0.stats.S1, r0.stats.S2) == (r1.stats.C, r1.stats.S1, r1.stats.S2)


def test_windowed_s1_matches_direct(engine):
    """The windowed S1 (s1win_kernel) and the sums kernel's direct S1 split every S1
    lookup between them; with the window switched off the sums kernel takes them
    all.  Both give the same M(X), the same C/S1/S2 checksums and the same S1 op
    count, for every window length and for inputs that reach window 0."""
    cases = [(10**9 + 7, 12), (2 * 10**10 + 1, 13), (10**11, 14), (3 * 10**12, 15), (10**14, 16), (10**15, 15),
             (10**16, 15)]
    for X, wl in cases:
        p = dr_b200.default_params(X, dr_b200.POLICY_GPU)
        on = dr_b200.Params(**{**p.as_dict(), "s1_window_log2": wl})
        off = dr_b200.Params(**{**p.as_dict(), "s1_window_log2": -1})
        r1, r0 = engine.mertens(X, on), engine.mertens(X, off)
        got = (r1.M, r1.stats.C, r1.stats.S1, r1.stats.S2, r1.stats.s1_ops, r1.stats.s2_ops)
        want = (r0.M, r0.stats.C, r0.stats.S1, r0.stats.S2, r0.stats.s1_ops, r0.stats.s2_ops)
        assert got == want, (X, wl)
    # a dense tier smaller than two windows switches the windowed S1 off by itself
    X = 10**12
    p = dr_b200.default_params(X, dr_b200.POLICY_GPU)
    small = dr_b200.Params(**{**p.as_dict(), "u_dense": 40000, "s1_window_log2": 15})
    assert engine.mertens(X, small).M == 62366


def test_compressed_lookup_counter(engine):
    """s1_comp_ops counts the S1 lookups whose quotient lies above the dense tier:
    none with an all-dense table, all of them with no dense tier, in between
    otherwise, and M(X) is the same in all three."""
    X = 10**12
    p = dr_b200.default_params(X, dr_b200.POLICY_COMPRESSED)
    dense = dr_b200.Params(**{**p.as_dict(), "u_dense": p.u_total})
    none = dr_b200.Params(**{**p.as_dict(), "u_dense": 0})
    r_all, r_none, r_mid = engine.mertens(X, dense), engine.mertens(X, none), engine.mertens(X, p)
    assert r_all.M == r_none.M == r_mid.M == 62366
    assert r_all.stats.s1_comp_ops == 0
    assert r_none.stats.s1_comp_ops == r_none.stats.s1_ops > 0
    assert 0 < r_mid.stats.s1_comp_ops < r_mid.stats.s1_ops
    assert r_all.stats.s1_ops == r_none.stats.s1_ops == r_mid.stats.s1_ops
