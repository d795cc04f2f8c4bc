"""CPU: the C-ABI library loads, exports what include/*.h declares, and its host
logic (parameter policy, coverage check) matches the reference restatement.
No compute call needs a GPU here."""
import ctypes
import os
import re

import pytest

import dr_b200
from conftest import ROOT


def declared_symbols():
    names = set()
    inc = os.path.join(ROOT, "include")
    for fn in os.listdir(inc):
        if not fn.endswith(".h"):
            continue
        text = open(os.path.join(inc, fn)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names.update(re.findall(r"\b(dr_[a-z0-9_]+)\s*\(", text))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    L = dr_b200.lib()
    decl = declared_symbols()
    assert len(decl) >= 15
    for name in decl:
        assert hasattr(L, name), name
    assert set(decl) <= set(dr_b200.exported_symbols()) | set(decl)


def test_binding_covers_declared_symbols():
    assert set(declared_symbols()) == set(dr_b200.exported_symbols())


def test_library_is_sm100a_build():
    # the shared object must carry sm_100a device code (cuobjdump is not used:
    # the fatbin header names the architecture in the ELF note strings)
    data = open(dr_b200._LIB_PATH, "rb").read()
    assert b"sm_100a" in data or b"compute_100a" in data


POLICY_X = [1, 2, 3, 100, 10**5, 10**5 + 1, 5 * 10**7, 5 * 10**7 + 1, 10**9, 10**10, 10**11 - 1, 10**11,
            123456789012, 10**12, 10**13, 10**14, 10**15, 10**16, 3 * 10**16, 10**17, 10**18]


@pytest.mark.parametrize("env", [{}, {"MERTENS_CX": "1.2"}, {"MERTENS_USE_CHMT": "0"}, {"MERTENS_USE_CHMT": "1"},
                                 {"MERTENS_FX": "0.5"}, {"MERTENS_CHMT_U_CAP": "4000000000"},
                                 {"MERTENS_U_CAP": "200000000"}])
def test_reference_policy_matches_oracle(oracle, monkeypatch, env):
    for k in ("MERTENS_CX", "MERTENS_USE_CHMT", "MERTENS_FX", "MERTENS_CHMT_U_CAP", "MERTENS_U_CAP"):
        monkeypatch.delenv(k, raising=False)
    for k, v in env.items():
        monkeypatch.setenv(k, v)
    for X in POLICY_X:
        p = dr_b200.default_params(X, dr_b200.POLICY_REFERENCE)
        q = oracle.default_params(X, oracle.L.dro_use_compressed(X))
        assert (p.u_total, p.u_dense, p.cx, p.mu_limit) == (q.u_total, q.u_dense, q.cx, q.mu_limit), (X, env)
        pd = dr_b200.default_params(X, dr_b200.POLICY_DENSE)
        qd = oracle.default_params(X, False)
        assert (pd.u_total, pd.u_dense, pd.cx, pd.mu_limit) == (qd.u_total, qd.u_dense, qd.cx, qd.mu_limit)


def test_coverage_check_rejects_bad_params():
    X = 10**12
    p = dr_b200.default_params(X)
    assert dr_b200.check_params(X, p) == 0
    bad = dr_b200.Params(**{**p.as_dict(), "mu_limit": 10})  # A and N above mu_limit
    assert dr_b200.check_params(X, bad) == dr_b200.DR_ERR_PARAMS
    bad = dr_b200.Params(**{**p.as_dict(), "u_dense": p.u_total + 1})
    assert dr_b200.check_params(X, bad) == dr_b200.DR_ERR_PARAMS
    bad = dr_b200.Params(**{**p.as_dict(), "cx": 0.0})
    assert dr_b200.check_params(X, bad) == dr_b200.DR_ERR_PARAMS
    bad = dr_b200.Params(**{**p.as_dict(), "u_dense": 8 * 10**9, "u_total": 9 * 10**9})
    assert dr_b200.check_params(X, bad) == dr_b200.DR_ERR_PARAMS  # int16 prefix range
    # over budget
    assert dr_b200.check_params(X, p, budget=1000) == dr_b200.DR_ERR_NOMEM
    assert dr_b200.table_bytes(p.u_total, p.u_dense, p.mu_limit) > 2 * p.u_dense


def test_no_gpu_fails_loudly():
    # without a usable sm_100 device the engine raises instead of computing on the CPU
    try:
        import torch

        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    with pytest.raises(dr_b200.DRError):
        dr_b200.Engine(0)


@pytest.mark.parametrize("threads", [1, 2, 3, 16, 0])
def test_reference_gpu_policy_matches_reference_build(monkeypatch, threads):
    """dr_reference_gpu_params against choose_gpu_sieve_limit / cx / mu limit of the
    reference GPU engine compiled from its own header (oracle/_ref)."""
    from oracle_py import ReferenceGpuParams

    if not ReferenceGpuParams.available():
        pytest.skip("reference build absent")
    for k in ("MERTENS_CX", "OMP_NUM_THREADS"):
        monkeypatch.delenv(k, raising=False)
    ref = ReferenceGpuParams()
    # threads 0: the engine's default thread count, omp_get_max_threads() = the host's cores
    rt = threads if threads > 0 else (os.cpu_count() or 1)
    for X in [5 * 10**7 + 1, 10**8, 10**9, 10**10, 10**11, 10**12, 10**13, 10**14, 10**15 - 1, 10**15, 10**16 - 1,
              10**16, 10**17, 10**18]:
        p = dr_b200.reference_gpu_params(X, threads)
        u, cx, ml = ref.params(X, rt)
        assert (p.u_total, p.u_dense, p.cx, p.mu_limit) == (u, u, cx, ml), (X, threads)
        # where N = X/u exceeds the table (10^18 with u capped at 6e8 or 1.4e9) the
        # reference's term loop would read mu past its table; the coverage check refuses
        ok = X // u <= ml and int(cx * X ** 0.5) <= ml
        assert dr_b200.check_params(X, p) == (0 if ok else dr_b200.DR_ERR_PARAMS), (X, threads)
    # the policy constant uses the default thread count
    q = dr_b200.default_params(10**15, dr_b200.POLICY_REFERENCE_GPU)
    r = dr_b200.reference_gpu_params(10**15, 0)
    assert (q.u_total, q.cx, q.mu_limit) == (r.u_total, r.cx, r.mu_limit)
    # X <= 5e7: that engine hands X to the CPU engine's dense path
    small = dr_b200.reference_gpu_params(10**7, threads)
    dense = dr_b200.default_params(10**7, dr_b200.POLICY_DENSE)
    assert (small.u_total, small.cx, small.mu_limit) == (dense.u_total, dense.cx, dense.mu_limit)


def test_noalloc_rejects_sizes_beyond_its_scratch():
    """dr_table_build_noalloc checks its arguments before any CUDA call: u_total
    above DR_NOALLOC_MAX_U = 2^33 (the fixed scratch's limit) is DR_ERR_ARG."""
    import ctypes

    f = dr_b200.lib().dr_table_build_noalloc
    buf = ctypes.c_void_p(1 << 20)  # never dereferenced: the call fails first
    for ut, ud, ml in [((1 << 33) + 1, 0, 1000), (1 << 40, 1 << 20, 1000), (0, 0, 0), (100, 200, 10), (100, 10, 101)]:
        rc = f(0, None, ut, ud, ml, buf, buf, buf, buf)
        assert rc == dr_b200.DR_ERR_ARG, (ut, ud, ml, rc)
    assert b"2^33" in dr_b200.lib().dr_last_error() or b"u_" in dr_b200.lib().dr_last_error()
    rc = f(0, None, (1 << 33) + 1, 0, 1000, buf, buf, buf, buf)
    assert b"DR_NOALLOC_MAX_U" in dr_b200.lib().dr_last_error()
    rc = f(-1, None, 1000, 0, 10, buf, buf, buf, buf)
    assert rc == dr_b200.DR_ERR_ARG
