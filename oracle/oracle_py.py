"""ctypes bindings of the oracle (TEST INFRASTRUCTURE ONLY).

``Oracle``     -- the plain-C restatement (oracle/dr_oracle.c), built on demand.
``Reference``  -- the reference engine compiled from its own sources into
                  oracle/_ref/libdr_ref.so (present only where the reference
                  source tree was available when building; optional).

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg use this.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "lib", "libdr_oracle.so")
REF_SO = os.path.join(HERE, "_ref", "libdr_ref.so")
REF_BENCH = os.path.join(HERE, "_ref", "bench_dr")

i64, u64, c_int, c_double = ctypes.c_int64, ctypes.c_uint64, ctypes.c_int, ctypes.c_double


class OParams(ctypes.Structure):
    _fields_ = [("X", i64), ("u_total", i64), ("u_dense", i64), ("cx", c_double), ("mu_limit", i64)]


class OResult(ctypes.Structure):
    _fields_ = [("M", i64), ("C", u64), ("S1", u64), ("S2", u64), ("terms", i64), ("evals", i64),
                ("s1_lookups", u64), ("s2_candidates", u64)]


class OTable(ctypes.Structure):
    _fields_ = [("u_total", i64), ("u_dense", i64), ("mu_limit", i64), ("num_words", i64),
                ("dense_M", ctypes.POINTER(ctypes.c_int16)), ("mu", ctypes.POINTER(ctypes.c_int8)),
                ("nz", ctypes.POINTER(u64)), ("neg", ctypes.POINTER(u64)), ("ckpt", ctypes.POINTER(ctypes.c_int32))]


class OTableSums(ctypes.Structure):
    _fields_ = [(n, u64) for n in ("dense_sum", "dense_wsum", "mu_wsum", "nz_wsum", "neg_wsum", "ckpt_wsum")]


def _build_oracle():
    if not os.path.exists(ORACLE_SO):
        subprocess.run(["make", "-C", HERE, "-s", "all"], check=True)


class Oracle:
    def __init__(self):
        _build_oracle()
        L = ctypes.CDLL(ORACLE_SO)
        sig = {
            "dro_isqrt": (i64, [i64]),
            "dro_choose_cx": (c_double, [i64]),
            "dro_choose_sieve_limit": (i64, [i64]),
            "dro_choose_compressed_limit": (i64, [i64]),
            "dro_use_compressed": (c_int, [i64]),
            "dro_default_params": (None, [i64, c_int, ctypes.POINTER(OParams)]),
            "dro_table_build": (c_int, [ctypes.POINTER(OTable), i64, i64, i64, c_int]),
            "dro_table_free": (None, [ctypes.POINTER(OTable)]),
            "dro_table_M": (ctypes.c_int32, [ctypes.POINTER(OTable), i64]),
            "dro_table_mu": (ctypes.c_int8, [ctypes.POINTER(OTable), i64]),
            "dro_table_checksums": (None, [ctypes.POINTER(OTable), ctypes.POINTER(OTableSums)]),
            "dro_piece": (i64, [c_int, u64]),
            "dro_s2_interval": (i64, [c_int, i64, i64, u64, ctypes.POINTER(ctypes.c_int8)]),
            "dro_finalize_byte": (ctypes.c_int8, [ctypes.c_uint8, u64]),
            "dro_mertens_params": (c_int, [ctypes.POINTER(OParams), c_int, ctypes.POINTER(OResult)]),
            "dro_mertens": (i64, [i64, c_int]),
            "dro_mertens_direct": (i64, [i64]),
            "dro_mertens_dirichlet": (i64, [i64]),
        }
        for n, (r, a) in sig.items():
            f = getattr(L, n)
            f.restype = r
            f.argtypes = a
        self.L = L

    def default_params(self, X: int, compressed: bool) -> OParams:
        p = OParams()
        self.L.dro_default_params(int(X), int(bool(compressed)), ctypes.byref(p))
        return p

    def mertens(self, X: int, threads: int = 0) -> int:
        return int(self.L.dro_mertens(int(X), int(threads)))

    def mertens_direct(self, X: int) -> int:
        return int(self.L.dro_mertens_direct(int(X)))

    def mertens_dirichlet(self, X: int) -> int:
        """The independent second method (dirichlet_dp.c), not Deleglise-Rivat."""
        return int(self.L.dro_mertens_dirichlet(int(X)))

    def run(self, X: int, u_total: int, u_dense: int, cx: float, mu_limit: int, threads: int = 0) -> dict:
        p = OParams(int(X), int(u_total), int(u_dense), float(cx), int(mu_limit))
        r = OResult()
        rc = self.L.dro_mertens_params(ctypes.byref(p), int(threads), ctypes.byref(r))
        if rc:
            raise RuntimeError(f"oracle failed rc={rc}")
        return {f: getattr(r, f) for f, _ in r._fields_}

    def table(self, u_total: int, u_dense: int, mu_limit: int, threads: int = 0):
        """(M[0..u_total], mu[0..mu_limit], sums tuple) from the oracle table."""
        t = OTable()
        rc = self.L.dro_table_build(ctypes.byref(t), int(u_total), int(u_dense), int(mu_limit), int(threads))
        if rc:
            raise RuntimeError(f"oracle table failed rc={rc}")
        try:
            ud = t.u_dense
            dense = np.ctypeslib.as_array(t.dense_M, shape=(ud + 1,)).astype(np.int32)
            M = np.empty(t.u_total + 1, dtype=np.int32)
            M[: ud + 1] = dense
            if t.num_words:
                nz = np.ctypeslib.as_array(t.nz, shape=(t.num_words,)).copy()
                neg = np.ctypeslib.as_array(t.neg, shape=(t.num_words,)).copy()
                ck = np.ctypeslib.as_array(t.ckpt, shape=(t.num_words,)).astype(np.int64)
                off = np.arange(t.u_total - ud, dtype=np.int64)
                w = off >> 6
                b = (off & 63).astype(np.uint64)
                bit_nz = (nz[w] >> b) & np.uint64(1)
                bit_ng = (neg[w] >> b) & np.uint64(1)
                mu_c = bit_nz.astype(np.int64) - 2 * bit_ng.astype(np.int64)
                # prefix within each word on top of its checkpoint
                cs = np.cumsum(mu_c)
                word_start = w * 64
                base_cs = np.where(word_start > 0, cs[np.maximum(word_start - 1, 0)], 0)
                M[ud + 1:] = (ck[w] + cs - base_cs).astype(np.int32)
            mu = np.ctypeslib.as_array(t.mu, shape=(t.mu_limit + 1,)).copy()
            s = OTableSums()
            self.L.dro_table_checksums(ctypes.byref(t), ctypes.byref(s))
            sums = tuple(getattr(s, n) for n, _ in s._fields_)
            return M, mu, sums
        finally:
            self.L.dro_table_free(ctypes.byref(t))

    def piece(self, piece: int, q: int) -> int:
        return int(self.L.dro_piece(int(piece), int(q)))

    def s2_interval(self, piece: int, first: int, last: int, y: int, mu: np.ndarray) -> int:
        mu = np.ascontiguousarray(mu, dtype=np.int8)
        return int(self.L.dro_s2_interval(int(piece), int(first), int(last), int(y),
                                          mu.ctypes.data_as(ctypes.POINTER(ctypes.c_int8))))


REF_GPU_PARAMS_SO = os.path.join(HERE, "_ref", "libdr_ref_gpu_params.so")


class ReferenceGpuParams:
    """The reference GPU engine's parameter heuristic, compiled from mertens_cuda.cuh
    (choose_gpu_sieve_limit :421-436, cx :473, mu limit :492)."""

    @staticmethod
    def available() -> bool:
        return os.path.exists(REF_GPU_PARAMS_SO)

    def __init__(self):
        L = ctypes.CDLL(REF_GPU_PARAMS_SO)
        L.ref_gpu_sieve_limit.restype = i64
        L.ref_gpu_sieve_limit.argtypes = [i64, c_int]
        L.ref_gpu_cx.restype = c_double
        L.ref_gpu_cx.argtypes = [i64]
        L.ref_gpu_mu_limit.restype = i64
        L.ref_gpu_mu_limit.argtypes = [i64, i64]
        self.L = L

    def params(self, X: int, threads: int):
        u = int(self.L.ref_gpu_sieve_limit(int(X), int(threads)))
        return u, float(self.L.ref_gpu_cx(int(X))), int(self.L.ref_gpu_mu_limit(int(X), u))


class Reference:
    """The reference engine built from its own sources (oracle/_ref)."""

    @staticmethod
    def available() -> bool:
        return os.path.exists(REF_SO)

    def __init__(self):
        if not self.available():
            raise FileNotFoundError(REF_SO)
        L = ctypes.CDLL(REF_SO)
        vp = ctypes.c_void_p
        sig = {
            "ref_compute_mertens": (i64, [i64, c_int]),
            "ref_compute_compressed": (i64, [i64, c_int]),
            "ref_choose_cx": (c_double, [i64]),
            "ref_choose_sieve_limit": (i64, [i64]),
            "ref_choose_compressed_limit": (i64, [i64]),
            "ref_isqrt": (i64, [i64]),
            "ref_table_new": (vp, [i64, i64, i64, c_int]),
            "ref_table_free": (None, [vp]),
            "ref_table_info": (None, [vp, ctypes.POINTER(i64)]),
            "ref_table_get": (None, [vp, i64, i64, ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int8)]),
            "ref_table_checksums": (None, [vp, ctypes.POINTER(u64)]),
            "ref_sieve_new": (vp, [i64, i64, c_int]),
            "ref_sieve_free": (None, [vp]),
            "ref_sieve_get": (None, [vp, i64, i64, ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int8)]),
            "ref_s2_single": (i64, [i64, i64, ctypes.POINTER(ctypes.c_int8)]),
            "ref_s2_combined": (i64, [i64, i64, i64, ctypes.POINTER(ctypes.c_int8)]),
            "ref_s2_interval": (i64, [c_int, i64, i64, i64, ctypes.POINTER(ctypes.c_int8)]),
            "ref_piece": (i64, [c_int, i64]),
            "ref_finalize_bytes": (None, [ctypes.POINTER(ctypes.c_uint8), i64, i64, c_int]),
            "ref_dr_checksums": (c_int, [i64, i64, i64, c_double, i64, c_int, ctypes.POINTER(i64)]),
        }
        for n, (r, a) in sig.items():
            f = getattr(L, n)
            f.restype = r
            f.argtypes = a
        self.L = L

    def compute_mertens(self, X: int, threads: int = 0) -> int:
        return int(self.L.ref_compute_mertens(int(X), int(threads)))

    def compute_compressed(self, X: int, threads: int = 0) -> int:
        return int(self.L.ref_compute_compressed(int(X), int(threads)))

    def checksums(self, X: int, u_total: int, u_dense: int, cx: float, mu_limit: int, threads: int = 0) -> dict:
        out = (i64 * 5)()
        self.L.ref_dr_checksums(int(X), int(u_total), int(u_dense), float(cx), int(mu_limit), int(threads), out)
        m = (1 << 64) - 1
        return {"M": out[0], "C": out[1] & m, "S1": out[2] & m, "S2": out[3] & m, "terms": out[4]}

    def table(self, u_total: int, u_dense: int, mu_limit: int, threads: int = 0):
        h = self.L.ref_table_new(int(u_total), int(u_dense), int(mu_limit), int(threads))
        try:
            info = (i64 * 4)()
            self.L.ref_table_info(h, info)
            n = info[0] + 1
            M = np.zeros(n, dtype=np.int32)
            mu = np.zeros(n, dtype=np.int8)
            self.L.ref_table_get(h, 0, n, M.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                                 mu.ctypes.data_as(ctypes.POINTER(ctypes.c_int8)))
            s = (u64 * 6)()
            self.L.ref_table_checksums(h, s)
            return M, mu, tuple(s), tuple(info)
        finally:
            self.L.ref_table_free(h)

    def table_sums(self, u_total: int, u_dense: int, mu_limit: int, threads: int = 0):
        h = self.L.ref_table_new(int(u_total), int(u_dense), int(mu_limit), int(threads))
        try:
            s = (u64 * 6)()
            self.L.ref_table_checksums(h, s)
            info = (i64 * 4)()
            self.L.ref_table_info(h, info)
            return tuple(s), tuple(info)
        finally:
            self.L.ref_table_free(h)
