"""dr_b200 -- Python view of the B200 Deleglise-Rivat Mertens engine.

The engine itself is native: hand-written sm_100a kernels plus a C++20 host
engine behind the C ABI declared in include/dr_engine.h (libdrb200.so).  This
module only binds that ABI with ctypes so that tests and bench.py can call it.
Names follow the reference (ecreeth/deleglise-rivat): ``compute_mertens``,
``compute_compressed``, ``choose_cx``, ``SieveTable``-style table reads.

The library has no CPU fallback: if libdrb200.so cannot be loaded, or no
sm_100 device is present, every call raises ``DRError``.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import threading
from dataclasses import dataclass
from typing import Iterable, Optional, Sequence

_PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
_LIB_PATH = os.environ.get("DR_B200_LIB") or os.path.join(_PKG_DIR, "lib", "libdrb200.so")
_CSRC = os.path.join(_PKG_DIR, "csrc")

DR_OK = 0
DR_ERR_ARG = -1
DR_ERR_PARAMS = -2
DR_ERR_NOMEM = -3
DR_ERR_CUDA = -4
DR_ERR_DEVICE = -5

POLICY_REFERENCE = 0
POLICY_DENSE = 1
POLICY_COMPRESSED = 2
POLICY_GPU = 3
POLICY_REFERENCE_GPU = 4


class DRError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"dr error {code}: {msg}")
        self.code = code


class Params(ctypes.Structure):
    _fields_ = [
        ("u_total", ctypes.c_int64),
        ("u_dense", ctypes.c_int64),
        ("cx", ctypes.c_double),
        ("mu_limit", ctypes.c_int64),
        ("segment_log2", ctypes.c_int32),
        ("block_threads", ctypes.c_int32),
        ("chunk_log2", ctypes.c_int32),
        ("s1_window_log2", ctypes.c_int32),
    ]

    def as_dict(self) -> dict:
        return {f: getattr(self, f) for f, _ in self._fields_}

    def __repr__(self) -> str:
        return f"Params({self.as_dict()})"


class Stats(ctypes.Structure):
    _fields_ = [
        ("M", ctypes.c_int64),
        ("C", ctypes.c_uint64),
        ("S1", ctypes.c_uint64),
        ("S2", ctypes.c_uint64),
        ("terms", ctypes.c_int64),
        ("evals", ctypes.c_int64),
        ("s1_ops", ctypes.c_uint64),
        ("s2_ops", ctypes.c_uint64),
        ("table_ms", ctypes.c_double),
        ("plan_ms", ctypes.c_double),
        ("sums_ms", ctypes.c_double),
        ("total_ms", ctypes.c_double),
        ("h2d_ms", ctypes.c_double),
        ("d2h_ms", ctypes.c_double),
        ("sieve_launches", ctypes.c_int32),
        ("sums_launches", ctypes.c_int32),
        ("kernel_launches", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
        ("h2d_bytes", ctypes.c_uint64),
        ("d2h_bytes", ctypes.c_uint64),
        ("s1_comp_ops", ctypes.c_uint64),
        ("band_table_ms", ctypes.c_double),
        ("band_sums_ms", ctypes.c_double),
        ("bands", ctypes.c_int64),
    ]

    def as_dict(self) -> dict:
        return {f: getattr(self, f) for f, _ in self._fields_ if f != "reserved"}


class TableSums(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint64) for n in ("dense_sum", "dense_wsum", "mu_wsum", "nz_wsum", "neg_wsum", "ckpt_wsum")]

    def as_tuple(self):
        return tuple(getattr(self, n) for n, _ in self._fields_)


_lib = None
_lib_lock = threading.Lock()


def build_library(force: bool = False) -> str:
    """Compile libdrb200.so in-tree with nvcc for sm_100a (make in csrc/)."""
    if force or not os.path.exists(_LIB_PATH):
        subprocess.run(["make", "-C", _CSRC, "-s"], check=True)
    return _LIB_PATH


def lib():
    """Load libdrb200.so (building it first if it is missing)."""
    global _lib
    with _lib_lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(_LIB_PATH):
            build_library()
        L = ctypes.CDLL(_LIB_PATH)
        P, S = ctypes.POINTER(Params), ctypes.POINTER(Stats)
        vp, i64, u64, i32 = ctypes.c_void_p, ctypes.c_int64, ctypes.c_uint64, ctypes.c_int
        sig = {
            "dr_ctx_create": (i32, [i32, vp, ctypes.POINTER(vp)]),
            "dr_ctx_destroy": (i32, [vp]),
            "dr_last_error": (ctypes.c_char_p, []),
            "dr_ctx_set_hbm_budget": (i32, [vp, u64]),
            "dr_ctx_set_resident_limit": (i32, [vp, i64, i64]),
            "dr_device_info": (i32, [i32, ctypes.POINTER(i32), ctypes.POINTER(u64)]),
            "dr_default_params": (i32, [i64, i32, P]),
            "dr_reference_gpu_params": (i32, [i64, i32, P]),
            "dr_check_params": (i32, [i64, P, u64]),
            "dr_table_bytes": (u64, [i64, i64, i64]),
            "dr_query_bytes": (u64, [i64, P]),
            "dr_mertens": (i32, [vp, i64, P, ctypes.POINTER(i64), S]),
            "dr_mertens_batch": (i32, [vp, ctypes.POINTER(i64), i64, P, ctypes.POINTER(i64), S]),
            "dr_batch_checksums": (i32, [vp, ctypes.POINTER(u64), i64]),
            "dr_table_build": (i32, [vp, i64, i64, i64, P, S]),
            "dr_table_read": (i32, [vp, i64, i64, ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int8)]),
            "dr_table_read_wheel": (i32, [vp, i64, i64, ctypes.POINTER(ctypes.c_int8)]),
            "dr_table_checksums": (i32, [vp, ctypes.POINTER(TableSums)]),
            "dr_debug_udiv": (i32, [vp, ctypes.POINTER(u64), ctypes.POINTER(u64), i64, ctypes.POINTER(u64)]),
            "dr_debug_udiv_rcp": (i32, [vp, ctypes.POINTER(u64), ctypes.POINTER(u64), i64, ctypes.POINTER(u64)]),
            "dr_debug_udiv32": (i32, [vp, ctypes.POINTER(u64), ctypes.POINTER(u64), i64, ctypes.POINTER(u64)]),
            "dr_debug_piece": (i32, [vp, ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(u64), i64,
                                     ctypes.POINTER(i64)]),
            "dr_debug_piece32": (i32, [vp, ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(u64), i64,
                                       ctypes.POINTER(i64)]),
            "dr_table_build_noalloc": (i32, [i32, vp, i64, i64, i64, vp, vp, vp, vp]),
            "dr_autotune_batch": (i32, [vp, ctypes.POINTER(i64), i64, i32, P, ctypes.POINTER(ctypes.c_double)]),
            "dr_mlp_create": (i32, [vp, u64, ctypes.POINTER(vp)]),
            "dr_mlp_destroy": (i32, [vp]),
            "dr_mlp_num_params": (i64, []),
            "dr_mlp_set_weights": (i32, [vp, ctypes.POINTER(ctypes.c_float), i64]),
            "dr_mlp_get_weights": (i32, [vp, ctypes.POINTER(ctypes.c_float), i64]),
            "dr_mlp_forward": (i32, [vp, ctypes.POINTER(ctypes.c_float), i64, ctypes.POINTER(ctypes.c_float)]),
            "dr_mlp_grad": (i32, [vp, ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float), i64,
                                  ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float)]),
            "dr_mlp_train": (i32, [vp, ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float), i64, i32,
                                   ctypes.c_float, ctypes.POINTER(ctypes.c_float)]),
            "dr_tuner_features": (i32, [i64, u64, i32, i32, ctypes.POINTER(ctypes.c_float)]),
            "dr_tuner_params": (i32, [i64, ctypes.POINTER(ctypes.c_float), P]),
            "dr_tuner_propose": (i32, [vp, i64, u64, i32, i32, P, ctypes.POINTER(i32)]),
            "dr_measure_peaks": (i32, [i32, ctypes.POINTER(Peaks)]),
            "dr_debug_sieve_plan": (i64, [i64, i64, i32, i64, ctypes.POINTER(i64), i64]),
            "dr_debug_stream_plan": (i64, [i64, i64, i32, i64, i64, ctypes.POINTER(i64), ctypes.POINTER(i64), i64]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
        return L


def exported_symbols() -> list:
    """Names of the C-ABI entry points this binding expects (for load tests)."""
    lib()
    return [
        "dr_ctx_create", "dr_ctx_destroy", "dr_last_error", "dr_ctx_set_hbm_budget", "dr_ctx_set_resident_limit",
        "dr_device_info",
        "dr_default_params", "dr_reference_gpu_params", "dr_check_params", "dr_table_bytes", "dr_query_bytes", "dr_mertens", "dr_mertens_batch",
        "dr_batch_checksums", "dr_table_build", "dr_table_read", "dr_table_read_wheel", "dr_table_checksums",
        "dr_debug_udiv", "dr_debug_udiv_rcp", "dr_debug_udiv32", "dr_debug_piece", "dr_debug_piece32",
        "dr_table_build_noalloc", "dr_autotune_batch",
        "dr_mlp_create", "dr_mlp_destroy", "dr_mlp_num_params", "dr_mlp_set_weights", "dr_mlp_get_weights",
        "dr_mlp_forward", "dr_mlp_grad", "dr_mlp_train", "dr_tuner_features", "dr_tuner_params", "dr_tuner_propose",
        "dr_measure_peaks", "dr_debug_sieve_plan", "dr_debug_stream_plan",
    ]


class Peaks(ctypes.Structure):
    """dr_peaks: measured ceilings, operations per second over the whole GPU."""
    _fields_ = [("smem_atomic_per_s", ctypes.c_double), ("smem_atomic_stride_per_s", ctypes.c_double),
                ("imad_per_s", ctypes.c_double), ("dfma_per_s", ctypes.c_double)]


def sieve_plan(u_total: int, u_dense: int, segment_log2: int, first_wave: int) -> list:
    """The table build's sieve launches: (first segment, end segment, odd mode) in stream order."""
    n = int(lib().dr_debug_sieve_plan(int(u_total), int(u_dense), int(segment_log2), int(first_wave), None, 0))
    if n < 0:
        _check(n)
    buf = (ctypes.c_int64 * (3 * max(n, 1)))()
    lib().dr_debug_sieve_plan(int(u_total), int(u_dense), int(segment_log2), int(first_wave), buf, n)
    return [(buf[3 * i], buf[3 * i + 1], bool(buf[3 * i + 2])) for i in range(n)]


def stream_plan(u_total: int, u_dense: int, segment_log2: int, u_resident: int, band_values: int = 0):
    """The bands of a streamed table: (u_res, [(vlo, vhi, odd mode), ...]); no bands when
    nothing streams."""
    ures = ctypes.c_int64()
    args = (int(u_total), int(u_dense), int(segment_log2), int(u_resident), int(band_values), ctypes.byref(ures))
    n = int(lib().dr_debug_stream_plan(*args, None, 0))
    if n < 0:
        _check(n)
    buf = (ctypes.c_int64 * (3 * max(n, 1)))()
    lib().dr_debug_stream_plan(*args, buf, n)
    return ures.value, [(buf[3 * i], buf[3 * i + 1], bool(buf[3 * i + 2])) for i in range(n)]


def measure_peaks(device: int = 0) -> dict:
    """Shared-memory atomic, IMAD and DFMA throughput ceilings of `device` (dr_measure_peaks)."""
    pk = Peaks()
    _check(lib().dr_measure_peaks(int(device), ctypes.byref(pk)))
    return {name: getattr(pk, name) for name, _ in Peaks._fields_}


def _check(rc: int):
    if rc != DR_OK:
        raise DRError(rc, lib().dr_last_error().decode(errors="replace"))


def default_params(X: int, policy: int = POLICY_REFERENCE) -> Params:
    """Reference parameter policy (choose_cx / choose_sieve_limit / choose_compressed_limit)."""
    p = Params()
    _check(lib().dr_default_params(int(X), int(policy), ctypes.byref(p)))
    return p


def reference_gpu_params(X: int, host_threads: int = 0) -> Params:
    """The reference GPU engine's parameters (choose_gpu_sieve_limit, mertens_cuda.cuh:421)."""
    p = Params()
    _check(lib().dr_reference_gpu_params(int(X), int(host_threads), ctypes.byref(p)))
    return p


def check_params(X: int, p: Params, budget: int = 0) -> int:
    """Endpoint-coverage check; returns the status code (0 = usable)."""
    return lib().dr_check_params(int(X), ctypes.byref(p), int(budget))


def table_bytes(u_total: int, u_dense: int, mu_limit: int) -> int:
    return int(lib().dr_table_bytes(int(u_total), int(u_dense), int(mu_limit)))


def query_bytes(X: int, p: Params) -> int:
    """Device bytes one query needs (table + reciprocal tables + work arrays)."""
    return int(lib().dr_query_bytes(int(X), ctypes.byref(p)))


def choose_cx(X: int) -> float:
    return default_params(X).cx


@dataclass
class Result:
    M: int
    stats: Stats


class Engine:
    """A device context (mirror of the reference engines' static entry points)."""

    def __init__(self, device: int = 0, stream: Optional[int] = None):
        self._ctx = ctypes.c_void_p()
        _check(lib().dr_ctx_create(int(device), ctypes.c_void_p(stream) if stream else None, ctypes.byref(self._ctx)))

    def close(self):
        if self._ctx:
            lib().dr_ctx_destroy(self._ctx)
            self._ctx = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_hbm_budget(self, nbytes: int):
        _check(lib().dr_ctx_set_hbm_budget(self._ctx, int(nbytes)))

    def set_resident_limit(self, u_resident: int, band_values: int = 0):
        """Stream the compressed tier of single-query tables above u_resident values in
        bands of band_values (0: the resident compressed tier's size); 0 holds every
        table whole."""
        _check(lib().dr_ctx_set_resident_limit(self._ctx, int(u_resident), int(band_values)))

    # --- reference-named entry points ---------------------------------------
    def compute_mertens(self, X: int, params: Optional[Params] = None) -> int:
        """DelégliseRivatEngine::compute_mertens (reference policy when params is None)."""
        return self.mertens(X, params).M

    def compute_compressed(self, X: int) -> int:
        """DelégliseRivatEngine::compute_compressed: the streamed-table parameters."""
        return self.mertens(X, default_params(X, POLICY_COMPRESSED)).M

    def mertens(self, X: int, params: Optional[Params] = None) -> Result:
        out = ctypes.c_int64()
        st = Stats()
        _check(lib().dr_mertens(self._ctx, int(X), ctypes.byref(params) if params is not None else None,
                                ctypes.byref(out), ctypes.byref(st)))
        return Result(out.value, st)

    def mertens_batch(self, Xs: Sequence[int], params: Optional[Sequence[Params]] = None):
        n = len(Xs)
        arr = (ctypes.c_int64 * n)(*[int(x) for x in Xs])
        out = (ctypes.c_int64 * n)()
        st = Stats()
        parr = None
        if params is not None:
            parr = (Params * n)(*params)
        _check(lib().dr_mertens_batch(self._ctx, arr, n, parr, out, ctypes.byref(st)))
        return list(out), st

    def autotune_batch(self, Xs: Sequence[int], max_trials: int = 24):
        """Batch autotuner: (per-query Params, best device ms)."""
        n = len(Xs)
        arr = (ctypes.c_int64 * n)(*[int(x) for x in Xs])
        out = (Params * n)()
        best = ctypes.c_double()
        _check(lib().dr_autotune_batch(self._ctx, arr, n, int(max_trials), out, ctypes.byref(best)))
        return list(out), best.value

    def batch_checksums(self, n: int):
        buf = (ctypes.c_uint64 * (3 * n))()
        _check(lib().dr_batch_checksums(self._ctx, buf, n))
        return [(buf[3 * i], buf[3 * i + 1], buf[3 * i + 2]) for i in range(n)]

    # --- tables ---------------------------------------------------------------
    def table_build(self, u_total: int, u_dense: int, mu_limit: int, tuning: Optional[Params] = None) -> Stats:
        st = Stats()
        _check(lib().dr_table_build(self._ctx, int(u_total), int(u_dense), int(mu_limit),
                                    ctypes.byref(tuning) if tuning is not None else None, ctypes.byref(st)))
        return st

    def table_read(self, first: int, count: int):
        """(M[first:first+count], mu[...]) as numpy arrays (get_M / get_mu)."""
        import numpy as np

        M = np.zeros(count, dtype=np.int32)
        mu = np.zeros(count, dtype=np.int8)
        _check(lib().dr_table_read(self._ctx, int(first), int(count),
                                   M.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                                   mu.ctypes.data_as(ctypes.POINTER(ctypes.c_int8))))
        return M, mu

    def table_read_wheel(self, first: int, count: int):
        import numpy as np

        mu = np.zeros(count, dtype=np.int8)
        _check(lib().dr_table_read_wheel(self._ctx, int(first), int(count),
                                         mu.ctypes.data_as(ctypes.POINTER(ctypes.c_int8))))
        return mu

    # --- device arithmetic (test support) --------------------------------------
    def debug_udiv(self, ys, ds, rcp=False):
        """floor(y/d) computed by a device quotient routine: the general one
        (rcp False), the 64-bit reciprocal-estimate one (rcp True or "64"), or
        the 32-bit one of the fast S1/S2 paths (rcp "32"); 2^64-1 outside the
        routine's domain."""
        n = len(ys)
        Y = (ctypes.c_uint64 * n)(*[int(v) for v in ys])
        D = (ctypes.c_uint64 * n)(*[int(v) for v in ds])
        Q = (ctypes.c_uint64 * n)()
        fn = lib().dr_debug_udiv32 if rcp == "32" else lib().dr_debug_udiv_rcp if rcp else lib().dr_debug_udiv
        _check(fn(self._ctx, Y, D, n, Q))
        return list(Q)

    def debug_piece(self, pieces, qs, fast: bool = False):
        """S2 summand piece(q): the 64-bit routine, or (fast) the 32-bit one of the
        fast S2 path (INT64_MIN for q >= 2^31)."""
        n = len(qs)
        P = (ctypes.c_int32 * n)(*[int(v) for v in pieces])
        Q = (ctypes.c_uint64 * n)(*[int(v) for v in qs])
        O = (ctypes.c_int64 * n)()
        _check((lib().dr_debug_piece32 if fast else lib().dr_debug_piece)(self._ctx, P, Q, n, O))
        return list(O)

    def table_checksums(self) -> tuple:
        s = TableSums()
        _check(lib().dr_table_checksums(self._ctx, ctypes.byref(s)))
        return s.as_tuple()


def device_info(device: int = 0):
    sm = ctypes.c_int()
    hbm = ctypes.c_uint64()
    _check(lib().dr_device_info(int(device), ctypes.byref(sm), ctypes.byref(hbm)))
    return sm.value, hbm.value


def _fptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def tuner_features(X: int, budget: int, sms: int = 148, batch: int = 1):
    import numpy as np

    f = np.zeros(4, dtype=np.float32)
    _check(lib().dr_tuner_features(int(X), int(budget), int(sms), int(batch), _fptr(f)))
    return f


def tuner_params(X: int, y_normalised) -> Params:
    import numpy as np

    y = np.ascontiguousarray(y_normalised, dtype=np.float32)
    p = Params()
    _check(lib().dr_tuner_params(int(X), _fptr(y), ctypes.byref(p)))
    return p


class MLP:
    """The learned tuner's network on the device (dr_mlp_*)."""

    def __init__(self, engine: Engine, seed: int = 1):
        self._h = ctypes.c_void_p()
        _check(lib().dr_mlp_create(engine._ctx, int(seed), ctypes.byref(self._h)))
        self.n_params = int(lib().dr_mlp_num_params())

    def close(self):
        if self._h:
            lib().dr_mlp_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def get_weights(self):
        import numpy as np

        w = np.zeros(self.n_params, dtype=np.float32)
        _check(lib().dr_mlp_get_weights(self._h, _fptr(w), self.n_params))
        return w

    def set_weights(self, w):
        import numpy as np

        w = np.ascontiguousarray(w, dtype=np.float32)
        _check(lib().dr_mlp_set_weights(self._h, _fptr(w), len(w)))

    def forward(self, x):
        import numpy as np

        x = np.ascontiguousarray(x, dtype=np.float32)
        y = np.zeros((x.shape[0], 4), dtype=np.float32)
        _check(lib().dr_mlp_forward(self._h, _fptr(x), x.shape[0], _fptr(y)))
        return y

    def grad(self, x, t):
        import numpy as np

        x = np.ascontiguousarray(x, dtype=np.float32)
        t = np.ascontiguousarray(t, dtype=np.float32)
        g = np.zeros(self.n_params, dtype=np.float32)
        loss = ctypes.c_float()
        _check(lib().dr_mlp_grad(self._h, _fptr(x), _fptr(t), x.shape[0], _fptr(g), ctypes.byref(loss)))
        return g, loss.value

    def train(self, x, t, steps: int, lr: float = 3e-3) -> float:
        import numpy as np

        x = np.ascontiguousarray(x, dtype=np.float32)
        t = np.ascontiguousarray(t, dtype=np.float32)
        loss = ctypes.c_float()
        _check(lib().dr_mlp_train(self._h, _fptr(x), _fptr(t), x.shape[0], int(steps), float(lr), ctypes.byref(loss)))
        return loss.value

    def propose(self, X: int, budget: int, sms: int = 148, batch: int = 1):
        """(Params, used_fallback) for X: inference + coverage check + fallback."""
        p = Params()
        fb = ctypes.c_int()
        _check(lib().dr_tuner_propose(self._h, int(X), int(budget), int(sms), int(batch), ctypes.byref(p),
                                      ctypes.byref(fb)))
        return p, bool(fb.value)
