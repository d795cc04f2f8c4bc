"""Generate the golden fixtures under tests/golden/ from the reference engine.

Run from the repository root where the reference source tree is available:

    make -C oracle ref            # builds oracle/_ref/ from the reference sources
    python tests/golden/make_golden.py [--skip-big]

Everything written here is computed by the reference itself (oracle/_ref,
compiled from mertens_dr.hpp) -- M(X), the C/S1/S2 checksums of
ref_dr_checksums() at the reference's own default parameters, table
checksums of CompressedMertensTable -- except kat.json, whose values are the
reference's published known answers (cited per entry).
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
from oracle_py import Oracle, Reference  # noqa: E402

BATCH_SEED = 20261203

# Published known answers of the reference (values, then where they are pinned).
KAT = [
    (1, 1, "test_dr.cpp:27"), (2, 0, "test_dr.cpp:28"), (3, -1, "test_dr.cpp:29"),
    (4, -1, "test_dr.cpp:30"), (5, -2, "test_dr.cpp:31"), (10, -1, "test_dr.cpp:32"),
    (100, 1, "test_dr.cpp:33"), (1000, 2, "test_dr.cpp:34"), (10**4, -23, "test_dr.cpp:35"),
    (10**5, -48, "test_dr.cpp:36"), (10**6, 212, "test_dr.cpp:37"), (10**7, 1037, "test_dr.cpp:38"),
    (10**8, 1928, "test_dr.cpp:39"), (10**9, -222, "test_dr.cpp:40"), (10**10, -33722, "test_dr.cpp:41"),
    (10**11, -87856, "test_dr.cpp:42"), (10**12, 62366, "test_dr.cpp:43"), (10**13, 599582, "test_dr.cpp:44"),
    (10**14, -875575, "test_dr.cpp:45"), (10**15, -3216373, "test_dr.cpp:46"),
    (10**16, -3195437, "test_cuda.cu:59"), (10**17, -21830254, "README.md:188"),
]


def batch_inputs(n: int = 256, seed: int = BATCH_SEED) -> list:
    """256 X = round(10^U), U ~ Uniform(9, 14) from numpy default_rng(seed)."""
    rng = np.random.default_rng(seed)
    return [int(round(10 ** u)) for u in rng.uniform(9.0, 14.0, size=n)]


def params_of(o: Oracle, X: int, compressed: bool) -> dict:
    p = o.default_params(X, compressed)
    return {"X": X, "u_total": p.u_total, "u_dense": p.u_dense, "cx": p.cx, "mu_limit": p.mu_limit}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--skip-big", action="store_true", help="skip 10^16 checksums and the batch")
    ap.add_argument("--threads", type=int, default=0)
    args = ap.parse_args()
    o, r = Oracle(), Reference()
    th = args.threads

    with open(os.path.join(HERE, "kat.json"), "w") as f:
        json.dump({"source": "reference known answers", "cases": [{"X": x, "M": m, "cite": c} for x, m, c in KAT]},
                  f, indent=1)

    # checksums at the reference's own default parameters
    cases = []
    dense_x = [54321, 987654, 12345678, 99975680, 987654321, 5 * 10**9, 10**9, 10**10, 10**11, 123456789012,
               10**12]
    comp_x = [10**11, 123456789012, 10**12, 10**13, 10**14, 10**15]
    if not args.skip_big:
        comp_x.append(10**16)
    for X in dense_x:
        cases.append(("dense", params_of(o, X, False)))
    for X in comp_x:
        cases.append(("compressed", params_of(o, X, True)))
    out = []
    for kind, p in cases:
        t0 = time.time()
        ck = r.checksums(p["X"], p["u_total"], p["u_dense"], p["cx"], p["mu_limit"], th)
        engine = r.compute_compressed(p["X"], th) if kind == "compressed" else None
        dt = time.time() - t0
        rec = dict(kind=kind, **p, **ck)
        if engine is not None:
            assert engine == ck["M"], (p, engine, ck)
        out.append(rec)
        print(kind, p["X"], ck["M"], f"{dt:.2f}s", flush=True)
    with open(os.path.join(HERE, "checksums.json"), "w") as f:
        json.dump({"source": "oracle/_ref ref_dr_checksums at reference default parameters",
                   "convention": "M = C - S1 - S2 (mod 2^64); see oracle/dr_oracle.h", "cases": out}, f, indent=1)

    # table checksums of CompressedMertensTable (raw members)
    tabs = []
    for ut, ud, ml in [(1048576, 1024, 1048576), (1000033, 131071, 1000033), (262147, 262147, 262147),
                       (17325, 7, 17325), (13861, 13860, 13861), (42696448, 10674176, 951000),
                       (195055360, 48763904, 3637619)]:
        sums, info = r.table_sums(ut, ud, ml, th)
        tabs.append({"u_total": ut, "u_dense": ud, "mu_limit": ml, "info": list(info), "sums": [int(s) for s in sums]})
    with open(os.path.join(HERE, "tables.json"), "w") as f:
        json.dump({"source": "oracle/_ref ref_table_checksums (CompressedMertensTable)",
                   "sums": "dense_sum, dense_wsum, mu_wsum, nz_wsum, neg_wsum, ckpt_wsum", "cases": tabs}, f, indent=1)

    if not args.skip_big:
        xs = batch_inputs()
        t0 = time.time()
        vals = [r.compute_mertens(x, th) for x in xs]
        with open(os.path.join(HERE, "batch256.json"), "w") as f:
            json.dump({"source": "oracle/_ref compute_mertens (default env)", "seed": BATCH_SEED,
                       "rule": "X = round(10**U), U ~ numpy default_rng(seed).uniform(9, 14, 256)",
                       "X": xs, "M": vals, "cpu_seconds": time.time() - t0}, f, indent=1)
        print("batch", time.time() - t0, flush=True)


if __name__ == "__main__":
    main()
