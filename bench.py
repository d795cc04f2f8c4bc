#!/usr/bin/env python
"""bench.py -- exact M(10^16) on B200 (seconds per M(X)) plus batched M(X)/s.

One "step" is one complete M(10^16) through the engine: segmented Mobius sieve,
dense + compressed Mertens tables, term planning, persistent S1/S2 kernel and
the reduction -- nothing cached between steps (the ~9 GB of tables and
reciprocals are rebuilt every step, far larger than the 126 MB L2).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl engine|reference]

N > 1 (torchrun, one process per GPU) runs N independent replicas: M(X) does
not need a collective.  Rank 0 prints one JSON line.  The reference arm times
the reference's own CPU engine (oracle/_ref, built from its sources) on this
host's cores.

Besides the contract's keys the line carries `phases_ms` (table, planning,
sums), `roofline` (the S1/S2 phase: against the HBM copy peak on its
algorithmic bytes, and in `roofline.issue` against its binding unit,
instruction issue), `table_roofline` (the table phase against instruction
issue, with the sieve's shared-memory atomics and the table's HBM writes
beside it), `int_peaks` (shared-memory atomic, IMAD and DFMA ceilings measured
on this GPU by dr_measure_peaks), `default_params` and `learned_tuner` (the
same step with the reference's parameters and with the learned tuner's
proposal) and `batched` (the 256-query batch: replay throughput, first-call
cost, launches per batch).

Profiling cases: `--x X` times M(X) instead of M(10^16), `--u U` sets the table
size, and `--resident R --band B` streams the table above R values in bands of B
(the line then carries `stream` and the bands' share of the sums phase).
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "deleglise-rivat_b200"))

X_HEADLINE = 10**16
M_HEADLINE = -3195437  # test_cuda.cu:59
BATCH_SEED = 20261203


def batch_inputs(n=256, seed=BATCH_SEED):
    import numpy as np

    rng = np.random.default_rng(seed)
    return [int(round(10**u)) for u in rng.uniform(9.0, 14.0, size=n)]


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.rows = []
        self.proc = None
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            if self.thread:
                self.thread.join(timeout=2)

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
                for name, v in zip(names, r[5:9]):
                    if v.strip().lower() == "active":
                        reasons.add(name)
            except Exception:
                continue
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist

        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        backend = os.environ.get("DR_DIST_BACKEND", "nccl")
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over_ranks(v, world):
    """Max of a per-rank time over all ranks (NCCL on GPUs, gloo on CPU)."""
    if world == 1:
        return v
    import torch
    import torch.distributed as dist

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def cpu_reference_sample(seconds_budget=40.0):
    """Reference CPU engine (oracle/_ref) on this host: one M(10^16) with all cores."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle_py import Reference

    cores = os.cpu_count() or 1
    if not Reference.available():
        from oracle_py import Oracle

        o = Oracle()
        t0 = time.perf_counter()
        m = o.mertens(10**13, cores)
        dt = time.perf_counter() - t0
        return {"value": dt, "unit": "s per M(10^13)", "cores": cores, "kind": "port",
                "sample": "oracle port M(10^13), reference build absent", "M": m}
    r = Reference()
    r.compute_mertens(10**8, cores)  # warm-up, as the reference's benchmarks do
    t0 = time.perf_counter()
    m = r.compute_mertens(X_HEADLINE, cores)
    dt = time.perf_counter() - t0
    return {"value": dt, "unit": "s per M(10^16)", "cores": cores, "kind": "reference",
            "sample": "one full M(10^16) by the reference engine (default env: streamed table)", "M": m}


def run_reference(args, world, rank):
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle_py import Reference

    cores = os.cpu_count() or 1
    if not Reference.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref was not built (reference sources absent)"}))
        return
    r = Reference()
    for _ in range(max(1, args.warmup)):
        r.compute_mertens(10**8, cores)
    times = []
    t_start = time.perf_counter()
    for _ in range(args.steps):
        t0 = time.perf_counter()
        m = r.compute_mertens(X_HEADLINE, cores)
        times.append(time.perf_counter() - t0)
        assert m == M_HEADLINE, m
        if time.perf_counter() - t_start > 150:
            break
    v = statistics.median(times)
    line = {
        "impl": "reference", "metric": "sec per M(10^16)", "value": v, "unit": "s", "n_gpus": args.gpus,
        "steps": len(times), "warmup": args.warmup, "ms_per_step": v * 1e3, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "int64", "data": "synthetic (the single input X=10^16)",
        "config": {"workload": "M(10^16), reference default parameters (streamed table)", "X": X_HEADLINE},
        "cpu_baseline": {"value": v, "unit": "s", "cores": cores, "kind": "reference",
                         "sample": f"{len(times)} full M(10^16) runs (capped at ~150 s), median"},
        "e2e": {"value": v, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


KNOWN = {10**k: m for k, m in [(9, -222), (10, -33722), (11, -87856), (12, 62366), (13, 599582), (14, -875575),
                                    (15, -3216373), (16, -3195437), (17, -21830254), (18, -46758740)]}
# test_dr.cpp, test_cuda.cu, README; 10^18 pinned by the reference engine built from its own sources
KNOWN[(1 << 63) - 1] = 580197744  # this engine's value, agreed by two parameter sets (no reference value)


def with_table_size(p, X, u):
    """The B200 policy's parameters with the table size set to u: the dense tier by the
    policy's rule (max(1.28e8, u/16), at most 4e9) and mu_limit covering A and X/u."""
    import dr_b200

    dense = min(4000000000, max(128000000, u // 16))
    dense = min(u, (dense + 255) & ~255)
    a_max = int(p.cx * X**0.5) + 1000
    return dr_b200.Params(**{**p.as_dict(), "u_total": u, "u_dense": dense, "mu_limit": min(u, max(a_max, X // u + 1000))})


def sieve_marks(u_total, u_dense, sm_count, S=1 << 17):
    """Shared-memory atomics the table build issues: one per multiple of a prime
    13 <= p <= sqrt(u) (log weight) and per multiple of p^2, p >= 5 (square flag),
    every multiple in the first wave of full-mode segments (sm_count segments of S
    values) and the odd multiples above it (odd mode, when u_dense is on a 64-value
    word).  Counted on the host from the primes."""
    import numpy as np

    r = int(np.sqrt(u_total)) + 1
    sieve = np.ones(r + 1, dtype=bool)
    sieve[:2] = False
    for i in range(2, int(r ** 0.5) + 1):
        if sieve[i]:
            sieve[i * i::i] = False
    pr = np.nonzero(sieve)[0].astype(np.int64)
    pr = pr[pr * pr <= u_total]
    vf = min(u_total, sm_count * S) if u_dense % 64 == 0 else u_total
    mods = np.concatenate([pr[pr >= 13], pr[pr >= 5] ** 2])
    full = vf // mods
    odd = (u_total // mods + 1) // 2 - (vf // mods + 1) // 2
    return int(full.sum() + odd.sum())


# Warp instructions per unit of work, from ncu smsp__inst_executed.sum of one launch
# divided by that launch's work:
#   sums_kernel at M(10^15) (B200 policy): 7.05e9 instructions for 5.98e9 S1 lookups +
#     2.40e9 S2 wheel positions; the S2 positions at 1.50 each (timing-only capture that
#     keeps only the S2 part), the rest, 0.58 per lookup, to S1;
#   sieve_kernel, odd mode, on the M(10^15) table: 5.63e7 instructions for 1.01e8 values.
SUMS_INST_PER_S1 = 0.58
SUMS_INST_PER_S2 = 1.50
SIEVE_INST_PER_VALUE = 0.556
# DRAM bytes per op of sums_kernel (dram__bytes_read.sum + dram__bytes_write.sum of one
# launch over its S1 lookups + S2 positions) at M(10^15): 10.71 GB / 8.38e9 ops.
SUMS_DRAM_PER_OP = 1.28


def sums_roofline(st, sums_ms, peak, peak_kind, issue_peak, f_mhz):
    """S1/S2 phase (sums_kernel) against HBM on the algorithmic bytes -- 2 B per
    dense-tier S1 lookup, 20 B per compressed-tier lookup (16 B plane pair + 4 B
    checkpoint), 1 B of Mobius value per S2 candidate j (two per wheel position) --
    and against its binding unit, instruction issue."""
    t = sums_ms / 1e3
    dense = st.s1_ops - st.s1_comp_ops
    alg = 2.0 * dense + 20.0 * st.s1_comp_ops + 2.0 * st.s2_ops
    inst = SUMS_INST_PER_S1 * st.s1_ops + SUMS_INST_PER_S2 * st.s2_ops
    return {
        "bound": "hbm", "kernel": "sums_kernel (S1/S2 phase)", "achieved": alg / t / 1e9, "peak": peak,
        "unit": "GB/s", "frac": alg / t / 1e9 / peak, "peak_kind": peak_kind,
        "traffic": SUMS_DRAM_PER_OP * (st.s1_ops + st.s2_ops),
        "traffic_basis": "ncu DRAM bytes per op of one sums_kernel launch at M(10^15), times this call's op count",
        "alg_bytes": alg,
        "ops": {"s1_lookups": st.s1_ops, "s1_compressed": st.s1_comp_ops, "s2_positions": st.s2_ops},
        "ops_per_s": (st.s1_ops + st.s2_ops) / t,
        "issue": {"bound": "instruction issue (binding)", "warp_inst": inst, "achieved": inst / t,
                  "peak": issue_peak, "unit": "warp instructions/s", "frac": inst / t / issue_peak,
                  "basis": f"{SUMS_INST_PER_S1} warp instructions per S1 lookup + {SUMS_INST_PER_S2} per S2 "
                           f"position (ncu at M(10^15)); peak = SMs x 4 x {f_mhz:.0f} MHz"},
    }


def sieve_roofline(p, tab_ms, peak, peaks_int, issue_peak, sms):
    """Table phase against its binding unit (instruction issue), the shared-memory
    atomics it issues, and HBM on the table's algorithmic bytes."""
    t = tab_ms / 1e3
    seg = 1 << (p.segment_log2 or 18)
    marks = sieve_marks(p.u_total, p.u_dense, sms, seg)
    tbytes = 2 * p.u_dense + 0.3125 * (p.u_total - p.u_dense) + p.mu_limit / 4
    inst = SIEVE_INST_PER_VALUE * p.u_total
    return {
        "kernel": "sieve_kernel (whole table phase: sieve, bucket, scan and fixup launches)",
        "bound": "instruction issue", "achieved": inst / t, "peak": issue_peak, "unit": "warp instructions/s",
        "frac": inst / t / issue_peak,
        "basis": f"{SIEVE_INST_PER_VALUE} warp instructions per table value (ncu, odd-mode sieve on the "
                 f"M(10^15) table); peak = SMs x 4 x the median SM clock of the timed region",
        "atomics": {"marks": marks, "achieved": marks / t, "peak": peaks_int["smem_atomic_per_s"],
                    "peak_sieve_pattern": peaks_int["smem_atomic_stride_per_s"], "unit": "atomics/s",
                    "frac": marks / t / peaks_int["smem_atomic_per_s"],
                    "frac_of_sieve_pattern": marks / t / peaks_int["smem_atomic_stride_per_s"],
                    "peak_kind": "measured on this GPU by dr_measure_peaks (synthetic kernels)"},
        "hbm": {"bytes": tbytes, "achieved": tbytes / t / 1e9, "peak": peak, "unit": "GB/s",
                "frac": tbytes / t / 1e9 / peak},
    }


def run_table_only(args, eng, stream):
    """Time the table build alone (sieve + prefix + compressed tier): --table u_total[,u_dense[,mu_limit]]."""
    import torch

    import dr_b200

    parts = [int(float(v)) for v in args.table.split(",")]
    ut = parts[0]
    ud = parts[1] if len(parts) > 1 else min(ut, 7600000000)
    ml = parts[2] if len(parts) > 2 else min(ut, 135001000)
    tun = dr_b200.Params(segment_log2=args.seg, block_threads=args.block)
    for _ in range(args.warmup):
        eng.table_build(ut, ud, ml, tun)
    ms = []
    for _ in range(args.steps):
        ms.append(eng.table_build(ut, ud, ml, tun).table_ms)
    torch.cuda.synchronize()
    out_bytes = 2 * ud + 20 * ((ut - ud + 63) // 64) + 16 * (ml // 192 + 2)
    t = statistics.median(ms) / 1e3
    peak, kind = load_peaks()
    print(json.dumps({"metric": "table build", "u_total": ut, "u_dense": ud, "mu_limit": ml, "seg_log2": args.seg,
                      "block": args.block, "ms": t * 1e3, "values_per_s": ut / t,
                      "write_GBps": out_bytes / t / 1e9, "hbm_frac": out_bytes / t / 1e9 / peak, "peak_kind": kind}))


def run_engine(args, world, rank, local):
    import torch

    import dr_b200

    torch.cuda.set_device(local)
    stream = torch.cuda.current_stream()
    eng = dr_b200.Engine(local, stream.cuda_stream)
    if args.table:
        run_table_only(args, eng, stream)
        eng.close()
        return
    X = int(float(args.x)) if "e" in str(args.x) else int(args.x)
    want = KNOWN.get(X)
    tuned = dr_b200.default_params(X, dr_b200.POLICY_REFERENCE if args.policy == "reference" else dr_b200.POLICY_GPU)
    default = dr_b200.default_params(X, dr_b200.POLICY_REFERENCE)
    if args.u:
        tuned = with_table_size(tuned, X, int(float(args.u)))
    streamed = None
    if args.resident:
        # streamed table: M held up to the resident limit, the rest sieved band by band
        streamed = {"u_resident": int(float(args.resident)), "band_values": int(float(args.band or 0))}
        eng.set_resident_limit(streamed["u_resident"], streamed["band_values"])

    def check(m):
        if want is not None and m != want:
            raise SystemExit(f"M({X}) mismatch: {m} != {want}")

    def timed(p, steps, clocks=None):
        """Device time (CUDA events on the engine's stream) and host time per call."""
        barrier(world)
        torch.cuda.synchronize()
        if clocks:
            clocks.start()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        stats = []
        host_t0 = time.perf_counter()
        ev0.record(stream)
        for _ in range(steps):
            r = eng.mertens(X, p)
            stats.append(r.stats)
            check(r.M)
        ev1.record(stream)
        torch.cuda.synchronize()
        host_dt = time.perf_counter() - host_t0
        barrier(world)
        if clocks:
            clocks.stop()
        dev = max_over_ranks(ev0.elapsed_time(ev1) / 1e3, world) / steps
        host = max_over_ranks(host_dt, world) / steps
        return dev, host, stats

    # ceilings of the units the kernels are bound by (shared atomics, IMAD, DFMA),
    # measured here on this GPU before anything is timed
    peaks_int = dr_b200.measure_peaks(local)
    # warm-up (also the correctness gate)
    for _ in range(args.warmup):
        check(eng.mertens(X, tuned).M)
    clocks = ClockSampler(local)
    sec_per, host_per, stats = timed(tuned, args.steps, clocks)
    value = sec_per / world  # whole job: N replicas finish N results in sec_per

    if streamed:
        eng.set_resident_limit(0)  # the comparison arms hold their tables whole
    # the plain path with the reference's default parameters, same run
    dsec = dhost = None
    if not args.no_compare:
        check(eng.mertens(X, default).M)
        dsec, dhost, dstats = timed(default, max(1, args.steps // 2))

    # the learned tuner's proposal (committed weights), same run
    learned = None
    wpath = os.path.join(ROOT, "deleglise-rivat_b200", "dr_b200", "tuner_weights.json")
    if os.path.exists(wpath) and not args.no_compare:
        import numpy as np

        mlp = dr_b200.MLP(eng)
        with open(wpath) as f:
            mlp.set_weights(np.array(json.load(f)["weights"], dtype=np.float32))
        _, hbm = dr_b200.device_info(local)
        lp, fb = mlp.propose(X, int(hbm * 0.9), 148, 1)
        check(eng.mertens(X, lp).M)
        lsec, _, _ = timed(lp, max(1, args.steps // 2))
        learned = {"ms_per_step": lsec * 1e3, "u_total": lp.u_total, "cx": lp.cx, "segment_log2": lp.segment_log2,
                   "fallback": fb, "speedup_vs_default": dsec / lsec}
        mlp.close()

    tab = statistics.mean(s.table_ms for s in stats)
    plan = statistics.mean(s.plan_ms for s in stats)
    sums = statistics.mean(s.sums_ms for s in stats)
    launches = sum(s.kernel_launches for s in stats)

    # batched config (256 uneven X in one table build + one persistent launch)
    batch = None
    if not args.no_batch:
        xs = batch_inputs()

        def batch_time(bp, reps=3):
            """(replay seconds per batch, results, replay stats, first-call seconds):
            the first call of a new batch runs eagerly and captures the graph (host
            wall time, synchronised); identical calls then replay it."""
            torch.cuda.synchronize()
            f0 = time.perf_counter()
            got, _ = eng.mertens_batch(xs, bp)  # eager run; captures the graph
            torch.cuda.synchronize()
            first = time.perf_counter() - f0
            t0 = torch.cuda.Event(enable_timing=True)
            t1 = torch.cuda.Event(enable_timing=True)
            t0.record(stream)
            for _ in range(reps):
                got, bst = eng.mertens_batch(xs, bp)  # graph replays
            t1.record(stream)
            torch.cuda.synchronize()
            return t0.elapsed_time(t1) / 1e3 / reps, got, bst, first

        untuned_s, _, _, _ = batch_time([dr_b200.default_params(x, dr_b200.POLICY_GPU) for x in xs])
        tt0 = time.perf_counter()
        bp, _ = eng.autotune_batch(xs, 24)
        tune_s = time.perf_counter() - tt0
        bs, got, bst, first_s = batch_time(bp)
        # baseline: 256 sequential plain single-query calls with default parameters
        s0 = torch.cuda.Event(enable_timing=True)
        s1 = torch.cuda.Event(enable_timing=True)
        s0.record(stream)
        seq = [eng.mertens(x).M for x in xs]
        s1.record(stream)
        torch.cuda.synchronize()
        ss = s0.elapsed_time(s1) / 1e3
        if seq != got:
            raise SystemExit("batched and single-query results differ")
        kern_ms = bst.table_ms + bst.plan_ms + bst.sums_ms
        batch = {"queries": len(xs), "M_per_s": len(xs) / bs, "s_per_batch": bs,
                 "replay_M_per_s": len(xs) / bs, "first_call_s": first_s,
                 "first_call_M_per_s": len(xs) / first_s,
                 "sequential_plain_M_per_s": len(xs) / ss, "speedup_vs_sequential": ss / bs,
                 "untuned_batch_M_per_s": len(xs) / untuned_s, "launches_per_batch": bst.kernel_launches,
                 "replay_kernel_ms": kern_ms, "replay_gap_ms": bs * 1e3 - kern_ms,
                 "cuda_graph": True,
                 "autotune": {"seconds": tune_s, "u_total": bp[0].u_total, "cx": bp[0].cx,
                              "segment_log2": bp[0].segment_log2, "block_threads": bp[0].block_threads,
                              "chunk_log2": bp[0].chunk_log2},
                 "seed": BATCH_SEED, "X": "round(10**U), U~U(9,14)"}

    peak, peak_kind = load_peaks()
    s0_ = stats[0]
    phases = {"table_ms": tab, "plan_ms": plan, "sums_ms": sums}
    if streamed:  # both within sums_ms
        phases.update({"band_table_ms": statistics.mean(s.band_table_ms for s in stats),
                       "band_sums_ms": statistics.mean(s.band_sums_ms for s in stats), "bands": stats[0].bands})
    clk = clocks.summary()
    sms = torch.cuda.get_device_properties(local).multi_processor_count
    # issue ceiling: 4 warp instructions per SM and clock at the median SM clock
    # sampled during the timed region (the maximum clock where none was sampled)
    f_mhz = clk["sm_mhz"] or clk["sm_max_mhz"] or 1965.0
    issue_peak = sms * 4 * f_mhz * 1e6
    roofline = sums_roofline(s0_, sums, peak, peak_kind, issue_peak, f_mhz)
    # a streamed table's bands are built inside the sums phase: no table-phase roofline
    table_roofline = None if streamed else sieve_roofline(tuned, tab, peak, peaks_int, issue_peak, sms)
    line = {
        "metric": "sec per M(10^16)" if X == X_HEADLINE else f"sec per M({X})", "value": value, "unit": "s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": sec_per * 1e3,
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "int64",
        "data": f"synthetic (the single input X={X})",
        "config": {"workload": f"M({X}), {args.policy} (tuned) parameters", "X": X, "u_total": tuned.u_total,
                   "u_dense": tuned.u_dense, "cx": tuned.cx, "mu_limit": tuned.mu_limit,
                   "l2": "inputs larger than L2 (table and reciprocals rebuilt each step)",
                   "parallelism": f"replicas x{world}"},
        "phases_ms": phases,
        "default_params": None if dsec is None else {"ms_per_step": dsec * 1e3, "u_total": default.u_total,
                                                     "cx": default.cx, "tuned_speedup": dsec / sec_per, "e2e_s": dhost},
        "stream": streamed,
        "learned_tuner": learned,
        "gpu_launches": launches,
        "e2e": {"value": host_per / world, "unit": "s", "h2d_bytes_per_step": int(s0_.h2d_bytes),
                "d2h_bytes_per_step": int(s0_.d2h_bytes)},
        "roofline": roofline,
        "table_roofline": table_roofline,
        "int_peaks": peaks_int,
        "clocks": clk,
        "batched": batch,
    }
    if rank == 0 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_reference_sample()
    if rank == 0:
        print(json.dumps(line))
    eng.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["engine", "reference"], default="engine")
    ap.add_argument("--policy", choices=["reference", "gpu"], default="gpu",
                    help="parameters of the timed path (the reference's defaults are always timed beside it)")
    ap.add_argument("--x", default="1e16", help="X of the single-query workload (profiling cases)")
    ap.add_argument("--table", default=None, help="time the table build only: u_total[,u_dense[,mu_limit]]")
    ap.add_argument("--seg", type=int, default=0, help="sieve segment = 2^seg values (0: default)")
    ap.add_argument("--block", type=int, default=0, help="sieve threads per CTA (0: default)")
    ap.add_argument("--u", default=None, help="table size u_total (dense tier and mu_limit by the B200 policy's rule)")
    ap.add_argument("--resident", default=None, help="stream the table above this many values (dr_ctx_set_resident_limit)")
    ap.add_argument("--band", default=None, help="values per streamed band (0: the resident compressed tier's size)")
    ap.add_argument("--no-compare", action="store_true", help="skip the default-parameter and learned-tuner arms")
    ap.add_argument("--no-batch", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    world, rank, local = dist_setup()
    try:
        if args.impl == "reference":
            run_reference(args, world, rank)
        else:
            run_engine(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
