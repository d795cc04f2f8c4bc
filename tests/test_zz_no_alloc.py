"""GPU: the table build that allocates nothing (dr_table_build_noalloc).

Some callers cannot let this library call cudaMalloc: their device memory
belongs to their own allocator (here torch's caching allocator stands in for
it), or they must not allocate once they are serving.  They allocate the table
buffers themselves and the build keeps its scratch in a fixed array inside
libdrb200.so.  This test calls that entry point through the C ABI twice in a
row with different sizes (the second smaller, so stale scratch or stale
buffer contents would show) and checks each table bit for bit against the one
the allocating entry point dr_table_build() produces.  The file sorts last so
that a run stopping at the first failure has run every other test already.
"""
import ctypes

import numpy as np
import pytest

import dr_b200

pytestmark = pytest.mark.gpu

# the last case has its dense cutoff on a 64-value word: the allocating build then
# sieves most segments on their odd values (halves from earlier launches) while the
# no-alloc build sieves every value
CASES = [(300000007, 40000003, 5000000), (1000033, 1024, 1000033), (300000007, 40000000, 5000000)]


def _wheel_mu(words, n):
    m = n // 6
    five = (n % 6) == 5
    g, b = m >> 5, (m & 31).astype(np.uint32)
    w = words.view(np.uint32).reshape(-1, 4)
    nz = np.where(five, w[g, 2], w[g, 0])
    ng = np.where(five, w[g, 3], w[g, 1])
    bit_nz = (nz >> b) & 1
    bit_ng = (ng >> b) & 1
    return (bit_nz.astype(np.int8) * (1 - 2 * bit_ng.astype(np.int8))).astype(np.int8)


def _compressed_M(planes, ckpt, ud, ut):
    off = np.arange(ut - ud, dtype=np.int64)
    w = off >> 6
    mask = np.uint64(0xFFFFFFFFFFFFFFFF) >> (np.uint64(63) - (off & 63).astype(np.uint64))
    pw = planes.view(np.uint64).reshape(-1, 2)
    nz = np.bitwise_count(pw[w, 0] & mask).astype(np.int64)
    ng = np.bitwise_count(pw[w, 1] & mask).astype(np.int64)
    return (ckpt[w].astype(np.int64) + nz - 2 * ng).astype(np.int32)


def test_noalloc_table_matches_allocating_build():
    import torch

    f = dr_b200.lib().dr_table_build_noalloc
    eng = dr_b200.Engine(0)
    stream = torch.cuda.current_stream()
    for ut, ud, ml in CASES:
        W = (ut - ud + 63) // 64
        G = ml // 192 + 2
        dM = torch.empty(max(ud, 8), dtype=torch.int16, device="cuda")
        planes = torch.empty(max(2 * W, 2), dtype=torch.int64, device="cuda")
        ckpt = torch.empty(max(W, 1), dtype=torch.int32, device="cuda")
        wheel = torch.full((4 * G,), -1, dtype=torch.int32, device="cuda")  # the call must clear it
        rc = f(0, ctypes.c_void_p(stream.cuda_stream), ut, ud, ml, ctypes.c_void_p(dM.data_ptr()),
               ctypes.c_void_p(planes.data_ptr()), ctypes.c_void_p(ckpt.data_ptr()), ctypes.c_void_p(wheel.data_ptr()))
        assert rc == 0, dr_b200.lib().dr_last_error().decode()
        torch.cuda.synchronize()
        dM_h = dM.cpu().numpy()[:ud]
        planes_h = planes.cpu().numpy()[: 2 * W]
        ckpt_h = ckpt.cpu().numpy()[:W]
        wheel_h = wheel.cpu().numpy()

        eng.table_build(ut, ud, ml)  # the allocating entry point, same limits
        ref = eng.table_checksums()
        n = np.arange(1, ud + 1, dtype=np.uint64)
        d64 = dM_h.astype(np.int64).astype(np.uint64)
        k = np.arange(W, dtype=np.uint64) * np.uint64(2) + np.uint64(1)
        pw = planes_h.view(np.uint64).reshape(-1, 2)
        with np.errstate(over="ignore"):
            mine = (int(d64.sum(dtype=np.uint64)), int((d64 * (np.uint64(2) * n + np.uint64(1))).sum(dtype=np.uint64)),
                    int((pw[:, 0] * k).sum(dtype=np.uint64)), int((pw[:, 1] * k).sum(dtype=np.uint64)),
                    int((ckpt_h.astype(np.int64).astype(np.uint64) * k).sum(dtype=np.uint64)))
        assert mine == (ref[0], ref[1], ref[3], ref[4], ref[5]), (ut, ud, ml)

        # Mobius wheel, every n <= mu_limit coprime to 6
        nn = np.arange(1, ml + 1, dtype=np.int64)
        cop = (nn % 2 == 1) & (nn % 3 != 0)
        want = eng.table_read_wheel(1, ml)
        assert np.array_equal(_wheel_mu(wheel_h, nn[cop]), want[cop]), (ut, ud, ml)

        # M(n) element by element: all of the small case, samples of the large one
        if ut <= 2_000_000:
            M_ref, _ = eng.table_read(0, ut + 1)
            M = np.concatenate([[0], dM_h.astype(np.int32), _compressed_M(planes_h, ckpt_h, ud, ut)])
            assert np.array_equal(M, M_ref)
        else:
            M_ref, _ = eng.table_read(1, 200000)
            assert np.array_equal(dM_h[:200000].astype(np.int32), M_ref)
            M_ref, _ = eng.table_read(ut - 199999, 200000)
            assert np.array_equal(_compressed_M(planes_h, ckpt_h, ud, ut)[-200000:], M_ref)
    eng.close()


def test_noalloc_at_its_size_limit():
    """u_total = DR_NOALLOC_MAX_U = 2^33 with a small dense tier (about 2.7 GB of
    caller buffers): 65,537 segments of scratch sums, all 8,952 sieving primes up to
    92,681 and squares p^2 above 2^32 -- the upper bounds of the fixed scratch.  The
    table checksums and sampled M(n) windows equal dr_table_build's at the same limits."""
    import torch

    f = dr_b200.lib().dr_table_build_noalloc
    ut, ud, ml = 1 << 33, 1 << 20, 3000000
    W = (ut - ud + 63) // 64
    G = ml // 192 + 2
    dM = torch.empty(ud, dtype=torch.int16, device="cuda")
    planes = torch.empty(2 * W, dtype=torch.int64, device="cuda")
    ckpt = torch.empty(W, dtype=torch.int32, device="cuda")
    wheel = torch.full((4 * G,), -1, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream()
    rc = f(0, ctypes.c_void_p(stream.cuda_stream), ut, ud, ml, ctypes.c_void_p(dM.data_ptr()),
           ctypes.c_void_p(planes.data_ptr()), ctypes.c_void_p(ckpt.data_ptr()), ctypes.c_void_p(wheel.data_ptr()))
    assert rc == 0, dr_b200.lib().dr_last_error().decode()
    torch.cuda.synchronize()
    # the checksums of dr_table_sums, computed on the device (int64 arithmetic wraps mod 2^64)
    mask = (1 << 64) - 1
    n = torch.arange(1, ud + 1, dtype=torch.int64, device="cuda")
    d64 = dM.to(torch.int64)
    k = torch.arange(W, dtype=torch.int64, device="cuda") * 2 + 1
    pw = planes.view(-1, 2)
    mine = (int(d64.sum()) & mask, int((d64 * (2 * n + 1)).sum()) & mask, int((pw[:, 0] * k).sum()) & mask,
            int((pw[:, 1] * k).sum()) & mask, int((ckpt.to(torch.int64) * k).sum()) & mask)
    del n, d64, k, pw
    dM_h = dM.cpu().numpy()
    tail = 200000
    planes_t = planes[-2 * ((tail + 63) // 64 + 1):].cpu().numpy()
    ckpt_t = ckpt[-((tail + 63) // 64 + 1):].cpu().numpy()
    wheel_h = wheel.cpu().numpy()
    del dM, planes, ckpt, wheel
    torch.cuda.empty_cache()

    eng = dr_b200.Engine(0)
    try:
        eng.table_build(ut, ud, ml)
        ref = eng.table_checksums()
        assert mine == (ref[0], ref[1], ref[3], ref[4], ref[5])
        M_ref, _ = eng.table_read(1, 100000)
        assert np.array_equal(dM_h[:100000].astype(np.int32), M_ref)
        # the last values of the compressed tier: the planes and checkpoints of the tail words
        wt = len(ckpt_t)
        first_word = W - wt
        off0 = first_word * 64
        M_tail = _compressed_M(planes_t, ckpt_t, ud + off0, ut)
        M_ref, _ = eng.table_read(ut - tail + 1, tail)
        assert np.array_equal(M_tail[-tail:], M_ref)
        nn = np.arange(1, ml + 1, dtype=np.int64)
        cop = (nn % 2 == 1) & (nn % 3 != 0)
        assert np.array_equal(_wheel_mu(wheel_h, nn[cop]), eng.table_read_wheel(1, ml)[cop])
    finally:
        eng.close()
