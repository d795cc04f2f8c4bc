"""CPU: the bands of a streamed table (host logic of the library, no GPU).

Under a resident limit the table keeps M up to u_res -- the dense tier and whole
compressed segments of the full table's layout, at least one -- and the compressed tier
above is built in bands of whole segments, the last one ending at u_total.  The bands must
cover (u_res, u_total] once, in order; a band sieved in odd mode must find every half
floor(v/2) of its even values in the resident compressed tier, (u_dense, u_res].
"""
import random

import dr_b200


def _check(u_total, u_dense, lg, u_resident, band_values):
    S = 1 << lg
    u_res, bands = dr_b200.stream_plan(u_total, u_dense, lg, u_resident, band_values)
    if not bands:
        # nothing streams: no limit, a table within it, or no whole segment to leave out
        assert u_res == u_total
        assert u_resident <= 0 or u_total <= u_resident or u_dense + max(1, (u_resident - u_dense) // S) * S >= u_total
        return 0
    assert (u_res - u_dense) % S == 0 and u_res - u_dense >= S
    assert u_res <= max(u_resident, u_dense + S)
    assert u_res < u_total
    width = max(1, band_values // S) * S if band_values > 0 else u_res - u_dense
    lo = u_res
    for i, (vlo, vhi, odd) in enumerate(bands):
        assert vlo == lo and vhi > vlo
        if i + 1 < len(bands):
            assert vhi - vlo == width
        else:
            assert vhi == u_total and vhi - vlo <= width
        if odd:
            assert u_dense % 64 == 0
            first_half, last_half = (vlo + 2) // 2, vhi // 2
            assert u_dense < first_half and last_half + 64 <= u_res  # halves in resident words
        lo = vhi
    assert lo == u_total
    return len(bands)


def test_stream_plan_cases():
    # the configurations the GPU tests and the int64-max measurement use
    assert _check(42696448, 10674176, 14, 20000000, 1 << 16) > 100
    assert _check(5379446016, 128000000, 18, 3 * 10**9, 10**9) == 3
    u_res, bands = dr_b200.stream_plan(5379446016, 128000000, 18, 3 * 10**9, 10**9)
    assert all(odd for _, _, odd in bands)  # every half below 3e9
    assert _check(10**12, 4 * 10**9, 18, 2.5e11, 6.4e10) == 12
    u_res, bands = dr_b200.stream_plan(10**12, 4 * 10**9, 18, int(2.5e11), int(6.4e10))
    assert [odd for _, _, odd in bands][:3] == [True, True, True] and not bands[4][2]
    # nothing streams: no limit, or a table within the limit
    assert _check(10**9, 10**6, 18, 0, 0) == 0
    assert _check(10**9, 10**6, 18, 2 * 10**9, 0) == 0


def test_stream_plan_random():
    rng = random.Random(20261204)
    for _ in range(400):
        lg = rng.choice([12, 13, 14, 16, 17, 18])
        u_dense = rng.randint(0, 10**8) // 64 * 64 if rng.random() < 0.8 else rng.randint(0, 10**8)
        u_total = u_dense + rng.randint(1, 3 * 10**9)
        u_resident = rng.randint(0, u_total + 10**6)
        band = rng.choice([0, 1, rng.randint(1, 10**9)])
        _check(u_total, u_dense, lg, u_resident, band)
