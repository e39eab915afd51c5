"""Cases driver, host-only parts: combining per-case results the way the
reference's per-line runs combine, and reading the resume journal (including
a last line cut short by a crash, and a journal that belongs to other
cases)."""
import ctypes as C

import pytest


def _res(h, seeds, E, Es, st, sts, ov=()):
    import collatz_b200 as cb
    r = cb.CaseResultC()
    r.hash, r.seeds_checked, r.launches, r.pairs, r.n_overflow = h, seeds, 2, 10, len(ov)
    for i in range(4):
        r.max_excursion[i] = (E >> (32 * i)) & 0xFFFFFFFF
        r.max_excursion_seed[i] = (Es >> (32 * i)) & 0xFFFFFFFF
        r.max_stopping_time_seed[i] = (sts >> (32 * i)) & 0xFFFFFFFF
    r.max_stopping_time = st
    buf = (C.c_uint32 * (4 * max(1, len(ov))))()
    for j, s in enumerate(ov):
        for i in range(4):
            buf[4 * j + i] = (s >> (32 * i)) & 0xFFFFFFFF
    r.overflow_seeds = C.cast(buf, C.POINTER(C.c_uint32))
    r.overflow_cap = len(ov)
    return r, buf


def test_combine_case_results():
    import collatz_b200 as cb
    parts = [_res(0x1234, 100, 5000, 77, 90, 41, ov=[1 << 70, 5]),
             _res(0xFF00, 50, 5000, 33, 120, 99),         # same E, smaller seed wins
             _res(0x0001, 0, 0, 0, 0, 0),                 # an empty case
             _res(0x00F0, 7, 4000, 11, 120, 12, ov=[9])]  # same sigma, smaller seed wins
    arr = (cb.CaseResultC * 4)(*[p[0] for p in parts])
    out = cb.CaseResultC()
    ovb = (C.c_uint32 * 64)()
    out.overflow_seeds = C.cast(ovb, C.POINTER(C.c_uint32))
    out.overflow_cap = 16
    assert cb.lib().collatz_combine_case_results(arr, 4, C.byref(out)) == 0
    r = cb._case_result(out, ovb, 16)
    assert r.hash == 0x1234 ^ 0xFF00 ^ 0x0001 ^ 0x00F0
    assert (r.seeds_checked, r.launches, r.pairs, r.n_overflow) == (157, 8, 40, 3)
    assert (r.max_excursion, r.max_excursion_seed) == (5000, 33)
    assert (r.max_stopping_time, r.max_stopping_time_seed) == (120, 12)
    assert r.overflow == [5, 9, 1 << 70]


def _line(i, t, h, seeds, end=True):
    base, sf, tp, num, de, ne = t
    fields = ["case", i, base & (2**64 - 1), base >> 64, sf, tp, num & (2**64 - 1), num >> 64, de, ne, h, seeds,
              3, 4, 0, 1] + [7, 0, 0, 0] + [base, 0, 0, 0] + [55] + [base, 0, 0, 0] + [0, "1.5", 1, 99, 0, 0, 0]
    s = " ".join(str(x) for x in fields)
    return s + (" end\n" if end else "\n")


def test_journal_load(tmp_path):
    import collatz_b200 as cb
    cases = [(27, 10, 8, 183, 0, 0), (283, 10, 8, 1823, 2, 1), (795, 11, 9, 7655, 2, 1)]
    j = tmp_path / "j.txt"
    assert cb.journal_load(str(j), cases) == {}  # no journal yet
    j.write_text(_line(0, cases[0], 111, 1000) + _line(2, cases[2], 333, 3000)
                 + _line(1, cases[1], 222, 2000, end=False)[:40])  # a write cut short
    got = cb.journal_load(str(j), cases)
    assert sorted(got) == [0, 2]
    assert (got[0].hash, got[0].seeds_checked, got[2].hash, got[2].seeds_checked) == (111, 1000, 333, 3000)
    assert got[0].overflow == [99] and got[0].max_stopping_time == 55 and got[0].max_excursion == 7
    # a journal written for other cases is refused
    other = [(27, 10, 8, 184, 0, 0)] + cases[1:]
    with pytest.raises(cb.CollatzError) as e:
        cb.journal_load(str(j), other)
    assert e.value.status == cb.E_STATE
