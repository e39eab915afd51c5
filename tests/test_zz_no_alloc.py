"""collatz_verify_pairs_noalloc, the entry point for callers that cannot
allocate memory while they verify (their device buffers come from their own
pool, or their loop may not call cudaMalloc/cudaFree): called through the C ABI
with pairs already in device memory, it must give the same result as
collatz_verify_pairs, twice in a row (its scratch array keeps the previous
call's contents and has to be cleared by each call).

This file is named so that pytest collects it last."""
import ctypes as C

import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu

NOALLOC_OVERFLOW_MAX = 4064


def _lib():
    import collatz_b200 as cb
    L = cb.lib()
    f = L.collatz_verify_pairs_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32, C.POINTER(cb.CaseResultC)]
    return cb, f


def _noalloc(cb, f, v, bigindex, dev_pairs, npairs, cap):
    out = cb.CaseResultC()
    ov = (C.c_uint32 * (4 * max(1, cap)))()
    out.overflow_seeds = C.cast(ov, C.POINTER(C.c_uint32))
    out.overflow_cap = cap
    rc = f(v.handle, bigindex, C.c_void_p(dev_pairs), npairs, C.byref(out))
    return rc, cb._case_result(out, ov, cap)


def _key(r):
    return (r.hash, r.seeds_checked, r.launches, r.pairs, r.cpu_pairs, r.n_overflow, sorted(r.overflow),
            r.max_excursion, r.max_excursion_seed, r.max_stopping_time, r.max_stopping_time_seed, r.errors)


def test_noalloc_matches_verify_pairs_twice():
    import torch
    cb, f = _lib()
    v = cb.Verifier(45)
    fx = load_golden("pairs_N45.json")
    batches = [b for b in fx["batches"] if len(b["overflow"]) <= NOALLOC_OVERFLOW_MAX]
    assert any(b["overflow"] for b in batches)
    for b in batches:
        pairs = [(int(x), int(y)) for x, y in b["pairs"]]
        ref = v.launchkernel(b["bigindex"], pairs)
        packed = cb.pack_pairs(pairs)
        dev = torch.tensor(list(packed), dtype=torch.int64).to(torch.int32).cuda()
        torch.cuda.synchronize()
        for _ in range(2):
            rc, got = _noalloc(cb, f, v, b["bigindex"], dev.data_ptr(), len(pairs), NOALLOC_OVERFLOW_MAX)
            assert rc == 0
            assert _key(got) == _key(ref), (b["kind"], b["bigindex"])
            assert f"{got.hash:X}" == b["hash"]
    v.close()


def test_noalloc_rejects_oversized_report():
    import torch
    cb, f = _lib()
    v = cb.Verifier(26)
    dev = torch.zeros(8, dtype=torch.int32, device="cuda")
    rc, _ = _noalloc(cb, f, v, 0, dev.data_ptr(), 1, NOALLOC_OVERFLOW_MAX + 1)
    assert rc == cb.E_LIMIT
    assert "4064" in cb.lib().collatz_last_error(v.handle).decode()
    v.close()


def test_noalloc_small_cap_returns_the_smallest_seeds():
    """With an overflow_cap of 1 or 2 and more overflow seeds than that, both
    entry points return the smallest seeds, twice in a row."""
    import torch
    cb, f = _lib()
    v = cb.Verifier(45)
    fx = load_golden("pairs_N45.json")
    batches = [b for b in fx["batches"] if 2 < len(b["overflow"]) <= NOALLOC_OVERFLOW_MAX]
    assert batches
    for b in batches[:2]:
        pairs = [(int(x), int(y)) for x, y in b["pairs"]]
        packed = cb.pack_pairs(pairs)
        dev = torch.tensor(list(packed), dtype=torch.int64).to(torch.int32).cuda()
        torch.cuda.synchronize()
        for cap in (1, 2):
            ref = v.launchkernel(b["bigindex"], pairs, overflow_cap=cap)
            assert ref.n_overflow == len(b["overflow"]) > cap
            for _ in range(2):
                rc, got = _noalloc(cb, f, v, b["bigindex"], dev.data_ptr(), len(pairs), cap)
                assert rc == 0
                assert got.overflow == ref.overflow and len(got.overflow) == cap
                assert _key(got) == _key(ref)
    v.close()


def test_noalloc_rejects_null_report_buffer():
    import torch
    cb, f = _lib()
    v = cb.Verifier(26)
    dev = torch.zeros(8, dtype=torch.int32, device="cuda")
    out = cb.CaseResultC()
    out.overflow_cap = 4
    rc = f(v.handle, 0, C.c_void_p(dev.data_ptr()), 1, C.byref(out))
    assert rc == cb.E_ARG
    v.close()
