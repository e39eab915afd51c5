"""ctypes wrapper of the CPU oracle (oracle/collatz_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
cpu_baseline / reference legs of bench.py, always as the checker.  The
product package collatz_b200 never imports this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "collatz_oracle.c")
LIB = os.path.join(HERE, "_build", "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")

U128 = int


def build(force: bool = False) -> str:
    """Compile the oracle with gcc into oracle/_build/liboracle.so."""
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    hdr = os.path.join(HERE, "collatz_oracle.h")
    if not force and os.path.exists(LIB):
        mt = os.path.getmtime(LIB)
        if mt >= os.path.getmtime(SRC) and mt >= os.path.getmtime(hdr):
            return LIB
    # a private temporary per process: concurrent builders (e.g. two ranks of
    # a multi-process test) each rename a complete library into place
    tmp = f"{LIB}.tmp{os.getpid()}"
    subprocess.check_call(["gcc", "-std=gnu11", "-O2", "-fPIC", "-shared", "-pthread",
                           "-Wall", "-o", tmp, SRC])
    os.replace(tmp, LIB)
    return LIB


class _Tables(C.Structure):
    _fields_ = [("maxbits", C.c_uint32), ("mbi", C.c_uint32), ("tpo", C.c_uint32),
                ("magic", C.c_uint32 * 16), ("bv", C.POINTER(C.c_uint32)),
                ("mod9", (C.c_uint32 * 32) * 9)]


class _U128(C.Structure):
    # 128-bit values are stored as (lo, hi) u64 pairs in the C structs
    _fields_ = [("lo", C.c_uint64), ("hi", C.c_uint64)]


class _CaseResult(C.Structure):
    _fields_ = [("hash", C.c_uint32), ("seeds", C.c_uint64), ("pairs", C.c_uint64),
                ("cpu_pairs", C.c_uint64), ("launches", C.c_uint64),
                ("checkpoints", C.c_uint64), ("n_overflow", C.c_uint64),
                ("overflow", C.c_void_p), ("overflow_cap", C.c_uint64),
                ("max_exc", _U128), ("max_exc_seed", _U128), ("max_st", C.c_uint64),
                ("max_st_seed", _U128), ("seeds_done", C.c_uint64)]


class _RangeResult(C.Structure):
    _fields_ = [("seeds", C.c_uint64), ("failures", C.c_uint64),
                ("max_exc", C.c_uint32 * 16), ("max_exc_seed", C.c_uint32 * 4),
                ("max_st", C.c_uint64), ("max_st_seed", C.c_uint32 * 4),
                ("steps", C.c_uint64), ("odd_runs", C.c_uint64), ("even_runs", C.c_uint64),
                ("wide64", C.c_uint64)]


def _u128(x: _U128) -> int:
    return x.lo | (x.hi << 64)


def _limbs(arr) -> int:
    return sum(int(w) << (32 * i) for i, w in enumerate(arr))


_lib = None


def lib():
    global _lib
    if _lib is None:
        path = build()
        L = C.CDLL(path)
        # 128-bit values cross the boundary as (lo, hi) u64 pairs.
        L.orc_tables_init.argtypes = [C.POINTER(_Tables), C.c_uint32]
        L.orc_tables_free.argtypes = [C.POINTER(_Tables)]
        L.orc_case_result_init.argtypes = [C.POINTER(_CaseResult)]
        L.orc_pair.argtypes = [C.POINTER(_Tables), C.c_uint32, C.c_uint64, C.c_uint64,
                               C.c_uint64, C.c_uint64, C.c_int, C.POINTER(_CaseResult)]
        L.orc_pair.restype = C.c_uint32
        L.orc_run_case.argtypes = [C.POINTER(_Tables), C.c_uint64, C.c_uint64, C.c_uint32,
                                   C.c_uint32, C.c_uint64, C.c_uint64, C.c_uint32, C.c_uint32,
                                   C.POINTER(_CaseResult)]
        L.orc_search1.argtypes = [C.POINTER(_Tables), C.c_uint64, C.c_uint64, C.c_uint32,
                                  C.c_uint32, C.c_uint64, C.c_uint64, C.c_uint32, C.c_uint32,
                                  C.c_void_p, C.c_void_p]
        L.orc_split.argtypes = [C.POINTER(_Tables), C.c_uint64, C.c_uint64, C.c_uint32,
                                C.c_uint32, C.c_uint64, C.c_uint64, C.c_uint32, C.c_uint32,
                                C.c_uint32, C.c_void_p, C.c_void_p]
        L.orc_range.restype = C.c_int
        L.orc_range_sieve.argtypes = [C.c_uint32, C.c_void_p]
        L.orc_range_sieve.restype = C.c_uint64
        L.orc_range_sieve_validate.argtypes = [C.c_uint32]
        L.orc_range_sieve_validate.restype = C.c_uint64
        L.orc_range.argtypes = [C.c_uint64, C.c_uint64, C.c_uint64, C.c_uint32, C.c_int,
                                C.c_int, C.c_int, C.POINTER(_RangeResult)]
        L.orc_range_ex.restype = C.c_int
        L.orc_range_ex.argtypes = [C.c_uint64, C.c_uint64, C.c_uint64, C.c_uint32, C.c_int,
                                   C.c_int, C.c_int, C.c_int, C.POINTER(_RangeResult)]
        L.orc_trajectory.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p,
                                     C.c_void_p, C.c_void_p]
        _lib = L
    return _lib


def _split(x: int):
    return x & ((1 << 64) - 1), x >> 64


LEAF_CB = C.CFUNCTYPE(None, C.c_void_p, C.c_uint32, C.c_uint64, C.c_uint64, C.c_uint64,
                      C.c_uint64)
ROOT_CB = C.CFUNCTYPE(None, C.c_void_p, C.c_uint64, C.c_uint64, C.c_uint32, C.c_uint32,
                      C.c_uint64, C.c_uint64, C.c_uint32, C.c_uint32)


@dataclass
class CaseResult:
    hash: int
    seeds: int
    pairs: int
    cpu_pairs: int
    launches: int
    checkpoints: int
    overflow: list
    max_exc: int
    max_exc_seed: int
    max_st: int
    max_st_seed: int


class Tables:
    """Reference tables for one N (precompute, cu:423-495)."""

    def __init__(self, maxbits: int):
        self._t = _Tables()
        rc = lib().orc_tables_init(C.byref(self._t), maxbits)
        if rc:
            raise ValueError(f"orc_tables_init({maxbits}) = {rc}")
        self.maxbits = maxbits
        self.mbi = self._t.mbi
        self.tpo = self._t.tpo

    def __del__(self):
        try:
            lib().orc_tables_free(C.byref(self._t))
        except Exception:
            pass

    @property
    def magic(self):
        return list(self._t.magic)

    def bv_bytes(self) -> bytes:
        n = 16 * ((1 << 19) + 32)
        return C.string_at(self._t.bv, 4 * n)

    def mod9_bytes(self) -> bytes:
        return bytes(self._t.mod9)

    def _result(self, cap=1 << 16):
        buf = (C.c_uint64 * (2 * cap))()
        r = _CaseResult()
        r.overflow = C.cast(buf, C.c_void_p)
        r.overflow_cap = cap
        lib().orc_case_result_init(C.byref(r))
        return r, buf

    @staticmethod
    def _convert(r, buf) -> CaseResult:
        n = min(r.n_overflow, r.overflow_cap)
        ov = [buf[2 * i] | (buf[2 * i + 1] << 64) for i in range(n)]
        return CaseResult(r.hash, r.seeds, r.pairs, r.cpu_pairs, r.launches, r.checkpoints, ov,
                          _u128(r.max_exc), _u128(r.max_exc_seed), r.max_st,
                          _u128(r.max_st_seed))

    def run_case(self, base, sigfig, threepower, number, doubleeven, numevens) -> CaseResult:
        r, buf = self._result()
        rc = lib().orc_run_case(C.byref(self._t), *_split(base), sigfig, threepower,
                                *_split(number), doubleeven, numevens, C.byref(r))
        if rc:
            raise ValueError("sigfig > N - A")
        return self._convert(r, buf)

    def pairs_result(self, bigindex: int, pairs, cpu_sem: bool = False) -> CaseResult:
        """pairs: iterable of (base, number) ints.  Hash = XOR over pairs."""
        r, buf = self._result()
        h = 0
        for base, number in pairs:
            h ^= lib().orc_pair(C.byref(self._t), bigindex, *_split(base), *_split(number),
                                1 if cpu_sem else 0, C.byref(r))
        out = self._convert(r, buf)
        out.hash = h
        return out

    def leaves(self, base, sigfig, threepower, number, doubleeven, numevens):
        """Step-1 leaves [(bigindex, base, number)] in the reference's order."""
        out = []

        def cb(_ctx, bi, blo, bhi, nlo, nhi):
            out.append((bi, blo | (bhi << 64), nlo | (nhi << 64)))

        f = LEAF_CB(cb)
        rc = lib().orc_search1(C.byref(self._t), *_split(base), sigfig, threepower,
                               *_split(number), doubleeven, numevens,
                               C.cast(f, C.c_void_p), None)
        if rc:
            raise ValueError("sigfig > N - A")
        return out

    def split(self, base, sigfig, threepower, number, doubleeven, numevens, cut):
        out = []

        def cb(_ctx, blo, bhi, sf, tp, nlo, nhi, de, ne):
            out.append((blo | (bhi << 64), sf, tp, nlo | (nhi << 64), de, ne))

        f = ROOT_CB(cb)
        rc = lib().orc_split(C.byref(self._t), *_split(base), sigfig, threepower,
                             *_split(number), doubleeven, numevens, cut,
                             C.cast(f, C.c_void_p), None)
        if rc:
            raise ValueError("bad cut")
        return out


def split_case(maxbits: int, tup, cut: int):
    """Step-1 subtree roots at sigfig == cut (only N matters, no tables needed)."""
    t = _Tables()
    t.maxbits = maxbits
    t.mbi = maxbits - 10
    t.tpo = t.mbi * 306 // 485 + 1
    out = []

    def cb(_ctx, blo, bhi, sf, tp, nlo, nhi, de, ne):
        out.append((blo | (bhi << 64), sf, tp, nlo | (nhi << 64), de, ne))

    f = ROOT_CB(cb)
    base, sigfig, threepower, number, doubleeven, numevens = tup
    rc = lib().orc_split(C.byref(t), *_split(base), sigfig, threepower, *_split(number),
                         doubleeven, numevens, cut, C.cast(f, C.c_void_p), None)
    if rc:
        raise ValueError("bad cut")
    return out


def leaves(maxbits: int, tup):
    """Step-1 leaves [(bigindex, base, number)] (only N matters)."""
    t = _Tables()
    t.maxbits = maxbits
    t.mbi = maxbits - 10
    t.tpo = t.mbi * 306 // 485 + 1
    out = []

    def cb(_ctx, bi, blo, bhi, nlo, nhi):
        out.append((bi, blo | (bhi << 64), nlo | (nhi << 64)))

    f = LEAF_CB(cb)
    base, sigfig, threepower, number, doubleeven, numevens = tup
    rc = lib().orc_search1(C.byref(t), *_split(base), sigfig, threepower, *_split(number),
                           doubleeven, numevens, C.cast(f, C.c_void_p), None)
    if rc:
        raise ValueError("sigfig > N - A")
    return out


@dataclass
class RangeResult:
    seeds: int
    failures: int
    max_exc: int
    max_exc_seed: int
    max_st: int
    max_st_seed: int
    steps: int
    odd_runs: int
    even_runs: int
    wide64: int = 0


def range_verify(offset: int, size: int, k: int, use_mod9: bool = True, method: int = 1,
                 nthreads: int = 1, direct_sieve: bool | None = None,
                 negative: bool = False) -> RangeResult:
    """orc_range; direct_sieve None = the oracle's choice (table for small k);
    negative: the negative-integer variant T'(m) = (3m-1)/2, m/2."""
    r = _RangeResult()
    if direct_sieve is None and not negative:
        rc = lib().orc_range(*_split(offset), size, k, 1 if use_mod9 else 0, method, nthreads,
                             C.byref(r))
    else:
        flags = (1 if direct_sieve else 0) | (2 if negative else 0)
        rc = lib().orc_range_ex(*_split(offset), size, k, 1 if use_mod9 else 0, method, nthreads,
                                flags, C.byref(r))
    if rc:
        raise ValueError(f"orc_range rc={rc}")
    return RangeResult(r.seeds, r.failures, _limbs(r.max_exc), _limbs(r.max_exc_seed),
                       r.max_st, _limbs(r.max_st_seed), r.steps, r.odd_runs, r.even_runs, r.wide64)


def range_sieve(k: int) -> tuple[int, bytes]:
    nbytes = ((1 << k) + 7) // 8
    buf = (C.c_uint8 * nbytes)()
    n = lib().orc_range_sieve(k, buf)
    return int(n), bytes(buf)


def range_sieve_validate(k: int) -> int:
    return int(lib().orc_range_sieve_validate(k))


def trajectory(seeds, seed_limbs: int = 8):
    """Returns [(status, stopping_time, excursion)] per seed."""
    n = len(seeds)
    arr = (C.c_uint32 * (n * seed_limbs))()
    for i, s in enumerate(seeds):
        for j in range(seed_limbs):
            arr[i * seed_limbs + j] = (s >> (32 * j)) & 0xFFFFFFFF
    st = (C.c_uint64 * n)()
    exc = (C.c_uint32 * (16 * n))()
    status = (C.c_uint32 * n)()
    rc = lib().orc_trajectory(arr, n, seed_limbs, st, exc, status)
    if rc:
        raise ValueError("orc_trajectory")
    return [(int(status[i]), int(st[i]), _limbs(exc[16 * i:16 * i + 16])) for i in range(n)]
