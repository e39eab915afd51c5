"""collatz_b200 -- B200-native Collatz verifier (Python mirror of the C ABI).

The compute path is the CUDA library libcollatz_b200.so (include/collatz.h);
this module only marshals arguments through ctypes.  There is no CPU
fallback: if the library or a usable sm_100 device is missing, calls raise.

Reference interface mirrored (vigleik0/collatz, collatz_cudav7.cu):
  run_case(...)        main() on one stdin 6-tuple            (cu:95-183)
  launchkernel(...)    one batch of Step-1 pairs of a bucket  (cu:565-649)
  step1_pairs(...)     the leaves of search1                  (cu:497-563)
New entry modes: verify_range, verify_batch, trajectory, plans and the server.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libcollatz_b200.so")

OK = 0
E_ARG, E_CUDA, E_NOMEM, E_LIMIT, E_DEVICE, E_TIMEOUT, E_STATE, E_ADMISSION, E_NODEV = \
    -1, -2, -3, -4, -5, -6, -7, -8, -9
RANGE_NO_MOD9 = 0x1
RANGE_NEGATIVE = 0x2
VARIANT_AUTO = 0xFFFFFFFF
BV_WORDS = (1 << 19) + 32


class CollatzError(RuntimeError):
    def __init__(self, status: int, msg: str = ""):
        super().__init__(f"collatz status {status}: {msg}")
        self.status = status


class Config(C.Structure):
    _fields_ = [("maxbits", C.c_uint32), ("range_k", C.c_uint32), ("device", C.c_int32),
                ("variant", C.c_uint32), ("iter_cap", C.c_uint32), ("flags", C.c_uint32),
                ("reserved", C.c_uint32 * 10)]


CFG_HOST_STEP1 = 0x1  # collatz_run_case: Step 1 on the host threads instead of the device


class Case(C.Structure):
    _fields_ = [("base", C.c_uint64 * 2), ("sigfig", C.c_uint32), ("threepower", C.c_uint32),
                ("number", C.c_uint64 * 2), ("doubleeven", C.c_uint32), ("numevens", C.c_uint32)]


class CaseResultC(C.Structure):
    _fields_ = [("hash", C.c_uint32), ("spot_checks", C.c_uint32), ("launches", C.c_uint64),
                ("seeds_checked", C.c_uint64), ("pairs", C.c_uint64), ("cpu_pairs", C.c_uint64),
                ("n_overflow", C.c_uint64), ("overflow_seeds", C.POINTER(C.c_uint32)),
                ("overflow_cap", C.c_uint64), ("max_excursion", C.c_uint32 * 4),
                ("max_excursion_seed", C.c_uint32 * 4), ("max_stopping_time", C.c_uint64),
                ("max_stopping_time_seed", C.c_uint32 * 4), ("errors", C.c_uint32),
                ("reserved", C.c_uint32), ("device_ms", C.c_double)]


class Range(C.Structure):
    _fields_ = [("offset", C.c_uint64 * 2), ("size", C.c_uint64), ("k", C.c_uint32),
                ("flags", C.c_uint32)]


class RangeResultC(C.Structure):
    _fields_ = [("seeds_checked", C.c_uint64), ("failures", C.c_uint64), ("widened", C.c_uint64),
                ("max_excursion", C.c_uint32 * 8), ("max_excursion_seed", C.c_uint32 * 4),
                ("max_stopping_time", C.c_uint64), ("max_stopping_time_seed", C.c_uint32 * 4),
                ("errors", C.c_uint32), ("status", C.c_int32), ("device_ms", C.c_double)]


REQ_RANGE, REQ_TRAJECTORY = 0, 1
TUNE_RANGE, TUNE_CASES, TUNE_NO_CACHE = 0x1, 0x2, 0x4
# collatz_set_variant modes: cases kernel, four-limb range kernel, 64-bit range
# kernel, and the limb width (largest seed bit length run by the 64-bit kernel)
MODE_CASES, MODE_RANGE, MODE_RANGE64, MODE_RANGE64_BITS = 0, 1, 2, 3
RANGE64_BITS_DEFAULT = 48


class TuneResultC(C.Structure):
    _fields_ = [("range_variant", C.c_int32), ("cases_variant", C.c_int32),
                ("range_ms", C.c_float * 8), ("cases_ms", C.c_float * 8),
                ("range64_variant", C.c_int32), ("range64_bits", C.c_uint32),
                ("range64_ms", C.c_float * 8), ("width_ms", C.c_float * 4)]


class IntPeakC(C.Structure):
    _fields_ = [("ops", C.c_uint64), ("ms", C.c_float), ("mix", C.c_uint32), ("sm_count", C.c_uint32),
                ("ops_per_s", C.c_double), ("sm_mhz", C.c_double), ("ops_per_clk_sm", C.c_double)]


class ServerConfig(C.Structure):
    _fields_ = [("max_active", C.c_uint32), ("slice_items", C.c_uint32), ("hbm_reserve", C.c_uint64),
                ("traj_batch_seeds", C.c_uint32), ("reserved", C.c_uint32 * 7)]


class RequestC(C.Structure):
    _fields_ = [("kind", C.c_uint32), ("nseeds", C.c_uint32), ("range", Range),
                ("seeds", C.c_void_p), ("stopping_time", C.c_void_p), ("excursion", C.c_void_p),
                ("status", C.c_void_p)]


class ResponseC(C.Structure):
    _fields_ = [("ticket", C.c_uint64), ("status", C.c_int32), ("kind", C.c_uint32),
                ("range", RangeResultC), ("submit_s", C.c_double), ("admit_s", C.c_double),
                ("done_s", C.c_double)]


class ServerInfoC(C.Structure):
    _fields_ = [("submitted", C.c_uint64), ("admitted", C.c_uint64), ("completed", C.c_uint64),
                ("refused", C.c_uint64), ("range_slices", C.c_uint64), ("traj_batches", C.c_uint64),
                ("range_seeds_checked", C.c_uint64), ("traj_seeds", C.c_uint64),
                ("active", C.c_uint32), ("pending", C.c_uint32), ("hbm_free", C.c_uint64),
                ("hbm_admitted", C.c_uint64), ("device_busy_s", C.c_double), ("loops", C.c_uint64),
                ("host_admit_s", C.c_double), ("host_slice_s", C.c_double), ("host_batch_s", C.c_double),
                ("host_complete_s", C.c_double), ("host_idle_s", C.c_double)]


def _limbs(arr) -> int:
    return sum(int(w) << (32 * i) for i, w in enumerate(arr))


_lib = None


def lib() -> C.CDLL:
    """Loads libcollatz_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: run collatz_b200/build.py")
        L = C.CDLL(LIB_PATH)
        P = C.c_void_p
        sigs = {
            "collatz_config_default": (None, [C.POINTER(Config)]),
            "collatz_create": (C.c_int, [C.POINTER(Config), C.POINTER(P)]),
            "collatz_destroy": (None, [P]),
            "collatz_status_string": (C.c_char_p, [C.c_int]),
            "collatz_last_error": (C.c_char_p, [P]),
            "collatz_set_stream": (C.c_int, [P, P]),
            "collatz_device_info": (C.c_int, [P, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
            "collatz_run_case": (C.c_int, [P, C.POINTER(Case), C.POINTER(CaseResultC)]),
            "collatz_verify_pairs": (C.c_int, [P, C.c_uint32, P, C.c_uint32, C.POINTER(CaseResultC)]),
            "collatz_step1_pairs": (C.c_int, [C.c_uint32, C.POINTER(Case), P, C.c_uint64,
                                              C.POINTER(C.c_uint64)]),
            "collatz_step1_pairs_device": (C.c_int, [P, C.POINTER(Case), P, C.c_uint64,
                                                     C.POINTER(C.c_uint64)]),
            "collatz_case_tables": (C.c_int, [P, P, P]),
            "collatz_range_sieve": (C.c_int, [P, C.c_uint32, P, C.POINTER(C.c_uint64)]),
            "collatz_verify_range": (C.c_int, [P, C.POINTER(Range), C.POINTER(RangeResultC)]),
            "collatz_verify_batch": (C.c_int, [P, P, C.c_uint32, P]),
            "collatz_plan_create": (C.c_int, [P, P, C.c_uint32, C.POINTER(P)]),
            "collatz_plan_launch": (C.c_int, [P]),
            "collatz_plan_results": (C.c_int, [P, P]),
            "collatz_plan_destroy": (None, [P]),
            "collatz_trajectory": (C.c_int, [P, P, C.c_uint32, P, P, P]),
            "collatz_server_config_default": (None, [C.POINTER(ServerConfig)]),
            "collatz_server_start": (C.c_int, [C.POINTER(Config), C.POINTER(ServerConfig), C.POINTER(P)]),
            "collatz_server_submit": (C.c_int, [P, C.POINTER(RequestC), C.POINTER(C.c_uint64)]),
            "collatz_server_wait": (C.c_int, [P, C.c_uint64, C.c_double, C.POINTER(ResponseC)]),
            "collatz_server_info": (C.c_int, [P, C.POINTER(ServerInfoC)]),
            "collatz_server_stop": (C.c_int, [P]),
            "collatz_autotune": (C.c_int, [P, C.c_uint32, C.POINTER(TuneResultC)]),
            "collatz_int_peak": (C.c_int, [P, C.c_int, C.POINTER(IntPeakC)]),
            "collatz_combine_case_results": (C.c_int, [P, C.c_uint32, C.POINTER(CaseResultC)]),
            "collatz_run_cases": (C.c_int, [P, P, C.c_uint32, C.c_char_p, P, C.POINTER(CaseResultC),
                                            C.POINTER(C.c_uint32)]),
            "collatz_run_case_batch": (C.c_int, [P, P, C.c_uint32, P, P, C.c_uint64]),
            "collatz_step1_split": (C.c_int, [C.c_uint32, C.POINTER(Case), C.c_uint32, P, C.c_uint64,
                                              C.POINTER(C.c_uint64)]),
            "collatz_journal_load": (C.c_int, [C.c_char_p, P, C.c_uint32, P, P]),
            "collatz_variant_count": (C.c_int, [C.c_int]),
            "collatz_set_variant": (C.c_int, [P, C.c_int, C.c_int]),
        }
        for name, (res, args) in sigs.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def status_string(s: int) -> str:
    return lib().collatz_status_string(s).decode()


# ----------------------------------------------------------------------------
# results
# ----------------------------------------------------------------------------

@dataclass
class CaseResult:
    hash: int
    launches: int
    spot_checks: int
    seeds_checked: int
    pairs: int
    cpu_pairs: int
    n_overflow: int
    overflow: list
    max_excursion: int
    max_excursion_seed: int
    max_stopping_time: int
    max_stopping_time_seed: int
    errors: int
    device_ms: float

    def summary_line(self) -> str:
        """The reference's stderr line (cu:181-182)."""
        return (f"Number of kernel launches = {self.launches}. Spot checks = {self.spot_checks}. "
                f"Complete hash = {self.hash:X}.")


@dataclass
class RangeResult:
    seeds_checked: int
    failures: int
    widened: int
    max_excursion: int
    max_excursion_seed: int
    max_stopping_time: int
    max_stopping_time_seed: int
    errors: int = 0
    status: int = 0
    device_ms: float = 0.0


def _case_result(r: CaseResultC, ovbuf, cap) -> CaseResult:
    n = min(r.n_overflow, cap)
    ov = [_limbs(ovbuf[4 * i:4 * i + 4]) for i in range(n)] if ovbuf is not None else []
    return CaseResult(r.hash, r.launches, r.spot_checks, r.seeds_checked, r.pairs, r.cpu_pairs,
                      r.n_overflow, ov, _limbs(r.max_excursion), _limbs(r.max_excursion_seed),
                      r.max_stopping_time, _limbs(r.max_stopping_time_seed), r.errors, r.device_ms)


def _range_result(r: RangeResultC) -> RangeResult:
    return RangeResult(r.seeds_checked, r.failures, r.widened, _limbs(r.max_excursion),
                       _limbs(r.max_excursion_seed), r.max_stopping_time,
                       _limbs(r.max_stopping_time_seed), r.errors, r.status, r.device_ms)


def make_case(base, sigfig, threepower, number, doubleeven, numevens) -> Case:
    c = Case()
    c.base[0], c.base[1] = base & (2**64 - 1), base >> 64
    c.sigfig, c.threepower = sigfig, threepower
    c.number[0], c.number[1] = number & (2**64 - 1), number >> 64
    c.doubleeven, c.numevens = doubleeven, numevens
    return c


def make_range(offset: int, size: int, k: int = 0, mod9: bool = True, negative: bool = False) -> Range:
    """negative: seeds m stand for -m (the map T'(m) = (3m-1)/2, m/2)."""
    r = Range()
    r.offset[0], r.offset[1] = offset & (2**64 - 1), offset >> 64
    r.size, r.k = size, k
    r.flags = (0 if mod9 else RANGE_NO_MOD9) | (RANGE_NEGATIVE if negative else 0)
    return r


def pack_pairs(pairs) -> "C.Array":
    """[(base, number)] -> npairs x 8 uint32 (cu:521-528 layout)."""
    buf = (C.c_uint32 * (8 * len(pairs)))()
    for i, (b, m) in enumerate(pairs):
        for j in range(4):
            buf[8 * i + j] = (b >> (32 * j)) & 0xFFFFFFFF
            buf[8 * i + 4 + j] = (m >> (32 * j)) & 0xFFFFFFFF
    return buf


def journal_load(journal: str, tuples, overflow_cap: int = 1 << 10):
    """Host-only: {case index: CaseResult} for the cases a journal records."""
    n = len(tuples)
    arr = (Case * max(1, n))()
    for i, t in enumerate(tuples):
        arr[i] = make_case(*t)
    res = (CaseResultC * max(1, n))()
    bufs = []
    for i in range(n):
        b = (C.c_uint32 * (4 * overflow_cap))()
        bufs.append(b)
        res[i].overflow_seeds = C.cast(b, C.POINTER(C.c_uint32))
        res[i].overflow_cap = overflow_cap
    done = (C.c_uint8 * max(1, n))()
    rc = lib().collatz_journal_load(journal.encode(), arr, n, res, done)
    if rc:
        raise CollatzError(rc, f"journal_load: {status_string(rc)}")
    return {i: _case_result(res[i], bufs[i], overflow_cap) for i in range(n) if done[i]}


def split_cases(maxbits: int, case, cut: int):
    """The Step-1 tree nodes of `case` (a 6-tuple) at sigfig = cut, in the reference's
    order (collatz_step1_split), as a ctypes Case array for Verifier.run_cases."""
    c = make_case(*case)
    cnt = C.c_uint64()
    rc = lib().collatz_step1_split(maxbits, C.byref(c), cut, None, 0, C.byref(cnt))
    if rc:
        raise CollatzError(rc, "step1_split")
    arr = (Case * max(1, cnt.value))()
    rc = lib().collatz_step1_split(maxbits, C.byref(c), cut, arr, cnt.value, C.byref(cnt))
    if rc:
        raise CollatzError(rc, "step1_split")
    return arr if cnt.value else (Case * 0)()


def case_tuple(c: Case) -> tuple:
    return (c.base[0] | (c.base[1] << 64), c.sigfig, c.threepower, c.number[0] | (c.number[1] << 64),
            c.doubleeven, c.numevens)


def step1_pairs(maxbits: int, base, sigfig, threepower, number, doubleeven, numevens, cap=None):
    """Step-1 leaves [(bigindex, base, number)] (host only, no device)."""
    c = make_case(base, sigfig, threepower, number, doubleeven, numevens)
    cnt = C.c_uint64()
    rc = lib().collatz_step1_pairs(maxbits, C.byref(c), None, 0, C.byref(cnt))
    if rc:
        raise CollatzError(rc, "step1_pairs")
    n = cnt.value if cap is None else min(cap, cnt.value)
    buf = (C.c_uint32 * (8 * max(1, n)))()
    rc = lib().collatz_step1_pairs(maxbits, C.byref(c), buf, n, C.byref(cnt))
    if rc:
        raise CollatzError(rc, "step1_pairs")
    out = []
    for i in range(n):
        w = buf[8 * i:8 * i + 8]
        out.append((w[3], w[0] | (w[1] << 32) | (w[2] << 64), _limbs(w[4:8])))
    return out


class Verifier:
    """One device context (tables resident in HBM)."""

    def __init__(self, maxbits: int = 45, range_k: int = 24, device: int = 0,
                 variant: int | None = None, iter_cap: int = 0, host_step1: bool = False):
        """host_step1: run_case runs Step 1 on the host threads (the default
        is the device)."""
        cfg = Config()
        lib().collatz_config_default(C.byref(cfg))
        cfg.maxbits, cfg.range_k, cfg.device = maxbits, range_k, device
        cfg.iter_cap = iter_cap
        cfg.flags = CFG_HOST_STEP1 if host_step1 else 0
        if variant is not None:
            cfg.variant = variant
        h = C.c_void_p()
        rc = lib().collatz_create(C.byref(cfg), C.byref(h))
        if rc:
            raise CollatzError(rc, status_string(rc))
        self._h = h
        self.maxbits = maxbits
        self.range_k = range_k

    def close(self):
        if getattr(self, "_h", None):
            lib().collatz_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, rc: int, what: str):
        if rc:
            raise CollatzError(rc, f"{what}: {status_string(rc)}: "
                                   f"{lib().collatz_last_error(self._h).decode()}")

    @property
    def handle(self):
        return self._h

    def device_info(self):
        sm, clk = C.c_int(), C.c_int()
        self._check(lib().collatz_device_info(self._h, C.byref(sm), C.byref(clk)), "device_info")
        return sm.value, clk.value

    def set_stream(self, stream_handle: int | None):
        self._check(lib().collatz_set_stream(self._h, C.c_void_p(stream_handle or 0)), "set_stream")

    def set_variant(self, mode: int, variant: int):
        self._check(lib().collatz_set_variant(self._h, mode, variant), "set_variant")

    def autotune(self, range_mode: bool = True, cases_mode: bool = True, cache: bool = True) -> dict:
        """Times every kernel variant on this device (collatz_autotune) and keeps the fastest."""
        flags = (TUNE_RANGE if range_mode else 0) | (TUNE_CASES if cases_mode else 0) | \
            (0 if cache else TUNE_NO_CACHE)
        r = TuneResultC()
        self._check(lib().collatz_autotune(self._h, flags, C.byref(r)), "autotune")
        return {"range_variant": r.range_variant, "cases_variant": r.cases_variant,
                "range_ms": [x for x in r.range_ms if x >= 0], "cases_ms": [x for x in r.cases_ms if x >= 0],
                "range64_variant": r.range64_variant, "range64_bits": r.range64_bits,
                "range64_ms": [x for x in r.range64_ms if x >= 0], "width_ms": list(r.width_ms)}

    def int_peak(self, mix: int = 1) -> dict:
        """Measured 32-bit integer peak of this device (collatz_int_peak): mix 0 is
        ALU-pipe operations only, mix 1 two ALU operations to one multiply-add."""
        r = IntPeakC()
        self._check(lib().collatz_int_peak(self._h, mix, C.byref(r)), "int_peak")
        return {"mix": r.mix, "ops": r.ops, "ms": r.ms, "ops_per_s": r.ops_per_s, "sm_mhz": r.sm_mhz,
                "ops_per_clk_sm": r.ops_per_clk_sm, "sm_count": r.sm_count}

    # ---- cases mode ----
    def run_case(self, base, sigfig, threepower, number, doubleeven, numevens,
                 overflow_cap: int = 1 << 16, check: bool = True) -> CaseResult:
        c = make_case(base, sigfig, threepower, number, doubleeven, numevens)
        r = CaseResultC()
        ov = (C.c_uint32 * (4 * overflow_cap))()
        r.overflow_seeds = C.cast(ov, C.POINTER(C.c_uint32))
        r.overflow_cap = overflow_cap
        rc = lib().collatz_run_case(self._h, C.byref(c), C.byref(r))
        if check:
            self._check(rc, "run_case")
        return _case_result(r, ov, overflow_cap)

    def run_case_batch(self, tuples, pool_cap: int = 1 << 16, check: bool = True) -> list[CaseResult]:
        """Cases [(base, sigfig, threepower, number, doubleeven, numevens)] in one
        device pass (collatz_run_case_batch); one CaseResult per case, as
        run_case would give it."""
        n = len(tuples)
        if n == 0:
            return []
        arr = (Case * n)()
        for i, t in enumerate(tuples):
            arr[i] = make_case(*t)
        res = (CaseResultC * n)()
        pool = (C.c_uint32 * (4 * max(1, pool_cap)))()
        rc = lib().collatz_run_case_batch(self._h, arr, n, res, pool, pool_cap)
        if check:
            self._check(rc, "run_case_batch")
        out = []
        for r in res:
            k = r.overflow_cap if r.overflow_seeds else 0
            ov = [_limbs(r.overflow_seeds[4 * j:4 * j + 4]) for j in range(k)]
            out.append(CaseResult(r.hash, r.launches, r.spot_checks, r.seeds_checked, r.pairs, r.cpu_pairs,
                                  r.n_overflow, ov, _limbs(r.max_excursion), _limbs(r.max_excursion_seed),
                                  r.max_stopping_time, _limbs(r.max_stopping_time_seed), r.errors,
                                  r.device_ms))
        return out

    def step1_pairs_device(self, base, sigfig, threepower, number, doubleeven, numevens, cap=None):
        """Step-1 leaves [(bigindex, base, number)] from the device Step 1, in
        no particular order (compare with step1_pairs as sorted lists)."""
        c = make_case(base, sigfig, threepower, number, doubleeven, numevens)
        cnt = C.c_uint64()
        self._check(lib().collatz_step1_pairs_device(self._h, C.byref(c), None, 0, C.byref(cnt)),
                    "step1_pairs_device")
        n = cnt.value if cap is None else min(cap, cnt.value)
        import numpy as np
        buf = np.zeros((max(1, n), 8), dtype=np.uint32)
        self._check(lib().collatz_step1_pairs_device(self._h, C.byref(c), buf.ctypes.data, n, C.byref(cnt)),
                    "step1_pairs_device")
        out = []
        for w in buf[:n].tolist():
            out.append((w[3], w[0] | (w[1] << 32) | (w[2] << 64),
                        w[4] | (w[5] << 32) | (w[6] << 64) | (w[7] << 96)))
        return out

    def launchkernel(self, bigindex: int, pairs, overflow_cap: int = 1 << 16,
                     check: bool = True) -> CaseResult:
        """One batch of pairs [(base, number)] or a packed uint32 buffer."""
        if isinstance(pairs, (list, tuple)):
            buf, n = pack_pairs(pairs), len(pairs)
        else:
            buf, n = pairs, len(pairs) // 8
        r = CaseResultC()
        ov = (C.c_uint32 * (4 * overflow_cap))()
        r.overflow_seeds = C.cast(ov, C.POINTER(C.c_uint32))
        r.overflow_cap = overflow_cap
        rc = lib().collatz_verify_pairs(self._h, bigindex, buf, n, C.byref(r))
        if check:
            self._check(rc, "verify_pairs")
        return _case_result(r, ov, overflow_cap)

    verify_pairs = launchkernel

    def run_cases(self, tuples, journal: str | None = None, overflow_cap: int = 1 << 16,
                  per_case: bool = True):
        """Runs cases_* lines [(base, sigfig, threepower, number, doubleeven, numevens)], or a
        ctypes Case array (split_cases), in one process (collatz_run_cases); returns
        (combined CaseResult, [per-case CaseResult] or None, run now)."""
        if isinstance(tuples, C.Array):
            arr, n = tuples, len(tuples)
        else:
            n = len(tuples)
            arr = (Case * max(1, n))()
            for i, t in enumerate(tuples):
                arr[i] = make_case(*t)
        per = (CaseResultC * max(1, n))() if per_case else None
        comb = CaseResultC()
        ov = (C.c_uint32 * (4 * overflow_cap))()
        comb.overflow_seeds = C.cast(ov, C.POINTER(C.c_uint32))
        comb.overflow_cap = overflow_cap
        ran = C.c_uint32()
        rc = lib().collatz_run_cases(self._h, arr, n, journal.encode() if journal else None, per,
                                     C.byref(comb), C.byref(ran))
        self._check(rc, "run_cases")
        return (_case_result(comb, ov, overflow_cap),
                [_case_result(per[i], None, 0) for i in range(n)] if per_case else None, ran.value)

    def case_tables(self) -> tuple[bytes, bytes]:
        bv = (C.c_uint32 * (16 * BV_WORDS))()
        m9 = (C.c_uint32 * (9 * 32))()
        self._check(lib().collatz_case_tables(self._h, bv, m9), "case_tables")
        return bytes(bv), bytes(m9)

    # ---- range mode ----
    def range_sieve(self, k: int) -> tuple[int, bytes]:
        cnt = C.c_uint64()
        buf = (C.c_uint8 * ((1 << k) // 8))()
        self._check(lib().collatz_range_sieve(self._h, k, buf, C.byref(cnt)), "range_sieve")
        return cnt.value, bytes(buf)

    def verify_range(self, offset: int, size: int, k: int = 0, mod9: bool = True,
                     check: bool = True, negative: bool = False) -> RangeResult:
        r = make_range(offset, size, k, mod9, negative)
        out = RangeResultC()
        rc = lib().collatz_verify_range(self._h, C.byref(r), C.byref(out))
        if check:
            self._check(rc, "verify_range")
        return _range_result(out)

    def verify_batch(self, reqs, check: bool = True) -> list[RangeResult]:
        """reqs: [(offset, size)] or [(offset, size, k, mod9)]."""
        n = len(reqs)
        arr = (Range * n)()
        for i, q in enumerate(reqs):
            arr[i] = make_range(*q)
        out = (RangeResultC * n)()
        rc = lib().collatz_verify_batch(self._h, arr, n, out)
        if check:
            self._check(rc, "verify_batch")
        return [_range_result(out[i]) for i in range(n)]

    def plan(self, reqs) -> "Plan":
        return Plan(self, reqs)

    # ---- trajectory queries ----
    def trajectory(self, seeds) -> list[tuple[int, int, int]]:
        """[(status, stopping_time, excursion)] per seed (< 2^256)."""
        n = len(seeds)
        arr = (C.c_uint32 * (8 * max(1, n)))()
        for i, s in enumerate(seeds):
            if s < 0 or s >> 256:
                raise ValueError("seeds must be in [0, 2^256)")
            for j in range(8):
                arr[8 * i + j] = (s >> (32 * j)) & 0xFFFFFFFF
        st = (C.c_uint64 * max(1, n))()
        exc = (C.c_uint32 * (16 * max(1, n)))()
        status = (C.c_uint32 * max(1, n))()
        self._check(lib().collatz_trajectory(self._h, arr, n, st, exc, status), "trajectory")
        return [(status[i], st[i], _limbs(exc[16 * i:16 * i + 16])) for i in range(n)]

    def trajectory_array(self, seeds):
        """seeds: numpy (n, 8) uint32 limbs -> numpy (status, stopping_time, excursion (n, 16))."""
        import numpy as np
        seeds = np.ascontiguousarray(seeds, dtype=np.uint32)
        n = seeds.shape[0]
        st = np.zeros(max(1, n), dtype=np.uint64)
        exc = np.zeros((max(1, n), 16), dtype=np.uint32)
        status = np.zeros(max(1, n), dtype=np.uint32)
        self._check(lib().collatz_trajectory(self._h, seeds.ctypes.data, n, st.ctypes.data, exc.ctypes.data,
                                             status.ctypes.data), "trajectory")
        return status[:n], st[:n], exc[:n]


class Plan:
    """Lowered range requests + a captured CUDA graph, relaunchable."""

    def __init__(self, v: Verifier, reqs):
        self.v = v
        self.n = len(reqs)
        arr = (Range * self.n)()
        for i, q in enumerate(reqs):
            arr[i] = make_range(*q)
        h = C.c_void_p()
        v._check(lib().collatz_plan_create(v.handle, arr, self.n, C.byref(h)), "plan_create")
        self._h = h

    def launch(self):
        self.v._check(lib().collatz_plan_launch(self._h), "plan_launch")

    def results(self, check: bool = True) -> list[RangeResult]:
        out = (RangeResultC * self.n)()
        rc = lib().collatz_plan_results(self._h, out)
        if check:
            self.v._check(rc, "plan_results")
        return [_range_result(out[i]) for i in range(self.n)]

    def close(self):
        if getattr(self, "_h", None):
            lib().collatz_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@dataclass
class Response:
    """One served request's outcome (collatz_response)."""
    ticket: int
    status: int
    kind: int
    range: RangeResult | None = None
    # trajectory queries: numpy arrays status (n,), stopping_time (n,), excursion (n, 16) limbs
    traj_status: object = None
    traj_stopping_time: object = None
    traj_excursion: object = None
    submit_s: float = 0.0
    admit_s: float = 0.0
    done_s: float = 0.0

    @property
    def latency_s(self) -> float:
        return self.done_s - self.submit_s

    @property
    def queue_s(self) -> float:
        return self.admit_s - self.submit_s

    def trajectory(self) -> list[tuple[int, int, int]]:
        """[(status, stopping_time, excursion)] per seed, as Verifier.trajectory."""
        return [(int(self.traj_status[i]), int(self.traj_stopping_time[i]),
                 _limbs(self.traj_excursion[i])) for i in range(len(self.traj_status))]


def seeds_array(seeds):
    """[int] (each < 2^256) -> numpy (n, 8) uint32 little-endian limbs."""
    import numpy as np
    arr = np.zeros((len(seeds), 8), dtype=np.uint32)
    for i, s in enumerate(seeds):
        if s < 0 or s >> 256:
            raise ValueError("seeds must be in [0, 2^256)")
        for j in range(8):
            arr[i, j] = (s >> (32 * j)) & 0xFFFFFFFF
    return arr


class Server:
    """Continuous-batching server (collatz_server_*): submit from any thread,
    wait for each ticket.  Range requests and trajectory queries share the
    device; results equal the same request run alone."""

    def __init__(self, maxbits: int = 26, range_k: int = 24, device: int = 0, max_active: int = 256,
                 slice_items: int = 1 << 19, hbm_reserve: int = 1 << 30,
                 traj_batch_seeds: int = 1 << 20, iter_cap: int = 0, variant: int | None = None):
        import threading
        cfg = Config()
        lib().collatz_config_default(C.byref(cfg))
        cfg.maxbits, cfg.range_k, cfg.device, cfg.iter_cap = maxbits, range_k, device, iter_cap
        if variant is not None:
            cfg.variant = variant
        sc = ServerConfig()
        lib().collatz_server_config_default(C.byref(sc))
        sc.max_active, sc.slice_items, sc.hbm_reserve = max_active, slice_items, hbm_reserve
        sc.traj_batch_seeds = traj_batch_seeds
        h = C.c_void_p()
        rc = lib().collatz_server_start(C.byref(cfg), C.byref(sc), C.byref(h))
        if rc:
            raise CollatzError(rc, f"server_start: {status_string(rc)}")
        self._h = h
        self._bufs: dict[int, tuple] = {}
        self._lock = threading.Lock()

    def submit_range(self, offset: int, size: int, k: int = 0, mod9: bool = True, negative: bool = False) -> int:
        q = RequestC()
        q.kind = REQ_RANGE
        q.range = make_range(offset, size, k, mod9, negative)
        t = C.c_uint64()
        rc = lib().collatz_server_submit(self._h, C.byref(q), C.byref(t))
        if rc:
            raise CollatzError(rc, f"submit_range: {status_string(rc)}")
        return t.value

    def submit_trajectory_array(self, seeds) -> int:
        """seeds: numpy (n, 8) uint32 limbs (kept alive until wait)."""
        import numpy as np
        seeds = np.ascontiguousarray(seeds, dtype=np.uint32)
        n = seeds.shape[0]
        st = np.zeros(n, dtype=np.uint64)
        exc = np.zeros((n, 16), dtype=np.uint32)
        status = np.zeros(n, dtype=np.uint32)
        q = RequestC()
        q.kind, q.nseeds = REQ_TRAJECTORY, n
        q.seeds, q.stopping_time = seeds.ctypes.data, st.ctypes.data
        q.excursion, q.status = exc.ctypes.data, status.ctypes.data
        t = C.c_uint64()
        with self._lock:
            rc = lib().collatz_server_submit(self._h, C.byref(q), C.byref(t))
            if rc:
                raise CollatzError(rc, f"submit_trajectory: {status_string(rc)}")
            self._bufs[t.value] = (seeds, st, exc, status)
        return t.value

    def submit_trajectory(self, seeds) -> int:
        return self.submit_trajectory_array(seeds_array(seeds))

    def wait(self, ticket: int, timeout: float | None = None) -> Response:
        r = ResponseC()
        rc = lib().collatz_server_wait(self._h, ticket, -1.0 if timeout is None else timeout, C.byref(r))
        if rc == E_TIMEOUT or rc == E_ARG:
            raise CollatzError(rc, f"wait({ticket}): {status_string(rc)}")
        with self._lock:
            bufs = self._bufs.pop(ticket, None)
        out = Response(r.ticket, r.status, r.kind, submit_s=r.submit_s, admit_s=r.admit_s, done_s=r.done_s)
        if r.kind == REQ_RANGE:
            out.range = _range_result(r.range)
        elif bufs is not None:
            out.traj_status, out.traj_stopping_time, out.traj_excursion = bufs[3], bufs[1], bufs[2]
        return out

    def info(self) -> dict:
        i = ServerInfoC()
        rc = lib().collatz_server_info(self._h, C.byref(i))
        if rc:
            raise CollatzError(rc, "server_info")
        return {name: getattr(i, name) for name, _ in ServerInfoC._fields_}

    def stop(self):
        if getattr(self, "_h", None):
            lib().collatz_server_stop(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.stop()

    def __del__(self):
        try:
            self.stop()
        except Exception:
            pass


def combine_range_results(parts: list[RangeResult]) -> RangeResult:
    """Merges results of disjoint sub-ranges (sum, max with the smaller seed on ties)."""
    out = RangeResult(0, 0, 0, 0, 0, 0, 0)
    have = False
    for p in parts:
        out.seeds_checked += p.seeds_checked
        out.failures += p.failures
        out.widened += p.widened
        out.errors |= p.errors
        if p.seeds_checked == 0:
            continue
        if not have or (p.max_excursion, -p.max_excursion_seed) > (out.max_excursion, -out.max_excursion_seed):
            out.max_excursion, out.max_excursion_seed = p.max_excursion, p.max_excursion_seed
        if not have or (p.max_stopping_time, -p.max_stopping_time_seed) > \
                (out.max_stopping_time, -out.max_stopping_time_seed):
            out.max_stopping_time, out.max_stopping_time_seed = p.max_stopping_time, p.max_stopping_time_seed
        have = True
    return out
