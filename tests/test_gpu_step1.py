"""Device Step 1 (search1, collatz_cudav7.cu:497-563, on the GPU) against the
oracle's restatement of search1 and against the product's host Step 1.

The device visits the same tree but writes the leaves in no particular
order, so leaves compare as sorted lists (multisets)."""
import ctypes as C

import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu

RUNS = load_golden("cases_runs.json")["runs"]

# (N, tuple): reference inputs, plus trees whose root is pruned, whose root
# is a leaf, and with doubleeven/numevens values the cases files never hold.
LEAF_CASES = [
    (26, (3, 2, 2, 9, 1, 0)),
    (36, (27, 10, 8, 183, 0, 0)),
    (45, (27, 25, 18, 335, 0, 1)),
    (30, (3, 2, 2, 9, 1, 0)),
    (26, (0, 5, 0, 1, 0, 0)),           # induction sieve prunes the root
    (26, (3, 16, 12, 9, 0, 0)),         # sigfig == N - A: the root is the leaf
    (30, (3, 2, 2, 9, 5, 0)),           # doubleeven >= 2: no even branches at all
    (30, (3, 2, 2, 9, 0, 7)),           # odd numevens carried in
    (30, (3, 2, 2, 9, 0, 0xFFFFFFFF)),  # numevens + 1 wraps like the reference's u32
    (40, (27, 10, 8, 183, 0, 0)),
]


@pytest.mark.parametrize("n,tup", LEAF_CASES, ids=lambda x: str(x))
def test_device_leaves_match_oracle(verifier, n, tup):
    from oracle import oracle as O
    dev = verifier(n).step1_pairs_device(*tup)
    ref = O.leaves(n, tup)
    assert sorted(dev) == sorted(ref)


def _host_pairs(n, tup):
    import collatz_b200 as cb
    c = cb.make_case(*tup)
    cnt = C.c_uint64()
    assert cb.lib().collatz_step1_pairs(n, C.byref(c), None, 0, C.byref(cnt)) == 0
    buf = np.zeros((max(1, cnt.value), 8), dtype=np.uint32)
    assert cb.lib().collatz_step1_pairs(n, C.byref(c), buf.ctypes.data, cnt.value, C.byref(cnt)) == 0
    return buf[:cnt.value]


def _device_pairs(v, tup, cap=None):
    import collatz_b200 as cb
    c = cb.make_case(*tup)
    cnt = C.c_uint64()
    assert cb.lib().collatz_step1_pairs_device(v._h, C.byref(c), None, 0, C.byref(cnt)) == 0
    n = cnt.value if cap is None else min(cap, cnt.value)
    buf = np.zeros((max(1, n), 8), dtype=np.uint32)
    assert cb.lib().collatz_step1_pairs_device(v._h, C.byref(c), buf.ctypes.data, n, C.byref(cnt)) == 0
    return buf[:n], cnt.value


def _sorted_rows(a):
    return a[np.lexsort(a.T[::-1])]


def test_device_leaves_n45_line1_equal_host(verifier):
    """All 4 057 442 leaves of the reference's default run (N = 45,
    cases_tiny line 1), as a multiset, equal the host Step 1's."""
    tup = (27, 10, 8, 183, 0, 0)
    host = _host_pairs(45, tup)
    dev, total = _device_pairs(verifier(45), tup)
    assert total == len(host) == 4057442
    assert np.array_equal(_sorted_rows(dev), _sorted_rows(host))
    # a capped call returns the first leaves of the same multiset
    part, total2 = _device_pairs(verifier(45), tup, cap=1000)
    assert total2 == total and len(part) == 1000
    assert len(np.unique(np.concatenate([part, dev]), axis=0)) == len(np.unique(dev, axis=0))


def _same(a, b):
    assert f"{a.hash:X}" == f"{b.hash:X}"
    assert (a.launches, a.seeds_checked, a.pairs, a.cpu_pairs) == (b.launches, b.seeds_checked, b.pairs,
                                                                     b.cpu_pairs)
    assert sorted(a.overflow) == sorted(b.overflow) and a.n_overflow == b.n_overflow
    assert (a.max_stopping_time, a.max_stopping_time_seed) == (b.max_stopping_time, b.max_stopping_time_seed)
    assert (a.max_excursion, a.max_excursion_seed) == (b.max_excursion, b.max_excursion_seed)
    assert a.errors == b.errors == 0


@pytest.mark.parametrize("n,tup", [(26, (3, 2, 2, 9, 1, 0)), (36, (3, 2, 2, 9, 1, 0)),
                                   (42, (27, 10, 8, 183, 0, 0)), (26, (0, 5, 0, 1, 0, 0)),
                                   (26, (3, 16, 12, 9, 0, 0))], ids=str)
def test_run_case_device_equals_host(verifier, n, tup):
    _same(verifier(n).run_case(*tup), verifier(n, host_step1=True).run_case(*tup))


def test_run_case_in_several_emit_chunks(verifier):
    """N = 46, cases_tiny line 1 has about 8 M leaves: the device Step 1 emits
    them in two windows of 2^22 pairs, each verified by its own cases launch;
    the result equals the host Step 1 run."""
    tup = (27, 10, 8, 183, 0, 0)
    d = verifier(46).run_case(*tup)
    assert d.pairs + d.cpu_pairs > 1 << 22
    _same(d, verifier(46, host_step1=True).run_case(*tup))


@pytest.mark.parametrize("run", [r for r in RUNS if r["N"] == 45 and r["tuple"][1] < 20][:2],
                         ids=lambda r: "N45-" + "_".join(map(str, r["tuple"])))
def test_host_step1_mode_matches_reference(verifier, run):
    """The host Step 1 mode stays bit-exact with the reference too."""
    r = verifier(45, host_step1=True).run_case(*run["tuple"])
    assert f"{r.hash:X}" == run["hash"]
    assert r.launches == run["launches"]
    assert r.seeds_checked == run["seeds"]
