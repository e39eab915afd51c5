"""The CPU oracle pinned against the reference's own outputs (golden fixtures
from collatz_cudav7.cu built through the CPU shim) and against brute force."""
import hashlib
import random

import pytest

from conftest import load_golden

RUNS = load_golden("cases_runs.json")["runs"]
TABLES = load_golden("tables.json")["tables"]


def T_step(n):
    return (3 * n + 1) // 2 if n & 1 else n // 2


def brute(n):
    """(stopping time, excursion) by single steps."""
    x, E, k = n, n, 0
    while True:
        x = T_step(x)
        k += 1
        E = max(E, x)
        if x < n:
            return k, E


@pytest.mark.parametrize("t", [t for t in TABLES if t["N"] in (26, 45)], ids=lambda t: f"N{t['N']}")
def test_oracle_tables_match_reference(oracle_tables, t):
    T = oracle_tables(t["N"])
    assert hashlib.sha256(T.bv_bytes()).hexdigest() == t["bv_sha256"]
    assert hashlib.sha256(T.mod9_bytes()).hexdigest() == t["mod9_sha256"]


@pytest.mark.parametrize("n", [26, 45])
def test_oracle_pairs_match_reference(oracle_tables, n):
    fx = load_golden(f"pairs_N{n}.json")
    T = oracle_tables(n)
    for b in fx["batches"]:
        pairs = [(int(x), int(y)) for x, y in b["pairs"]]
        o = T.pairs_result(b["bigindex"], pairs)
        assert f"{o.hash:X}" == b["hash"]
        assert o.seeds == b["seeds"]
        assert sorted(o.overflow) == sorted(int(x) for x in b["overflow"])
    for d in fx["search2"]:
        o = T.pairs_result(d["bigindex"], [(int(d["base"]), int(d["number"]))], cpu_sem=True)
        assert f"{o.hash:X}" == d["hash"]


@pytest.mark.parametrize("run", [r for r in RUNS if r["N"] <= 30 or (r["N"] == 36 and r["tuple"][1] >= 10)
                                 or r["tuple"][1] >= 20],
                         ids=lambda r: f"N{r['N']}-" + "_".join(map(str, r["tuple"])))
def test_oracle_runs_match_reference(oracle_tables, run):
    o = oracle_tables(run["N"]).run_case(*run["tuple"])
    assert f"{o.hash:X}" == run["hash"]
    assert o.launches == run["launches"]
    assert o.seeds == run["seeds"]
    assert sorted(o.overflow) == sorted(int(x) for x in run["overflow"])


def test_oracle_case_maxima_brute(oracle_tables):
    """sigma counts from n; E is the maximum over k >= N - A (Step 1 carries
    no history) -- equal to the brute-force maximum whenever the peak comes
    after step N - A."""
    o = oracle_tables(26).run_case(3, 2, 2, 9, 1, 0)
    st, _ = brute(o.max_st_seed)
    assert st == o.max_st
    n = o.max_exc_seed
    x, E = n, 0
    for k in range(1, brute(n)[0] + 1):
        x = T_step(x)
        if k >= 16:
            E = max(E, x)
    assert E == o.max_exc


def test_step1_leaves_match_product(oracle_tables):
    """The product's host Step 1 (collatz_step1_pairs) visits the same leaves
    in the same order as the oracle's restatement of search1."""
    import collatz_b200 as cb
    from oracle import oracle as O
    for n, tup in ((26, (3, 2, 2, 9, 1, 0)), (36, (27, 10, 8, 183, 0, 0)), (45, (27, 25, 18, 335, 0, 1)),
                   (26, (0, 5, 0, 1, 0, 0)), (26, (3, 16, 12, 9, 0, 0)), (30, (3, 2, 2, 9, 5, 0)),
                   (30, (3, 2, 2, 9, 0, 7)), (30, (3, 2, 2, 9, 0, 0xFFFFFFFF))):
        assert cb.step1_pairs(n, *tup) == O.leaves(n, tup)


@pytest.mark.parametrize("k", [8, 10, 12, 14, 16, 18, 20])
def test_range_sieve_valid_from_2k(k):
    """Every removed residue r descends within its tau steps from 2^k + r,
    hence (T^tau affine with slope < 1 on the class) for every n >= 2^k."""
    from oracle import oracle as O
    assert O.range_sieve_validate(k) == 0


def test_range_sieve_bruteforce():
    from oracle import oracle as O
    k = 12
    n, bits = O.range_sieve(k)
    cnt = 0
    for r in range(1 << k):
        x, f, ok = r, 0, True
        for j in range(1, k + 1):
            if x & 1:
                f += 1
            x = T_step(x)
            if 3 ** f < 2 ** j:
                ok = False
                break
        assert ok == bool((bits[r >> 3] >> (r & 7)) & 1)
        cnt += ok
    assert cnt == n


@pytest.mark.parametrize("case", [((1 << 20) + 7, 3000, 12), (2, 4000, 16), ((1 << 33) + 11, 5000, 16)])
def test_range_oracle_bruteforce(case):
    from oracle import oracle as O
    off, size, k = case
    o = O.range_verify(off, size, k, True, method=0)
    _, bits = O.range_sieve(k)
    best_st, best_e, seeds = (-1, 0), (-1, 0), 0
    for n in range(off, off + size):
        if n < 2 or n % 9 not in (0, 1, 3, 6, 7):
            continue
        if n >= (1 << k):
            r = n % (1 << k)
            if not (bits[r >> 3] >> (r & 7)) & 1:
                continue
        seeds += 1
        st, E = brute(n)
        best_st = max(best_st, (st, -n))
        best_e = max(best_e, (E, -n))
    assert o.seeds == seeds
    assert (o.max_st, o.max_st_seed) == (best_st[0], -best_st[1])
    assert (o.max_exc, o.max_exc_seed) == (best_e[0], -best_e[1])


@pytest.mark.parametrize("case", [(1 << 40, 1 << 20, 24), ((1 << 60) + 3, 1 << 18, 16), (0, 1 << 16, 12),
                                  ((1 << 90) + 5, 1 << 14, 16)])
def test_range_methods_agree(case):
    """Single steps, the reference's run-length loop and the GPU's jump +
    runs structure give identical results."""
    from oracle import oracle as O
    off, size, k = case
    rs = [O.range_verify(off, size, k, True, method=m, nthreads=4) for m in (0, 1, 2)]
    keys = [(r.seeds, r.max_st, r.max_st_seed, r.max_exc, r.max_exc_seed) for r in rs]
    assert keys[0] == keys[1] == keys[2]


@pytest.mark.parametrize("case", [(0, 1 << 22, 16), ((1 << 32) - (1 << 20), 1 << 20, 16),
                                  ((1 << 62) + 1, 1 << 16, 16), ((1 << 64) - (1 << 17), 1 << 18, 16)])
def test_range_u64_method_equals_u128(case):
    """The 64-bit loop with overflow detection (the plain verification of
    n < 2^32 in 64-bit arithmetic) gives the 128-bit loop's results; near
    2^62..2^64 some seeds leave 64 bits and are re-run in 128 bits."""
    from oracle import oracle as O
    off, size, k = case
    a = O.range_verify(off, size, k, True, method=1, nthreads=4)
    b = O.range_verify(off, size, k, True, method=3, nthreads=4)
    assert (a.seeds, a.failures, a.max_st, a.max_st_seed, a.max_exc, a.max_exc_seed) == \
        (b.seeds, b.failures, b.max_st, b.max_st_seed, b.max_exc, b.max_exc_seed)
    assert (b.wide64 > 0) == (off >= 1 << 62)


@pytest.mark.parametrize("case", [(1 << 40, 1 << 18, 16), ((1 << 60) + 12345, 1 << 17, 20), (3, 1 << 16, 12),
                                  ((1 << 50) - 4096, 1 << 16, 24)])
def test_range_direct_sieve_equals_table(case):
    """Testing each seed's residue against the sieve definition gives the
    same results as the 2^k-bit table (the direct test is what the oracle
    uses for k > 26, e.g. the k = 34 frontier configuration)."""
    from oracle import oracle as O
    off, size, k = case
    a = O.range_verify(off, size, k, True, method=2, nthreads=4, direct_sieve=False)
    b = O.range_verify(off, size, k, True, method=2, nthreads=4, direct_sieve=True)
    assert (a.seeds, a.max_st, a.max_st_seed, a.max_exc, a.max_exc_seed, a.odd_runs) == \
        (b.seeds, b.max_st, b.max_st_seed, b.max_exc, b.max_exc_seed, b.odd_runs)


def test_range_k34_bruteforce():
    from oracle import oracle as O
    k, off, size = 34, (1 << 60) + (7 << 34) + 99991, 2500
    o = O.range_verify(off, size, k, True, method=2)
    best_st, best_e, seeds = (-1, 0), (-1, 0), 0
    for n in range(off, off + size):
        if n % 9 not in (0, 1, 3, 6, 7):
            continue
        x, f, ok = n % (1 << k), 0, True
        for j in range(1, k + 1):
            if x & 1:
                f += 1
            x = T_step(x)
            if 3 ** f < 2 ** j:
                ok = False
                break
        if not ok:
            continue
        seeds += 1
        st, E = brute(n)
        best_st = max(best_st, (st, -n))
        best_e = max(best_e, (E, -n))
    assert o.seeds == seeds
    assert (o.max_st, o.max_st_seed) == (best_st[0], -best_st[1])
    assert (o.max_exc, o.max_exc_seed) == (best_e[0], -best_e[1])


def T_neg(m):
    """T acting on -m, written for m: (3m-1)/2 for odd m, m/2 for even m."""
    return (3 * m - 1) // 2 if m & 1 else m // 2


def brute_neg(m, cap=10000):
    """(stopping time, excursion), or None when m returns to itself or runs cap steps."""
    x, E, k = m, m, 0
    while True:
        x = T_neg(x)
        k += 1
        E = max(E, x)
        if x < m:
            return k, E
        if x == m or k >= cap:
            return None


def test_negative_merge_rules():
    """The negative variant's mod-9 sieve drops m = 1 (mod 3), m > 1, and
    m = 5 (mod 9), m > 5, because a smaller seed reaches them first."""
    for m in range(2, 3000):
        if m % 3 == 1:
            p = (2 * m + 1) // 3
            assert (2 * m + 1) % 3 == 0 and p % 2 == 1 and T_neg(p) == m and p < m
        if m % 9 == 5 and m > 5:
            x = (8 * m + 5) // 9
            assert (8 * m + 5) % 9 == 0 and T_neg(T_neg(T_neg(x))) == m and x < m


@pytest.mark.parametrize("case", [(2, 4000, 8, True), (2, 3000, 12, False), ((1 << 30) + 17, 3000, 12, True),
                                  ((1 << 34) + 5, 2000, 16, True)])
def test_range_negative_bruteforce(case):
    from oracle import oracle as O
    off, size, k, mod9 = case
    o = O.range_verify(off, size, k, mod9, method=0, negative=True)
    best_st, best_e, seeds, fails = (-1, 0), (-1, 0), 0, 0
    for m in range(off, off + size):
        if m < 2 or (mod9 and not (m % 9 in (0, 2, 3, 6, 8) or m == 5)):
            continue
        if m >= (1 << k):
            x, f, ok = m % (1 << k), 0, True
            for j in range(1, k + 1):
                if x & 1:
                    f += 1
                x = T_neg(x)
                if 3 ** f < 2 ** j:
                    ok = False
                    break
            if not ok:
                continue
        seeds += 1
        b = brute_neg(m)
        if b is None:
            fails += 1
            continue
        best_st = max(best_st, (b[0], -m))
        best_e = max(best_e, (b[1], -m))
    assert (o.seeds, o.failures) == (seeds, fails)
    assert (o.max_st, o.max_st_seed) == (best_st[0], -best_st[1])
    assert (o.max_exc, o.max_exc_seed) == (best_e[0], -best_e[1])
    if off <= 17 < off + size:
        assert fails == 2  # the cycle minima 5 and 17


@pytest.mark.parametrize("case", [(2, 1 << 18, 16), ((1 << 40) + 3, 1 << 18, 20), ((1 << 62) - 999, 1 << 16, 24)])
def test_range_negative_methods_agree(case):
    from oracle import oracle as O
    off, size, k = case
    rs = [O.range_verify(off, size, k, True, method=m, nthreads=4, negative=True) for m in (0, 1, 2)]
    keys = [(r.seeds, r.failures, r.max_st, r.max_st_seed, r.max_exc, r.max_exc_seed) for r in rs]
    assert keys[0] == keys[1] == keys[2]


def test_trajectory_bruteforce():
    from oracle import oracle as O
    rng = random.Random(3)
    seeds = [0, 1, 2, 3, 27, 97] + [rng.getrandbits(rng.randint(2, 80)) for _ in range(300)]
    out = O.trajectory(seeds)
    for s, (status, st, E) in zip(seeds, out):
        if s < 2:
            assert (status, st, E) == (1, 0, s)
        else:
            assert (status, st, E) == (0, *brute(s))


def test_split_matches_oracle():
    """collatz_step1_split (the product's cut of a case into cases_* lines)
    gives the oracle's nodes in the oracle's order, edge tuples included."""
    import collatz_b200 as cb
    from oracle import oracle as O
    for n, tup, cut in ((36, (3, 2, 2, 9, 1, 0), 12), (36, (3, 2, 2, 9, 1, 0), 20), (45, (27, 10, 8, 183, 0, 0), 23),
                        (30, (3, 2, 2, 9, 0, 7), 19), (26, (0, 5, 0, 1, 0, 0), 10), (26, (3, 15, 11, 9, 0, 0), 15),
                        (26, (3, 2, 2, 9, 1, 0), 2)):
        assert [cb.case_tuple(c) for c in cb.split_cases(n, tup, cut)] == O.split_case(n, tup, cut), (n, tup, cut)
    # at cut = N - A the nodes are the leaves (the oracle's split stops above them)
    nodes = [cb.case_tuple(c) for c in cb.split_cases(30, (3, 2, 2, 9, 1, 0), 20)]
    assert [(b, num) for b, _, _, num, _, _ in nodes] == [(b, num) for _, b, num in O.leaves(30, (3, 2, 2, 9, 1, 0))]


def test_split_rejects_bad_cut():
    import collatz_b200 as cb
    for n, tup, cut in ((26, (3, 2, 2, 9, 1, 0), 1), (26, (3, 2, 2, 9, 1, 0), 17), (15, (3, 2, 2, 9, 1, 0), 4)):
        with pytest.raises(cb.CollatzError):
            cb.split_cases(n, tup, cut)


@pytest.mark.parametrize("j", [8, 10, 11])
def test_jump_table_bounds(j):
    """The range kernels' j-step windows rest on 0 <= T^i(r) < 2^(j-i) 3^(f_i)
    for every r < 2^j and 1 <= i <= j (f_i: odd steps among the first i), so
    that for x = a 2^j + r, a g(r) <= T^i(x) < (a + 1) h(r) with g, h the least
    and largest of the j multipliers 2^(j-i) 3^(f_i).  Also checks that the
    table entry fits its fields: T^j(r) in 18 bits, f_j in 4, bit lengths of g
    and h in 5."""
    for r in range(1 << j):
        x, f, ms = r, 0, []
        for i in range(1, j + 1):
            if x & 1:
                x, f = (3 * x + 1) // 2, f + 1
            else:
                x //= 2
            m = (1 << (j - i)) * 3 ** f
            assert 0 <= x < m
            ms.append(m)
        assert x < 1 << 18 and f < 16 and max(ms).bit_length() < 32
        for a in (1, 2, 3, 1 << 40, (1 << 40) + 12345):
            y = a * (1 << j) + r
            for i in range(1, j + 1):
                y = (3 * y + 1) // 2 if y & 1 else y // 2
                assert a * min(ms) <= y < (a + 1) * max(ms)
