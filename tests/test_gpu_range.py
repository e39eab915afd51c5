"""Range mode and batches on the GPU against the oracle (oracle/collatz_oracle.c:
orc_range, the reference's run-length loop of search3, cu:684-715, with exact
stopping time and excursion)."""
import os

import pytest

pytestmark = pytest.mark.gpu

NT = max(1, min(32, os.cpu_count() or 1))

CASES = [
    # (offset, size, k, mod9)
    (1 << 40, 1 << 22, 16, True),
    (1 << 40, 1 << 22, 24, True),
    ((1 << 60) + (5 << 24), 1 << 21, 24, True),
    ((1 << 40) + 12345, 300001, 20, True),      # unaligned both ends, within one block
    ((1 << 40) - 77777, 3 << 20, 20, True),     # unaligned, spans blocks
    (0, 1 << 20, 16, True),                     # seeds below 2^k: unsieved (dense) region
    (1000, 5000, 12, False),                    # no mod-9 sieve
    ((1 << 64) - (1 << 20), 1 << 21, 24, True),  # crosses 2^64
    ((1 << 90) + 3, 1 << 17, 16, True),         # 91-bit seeds
    ((1 << 60) + (3 << 34), 1 << 22, 34, True),  # frontier sieve (2 GiB bit array), aligned
    ((1 << 60) + (5 << 34) - 100000, 300000, 34, True),  # crosses a 2^34 block boundary
    ((1 << 60) + 77777, 1 << 21, 30, True),     # k = 30, unaligned
    ((1 << 57) + 3, 1 << 20, 20, True),         # values cross 2^59 (the 64-bit body's limit) both ways
]


def _cmp(g, o):
    assert g.errors == 0 and g.failures == 0
    assert g.seeds_checked == o.seeds
    assert (g.max_stopping_time, g.max_stopping_time_seed) == (o.max_st, o.max_st_seed)
    assert (g.max_excursion, g.max_excursion_seed) == (o.max_exc, o.max_exc_seed)


@pytest.mark.parametrize("k", [8, 12, 16, 20, 24, 27])
def test_range_sieve_matches_oracle(verifier, k):
    from oracle import oracle as O
    n, bits = verifier(26).range_sieve(k)
    on, obits = O.range_sieve(k)
    assert n == on
    assert bits == obits


@pytest.mark.parametrize("case", CASES, ids=lambda c: f"o{c[0]:x}-s{c[1]}-k{c[2]}-m{int(c[3])}")
def test_range_matches_oracle(verifier, case):
    from oracle import oracle as O
    off, size, k, mod9 = case
    g = verifier(26).verify_range(off, size, k, mod9)
    o = O.range_verify(off, size, k, mod9, method=1, nthreads=NT)
    _cmp(g, o)


VARIANT_CASES = [CASES[i] for i in (0, 3, 4, 5, 6, 7, 8, 10, 12)]


@pytest.mark.parametrize("variant", range(8))
def test_range_variants_match_oracle(verifier, variant):
    """Every range-kernel variant (block shape; 4 and 5 add the 8-step window
    after the k-step jump) gives the oracle's results."""
    import collatz_b200 as cb
    from oracle import oracle as O
    assert cb.lib().collatz_variant_count(1) == 8
    v = verifier(26)
    v.set_variant(1, variant)
    v.set_variant(cb.MODE_RANGE64_BITS, 0)  # every launch on the four-limb kernel
    try:
        for off, size, k, mod9 in VARIANT_CASES:
            g = v.verify_range(off, size, k, mod9)
            o = O.range_verify(off, size, k, mod9, method=1, nthreads=NT)
            _cmp(g, o)
        reqs = [((1 << 40) + i * (1 << 24) + 9 * i, (1 << 18) + 1000 * i, 24, True) for i in range(6)]
        reqs.append((17, 40000, 24, True))
        for q, m in zip(reqs, v.verify_batch(reqs)):
            o = O.range_verify(*q, method=1, nthreads=NT)
            _cmp(m, o)
    finally:
        v.set_variant(1, 0)  # the defaults
        v.set_variant(cb.MODE_RANGE64_BITS, cb.RANGE64_BITS_DEFAULT)


VARIANT64_CASES = [CASES[i] for i in (0, 1, 3, 4, 5, 6)] + [
    ((1 << 46) + 999, 1 << 21, 24, True),       # values cross 2^59 lane by lane
    ((1 << 48) - (3 << 24), 1 << 21, 24, True),  # at the kernel's seed limit
    ((1 << 44) + 5, 1 << 21, 34, True),         # k = 34 (q < 2^14)
    (3, 1 << 18, 16, False),                    # below 2^k, no mod-9 sieve: every n, even ones too
]


RANGE64_VARIANTS = 8


@pytest.mark.parametrize("variant", range(RANGE64_VARIANTS))
def test_range64_variants_match_oracle(verifier, variant):
    """Every variant of the 64-bit range kernel (run pairs per pass, blocks per
    SM, in-loop table steps J, expansion windows of 8, 10 or 11 steps and run
    pairs at expansion) gives the oracle's results, for single ranges and a
    batch, with the limb width at its maximum (48 bits)."""
    import collatz_b200 as cb
    from oracle import oracle as O
    assert cb.lib().collatz_variant_count(cb.MODE_RANGE64) == RANGE64_VARIANTS
    v = verifier(26)
    v.set_variant(cb.MODE_RANGE64, variant)
    v.set_variant(cb.MODE_RANGE64_BITS, 48)
    try:
        for off, size, k, mod9 in VARIANT64_CASES:
            g = v.verify_range(off, size, k, mod9)
            o = O.range_verify(off, size, k, mod9, method=1, nthreads=NT)
            _cmp(g, o)
        reqs = [((1 << 40) + i * (1 << 24) + 9 * i, (1 << 18) + 1000 * i, 24, True) for i in range(6)]
        reqs.append((17, 40000, 24, True))
        for q, m in zip(reqs, v.verify_batch(reqs)):
            o = O.range_verify(*q, method=1, nthreads=NT)
            _cmp(m, o)
    finally:
        v.set_variant(cb.MODE_RANGE64, 0)
        v.set_variant(cb.MODE_RANGE64_BITS, cb.RANGE64_BITS_DEFAULT)


@pytest.mark.parametrize("off,size,k", [((1 << 40) + 777, 1 << 34, 24), ((1 << 46) + 12345, 1 << 32, 24),
                                        ((1 << 47) + (7 << 24), 1 << 31, 24), ((1 << 44) + (3 << 34), 1 << 34, 34)])
def test_range64_equals_four_limbs(verifier, off, size, k):
    """On large ranges the 64-bit kernel (every variant) and the four-limb
    kernel give the same seeds, maxima with their seeds, failures and widened
    seeds."""
    import collatz_b200 as cb
    v = verifier(26, range_k=k)
    try:
        v.set_variant(cb.MODE_RANGE64_BITS, 0)
        p = v.verify_range(off, size, k)
        v.set_variant(cb.MODE_RANGE64_BITS, 48)
        for var in range(cb.lib().collatz_variant_count(cb.MODE_RANGE64)):
            v.set_variant(cb.MODE_RANGE64, var)
            w = v.verify_range(off, size, k)
            assert (w.seeds_checked, w.failures, w.widened, w.errors) == \
                (p.seeds_checked, p.failures, p.widened, p.errors), var
            assert (w.max_stopping_time, w.max_stopping_time_seed) == \
                (p.max_stopping_time, p.max_stopping_time_seed), var
            assert (w.max_excursion, w.max_excursion_seed) == (p.max_excursion, p.max_excursion_seed), var
    finally:
        v.set_variant(cb.MODE_RANGE64, 0)
        v.set_variant(cb.MODE_RANGE64_BITS, cb.RANGE64_BITS_DEFAULT)


def test_batch_of_tiny_requests(verifier):
    """Hundreds of requests of 1..400 seeds in one launch: work items of one
    or two seeds each, so a warp's seed queue holds seeds of far more items
    than it has item slots; every request must still get exactly its own
    seeds and maxima."""
    import random
    from oracle import oracle as O
    rng = random.Random(77)
    reqs = []
    for _ in range(600):
        off = rng.randrange(1 << 40, 1 << 50)
        reqs.append((off, rng.randint(1, 400), 24, True))
    reqs.append((3, 300, 24, True))  # below 2^k
    v = verifier(26)
    got = v.verify_batch(reqs)
    for q, g in zip(reqs, got):
        o = O.range_verify(*q, method=1)
        _cmp(g, o)


NEG_CASES = [
    (2, 1 << 20, 16, True),                     # dense part and sieved part; the cycle minima 5, 17
    ((1 << 40) + 12345, 1 << 21, 24, True),     # unaligned
    (1 << 40, 1 << 22, 20, False),              # no mod-9 sieve
    ((1 << 62) - 999, 1 << 20, 24, True),
    ((1 << 60) + (3 << 34) - 5000, 300000, 34, True),  # frontier sieve, crosses a block
]


@pytest.mark.parametrize("case", NEG_CASES, ids=lambda c: f"neg-o{c[0]:x}-s{c[1]}-k{c[2]}-m{int(c[3])}")
def test_negative_range_matches_oracle(verifier, case):
    """The negative-integer variant T'(m) = (3m-1)/2, m/2 against the oracle's
    run-length formulation; the cycle minima count as failures."""
    from oracle import oracle as O
    off, size, k, mod9 = case
    g = verifier(26).verify_range(off, size, k, mod9, negative=True)
    o = O.range_verify(off, size, k, mod9, method=1, nthreads=NT, negative=True)
    assert g.errors == 0
    assert (g.seeds_checked, g.failures) == (o.seeds, o.failures)
    assert (g.max_stopping_time, g.max_stopping_time_seed) == (o.max_st, o.max_st_seed)
    assert (g.max_excursion, g.max_excursion_seed) == (o.max_exc, o.max_exc_seed)
    if off <= 5 and off + size > 17:
        assert g.failures == 2


def test_negative_batch_and_mixed_plan_rules(verifier):
    import collatz_b200 as cb
    v = verifier(26)
    reqs = [((1 << 44) + 7 * i, 5000 + 100 * i, 24, True, True) for i in range(8)]
    got = v.verify_batch(reqs)
    for q, g in zip(reqs, got):
        alone = v.verify_range(*q[:4], negative=True)
        assert _key(g) == _key(alone)
    with pytest.raises(cb.CollatzError):  # one sieve (k, sign) per launch
        v.verify_batch([(1 << 44, 1000, 24, True, True), (1 << 44, 1000, 24, True, False)])


def test_batch_equals_alone(verifier):
    """Each request's result is the same alone and in a mixed batch."""
    v = verifier(26)
    reqs = [((1 << 40) + i * (1 << 24) + 9 * i, (1 << 18) + 1000 * i, 24, True) for i in range(12)]
    reqs.append((1 << 50, 1 << 23, 24, True))
    reqs.append((17, 40000, 24, True))
    mixed = v.verify_batch(reqs)
    for q, m in zip(reqs, mixed):
        assert _key(v.verify_range(*q)) == _key(m)


def _key(r):
    return (r.seeds_checked, r.failures, r.max_stopping_time, r.max_stopping_time_seed, r.max_excursion,
            r.max_excursion_seed, r.errors)


def test_plan_relaunch_is_deterministic(verifier):
    v = verifier(26)
    p = v.plan([(1 << 44, 1 << 24, 24, True), ((1 << 52) + 1, 1 << 22, 24, True)])
    p.launch()
    a = p.results()
    p.launch()
    b = p.results()
    for x, y in zip(a, b):
        assert (x.seeds_checked, x.max_excursion, x.max_excursion_seed, x.max_stopping_time,
                x.max_stopping_time_seed) == (y.seeds_checked, y.max_excursion, y.max_excursion_seed,
                                              y.max_stopping_time, y.max_stopping_time_seed)
    p.close()


def test_shards_combine(verifier):
    """Disjoint shards (the multi-GPU split) combine to the whole range."""
    import collatz_b200 as cb
    v = verifier(26)
    off, size = (1 << 41) + 3, 5 << 22
    whole = v.verify_range(off, size, 24)
    parts = [v.verify_range(off + i * (size // 4), size // 4, 24) for i in range(4)]
    c = cb.combine_range_results(parts)
    assert (c.seeds_checked, c.max_excursion, c.max_excursion_seed, c.max_stopping_time,
            c.max_stopping_time_seed) == (whole.seeds_checked, whole.max_excursion,
                                          whole.max_excursion_seed, whole.max_stopping_time,
                                          whole.max_stopping_time_seed)


def test_limits_rejected(verifier):
    import collatz_b200 as cb
    v = verifier(26)
    with pytest.raises(cb.CollatzError):
        v.verify_range((1 << 96) - 10, 100, 24)
    with pytest.raises(cb.CollatzError):
        v.verify_range(1 << 40, 1 << 49, 24)


@pytest.mark.parametrize("off,size,k", [((1 << 40) + 12345, 1 << 32, 24), ((1 << 60) + (5 << 34), 1 << 34, 34),
                                        ((1 << 90) + 777, 1 << 30, 24)])
def test_window_variant_equals_plain(verifier, off, size, k):
    """The 8-step window after the k-step jump (variant 4) leaves every output
    unchanged on large ranges, where most seeds take it: seeds, maxima with
    their seeds, failures and widened seeds equal the plain variant's."""
    v = verifier(26, range_k=k)
    import collatz_b200 as cb
    v.set_variant(cb.MODE_RANGE64_BITS, 0)  # the four-limb kernel
    try:
        v.set_variant(1, 4)
        w = v.verify_range(off, size, k)
        v.set_variant(1, 2)
        p = v.verify_range(off, size, k)
    finally:
        v.set_variant(1, 0)  # the defaults
        v.set_variant(cb.MODE_RANGE64_BITS, cb.RANGE64_BITS_DEFAULT)
    assert (w.seeds_checked, w.failures, w.widened, w.errors) == (p.seeds_checked, p.failures, p.widened, p.errors)
    assert (w.max_stopping_time, w.max_stopping_time_seed) == (p.max_stopping_time, p.max_stopping_time_seed)
    assert (w.max_excursion, w.max_excursion_seed) == (p.max_excursion, p.max_excursion_seed)


@pytest.mark.parametrize("off,size,k", [((1 << 40) + 777, 1 << 33, 24), ((1 << 56) + 12345, 1 << 30, 24),
                                        ((1 << 58) + (7 << 24), 1 << 30, 24), ((1 << 63) + 5, 1 << 28, 24)])
def test_narrow_variant_equals_plain(verifier, off, size, k):
    """The 64-bit body (variant 6: taken while every active lane's value is below
    2^59) leaves every output unchanged: at 2^40 nearly all steps take it, at
    2^56-2^58 warps switch between the bodies, at 2^63 the seeds start above
    its limit."""
    v = verifier(26, range_k=k)
    import collatz_b200 as cb
    v.set_variant(cb.MODE_RANGE64_BITS, 0)  # the four-limb kernel
    try:
        v.set_variant(1, 6)
        w = v.verify_range(off, size, k)
        v.set_variant(1, 2)
        p = v.verify_range(off, size, k)
    finally:
        v.set_variant(1, 0)  # the defaults
        v.set_variant(cb.MODE_RANGE64_BITS, cb.RANGE64_BITS_DEFAULT)
    assert (w.seeds_checked, w.failures, w.widened, w.errors) == (p.seeds_checked, p.failures, p.widened, p.errors)
    assert (w.max_stopping_time, w.max_stopping_time_seed) == (p.max_stopping_time, p.max_stopping_time_seed)
    assert (w.max_excursion, w.max_excursion_seed) == (p.max_excursion, p.max_excursion_seed)


@pytest.mark.parametrize("width", [0, 48])
def test_range_edges_both_kernels(verifier, width):
    """Empty and one-seed ranges, a range of the smallest kept seeds, and a range
    straddling 2^48 (its launch has 49-bit seeds, so it runs four limbs even
    with the 64-bit kernel enabled) give the oracle's results with the limb
    width at 0 (four limbs only) and at 48."""
    import collatz_b200 as cb
    from oracle import oracle as O
    v = verifier(26)
    v.set_variant(cb.MODE_RANGE64_BITS, width)
    try:
        for off, size, k in [(1 << 40, 0, 24), ((1 << 40) + 27, 1, 24), ((1 << 40) + 28, 1, 24), (2, 1, 16),
                             (0, 10, 16), ((1 << 48) - (1 << 20), 1 << 21, 24)]:
            g = v.verify_range(off, size, k)
            o = O.range_verify(off, size, k, True, method=1, nthreads=NT)
            assert g.errors == 0 and g.failures == 0
            assert g.seeds_checked == o.seeds, (off, size)
            if o.seeds:
                assert (g.max_stopping_time, g.max_stopping_time_seed) == (o.max_st, o.max_st_seed)
                assert (g.max_excursion, g.max_excursion_seed) == (o.max_exc, o.max_exc_seed)
    finally:
        v.set_variant(cb.MODE_RANGE64_BITS, cb.RANGE64_BITS_DEFAULT)
