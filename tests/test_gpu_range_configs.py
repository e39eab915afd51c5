"""The benchmark configurations at their stated sizes against the CPU oracle's
fixtures (tests/golden/range_configs.json, made by
tests/golden/make_range_golden.py): the same seeds checked, failures, maximum
stopping time and maximum excursion with their seeds, on the product's range
path (collatz_verify_range / collatz_verify_batch) and, for the batch, its
plan (one persistent launch of a captured graph)."""
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu


def _key(r):
    return (r.seeds_checked, r.failures, r.max_stopping_time, r.max_stopping_time_seed, r.max_excursion,
            r.max_excursion_seed, r.errors)


def _want(g):
    return (g["seeds"], g["failures"], g["max_stopping_time"], int(g["max_stopping_time_seed"]),
            int(g["max_excursion"]), int(g["max_excursion_seed"]), 0)


@pytest.fixture(scope="module")
def fx():
    return load_golden("range_configs.json")


def test_config1_plain_all_below_2p32(verifier, fx):
    """Every n < 2^32, 2^16 sieve + mod-9: the oracle's 64-bit loop with
    overflow detection gives the reference answer."""
    c = fx["config1"]
    v = verifier(26, range_k=16)
    r = v.verify_range(int(c["offset"]), int(c["size"]), c["k"])
    assert _key(r) == _want(c["result"])


def test_config2_full_block(verifier, fx):
    """The headline workload: [2^40, 2^40 + 2^38), k = 24, one launch."""
    c = fx["config2"]
    v = verifier(26)
    r = v.verify_range(int(c["offset"]), int(c["size"]), c["k"])
    assert _key(r) == _want(c["result"])
    assert r.widened == 0


def test_config3_frontier_sub_block(verifier, fx):
    """2^36 seeds of the frontier block at 2^60 with the 2^34-bit sieve."""
    c = fx["config3"]
    v = verifier(26, range_k=34)
    r = v.verify_range(int(c["offset"]), int(c["size"]), c["k"])
    assert _key(r) == _want(c["result"])


def test_config4_batched_subset(verifier, fx):
    """516 requests of the batched configuration (sizes 2^20..2^31 at offsets
    up to 2^64) in one batch and in one plan launch, each request equal to
    the oracle's result for it alone."""
    reqs = fx["config4"]["requests"]
    v = verifier(26)
    qs = [(int(q["offset"]), int(q["size"]), q["k"], True) for q in reqs]
    got = v.verify_batch(qs)
    for q, r in zip(reqs, got):
        assert _key(r) == _want(q["result"]), q["index"]
    plan = v.plan(qs)
    try:
        plan.launch()
        for q, r in zip(reqs, plan.results()):
            assert _key(r) == _want(q["result"]), q["index"]
    finally:
        plan.close()
