"""Results of disjoint sub-ranges combine to the whole range's: the multi-GPU
split (one block per rank), batch segments and server slices all rely on it.
Random cut points (not aligned to the sieve modulus) over small ranges, each
piece run by the oracle, combined with collatz_b200.combine_range_results
(sums, maxima with the smaller seed on ties), against one oracle run over the
whole range."""
import pytest
from hypothesis import given, settings, strategies as st


def _rr(o):
    import collatz_b200 as cb
    return cb.RangeResult(o.seeds, o.failures, 0, o.max_exc, o.max_exc_seed, o.max_st, o.max_st_seed)


@settings(max_examples=25, deadline=None, derandomize=True)
@given(off_lo=st.integers(0, (1 << 20) - 1), size=st.integers(1, 1 << 16),
       cuts=st.lists(st.floats(0.0, 1.0), min_size=0, max_size=6), k=st.sampled_from([8, 12, 16]))
def test_split_anywhere_combines_to_whole(off_lo, size, cuts, k):
    import collatz_b200 as cb
    from oracle import oracle as O
    off = (1 << 40) + off_lo
    pts = sorted({0, size} | {int(c * size) for c in cuts})
    parts = [_rr(O.range_verify(off + a, b - a, k, True, 1, 1)) for a, b in zip(pts, pts[1:]) if b > a]
    c = cb.combine_range_results(parts)
    w = O.range_verify(off, size, k, True, 1, 1)
    assert (c.seeds_checked, c.failures) == (w.seeds, w.failures)
    if w.seeds:
        assert (c.max_stopping_time, c.max_stopping_time_seed) == (w.max_st, w.max_st_seed)
        assert (c.max_excursion, c.max_excursion_seed) == (w.max_exc, w.max_exc_seed)


def test_empty_parts_do_not_set_maxima():
    import collatz_b200 as cb
    empty = cb.RangeResult(0, 0, 0, 0, 0, 0, 0)
    one = cb.RangeResult(5, 0, 0, 1000, 27, 96, 27)
    c = cb.combine_range_results([empty, one, empty])
    assert (c.seeds_checked, c.max_excursion, c.max_excursion_seed, c.max_stopping_time,
            c.max_stopping_time_seed) == (5, 1000, 27, 96, 27)


def test_ties_keep_the_smaller_seed():
    import collatz_b200 as cb
    a = cb.RangeResult(3, 0, 0, 500, 91, 40, 91)
    b = cb.RangeResult(4, 0, 0, 500, 33, 40, 57)
    for parts in ([a, b], [b, a]):
        c = cb.combine_range_results(parts)
        assert (c.max_excursion_seed, c.max_stopping_time_seed, c.seeds_checked) == (33, 57, 7)
