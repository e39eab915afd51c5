"""Measured integer peak (collatz_int_peak): the loop performs the operations
it counts at a rate the device can issue, and reports the clock it ran at."""
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("mix", [0, 1])
def test_int_peak_plausible(verifier, mix):
    r = verifier(26).int_peak(mix)
    assert r["mix"] == mix
    # 8 blocks x 256 threads per SM, 2^17 iterations of 8 chains x 3 operations
    assert r["ops"] == r["sm_count"] * 8 * 256 * (1 << 17) * 8 * 3
    assert 200.0 < r["sm_mhz"] < 2500.0
    assert r["ms"] > 0.0
    # at most one warp instruction per SM sub-partition and clock: 128 lanes per SM
    assert 16.0 <= r["ops_per_clk_sm"] <= 128.0 * 1.03


def test_int_peak_rejects_unknown_mix(verifier):
    import collatz_b200 as cb
    with pytest.raises(cb.CollatzError):
        verifier(26).int_peak(2)
