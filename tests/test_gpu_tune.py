"""Autotuner (collatz_autotune): every variant gives the same results, the
tuner keeps the fastest, records it in its cache, and a new context created
with the automatic variant applies the cached choice."""
import pytest

pytestmark = pytest.mark.gpu


def _key(r):
    return (r.seeds_checked, r.failures, r.max_stopping_time, r.max_stopping_time_seed, r.max_excursion,
            r.max_excursion_seed, r.errors)


def test_every_variant_same_results(verifier):
    import collatz_b200 as cb
    v = verifier(36)
    ref_range = None
    v.set_variant(cb.MODE_RANGE64_BITS, 0)  # the four-limb kernel's variants first
    for var in range(cb.lib().collatz_variant_count(1)):
        v.set_variant(1, var)
        r = _key(v.verify_range((1 << 44) + 12345, 3 << 21, 24))
        assert ref_range is None or r == ref_range, var
        ref_range = r
    v.set_variant(cb.MODE_RANGE64_BITS, 48)  # then the 64-bit kernel's
    for var in range(cb.lib().collatz_variant_count(cb.MODE_RANGE64)):
        v.set_variant(cb.MODE_RANGE64, var)
        assert _key(v.verify_range((1 << 44) + 12345, 3 << 21, 24)) == ref_range, var
    v.set_variant(cb.MODE_RANGE64, 0)
    v.set_variant(cb.MODE_RANGE64_BITS, cb.RANGE64_BITS_DEFAULT)
    ref_case = None
    for var in range(cb.lib().collatz_variant_count(0)):
        v.set_variant(0, var)
        c = v.run_case(27, 10, 8, 183, 0, 0)
        got = (c.hash, c.seeds_checked, c.max_excursion, c.max_excursion_seed, c.max_stopping_time,
               c.max_stopping_time_seed)
        assert ref_case is None or got == ref_case, var
        ref_case = got
    v.set_variant(1, 0)  # the defaults
    v.set_variant(0, 4)


def test_autotune_records_and_reuses(tmp_path, monkeypatch):
    import collatz_b200 as cb
    cache = tmp_path / "tune.txt"
    monkeypatch.setenv("COLLATZ_TUNE_CACHE", str(cache))
    with cb.Verifier(36, range_k=20) as v:
        t = v.autotune()
    nr, nc = cb.lib().collatz_variant_count(1), cb.lib().collatz_variant_count(0)
    assert len(t["range_ms"]) == nr and len(t["cases_ms"]) == nc
    assert t["range_ms"][t["range_variant"]] == min(t["range_ms"])
    assert t["cases_ms"][t["cases_variant"]] == min(t["cases_ms"])
    n64 = cb.lib().collatz_variant_count(cb.MODE_RANGE64)
    assert len(t["range64_ms"]) == n64 and t["range64_ms"][t["range64_variant"]] == min(t["range64_ms"])
    assert t["range64_bits"] in (0, 44, 48) and all(x > 0 for x in t["width_ms"])
    lines = cache.read_text().splitlines()
    assert any(ln.startswith("range ") and f" 20 {t['range_variant']} " in ln for ln in lines)
    assert any(ln.startswith("cases ") and f" 36 {t['cases_variant']} " in ln for ln in lines)
    # a new context with the automatic variant picks up the cached choice
    with cb.Verifier(36, range_k=20) as v2:
        t2 = v2.autotune(range_mode=False, cases_mode=False)
        assert (t2["range_variant"], t2["cases_variant"]) == (t["range_variant"], t["cases_variant"])
        assert (t2["range64_variant"], t2["range64_bits"]) == (t["range64_variant"], t["range64_bits"])
