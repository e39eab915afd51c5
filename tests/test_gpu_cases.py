"""Cases mode on the GPU against the reference's own outputs (golden fixtures
made by running collatz_cudav7.cu through the CPU shim, tests/golden/) and
against the oracle for the outputs the reference does not define."""
import hashlib

import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu

RUNS = load_golden("cases_runs.json")["runs"]
TABLES = load_golden("tables.json")["tables"]


@pytest.mark.parametrize("t", TABLES, ids=lambda t: f"N{t['N']}")
def test_tables_bit_identical(verifier, t):
    """The 16 bit vectors and the mod-9 sieve built on the GPU equal the
    reference's precompute() (cu:423-495) byte for byte."""
    bv, m9 = verifier(t["N"]).case_tables()
    assert hashlib.sha256(m9).hexdigest() == t["mod9_sha256"]
    n = len(bv) // 16
    for i in range(16):
        assert hashlib.sha256(bv[i * n:(i + 1) * n]).hexdigest() == t["bv_each_sha256"][i], f"BV_{i}"
    assert hashlib.sha256(bv).hexdigest() == t["bv_sha256"]


@pytest.mark.parametrize("n", [26, 42, 45])
def test_pair_batches_match_reference_kernel(verifier, n):
    """launchkernel on explicit batches (Step-1 leaves and synthetic pairs
    that cross 2^100) reproduces compute_kernel's hash, seed count and
    overflow report."""
    fx = load_golden(f"pairs_N{n}.json")
    v = verifier(n)
    for b in fx["batches"]:
        pairs = [(int(x), int(y)) for x, y in b["pairs"]]
        r = v.launchkernel(b["bigindex"], pairs)
        assert f"{r.hash:X}" == b["hash"], (b["kind"], b["bigindex"])
        assert r.seeds_checked == b["seeds"], (b["kind"], b["bigindex"])
        assert sorted(r.overflow) == sorted(int(x) for x in b["overflow"])
        assert r.n_overflow == len(b["overflow"])
        assert r.launches == 1


@pytest.mark.parametrize("n", [26, 42, 45])
def test_search2_semantics(verifier, n):
    """Pairs with bigindex >= 16 take the reference's CPU path (search2,
    cu:654-715: mod-9 sieve only); bigindex < 16 through search2 is the
    spot-check path and must agree with the kernel."""
    fx = load_golden(f"pairs_N{n}.json")
    v = verifier(n)
    for d in fx["search2"]:
        r = v.launchkernel(d["bigindex"], [(int(d["base"]), int(d["number"]))])
        assert f"{r.hash:X}" == d["hash"], d
        assert sorted(r.overflow) == sorted(int(x) for x in d["overflow"])


def _fast_runs():
    return [r for r in RUNS if r["N"] <= 42 or r["tuple"][1] >= 20]


@pytest.mark.parametrize("run", _fast_runs(), ids=lambda r: f"N{r['N']}-" + "_".join(map(str, r["tuple"])))
def test_run_case_matches_reference(verifier, run):
    """Whole runs: hash, launch count, seeds checked and overflow list equal
    the reference program's (cu:95-183)."""
    r = verifier(run["N"]).run_case(*run["tuple"])
    assert f"{r.hash:X}" == run["hash"]
    assert r.launches == run["launches"]
    assert r.seeds_checked == run["seeds"]
    assert sorted(r.overflow) == sorted(int(x) for x in run["overflow"])
    assert r.errors == 0


@pytest.mark.parametrize("run", [r for r in RUNS if r["N"] == 45 and r["tuple"][1] < 20],
                         ids=lambda r: "N45-" + "_".join(map(str, r["tuple"])))
def test_run_case_n45_default(verifier, run):
    """The reference's default N = 45 on cases_tiny lines (555 M seeds for line 1)."""
    r = verifier(45).run_case(*run["tuple"])
    assert f"{r.hash:X}" == run["hash"]
    assert r.launches == run["launches"]
    assert r.seeds_checked == run["seeds"]


@pytest.mark.parametrize("n,tup", [(26, (3, 2, 2, 9, 1, 0)), (30, (3, 2, 2, 9, 1, 0)),
                                   (36, (27, 10, 8, 183, 0, 0))])
def test_case_maxima_match_oracle(verifier, oracle_tables, n, tup):
    """Maximum stopping time and excursion (with seeds, ties to the smaller
    seed) equal the oracle's; the hash doubles as a cross-check."""
    r = verifier(n).run_case(*tup)
    o = oracle_tables(n).run_case(*tup)
    assert r.hash == o.hash
    assert r.seeds_checked == o.seeds
    assert (r.max_stopping_time, r.max_stopping_time_seed) == (o.max_st, o.max_st_seed)
    assert (r.max_excursion, r.max_excursion_seed) == (o.max_exc, o.max_exc_seed)


@pytest.mark.parametrize("variant", range(5))
def test_every_cases_variant_matches_reference(verifier, oracle_tables, variant):
    """Each cases-kernel variant reproduces the reference's pair batches
    (overflow reports included), search2 pairs, and the oracle's maxima."""
    import collatz_b200 as cb
    assert cb.lib().collatz_variant_count(0) == 5
    v = verifier(45)
    v.set_variant(0, variant)
    try:
        fx = load_golden("pairs_N45.json")
        for b in fx["batches"]:
            r = v.launchkernel(b["bigindex"], [(int(x), int(y)) for x, y in b["pairs"]])
            assert f"{r.hash:X}" == b["hash"] and r.seeds_checked == b["seeds"], (variant, b["kind"])
            assert sorted(r.overflow) == sorted(int(x) for x in b["overflow"])
        for d in fx["search2"]:
            r = v.launchkernel(d["bigindex"], [(int(d["base"]), int(d["number"]))])
            assert f"{r.hash:X}" == d["hash"], (variant, d)
        v36 = verifier(36)
        v36.set_variant(0, variant)
        r = v36.run_case(27, 10, 8, 183, 0, 0)
        o = oracle_tables(36).run_case(27, 10, 8, 183, 0, 0)
        assert (r.hash, r.seeds_checked) == (o.hash, o.seeds)
        assert (r.max_stopping_time, r.max_stopping_time_seed) == (o.max_st, o.max_st_seed)
        assert (r.max_excursion, r.max_excursion_seed) == (o.max_exc, o.max_exc_seed)
    finally:  # back to the default variant
        v.set_variant(0, 4)
        verifier(36).set_variant(0, 4)


def test_pair_maxima_match_oracle(verifier, oracle_tables):
    fx = load_golden("pairs_N26.json")
    v, T = verifier(26), oracle_tables(26)
    for b in fx["batches"]:
        pairs = [(int(x), int(y)) for x, y in b["pairs"]]
        r = v.launchkernel(b["bigindex"], pairs)
        o = T.pairs_result(b["bigindex"], pairs)
        assert r.hash == o.hash
        assert (r.max_stopping_time, r.max_stopping_time_seed) == (o.max_st, o.max_st_seed)
        assert (r.max_excursion, r.max_excursion_seed) == (o.max_exc, o.max_exc_seed)


def test_xor_partition(verifier):
    """Splitting a case into sub-cases (as the cases_* files do) XOR-composes
    to the whole run's hash, and the seed counts add up."""
    from oracle import oracle as O
    v = verifier(36)
    whole = v.run_case(3, 2, 2, 9, 1, 0)
    roots = O.split_case(36, (3, 2, 2, 9, 1, 0), 12)
    assert len(roots) > 20
    h, seeds = 0, 0
    for rt in roots:
        r = v.run_case(*rt)
        h ^= r.hash
        seeds += r.seeds_checked
    assert h == whole.hash
    assert seeds == whole.seeds_checked
    assert f"{h:X}" == "AF103480"


def test_bad_case_rejected(verifier):
    import collatz_b200 as cb
    v = verifier(26)
    with pytest.raises(cb.CollatzError):
        v.run_case(3, 17, 12, 9, 1, 0)  # sigfig > N - A: the reference never terminates


@pytest.mark.parametrize("flags", [[], ["--host-step1"]], ids=["device-step1", "host-step1"])
def test_cli_drop_in_output(flags):
    """The CLI prints the reference's stderr summary (cu:181-182) and the
    overflow list on stdout (cu:298 format) for one stdin 6-tuple."""
    import os
    import subprocess
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    cli = os.path.join(root, "collatz_b200", "collatz_b200")
    p = subprocess.run([cli] + flags + ["26"], input="3 2 2 9 1 0\n", capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stderr
    lines = p.stderr.splitlines()
    assert lines[0] == "Number of kernel launches = 6. Spot checks = 0. Complete hash = 86E5527C."
    assert lines[1].startswith("# results {") and '"seeds_checked": 142133' in lines[1]
    assert p.stdout == ""


def test_iteration_cap_reports_instead_of_running_on():
    """A per-seed checkpoint cap that real seeds exceed ends those seeds with
    the ERR_ITER_CAP bit and a failure count (status COLLATZ_E_DEVICE); the
    launch finishes and the context stays usable."""
    import collatz_b200 as cb
    with cb.Verifier(26, iter_cap=2) as v:
        r = v.run_case(3, 2, 2, 9, 1, 0, check=False)
        assert r.errors & 0x2
        with pytest.raises(cb.CollatzError) as e:
            v.run_case(3, 2, 2, 9, 1, 0)
        assert e.value.status == cb.E_DEVICE
        assert v.trajectory([27, 97])[0][0] == 3  # trajectory queries: status 3, iteration cap
    # a fresh context computes the reference's answer
    assert f"{cb.Verifier(26).run_case(3, 2, 2, 9, 1, 0).hash:X}" == "86E5527C"


@pytest.mark.parametrize("n", [52, 53])
def test_narrow_body_matches_four_limbs_at_high_n(verifier, n):
    """N = 52 is the largest N that runs the 64-bit body: its seeds lie below
    2^52 and their values pass 2^59 often, so lanes switch bodies step by step.
    At N = 53 variant 4 falls back to the four-limb kernel.  Variant 4 and the
    four-limb variant 3 must give identical hashes, counts, overflow lists and
    maxima on lines of the N-bit tree."""
    import collatz_b200 as cb
    lines = cb.split_cases(n, (3, 2, 2, 9, 1, 0), 26)
    picks = [cb.case_tuple(lines[i]) for i in (0, 1, 1000, len(lines) // 2, len(lines) - 1)]
    v = verifier(n)
    try:
        for t in picks:
            v.set_variant(0, 4)
            a = v.run_case(*t)
            v.set_variant(0, 3)
            b = v.run_case(*t)
            assert (a.hash, a.seeds_checked, a.launches, a.n_overflow) == \
                (b.hash, b.seeds_checked, b.launches, b.n_overflow), t
            assert sorted(a.overflow) == sorted(b.overflow), t
            assert (a.max_stopping_time, a.max_stopping_time_seed) == (b.max_stopping_time, b.max_stopping_time_seed)
            assert (a.max_excursion, a.max_excursion_seed) == (b.max_excursion, b.max_excursion_seed)
            assert a.seeds_checked > 0
    finally:
        v.set_variant(0, 4)  # the default
