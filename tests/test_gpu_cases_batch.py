"""Line batches (collatz_run_case_batch): many cases_* lines verified in one
device pass with one record per line.  Every line's result must equal what
collatz_run_case gives for it alone, and the reference's own outputs where
the golden fixtures hold them."""
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu

RUNS = load_golden("cases_runs.json")["runs"]


def _key(r):
    return (f"{r.hash:X}", r.launches, r.seeds_checked, r.pairs, r.cpu_pairs, r.n_overflow, sorted(r.overflow),
            r.max_stopping_time, r.max_stopping_time_seed, r.max_excursion, r.max_excursion_seed, r.errors)


@pytest.mark.parametrize("n", sorted({r["N"] for r in RUNS}))
def test_batch_of_reference_runs(verifier, n):
    """All golden runs of one N in one batch: each line's hash, launch count,
    seed count and overflow list equal the reference program's."""
    runs = [r for r in RUNS if r["N"] == n]
    res = verifier(n).run_case_batch([r["tuple"] for r in runs])
    assert len(res) == len(runs)
    for run, r in zip(runs, res):
        assert f"{r.hash:X}" == run["hash"], run["tuple"]
        assert r.launches == run["launches"], run["tuple"]
        assert r.seeds_checked == run["seeds"], run["tuple"]
        assert sorted(r.overflow) == sorted(int(x) for x in run["overflow"])
        assert r.errors == 0


def test_batch_equals_alone(verifier):
    """Lines at different sigfigs (two cuts of the N = 36 tree), a root the
    induction sieve prunes, a root that is itself a leaf, and a line given
    twice: each result equals the line run alone."""
    from oracle import oracle as O
    v = verifier(36)
    lines = O.split_case(36, (3, 2, 2, 9, 1, 0), 12)[:20] + O.split_case(36, (3, 2, 2, 9, 1, 0), 16)[-60:]
    lines += [(0, 5, 0, 1, 0, 0), (3, 26, 17, 9, 0, 0), lines[3]]
    batch = v.run_case_batch(lines)
    for t, b in zip(lines, batch):
        assert _key(b) == _key(v.run_case(*t)), t
    assert _key(batch[-1]) == _key(batch[3])
    assert batch[-3].seeds_checked == 0 and batch[-3].launches == 0


def test_overflow_seeds_go_to_their_line(verifier, oracle_tables):
    """Synthetic lines whose numbers lie near 2^99 report hundreds of
    overflow seeds; in a batch with an ordinary line, each line gets exactly
    its own list (equal to the oracle's and to the line run alone)."""
    v, T = verifier(40), oracle_tables(40)
    lines = [(5, 28, 20, (1 << 99) - 12345, 0, 0), (27, 10, 8, 183, 0, 0),
             (7, 27, 19, (1 << 98) + 999, 0, 0), (3, 29, 21, (1 << 99) + (1 << 97), 0, 1)]
    batch = v.run_case_batch(lines)
    for t, b in zip(lines, batch):
        alone = v.run_case(*t)
        assert _key(b) == _key(alone), t
        o = T.run_case(*t)
        assert (b.hash, b.seeds_checked) == (o.hash, o.seeds)
        assert sorted(b.overflow) == sorted(o.overflow)
    assert [len(b.overflow) for b in batch] == [432, 0, 529, 281]


@pytest.mark.parametrize("cut", [20, 24])
def test_many_small_lines_compose_to_the_whole_run(verifier, cut):
    """The N = 36 root split into 16 264 (cut 20) or 178 304 (cut 24) lines,
    the shape of a cases_big file, in one batch: the XOR of the lines'
    hashes and the sum of their seeds equal the reference's whole run."""
    from oracle import oracle as O
    lines = O.split_case(36, (3, 2, 2, 9, 1, 0), cut)
    res = verifier(36).run_case_batch(lines)
    h, seeds, launches = 0, 0, 0
    for r in res:
        h ^= r.hash
        seeds += r.seeds_checked
        assert r.errors == 0
    assert f"{h:X}" == "AF103480"
    assert seeds == 76684750


def test_driver_runs_groups_and_resumes(verifier, tmp_path):
    """collatz_run_cases on 16 264 lines runs two device passes (8192 lines
    each at most), journals every line, and a rerun takes all of them from
    the journal."""
    from oracle import oracle as O
    lines = O.split_case(36, (3, 2, 2, 9, 1, 0), 20)
    j = str(tmp_path / "j.txt")
    v = verifier(36)
    comb, per, ran = v.run_cases(lines, journal=j)
    assert ran == len(lines) == 16264
    assert f"{comb.hash:X}" == "AF103480" and comb.seeds_checked == 76684750
    with open(j) as f:
        assert sum(1 for _ in f) == len(lines)
    comb2, _, ran2 = v.run_cases(lines, journal=j)
    assert ran2 == 0 and comb2.hash == comb.hash and comb2.seeds_checked == comb.seeds_checked


def test_batch_argument_checks(verifier):
    import collatz_b200 as cb
    v = verifier(26)
    with pytest.raises(cb.CollatzError):
        v.run_case_batch([(3, 2, 2, 9, 1, 0), (3, 17, 12, 9, 1, 0)])  # sigfig > N - A
    assert v.run_case_batch([]) == []


def test_overflow_pool_smaller_than_the_reports(verifier):
    """With an overflow pool of 500 seeds for 1 242 reports, every line still
    counts all its reports (n_overflow), the pool is filled line by line, and
    each line's part is a subset of its full list."""
    v = verifier(40)
    lines = [(5, 28, 20, (1 << 99) - 12345, 0, 0), (7, 27, 19, (1 << 98) + 999, 0, 0),
             (3, 29, 21, (1 << 99) + (1 << 97), 0, 1)]
    part = v.run_case_batch(lines, pool_cap=500)
    full = v.run_case_batch(lines)
    assert [r.n_overflow for r in part] == [432, 529, 281]
    assert [len(r.overflow) for r in part] == [432, 68, 0]
    for p, f in zip(part, full):
        assert set(p.overflow) <= set(f.overflow)
        assert (p.hash, p.seeds_checked) == (f.hash, f.seeds_checked)
