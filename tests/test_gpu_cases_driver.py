"""Cases driver on the GPU: the Step-1 subtrees of the N = 36 root case run
as separate cases_* lines combine to the reference's whole-run outputs
(hash AF103480, 76 684 750 seeds); a rerun with the journal runs nothing,
and a journal cut in half resumes with the rest."""
import os
import subprocess

import pytest

from conftest import ROOT, load_golden

pytestmark = pytest.mark.gpu


def _whole():
    return next(r for r in load_golden("cases_runs.json")["runs"]
                if r["N"] == 36 and r["tuple"] == [3, 2, 2, 9, 1, 0])


def _lines():
    from oracle import oracle as O
    return O.split_case(36, (3, 2, 2, 9, 1, 0), 12)


def test_driver_combines_and_resumes(verifier, tmp_path):
    whole = _whole()
    lines = _lines()
    assert len(lines) > 20
    v = verifier(36)
    j = str(tmp_path / "journal.txt")
    comb, per, ran = v.run_cases(lines, journal=j)
    assert ran == len(lines)
    assert f"{comb.hash:X}" == whole["hash"] and comb.seeds_checked == whole["seeds"]
    assert sum(p.seeds_checked for p in per) == whole["seeds"]
    # everything is in the journal: nothing runs again, same outputs
    comb2, _, ran2 = v.run_cases(lines, journal=j)
    assert ran2 == 0
    key = lambda c: (c.hash, c.seeds_checked, c.launches, c.max_excursion, c.max_excursion_seed,  # noqa: E731
                     c.max_stopping_time, c.max_stopping_time_seed)
    assert key(comb2) == key(comb)
    # keep the first half (plus a cut-short line): the rest runs, same outputs
    rows = open(j).read().splitlines(keepends=True)
    half = len(rows) // 2
    with open(j, "w") as f:
        f.writelines(rows[:half])
        f.write(rows[half][:25])
    comb3, _, ran3 = v.run_cases(lines, journal=j)
    assert ran3 == len(lines) - half
    assert key(comb3) == key(comb)
    # the combined maxima equal those of the whole run
    w = v.run_case(3, 2, 2, 9, 1, 0)
    assert key(comb)[3:] == key(w)[3:]


def test_cli_cases_file(tmp_path):
    whole = _whole()
    lines = _lines()
    cf = tmp_path / "cases_test"
    cf.write_text("".join(" ".join(str(x) for x in t) + "\n" for t in lines))
    cli = os.path.join(ROOT, "collatz_b200", "collatz_b200")
    p = subprocess.run([cli, "--cases", str(cf), "--journal", str(tmp_path / "j"), "36"],
                       capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stderr
    assert f"Complete hash = {whole['hash']}." in p.stderr
    assert '"cases_run": %d' % len(lines) in p.stderr
