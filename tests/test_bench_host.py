"""bench.py's host-side measurement of the reference's own program against the
drop-in CLI (cases_tiny line 1 at N = 45), with the two programs replaced by
fakes and a fake clock: the four runs (each program on line 1 and on the
start-up-only input) are interleaved, each keeps its best time, a start-up
subtracted run time is reported only when it is not negative, and a program
that fails raises."""
import types

import pytest

SUMMARY = "Number of kernel launches = 69. Spot checks = 0. Complete hash = 9F6332DF."
LINE1, EMPTY = "27 10 8 183 0 0\n", "0 5 0 1 0 0\n"


class _Proc:
    def __init__(self, rc, err):
        self.returncode = rc
        self.stderr = err


def _fake(monkeypatch, tmp_path, durations, rc=0):
    """durations[(program, input)] = list of seconds, one per repetition."""
    import bench
    for rel in ("oracle/_ref/ref_gpu_N45", "collatz_b200/collatz_b200"):
        p = tmp_path / rel
        p.parent.mkdir(parents=True, exist_ok=True)
        p.write_text("")
    monkeypatch.setattr(bench, "ROOT", str(tmp_path))
    clock = {"t": 100.0}
    calls = []

    def run(cmd, input, capture_output, text, timeout):  # noqa: A002
        prog = "cli" if cmd[0].endswith("collatz_b200") else "ref"
        key = (prog, "line" if input == LINE1 else "empty")
        i = sum(1 for c in calls if c == key)
        calls.append(key)
        clock["t"] += durations[key][i]
        err = SUMMARY + "\n"
        if prog == "cli":
            err += '# results {"run_ms": 35.5, "device_ms": 29.8}\n'
        return _Proc(rc, err)

    monkeypatch.setattr(bench, "subprocess", types.SimpleNamespace(run=run))
    monkeypatch.setattr(bench, "time", types.SimpleNamespace(perf_counter=lambda: clock["t"]))
    return bench, calls


def test_runs_are_interleaved_and_best_of(monkeypatch, tmp_path):
    d = {("ref", "line"): [4.6, 4.3, 4.4], ("ref", "empty"): [4.1, 4.0, 4.2],
         ("cli", "line"): [0.55, 0.50, 0.52], ("cli", "empty"): [0.49, 0.48, 0.47]}
    bench, calls = _fake(monkeypatch, tmp_path, d)
    r = bench.run_reference_gpu_program(reps=3)
    assert calls == [("ref", "line"), ("ref", "empty"), ("cli", "line"), ("cli", "empty")] * 3
    assert r["reference_s"] == pytest.approx(4.3) and r["reference_startup_s"] == pytest.approx(4.0)
    assert r["cli_s"] == pytest.approx(0.50) and r["cli_startup_s"] == pytest.approx(0.47)
    assert r["reference_run_s"] == pytest.approx(0.3) and r["cli_run_s"] == pytest.approx(0.03)
    assert r["same_summary_line"] and r["reference_summary"] == SUMMARY
    assert (r["cli_run_ms_inside"], r["cli_device_ms"]) == (35.5, 29.8)


def test_start_up_noise_gives_no_run_time(monkeypatch, tmp_path):
    # the start-up-only runs of the CLI happened to be slower than its line-1 runs
    d = {("ref", "line"): [4.3, 4.3], ("ref", "empty"): [4.0, 4.0],
         ("cli", "line"): [0.49, 0.50], ("cli", "empty"): [0.85, 0.90]}
    bench, _ = _fake(monkeypatch, tmp_path, d)
    r = bench.run_reference_gpu_program(reps=2)
    assert r["cli_run_s"] is None
    assert r["reference_run_s"] == pytest.approx(0.3)
    assert r["cli_s"] == pytest.approx(0.49)


def test_failing_program_raises(monkeypatch, tmp_path):
    d = {k: [1.0] for k in (("ref", "line"), ("ref", "empty"), ("cli", "line"), ("cli", "empty"))}
    bench, _ = _fake(monkeypatch, tmp_path, d, rc=1)
    with pytest.raises(RuntimeError):
        bench.run_reference_gpu_program(reps=1)


def test_missing_programs_are_reported(monkeypatch, tmp_path):
    import bench
    monkeypatch.setattr(bench, "ROOT", str(tmp_path))
    r = bench.run_reference_gpu_program(reps=1)
    assert "unavailable" in r
