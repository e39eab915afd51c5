#!/usr/bin/env python
"""Benchmark: seeds verified per second on B200 (range mode, plain kernel).

Workload (default): every seed in [2^40, 2^40 + 2^38) with the 2^24 residue
sieve and the mod-9 sieve, 128-bit limbs -- the "single large block, plain
kernel" configuration.  One step = one full verification of that block
(2^38 seeds covered, ~2.6e9 surviving seeds iterated).  With N GPUs each rank
verifies its own disjoint block of the same size (weak scaling, no data-path
collective; results combine by sum / max on the host).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Prints one JSON line (rank 0).  `value` is device-timed throughput with the
work list resident on the device (CUDA events around each launch on the
library's stream, L2 flushed between steps); `e2e` is the same metric through
the C ABI call collatz_verify_range (host request in, host result out).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

OFFSET = 1 << 40
SIZE_LOG2 = 38
K_SIEVE = 24
# Range workloads: the single large block (the headline) and the frontier
# block (2^40 seeds at 2^60 with the 2^34-bit sieve resident in HBM).
WORKLOADS = {
    "block": {"offset": OFFSET, "offset_log2": 40, "k": K_SIEVE, "size_log2": SIZE_LOG2,
              "name": "single large block"},
    "frontier": {"offset": 1 << 60, "offset_log2": 60, "k": 34, "size_log2": 40,
                 "name": "frontier block"},
}
METRIC = "seeds verified/s"
UNIT = "seeds/s"
# Algorithmic 32-bit integer operations per surviving seed (L = 4 limbs):
# one k-step jump (4L) plus, per odd run, 3L + 2 (L shifts, L multiply-adds,
# ctz, table, overflow test) and, per even run, 2L + 4 (decrement, ctz, L
# shifts, increment with carry, descent test).
OPS_JUMP, OPS_ODD, OPS_EVEN = 16, 14, 12
# Counters of one range-kernel launch taken with ncu, valid only for the
# sources of the kernel they were captured from: `src` is
# kernel_source_hash(workload) at capture time (the kernel's own file and the
# headers and table code it shares), and a line reports them only while those
# sources still hash to it.
#   block:    k_range64, 2^33 launch at 2^40, k = 24 (dram bytes per launch do
#             not grow with the block: the 4.6 MB survivor table is read from
#             DRAM once and from L2 after that);
#   frontier: k_range, 2^36 launch at 2^60, k = 34 (dram bytes per 2^34 block:
#             each block streams the 5 mod-9 classes it keeps of the 2.43 GB
#             table).
NCU_CAPTURES = {
    "block": {"src": "212c53bc6b1ae53d", "dram_bytes": 5.210368e6 + 0.406272e6, "per": "launch",
              "issue_slots_busy": 0.7923, "alu_pipe_busy": 0.6873, "kernel": "k_range64 (64-bit values)"},
    "frontier": {"src": "756669d9f18f48b4", "dram_bytes": (5.423305e9 + 9.317888e6) / 4, "per": "2^34 block",
                 "issue_slots_busy": 0.7581, "alu_pipe_busy": 0.6762, "kernel": "k_range (four limbs)"},
}
SHARED_KERNEL_SOURCES = ("range_shared.cuh", "common.cuh", "kernels.h", "tables.h", "tables.cu")
KERNEL_SOURCES = {"block": ("range64.cu",) + SHARED_KERNEL_SOURCES,
                  "frontier": ("range.cu",) + SHARED_KERNEL_SOURCES}
# CPU sample of the block workload, the same for the reference arm's steps and
# the cpu_baseline leg: 2^32 seeds at 2^40 + i 2^32 with the k = 24 sieve.
CPU_SAMPLE_LOG2 = 32


def kernel_source_hash(workload: str) -> str:
    """sha256 (first 16 hex digits) of the sources of the range kernel that
    runs the workload."""
    import hashlib
    h = hashlib.sha256()
    for name in KERNEL_SOURCES[workload]:
        with open(os.path.join(ROOT, "collatz_b200", "csrc", name), "rb") as f:
            h.update(f.read())
    return h.hexdigest()[:16]


def dist_env():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), \
        int(os.environ.get("LOCAL_RANK", "0"))


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines: list[str] = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def stop(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                smax.append(float(p[2]))
            except ValueError:
                continue
            for nm, val in zip(names, p[5:9]):
                if val.lower() in ("active", "1"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_reference_steps(base: int, size: int, k: int, nthreads: int, steps: int, warmup: int) -> list[float]:
    """Times the oracle's run-length loop (the reference's search3 shape,
    collatz_cudav7.cu:684-715) on `steps` samples [base + i size, base + (i+1)
    size) after `warmup` untimed ones, on nthreads host threads; returns the
    seconds per step.  The reference arm and the cpu_baseline leg both call
    this with the same sample, so their rates agree."""
    from oracle import oracle as O
    for i in range(warmup):
        O.range_verify(base + i * size, size, k, True, 1, nthreads)
    times = []
    for i in range(steps):
        t0 = time.perf_counter()
        O.range_verify(base + i * size, size, k, True, 1, nthreads)
        times.append(time.perf_counter() - t0)
    return times


def cpu_sample_desc(wl: dict, size: int, steps: int, nthreads: int) -> str:
    return (f"{steps} x {size} seeds at 2^{wl['offset_log2']} + i*{size}, k={wl['k']} sieve + mod-9 "
            f"(oracle/collatz_oracle.c run-length loop after cu:684-715, {nthreads} threads; the 2^{wl['k']} "
            "sieve table is built once per process, outside the timed steps)")


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    wl = WORKLOADS[args.workload]
    base, ksv = wl["offset"], wl["k"]
    nthreads = os.cpu_count() or 1
    # one step = a bounded sample of the workload (the full block takes CPU-minutes)
    size = 1 << CPU_SAMPLE_LOG2
    times = cpu_reference_steps(base, size, ksv, nthreads, args.steps, args.warmup)
    tot = sum(times)
    value = size * args.steps / tot
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u128",
            "data": "synthetic (deterministic seed range)",
            "config": {"workload": f"range [2^{wl['offset_log2']} + i*S, 2^{wl['offset_log2']} + (i+1)*S), "
                                   f"S = 2^{CPU_SAMPLE_LOG2} (bounded sample of the 2^{args.size_log2 or wl['size_log2']} "
                                   f"{wl['name']}), k={ksv} sieve + mod-9",
                       "k": ksv, "sample_size": size},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": nthreads, "kind": "port",
                             "sample": cpu_sample_desc(wl, size, args.steps, nthreads)},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def _range_key(r):
    return (r.seeds_checked, r.failures, r.widened, r.max_excursion, r.max_excursion_seed,
            r.max_stopping_time, r.max_stopping_time_seed, r.errors)


def batched_requests(n_req: int = 4096, seed: int = 4096, lo_log2: int = 20, hi_log2: int = 34):
    """The batched configuration's requests: n_req (offset, size, k, mod9)
    tuples, sizes log-uniform in [2^lo, 2^hi] seeds, offsets uniform in
    [2^40, 2^64) rounded down to a multiple of the 2^24 sieve modulus, drawn
    from numpy default_rng(seed)."""
    import numpy as np
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(lo_log2 * np.log(2), hi_log2 * np.log(2), n_req)).astype(np.uint64)
    reqs = []
    for s in sizes:
        off = int(rng.integers(1 << 40, 1 << 64, dtype=np.uint64))
        reqs.append((off - off % (1 << K_SIEVE), int(s), K_SIEVE, True))
    return reqs


def run_batched(v, n_req: int = 4096, seed: int = 4096, lo_log2: int = 20, hi_log2: int = 34) -> dict:
    """Batched configuration: n_req range requests, sizes log-uniform in
    [2^lo, 2^hi] seeds, offsets uniform in [2^40, 2^64) aligned to the 2^24
    sieve modulus (seeded), all in one persistent launch (a plan: lowered work
    list + captured graph), against the plain path that verifies the same
    requests one at a time (collatz_verify_range).  Bit-exact per request."""
    import torch
    reqs = batched_requests(n_req, seed, lo_log2, hi_log2)
    total = sum(q[1] for q in reqs)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    plan = v.plan(reqs)
    t_plan = time.perf_counter() - t0
    plan.launch()
    batched_warm = plan.results()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    plan.launch()
    batched = plan.results()
    t_batched = time.perf_counter() - t0
    dev_ms = batched[0].device_ms
    plan.close()
    t0 = time.perf_counter()
    plain = [v.verify_range(*q) for q in reqs]
    t_plain = time.perf_counter() - t0
    dev_plain = sum(p.device_ms for p in plain) / 1e3
    exact = all(_range_key(a) == _range_key(b) for a, b in zip(batched, plain)) and \
        all(_range_key(a) == _range_key(b) for a, b in zip(batched, batched_warm))
    return {"workload": f"{n_req} range requests, sizes log-uniform [2^{lo_log2}, 2^{hi_log2}], offsets "
                        "uniform [2^40, 2^64) aligned to 2^24, k=24, seeded (numpy default_rng"
                        f"({seed}))",
            "seeds": total, "batched_seeds_per_s": total / t_batched,
            "batched_device_seeds_per_s": total / (dev_ms / 1e3), "plan_build_s": t_plan,
            "plain_seeds_per_s": total / t_plain, "plain_device_seeds_per_s": total / dev_plain,
            "speedup_vs_plain_wall": t_plain / t_batched,
            "speedup_vs_plain_device": dev_plain / (dev_ms / 1e3),
            "bit_exact_vs_plain": bool(exact)}


def run_cases() -> dict:
    """Cases mode, the reference's own verification run (Algorithm 1: Step 1
    on the device, Steps 2-3), end to end through collatz_run_case on the
    golden tuples with more than 10^7 seeds (N = 36 root case; N = 45
    cases_tiny lines 1-3), each checked against the reference's hash and
    launch count.  `host_step1_s`: the same call with Step 1 on the host
    threads (COLLATZ_CFG_HOST_STEP1).  CPU: the oracle's restatement of the
    reference, one thread like the reference's host program, on the N = 36
    root case."""
    import collatz_b200 as cb
    from oracle import oracle as O
    with open(os.path.join(ROOT, "tests", "golden", "cases_runs.json")) as f:
        runs = [r for r in json.load(f)["runs"] if r["N"] in (36, 45) and r["seeds"] > 10 ** 7]
    verifiers, out = {}, []

    def timed(v, tup):
        v.run_case(*tup)  # warm-up (buffers, first launches)
        t0 = time.perf_counter()
        res = v.run_case(*tup)
        return res, time.perf_counter() - t0

    for r in runs:
        for host in (False, True):
            if (r["N"], host) not in verifiers:
                verifiers[(r["N"], host)] = cb.Verifier(r["N"], host_step1=host)
        res, dt = timed(verifiers[(r["N"], False)], r["tuple"])
        hres, hdt = timed(verifiers[(r["N"], True)], r["tuple"])
        out.append({"N": r["N"], "tuple": r["tuple"], "seeds": res.seeds_checked, "s": dt,
                    "seeds_per_s": res.seeds_checked / dt, "device_ms": res.device_ms, "host_step1_s": hdt,
                    "hash_ok": f"{res.hash:X}" == r["hash"] and hres.hash == res.hash,
                    "launches_ok": res.launches == r["launches"] == hres.launches,
                    "seeds_ok": res.seeds_checked == r["seeds"] == hres.seeds_checked})
    # many small lines, the shape of the reference's cases_big file: the whole
    # N = 45 tree cut at sigfig 24, run through the line-batched driver
    v45 = verifiers[(45, False)]
    lines = cb.split_cases(45, (3, 2, 2, 9, 1, 0), 24)
    t0 = time.perf_counter()
    whole = v45.run_case(3, 2, 2, 9, 1, 0)
    t_whole = time.perf_counter() - t0
    t0 = time.perf_counter()
    comb, _, _ = v45.run_cases(lines, per_case=False)
    t_lines = time.perf_counter() - t0
    sample = 1000
    t0 = time.perf_counter()
    for c in lines[:sample]:
        v45.run_case(*cb.case_tuple(c))
    per_line_s = (time.perf_counter() - t0) / sample
    many = {"workload": f"N=45 root case (3 2 2 9 1 0) cut at sigfig 24 into {len(lines)} lines "
                        "(collatz_step1_split; the shape of the reference's cases_big), one collatz_run_cases "
                        "call (groups of 8192 lines per device pass)",
            "lines": len(lines), "seeds": comb.seeds_checked, "s": t_lines,
            "seeds_per_s": comb.seeds_checked / t_lines, "lines_per_s": len(lines) / t_lines,
            "device_s": comb.device_ms / 1e3, "xor_of_lines_equals_whole_run": comb.hash == whole.hash
            and comb.seeds_checked == whole.seeds_checked,
            "whole_run": {"hash": f"{whole.hash:X}", "seeds": whole.seeds_checked, "s": t_whole,
                          "seeds_per_s": whole.seeds_checked / t_whole},
            "one_call_per_line_ms": per_line_s * 1e3,
            "vs_one_call_per_line": per_line_s * len(lines) / t_lines,
            "one_call_per_line_sample": f"first {sample} lines, collatz_run_case each"}
    for v in verifiers.values():
        v.close()
    T = O.Tables(36)
    t0 = time.perf_counter()
    c = T.run_case(3, 2, 2, 9, 1, 0)
    cdt = time.perf_counter() - t0
    n45 = [o for o in out if o["N"] == 45]
    try:
        refgpu = run_reference_gpu_program()
    except Exception as e:  # noqa: BLE001
        refgpu = {"error": f"{type(e).__name__}: {e}"}
    return {"reference_gpu_program": refgpu,"workload": "collatz_run_case (Step 1 and Steps 2-3 on the GPU) on the reference's golden tuples",
            "runs": out,
            "n45_seeds_per_s": sum(o["seeds"] for o in n45) / max(1e-9, sum(o["s"] for o in n45)),
            "all_match_reference": all(o["hash_ok"] and o["launches_ok"] and o["seeds_ok"] for o in out),
            "many_lines": many,
            "cpu_baseline": {"value": c.seeds / cdt, "unit": UNIT, "cores": 1, "kind": "port",
                             "sample": f"N=36 root case (3 2 2 9 1 0), {c.seeds} seeds in {cdt:.1f} s "
                                       "(oracle/collatz_oracle.c orc_run_case, the reference's kernel "
                                       "semantics cu:185-411 on one thread)"}}


def run_reference_gpu_program(reps: int = 3) -> dict:
    """The reference program itself -- collatz_cudav7.cu compiled unchanged
    for sm_100a (MAXBITS = 45, the source's own value; built from the
    reference's sources by oracle/build_ref_gpu.sh) -- against this
    repository's drop-in CLI, on the same box and from the same process tree:
    cases_tiny line 1 at N = 45, each a whole process (context creation,
    tables, Step 1, Steps 2-3), wall time, best of `reps`.  An input whose
    Step 1 has no leaves (start-up only) separates start-up from the run."""
    ref = os.path.join(ROOT, "oracle", "_ref", "ref_gpu_N45")
    cli = os.path.join(ROOT, "collatz_b200", "collatz_b200")
    if not (os.path.exists(ref) and os.path.exists(cli)):
        return {"unavailable": "oracle/_ref/ref_gpu_N45 or the CLI is not built (the reference sources were "
                               "absent at build time)"}
    line1, empty = "27 10 8 183 0 0\n", "0 5 0 1 0 0\n"
    best = {}
    info = {}

    def run(key, cmd, text):
        t0 = time.perf_counter()
        p = subprocess.run(cmd, input=text, capture_output=True, text=True, timeout=300)
        dt = time.perf_counter() - t0
        if p.returncode:
            raise RuntimeError(f"{os.path.basename(cmd[0])} rc={p.returncode}: {p.stderr[-200:]}")
        lines = p.stderr.splitlines()
        info[key] = (next((ln for ln in lines if ln.startswith("Number of kernel launches")), None),
                     next((json.loads(ln[len("# results "):]) for ln in lines if ln.startswith("# results ")),
                          None))
        best[key] = min(best.get(key, dt), dt)

    # interleaved, so that a slow stretch of the host hits every program and input alike
    for _ in range(reps):
        run("r_line", [ref], line1)
        run("r_empty", [ref], empty)
        run("c_line", [cli, "45"], line1)
        run("c_empty", [cli, "45"], empty)
    r_sum, c_sum, c_res = info["r_line"][0], info["c_line"][0], info["c_line"][1]

    def diff(a, b):
        d = best[a] - best[b]
        return d if d >= 0 else None

    return {"input": "27 10 8 183 0 0 (cases_tiny line 1, N = 45; the reference's own default run)",
            "reference_program": "oracle/_ref/ref_gpu_N45 (collatz_cudav7.cu, nvcc -O3 sm_100a, unchanged)",
            "reference_summary": r_sum, "cli_summary": c_sum, "same_summary_line": r_sum == c_sum,
            "reference_s": best["r_line"], "cli_s": best["c_line"], "reference_startup_s": best["r_empty"],
            "cli_startup_s": best["c_empty"], "reference_run_s": diff("r_line", "r_empty"),
            "cli_run_s": diff("c_line", "c_empty"),
            "cli_run_ms_inside": (c_res or {}).get("run_ms"), "cli_device_ms": (c_res or {}).get("device_ms"),
            "note": f"wall time of whole processes, best of {reps}, the four runs interleaved; *_run_s = line 1 "
                    "minus the start-up-only input (0 5 0 1 0 0, no Step-1 leaves), null when the start-up "
                    "spread (CUDA context creation varies by up to a second from process to process) exceeds "
                    "the run; the reference's start-up includes its CPU table precompute. cli_run_ms_inside: "
                    "the CLI's own timer around the run after set-up."}


def run_served(v, capacity: float, load: float = 0.7, duration: float = 1.0, seed: int = 5,
               slice_items: int = 1 << 19, plain_sample: int = 600, trace: str | None = None) -> dict:
    """Served configuration: Poisson arrivals at `load` x capacity (range seeds
    per second), 70 % range verifications (sizes log-uniform 2^16..2^32,
    offsets uniform [2^40, 2^64), unaligned) and 30 % trajectory queries
    (1..65536 seeds, log-uniform count, bit lengths uniform 64..256), through
    collatz_server_*; p50/p99 latency, throughput, and the plain path (each
    request alone, in arrival order) on a sample of the same stream."""
    import numpy as np
    import collatz_b200 as cb
    rng = np.random.default_rng(seed)
    mean_range = ((1 << 32) - (1 << 16)) / np.log(1 << 16)
    lam = load * capacity / (0.7 * mean_range)
    n = max(50, int(lam * duration))
    gaps = rng.exponential(1.0 / lam, n)
    arrivals = np.cumsum(gaps) - gaps[0]
    # seed pool for trajectory queries: random limbs, bit length uniform 64..256
    pool_n = 1 << 21
    pool = rng.integers(0, 1 << 32, size=(pool_n, 8), dtype=np.uint64).astype(np.uint32)
    bl = rng.integers(64, 257, pool_n)
    for j in range(8):
        keep = np.clip(bl - 32 * j, 0, 32)
        mask = np.where(keep >= 32, 0xFFFFFFFF, (1 << keep.astype(np.uint64)) - 1).astype(np.uint32)
        pool[:, j] &= mask
    top = (bl - 1) // 32
    pool[np.arange(pool_n), top] |= (1 << ((bl - 1) % 32)).astype(np.uint32)
    reqs = []
    for i in range(n):
        if rng.random() < 0.7:
            size = int(np.exp(rng.uniform(16 * np.log(2), 32 * np.log(2))))
            off = int(rng.integers(1 << 40, 1 << 64, dtype=np.uint64))
            reqs.append(("range", (off, size, K_SIEVE)))
        else:
            m = int(np.exp(rng.uniform(0, 16 * np.log(2))))
            m = max(1, min(m, 65536))
            a = int(rng.integers(0, pool_n - m))
            reqs.append(("traj", pool[a:a + m]))
    srv = cb.Server(26, range_k=K_SIEVE, slice_items=slice_items)
    # warm-up: tables, pools, first slices
    for t in [srv.submit_range(1 << 50, 1 << 30), srv.submit_trajectory_array(pool[:1000])]:
        srv.wait(t)
    tickets = [None] * n
    resps = [None] * n

    def waiter():
        for i in range(n):
            while tickets[i] is None:
                time.sleep(1e-4)
            resps[i] = srv.wait(tickets[i])

    wt = threading.Thread(target=waiter)
    wt.start()
    t0 = time.perf_counter()
    for i, (kind, arg) in enumerate(reqs):
        d = t0 + arrivals[i] - time.perf_counter()
        if d > 0:
            time.sleep(d)
        tickets[i] = srv.submit_range(*arg) if kind == "range" else srv.submit_trajectory_array(arg)
    wt.join()
    wall = max(r.done_s for r in resps) - min(r.submit_s for r in resps)
    if trace:  # per request: kind (0 range, 1 query), seeds, planned arrival, submit, admit, done (s)
        s0 = resps[0].submit_s
        np.save(trace, np.array([(0 if k == "range" else 1, a[1] if k == "range" else len(a), arrivals[i],
                                  r.submit_s - s0, r.admit_s - s0, r.done_s - s0)
                                 for i, ((k, a), r) in enumerate(zip(reqs, resps))], dtype=np.float64))
    info = srv.info()
    srv.stop()
    lat = np.array([r.latency_s for r in resps]) * 1e3
    lat_r = np.array([r.latency_s for r, (k, _) in zip(resps, reqs) if k == "range"]) * 1e3
    lat_t = np.array([r.latency_s for r, (k, _) in zip(resps, reqs) if k == "traj"]) * 1e3
    range_seeds = sum(a[1] for k, a in reqs if k == "range")
    traj_seeds = sum(len(a) for k, a in reqs if k == "traj")
    # plain path: plain_sample requests spread evenly over the stream (the same mix of kinds
    # and sizes), one at a time
    stride = max(1, n // plain_sample)
    pick = list(range(0, n, stride))[:plain_sample]
    sub = [reqs[i] for i in pick]
    t1 = time.perf_counter()
    exact = True
    t_kind = {"range": 0.0, "traj": 0.0}
    for (kind, arg), r in zip(sub, [resps[i] for i in pick]):
        tk = time.perf_counter()
        if kind == "range":
            got = v.verify_range(*arg)
            t_kind[kind] += time.perf_counter() - tk
            exact &= _range_key(got) == _range_key(r.range)
        else:
            status, st, exc = v.trajectory_array(arg)
            t_kind[kind] += time.perf_counter() - tk
            exact &= bool((status == r.traj_status).all() and (st == r.traj_stopping_time).all()
                          and (exc == r.traj_excursion).all())
    t_plain = time.perf_counter() - t1
    sub_seeds = sum(a[1] for k, a in sub if k == "range")
    return {"workload": f"Poisson arrivals for {duration:.1f} s at {load:.2f} x the batched "
                        f"configuration's capacity ({capacity:.3g} seeds/s, measured in the same run); 70% ranges (log-uniform 2^16..2^32 seeds, offsets uniform [2^40, 2^64)), "
                        "30% trajectory queries (log-uniform 1..65536 seeds of 64..256 bits); numpy "
                        f"default_rng({seed})",
            "requests": n, "lambda_per_s": lam, "range_seeds": range_seeds, "traj_seeds": traj_seeds,
            "seeds_per_s": range_seeds / wall, "traj_seeds_per_s": traj_seeds / wall,
            "offered_seeds_per_s": load * capacity,
            "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "range_p50_ms": float(np.percentile(lat_r, 50)), "range_p99_ms": float(np.percentile(lat_r, 99)),
            "traj_p50_ms": float(np.percentile(lat_t, 50)) if len(lat_t) else None,
            "traj_p99_ms": float(np.percentile(lat_t, 99)) if len(lat_t) else None,
            "statuses_ok": int(sum(r.status == 0 for r in resps)),
            "slices": info["range_slices"], "traj_batches": info["traj_batches"],
            "device_busy_frac": info["device_busy_s"] / wall,
            "plain_seeds_per_s_same_stream": sub_seeds / t_plain,
            "plain_sample": f"{len(sub)} requests, every {stride}th of the stream, one at a time "
                            "(verify_range / trajectory)",
            "plain_s": {"range": t_kind["range"], "traj": t_kind["traj"], "all": t_plain},
            "host_s": {"admit": info["host_admit_s"], "build_slices": info["host_slice_s"],
                       "build_batches": info["host_batch_s"], "complete": info["host_complete_s"],
                       "idle": info["host_idle_s"], "wall": wall},
            "served_vs_plain": (range_seeds / wall) / (sub_seeds / t_plain),
            "bit_exact_vs_plain_sample": bool(exact)}


def roofline(workload: str, base: int, k: int, survivors: int, mean_ms: float, size: int, sm_count: int,
             sm_mhz: float, ipk: dict) -> dict:
    """Integer roofline of one k_range launch: algorithmic 32-bit operations
    (per surviving seed: the jump plus the odd and even runs the oracle's
    jump+runs model counts on a 2^24-seed sample of the same workload) per
    second of device time, against the measured integer peak at the sampled
    SM clock.  ncu counters are attached only while the kernel sources still
    hash to those they were captured from."""
    from oracle import oracle as O
    samp = O.range_verify(base, 1 << 24, k, True, 2, min(8, os.cpu_count() or 1))
    odd_per = samp.odd_runs / samp.seeds
    even_per = samp.even_runs / samp.seeds
    ops_per_seed = OPS_JUMP + OPS_ODD * odd_per + OPS_EVEN * even_per
    achieved = survivors * ops_per_seed / (mean_ms / 1e3) / 1e12
    peak = ipk[1]["ops_per_clk_sm"] * sm_count * sm_mhz * 1e6 / 1e12
    issue_peak = sm_count * 128 * sm_mhz * 1e6 / 1e12
    cap = NCU_CAPTURES[workload]
    src = kernel_source_hash(workload)
    valid = cap["src"] == src
    traffic = None
    if valid:
        traffic = cap["dram_bytes"] * (1 if cap["per"] == "launch" else max(1, size >> k))
    d = {"bound": "int", "achieved": achieved, "peak": peak, "unit": "Tops/s (32-bit)", "frac": achieved / peak,
         "traffic": traffic,
         "traffic_basis": (f"ncu dram__bytes_read.sum + dram__bytes_write.sum per {cap['per']}, captured from "
                           f"kernel sources {cap['src']}" + (f" x {max(1, size >> k)} blocks" if cap["per"] != "launch"
                                                             else "")) if valid else
         f"null: the kernel sources ({src}) changed since the last ncu capture ({cap['src']})",
         "model": f"{ops_per_seed:.1f} algorithmic 32-bit ops per surviving seed ({OPS_JUMP} + {OPS_ODD} x "
                  f"{odd_per:.2f} odd runs + {OPS_EVEN} x {even_per:.2f} even runs) x {survivors} seeds per launch",
         "peak_basis": f"measured integer peak (collatz_int_peak mix 1: funnel shift, 3-input add, multiply-add "
                       f"chains on every SM): {ipk[1]['ops_per_clk_sm']:.1f} ops per SM clock x {sm_count} SMs x "
                       f"{sm_mhz:.0f} MHz (sampled median SM clock); MEASURED_PEAKS.json has no integer peak",
         "int_peak_measured": {
             "mix1_kernel_mix": {"tops": ipk[1]["ops_per_s"] / 1e12, "ops_per_clk_sm": ipk[1]["ops_per_clk_sm"],
                                 "sm_mhz": ipk[1]["sm_mhz"]},
             "mix0_alu_only": {"tops": ipk[0]["ops_per_s"] / 1e12, "ops_per_clk_sm": ipk[0]["ops_per_clk_sm"],
                               "sm_mhz": ipk[0]["sm_mhz"]}},
         "issue_peak": issue_peak, "frac_of_issue_peak": achieved / issue_peak}
    if valid:
        # every issued instruction (work distribution included), where achieved/peak counts only
        # the algorithmic operations
        d["ncu"] = {"kernel": cap["kernel"], "issue_slots_busy": cap["issue_slots_busy"],
                    "alu_pipe_busy": cap["alu_pipe_busy"], "kernel_sources": cap["src"],
                    "metrics": "sm__inst_issued.avg.pct_of_peak_sustained_active, "
                               "sm__pipe_alu_cycles_active.avg.pct_of_peak_sustained_active"}
    return d


def run_frontier(local: int, stream, flush, sm_count: int, ipk: dict, steps: int = 5, warmup: int = 3) -> dict:
    """Frontier configuration: [2^60, 2^60 + 2^40) with the 2^34-bit sieve and
    its class-major survivor table resident in HBM (built on the GPU first),
    one plan launch per step, L2 flushed between steps, CUDA events on the
    library's stream; clocks sampled during the timed steps."""
    import torch
    import collatz_b200 as cb
    wl = WORKLOADS["frontier"]
    size = 1 << wl["size_log2"]
    fv = cb.Verifier(26, range_k=wl["k"], device=local)
    try:
        fv.set_stream(stream.cuda_stream)
        t0 = time.perf_counter()
        plan = fv.plan([(wl["offset"], size, wl["k"], True)])
        t_tab = time.perf_counter() - t0

        def step():
            with torch.cuda.stream(stream):
                flush.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            plan.launch()
            e1.record(stream)
            return e0, e1

        for _ in range(warmup):
            step()
        torch.cuda.synchronize()
        clk = ClockSampler(local)
        clk.start()
        time.sleep(0.3)
        evs = [step() for _ in range(steps)]
        torch.cuda.synchronize()
        clocks = clk.stop()
        ms = [a.elapsed_time(b) for a, b in evs]
        res = plan.results()[0]
        plan.close()
        mean_ms = sum(ms) / len(ms)
        roof = roofline("frontier", wl["offset"], wl["k"], res.seeds_checked, mean_ms, size, sm_count,
                        clocks.get("sm_mhz") or 1965.0, ipk)
        return {"workload": f"range [2^60, 2^60 + 2^40), k={wl['k']} sieve (2^34-bit bit array + class-major "
                            "survivor table resident in HBM) + mod-9, 128-bit limbs widening to 192/256, plain kernel",
                "steps": steps, "warmup": warmup, "ms_per_step": mean_ms, "seeds_per_s": size / (mean_ms / 1e3),
                "survivors_per_step": res.seeds_checked, "table_build_s": t_tab,
                "results": {"seeds_checked": res.seeds_checked, "failures": res.failures, "widened": res.widened,
                            "max_stopping_time": res.max_stopping_time,
                            "max_stopping_time_seed": str(res.max_stopping_time_seed),
                            "max_excursion": str(res.max_excursion),
                            "max_excursion_seed": str(res.max_excursion_seed), "errors": res.errors},
                "roofline": roof, "clocks": clocks,
                "l2": "flushed between steps (256 MiB write, outside the timed events)"}
    finally:
        fv.close()


def run_config1(local: int, nthreads: int) -> dict:
    """Plain verification: every n in [0, 2^32) with the 2^16 residue sieve
    and the mod-9 sieve.  CPU: the oracle's run-length loop in 64-bit
    arithmetic with overflow detection (a seed that would leave 64 bits is
    re-run in 128 bits) on all host threads; GPU: collatz_verify_range on the
    same range.  Both must give the same outputs."""
    import collatz_b200 as cb
    from oracle import oracle as O
    n = 1 << 32
    v1 = cb.Verifier(26, range_k=16, device=local)
    try:
        v1.verify_range(0, n, 16)  # tables, buffers
        walls, devs = [], []
        for _ in range(3):
            t0 = time.perf_counter()
            g = v1.verify_range(0, n, 16)
            walls.append(time.perf_counter() - t0)
            devs.append(g.device_ms)
    finally:
        v1.close()
    t0 = time.perf_counter()
    c = O.range_verify(0, n, 16, True, 3, nthreads)
    cdt = time.perf_counter() - t0
    exact = (g.seeds_checked, g.failures, g.max_stopping_time, g.max_stopping_time_seed, g.max_excursion,
             g.max_excursion_seed) == (c.seeds, c.failures, c.max_st, c.max_st_seed, c.max_exc, c.max_exc_seed)
    return {"workload": "every n in [0, 2^32) (n >= 2), k=16 residue sieve (n >= 2^16) + mod-9 sieve",
            "results": {"seeds_checked": g.seeds_checked, "failures": g.failures,
                        "max_stopping_time": g.max_stopping_time,
                        "max_stopping_time_seed": str(g.max_stopping_time_seed),
                        "max_excursion": str(g.max_excursion), "max_excursion_seed": str(g.max_excursion_seed)},
            "cpu": {"value": n / cdt, "unit": UNIT, "s": cdt, "cores": nthreads, "kind": "port",
                    "arith": "u64, __builtin_mul_overflow on every odd run; seeds leaving 64 bits re-run in u128",
                    "seeds_leaving_64_bits": c.wide64,
                    "code": "oracle/collatz_oracle.c method 3 (run-length loop after cu:684-715)"},
            "gpu": {"value": n / statistics.median(walls), "unit": UNIT, "wall_s": statistics.median(walls),
                    "device_ms": statistics.median(devs), "call": "collatz_verify_range"},
            "bit_exact_gpu_vs_cpu": bool(exact)}


def _sig(x, d=4):
    return float(f"{x:.{d}g}") if isinstance(x, (int, float)) and not isinstance(x, bool) else x


def summary(line: dict) -> dict:
    """The figures of every leg in a few hundred bytes, printed last on the line."""
    def get(d, *ks):
        for k in ks:
            if not isinstance(d, dict):
                return None
            d = d.get(k)
        return _sig(d)
    s = {"block_seeds_per_s": get(line, "value"), "block_frac": get(line, "roofline", "frac"),
         "block_e2e": get(line, "e2e", "value"), "cpu_baseline": get(line, "cpu_baseline", "value"),
         "frontier_seeds_per_s": get(line, "frontier", "seeds_per_s"),
         "frontier_frac": get(line, "frontier", "roofline", "frac"),
         "frontier_widened": get(line, "frontier", "results", "widened"),
         "config1_cpu_seeds_per_s": get(line, "config1", "cpu", "value"),
         "config1_gpu_seeds_per_s": get(line, "config1", "gpu", "value"),
         "config1_bit_exact": get(line, "config1", "bit_exact_gpu_vs_cpu"),
         "batched_seeds_per_s": get(line, "batched", "batched_seeds_per_s"),
         "batched_vs_plain": get(line, "batched", "speedup_vs_plain_wall"),
         "batched_bit_exact": get(line, "batched", "bit_exact_vs_plain"),
         "served_seeds_per_s": get(line, "served", "seeds_per_s"),
         "served_vs_plain": get(line, "served", "served_vs_plain"),
         "served_p50_ms": get(line, "served", "p50_ms"), "served_p99_ms": get(line, "served", "p99_ms"),
         "served_range_p99_ms": get(line, "served", "range_p99_ms"),
         "served_traj_p99_ms": get(line, "served", "traj_p99_ms"),
         "served_bit_exact": get(line, "served", "bit_exact_vs_plain_sample"),
         "cases_n45_seeds_per_s": get(line, "cases", "n45_seeds_per_s"),
         "cases_match_reference": get(line, "cases", "all_match_reference"),
         "cases_ref_gpu_program_s": get(line, "cases", "reference_gpu_program", "reference_s"),
         "cases_cli_s": get(line, "cases", "reference_gpu_program", "cli_s"),
         "cases_ref_gpu_program_run_s": get(line, "cases", "reference_gpu_program", "reference_run_s"),
         "cases_cli_run_s": get(line, "cases", "reference_gpu_program", "cli_run_s"),
         "cases_cli_run_ms_inside": get(line, "cases", "reference_gpu_program", "cli_run_ms_inside")}
    errs = [k for k in ("frontier", "config1", "batched", "served", "cases")
            if isinstance(line.get(k), dict) and "error" in line[k]]
    if errs:
        s["errors_in"] = errs
    return {k: x for k, x in s.items() if x is not None}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="block", choices=sorted(WORKLOADS),
                    help="block: [2^40, 2^40 + 2^38), k = 24 (default); frontier: [2^60, 2^60 + 2^40), k = 34")
    ap.add_argument("--size-log2", type=int, default=None,
                    help="seeds per GPU as a power of two (default: the workload's, 38 or 40)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the batched and served measurements (run at N = 1 only)")
    ap.add_argument("--served-load", type=float, default=0.7)
    ap.add_argument("--served-duration", type=float, default=2.0)
    ap.add_argument("--variant", type=int, default=None)
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)

    rank, world, local = dist_env()
    import torch
    pg = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
        pg = dist
    torch.cuda.set_device(local)
    import collatz_b200 as cb

    wl = WORKLOADS[args.workload]
    base, ksv = wl["offset"], wl["k"]
    if args.size_log2 is None:
        args.size_log2 = wl["size_log2"]
    size = 1 << args.size_log2
    off = base + rank * size
    v = cb.Verifier(26, range_k=ksv, device=local, variant=args.variant)
    stream = torch.cuda.Stream(device=local)
    v.set_stream(stream.cuda_stream)
    t_tab = time.perf_counter()
    plan = v.plan([(off, size, ksv, True)])  # builds the k-sieve tables on first use
    t_tab = time.perf_counter() - t_tab
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{local}")
    sm_count, _ = v.device_info()

    def step():
        with torch.cuda.stream(stream):
            flush.zero_()  # L2 (126 MB) flushed between steps, outside the timed events
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        plan.launch()
        e1.record(stream)
        return e0, e1

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if pg:
        pg.barrier()
    clk = ClockSampler(local)
    clk.start()
    time.sleep(0.3)
    torch.cuda.synchronize()
    if pg:
        pg.barrier()
    w0 = time.perf_counter()
    evs = [step() for _ in range(args.steps)]
    torch.cuda.synchronize()
    wall = time.perf_counter() - w0
    if pg:
        pg.barrier()
    clocks = clk.stop()
    ms = [a.elapsed_time(b) for a, b in evs]
    res = plan.results()[0]
    dev_s = sum(ms) / 1e3
    if pg:
        t = torch.tensor([dev_s, wall], dtype=torch.float64, device=f"cuda:{local}")
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        dev_s, wall = float(t[0]), float(t[1])
    value = world * size * args.steps / dev_s

    # e2e: the public C-ABI call with a host request and a host result
    e2e_times = []
    e2e_res = None
    v.set_stream(None)
    for i in range(2 + max(1, min(args.steps, 3))):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e2e_res = v.verify_range(off, size, ksv)
        e2e_times.append(time.perf_counter() - t0)
    e2e_s = statistics.median(e2e_times[2:])
    if pg:
        t = torch.tensor([e2e_s], dtype=torch.float64, device=f"cuda:{local}")
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        e2e_s = float(t[0])
    e2e_value = world * size / e2e_s

    if rank == 0:
        sm_mhz = clocks.get("sm_mhz") or 1965.0
        # measured integer peak (collatz_int_peak, after the timed region): the
        # kernel mix's operations per SM clock, scaled to the clock sampled under load
        ipk = {m: v.int_peak(m) for m in (1, 0)}
        roof = roofline(args.workload, base, ksv, res.seeds_checked, sum(ms) / len(ms), size, sm_count, sm_mhz,
                        ipk)
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * dev_s / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u128 (4x u32 limbs)",
            "data": "synthetic (deterministic seed range)",
            "config": {"workload": f"range [2^{wl['offset_log2']} + r*2^{args.size_log2}, "
                                   f"2^{wl['offset_log2']} + (r+1)*2^{args.size_log2}) per rank r, k={ksv} "
                                   "residue sieve + mod-9 sieve, 128-bit limbs widening to 192/256, plain "
                                   f"kernel ({wl['name']})",
                       "offset": base, "size_per_gpu": size, "k": ksv,
                       "survivors_per_step_per_gpu": res.seeds_checked,
                       "table_build_s": t_tab,
                       "l2": "flushed between steps (256 MiB write, outside the timed events)",
                       "parallelism": f"replicas over disjoint blocks x{world}",
                       "kernel_variant": args.variant},
            "results": {"seeds_checked": res.seeds_checked, "failures": res.failures,
                        "widened": res.widened, "max_stopping_time": res.max_stopping_time,
                        "max_stopping_time_seed": str(res.max_stopping_time_seed),
                        "max_excursion": str(res.max_excursion),
                        "max_excursion_seed": str(res.max_excursion_seed), "errors": res.errors},
            "roofline": roof,
            # request (32 B) + its work list: an aligned range of many blocks lowers to 55
            # 64-byte segments (5 kept mod-9 classes of the first and last block, 9 x 5 for the
            # blocks between), and the request's 4-byte first-segment index (threshold scouts)
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 32 + 64 * 55 + 4,
                    "d2h_bytes_per_step": 136,
                    "call": "collatz_verify_range (lower + upload work list + launches + result copy)"},
            "clocks": clocks,
            # per step: k_range_scout, k_range and the two widening passes
            "gpu_launches": 4 * args.steps,
            "wall_s_timed": wall,
        }
        nthreads = os.cpu_count() or 1
        if not args.no_cpu_baseline:
            csize, csteps = 1 << CPU_SAMPLE_LOG2, 3
            ctimes = cpu_reference_steps(base, csize, ksv, nthreads, csteps, 1)
            line["cpu_baseline"] = {"value": csize * csteps / sum(ctimes), "unit": UNIT, "cores": nthreads,
                                    "kind": "port", "sample": cpu_sample_desc(wl, csize, csteps, nthreads)}
        if world == 1 and not args.no_extras and args.workload == "block":
            def extra(fn):
                try:
                    return fn()
                except Exception as e:  # noqa: BLE001 -- the headline line is printed regardless
                    return {"error": f"{type(e).__name__}: {e}"}
            line["frontier"] = extra(lambda: run_frontier(local, stream, flush, sm_count, ipk))
            line["config1"] = extra(lambda: run_config1(local, nthreads))
            line["batched"] = extra(lambda: run_batched(v))
            # served load: a fraction of the batched configuration's capacity (requests of the
            # same offsets and sizes), else of the headline block's
            cap = line["batched"].get("batched_seeds_per_s") or value
            line["served"] = extra(lambda: run_served(v, cap, load=args.served_load,
                                                      duration=args.served_duration))
            line["cases"] = extra(run_cases)
        line["summary"] = summary(line)
        print(json.dumps(line), flush=True)
    plan.close()
    v.close()
    if pg:
        pg.barrier()
        pg.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
