"""Generates tests/golden/range_configs.json: the outputs of the benchmark
configurations at their stated sizes, computed by the CPU oracle on all host
threads (about five minutes on 8 cores).

  config1  every n in [0, 2^32) with the 2^16 residue sieve and the mod-9
           sieve, in 64-bit arithmetic with overflow detection (oracle
           method 3), cross-checked against the 128-bit run-length loop
           (method 1, the reference's search3 shape, collatz_cudav7.cu:684-715);
  config2  the single large block [2^40, 2^40 + 2^38), k = 24 (method 1);
  config3  a 2^36 sub-block of the frontier, [2^60 + 3 2^34, 2^60 + 7 2^34),
           k = 34; the oracle tests each seed's residue against the sieve's
           definition (direct mode, a 2^20 table as an exact prefilter);
  config4  a subset of the batched configuration's 4096 requests (the
           generator bench.batched_requests, numpy default_rng(4096)): the 512
           smallest and the 4 smallest of size >= 2^30, each its own range.

The reference computes none of these outputs (it has no range mode, no
stopping time and no excursion), so they are pinned by the oracle alone; the
oracle's formulations are checked against each other and against brute force
in tests/test_oracle.py.

  python tests/golden/make_range_golden.py [--only config2,...] [--threads N]
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
from oracle import oracle as O  # noqa: E402

OUT = os.path.join(HERE, "range_configs.json")


def _res(r, dt: float, **extra) -> dict:
    d = {"seeds": r.seeds, "failures": r.failures, "max_stopping_time": r.max_st,
         "max_stopping_time_seed": str(r.max_st_seed), "max_excursion": str(r.max_exc),
         "max_excursion_seed": str(r.max_exc_seed), "oracle_s": round(dt, 1)}
    d.update(extra)
    return d


def _range(offset: int, size: int, k: int, method: int, threads: int, **kw):
    t0 = time.perf_counter()
    r = O.range_verify(offset, size, k, True, method, threads, **kw)
    return r, time.perf_counter() - t0


def config1(threads: int) -> dict:
    r, dt = _range(0, 1 << 32, 16, 3, threads)
    r1, _ = _range(0, 1 << 32, 16, 1, threads)
    key = lambda x: (x.seeds, x.failures, x.max_st, x.max_st_seed, x.max_exc, x.max_exc_seed)  # noqa: E731
    assert key(r) == key(r1), "64-bit and 128-bit oracle loops disagree"
    return {"offset": "0", "size": str(1 << 32), "k": 16,
            "result": _res(r, dt, wide64=r.wide64, method="u64 run-length loop with overflow detection")}


def config2(threads: int) -> dict:
    off, size = 1 << 40, 1 << 38
    r, dt = _range(off, size, 24, 1, threads)
    return {"offset": str(off), "size": str(size), "k": 24, "result": _res(r, dt)}


def config3(threads: int) -> dict:
    off, size = (1 << 60) + 3 * (1 << 34), 1 << 36
    r, dt = _range(off, size, 34, 1, threads, direct_sieve=True)
    return {"offset": str(off), "size": str(size), "k": 34, "result": _res(r, dt)}


def config4(threads: int) -> dict:
    import bench
    reqs = bench.batched_requests()
    order = sorted(range(len(reqs)), key=lambda i: (reqs[i][1], i))
    pick = order[:512] + [i for i in order if reqs[i][1] >= 1 << 30][:4]
    out = []
    t0 = time.perf_counter()
    for i in pick:
        off, size, k, _ = reqs[i]
        r, dt = _range(off, size, k, 1, threads)
        out.append({"index": i, "offset": str(off), "size": str(size), "k": k, "result": _res(r, dt)})
    return {"generator": "bench.batched_requests() (4096 requests, numpy default_rng(4096))",
            "selection": "the 512 smallest requests and the 4 smallest of size >= 2^30",
            "oracle_s": round(time.perf_counter() - t0, 1), "requests": out}


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--only", default="config1,config2,config3,config4")
    ap.add_argument("--threads", type=int, default=os.cpu_count() or 1)
    args = ap.parse_args()
    data = {}
    if os.path.exists(OUT):
        with open(OUT) as f:
            data = json.load(f)
    data["generated_by"] = "tests/golden/make_range_golden.py (CPU oracle, oracle/collatz_oracle.c)"
    fns = {"config1": config1, "config2": config2, "config3": config3, "config4": config4}
    for name in args.only.split(","):
        t0 = time.perf_counter()
        data[name] = fns[name](args.threads)
        print(f"{name}: {time.perf_counter() - t0:.1f} s", file=sys.stderr, flush=True)
        with open(OUT, "w") as f:
            json.dump(data, f, indent=1)
            f.write("\n")


if __name__ == "__main__":
    main()
