"""Generates the golden fixtures in tests/golden/ from the reference itself.

Runs where the reference sources are present ($REF_DIR, else the directory
"reference" beside this repository): oracle/build_ref.sh compiles collatz_cudav7.cu for the CPU
through oracle/ref_shim/, then this script records

  cases_runs.json   whole reference runs (stdin 6-tuple -> hash, launches,
                    seeds checked, overflow seeds) at several N;
  tables.json       sha256 of the reference's 16 bit vectors and mod-9 sieve
                    at several N (precompute, cu:423-495);
  pairs_N<N>.json   explicit pair batches (Step-1 leaves and synthetic pairs,
                    including pairs that cross 2^100) with the hash that the
                    reference's compute_kernel / search2 produce for them.

Usage:  python tests/golden/make_golden.py [--quick]
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import random
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
from oracle import oracle as O  # noqa: E402

# the reference project: $REF_DIR, else the directory "reference" beside this repository
REF = os.environ.get("REF_DIR", os.path.join(os.path.dirname(ROOT), "reference"))
OUT = os.path.join(ROOT, "oracle", "_ref")


def case_line(fname: str, i: int) -> list[int]:
    with open(os.path.join(REF, fname)) as f:
        for j, line in enumerate(f, 1):
            if j == i:
                return [int(x) for x in line.split()]
    raise IndexError(i)


def run_ref(n: int, tup: list[int]) -> dict:
    p = subprocess.run([os.path.join(OUT, f"ref_N{n}")], input=" ".join(map(str, tup)) + "\n",
                       capture_output=True, text=True, check=True)
    err = p.stderr
    launches = int(err.split("Number of kernel launches = ")[1].split(".")[0])
    h = err.split("Complete hash = ")[1].split(".")[0]
    seeds = int(err.split("shim seeds = ")[1].split()[0])
    over = sorted(int(x, 16) for x in p.stdout.split())
    return {"N": n, "tuple": tup, "hash": h, "launches": launches, "seeds": seeds,
            "overflow": [str(x) for x in over]}


def ref_tool(n: int, script: str) -> list[str]:
    p = subprocess.run([os.path.join(OUT, f"ref_tool_N{n}")], input=script, capture_output=True,
                       text=True, check=True, env={**os.environ, "SHIM_QUIET": "1"})
    return p.stdout.split("\n")


def parse_hash_blocks(lines: list[str]) -> list[dict]:
    out, ov = [], []
    for ln in lines:
        if not ln.strip():
            continue
        if ln.startswith("HASH"):
            parts = ln.split()
            d = {"hash": parts[1], "overflow": [str(x) for x in sorted(ov)]}
            if len(parts) > 2:
                d["seeds"] = int(parts[2])
            out.append(d)
            ov = []
        elif ln.startswith("TABLES"):
            continue
        else:
            ov.append(int(ln, 16))
    return out


def tables_digest(n: int) -> dict:
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "t.bin")
        ref_tool(n, f"T {path}\n")
        data = open(path, "rb").read()
    nbv = 16 * ((1 << 19) + 32) * 4
    bv, m9 = data[:nbv], data[nbv:]
    per = [hashlib.sha256(bv[i * (nbv // 16):(i + 1) * (nbv // 16)]).hexdigest()
           for i in range(16)]
    return {"N": n, "bv_sha256": hashlib.sha256(bv).hexdigest(), "bv_each_sha256": per,
            "mod9_sha256": hashlib.sha256(m9).hexdigest()}


def pair_words(base: int, number: int) -> list[int]:
    w = []
    for x in (base, number):
        for i in range(4):
            w.append((x >> (32 * i)) & 0xFFFFFFFF)
    return w


def pair_fixture(n: int, tup: list[int], per_bucket: int, rng: random.Random) -> dict:
    T = O.Tables(n)
    leaves = T.leaves(*tup)
    buckets: dict[int, list] = {}
    for bi, base, number in leaves:
        if bi < 16:
            buckets.setdefault(bi, []).append((base, number))
    batches = []
    script = []
    for bi in sorted(buckets):
        pairs = buckets[bi][:per_bucket]
        batches.append({"kind": "leaves", "bigindex": bi,
                        "pairs": [[str(b), str(m)] for b, m in pairs]})
        words = [w for b, m in pairs for w in pair_words(b, m)]
        script.append(f"K {bi} {len(pairs)} " + " ".join(map(str, words)))
    # synthetic pairs whose values cross 2^100 (overflow report + reset, cu:295-301)
    mbi = T.mbi
    for bi in (0, 3):
        pairs = []
        for _ in range(48):
            base = rng.randrange(3, 1 << mbi) | 1
            number = rng.randrange(1 << 96, 1 << 100)
            pairs.append((base, number))
        batches.append({"kind": "synthetic_high", "bigindex": bi,
                        "pairs": [[str(b), str(m)] for b, m in pairs]})
        words = [w for b, m in pairs for w in pair_words(b, m)]
        script.append(f"K {bi} {len(pairs)} " + " ".join(map(str, words)))
    res = parse_hash_blocks(ref_tool(n, "\n".join(script) + "\n"))
    assert len(res) == len(batches)
    for b, r in zip(batches, res):
        b.update(r)
    # search2 (CPU semantics, cu:654-715): bigindex >= 16 (mod-9 sieve only)
    # and bigindex < 16 (the spot-check path) on single pairs
    s2 = []
    script = []
    for bi in (16, 17, 20):
        for _ in range(6):
            base = rng.randrange(3, 1 << mbi) | 1
            number = rng.randrange(1 << 40, 1 << 64)
            s2.append({"bigindex": bi, "base": str(base), "number": str(number)})
            script.append(f"S {bi} {base & (2**64 - 1)} {base >> 64} {number & (2**64 - 1)} "
                          f"{number >> 64}")
    for bi in sorted(buckets)[:4]:
        for base, number in buckets[bi][:3]:
            s2.append({"bigindex": bi, "base": str(base), "number": str(number)})
            script.append(f"S {bi} {base & (2**64 - 1)} {base >> 64} {number & (2**64 - 1)} "
                          f"{number >> 64}")
    for _ in range(8):
        base = rng.randrange(3, 1 << mbi) | 1
        number = rng.randrange(1 << 97, 1 << 100)
        s2.append({"bigindex": 17, "base": str(base), "number": str(number)})
        script.append(f"S 17 {base & (2**64 - 1)} {base >> 64} {number & (2**64 - 1)} "
                      f"{number >> 64}")
    res = parse_hash_blocks(ref_tool(n, "\n".join(script) + "\n"))
    assert len(res) == len(s2)
    for d, r in zip(s2, res):
        d.update(r)
    return {"N": n, "tuple": tup, "batches": batches, "search2": s2}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--quick", action="store_true", help="skip the N=45 whole runs")
    args = ap.parse_args()
    subprocess.check_call([os.path.join(ROOT, "oracle", "build_ref.sh")],
                          env={**os.environ, "NS": "26 30 36 40 42 45"})
    rng = random.Random(20261203)

    runs = [run_ref(26, [3, 2, 2, 9, 1, 0]), run_ref(30, [3, 2, 2, 9, 1, 0]),
            run_ref(36, [3, 2, 2, 9, 1, 0])]
    for i in (1, 2, 3, 10, 55):
        runs.append(run_ref(36, case_line("cases_tiny", i)))
    runs.append(run_ref(40, case_line("cases_tiny", 1)))
    runs.append(run_ref(40, case_line("cases_small", 1)))
    runs.append(run_ref(42, case_line("cases_tiny", 1)))
    runs.append(run_ref(45, case_line("cases_big", 1)))
    if not args.quick:
        for i in (1, 2, 3):
            runs.append(run_ref(45, case_line("cases_tiny", i)))
    with open(os.path.join(HERE, "cases_runs.json"), "w") as f:
        json.dump({"generator": "tests/golden/make_golden.py", "runs": runs}, f, indent=1)

    tabs = [tables_digest(n) for n in (26, 36, 42, 45)]
    with open(os.path.join(HERE, "tables.json"), "w") as f:
        json.dump({"generator": "tests/golden/make_golden.py", "tables": tabs}, f, indent=1)

    for n, tup, per in ((26, [3, 2, 2, 9, 1, 0], 96), (42, case_line("cases_tiny", 1), 64),
                        (45, case_line("cases_tiny", 1), 64)):
        fx = pair_fixture(n, tup, per, rng)
        fx["generator"] = "tests/golden/make_golden.py"
        with open(os.path.join(HERE, f"pairs_N{n}.json"), "w") as f:
            json.dump(fx, f)
    print("golden fixtures written")


if __name__ == "__main__":
    main()
