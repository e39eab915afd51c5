"""Trajectory queries on the GPU against the oracle's single-step 512-bit
iteration (oracle/collatz_oracle.c: orc_trajectory)."""
import random

import pytest

pytestmark = pytest.mark.gpu


def test_trajectory_matches_oracle(verifier):
    from oracle import oracle as O
    rng = random.Random(7)
    seeds = [0, 1, 2, 3, 4, 5, 6, 7, 27, 97, 871, (1 << 64) - 1, 1 << 64, (1 << 256) - 1]
    # 2^b - 1 climbs to about 3^b: each of these outgrows its limb class at least once, so its
    # thread runs it again with the next width (4 -> 6 -> 8 -> 12 -> 16 limbs)
    seeds += [(1 << b) - 1 for b in (95, 96, 127, 160, 191, 224, 255)]
    for bits in (33, 64, 65, 96, 97, 128, 160, 161, 200, 224, 225, 255, 256):
        for _ in range(40):
            seeds.append(rng.getrandbits(bits - 1) | (1 << (bits - 1)))
    g = verifier(26).trajectory(seeds)
    o = O.trajectory(seeds)
    assert g == o


def test_trajectory_batch_large(verifier):
    from oracle import oracle as O
    rng = random.Random(11)
    seeds = [rng.getrandbits(rng.randint(64, 256)) | 1 for _ in range(5000)]
    g = verifier(26).trajectory(seeds)
    o = O.trajectory(seeds)
    assert g == o
