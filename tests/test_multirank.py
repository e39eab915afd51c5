"""The multi-GPU split (bench.py: one disjoint block per rank, results combined
on the host) on 2 gloo ranks on CPU, with the oracle standing in for the
device: the combined result equals the whole range's."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, off, size, k, q):
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import torch.distributed as dist
    from datetime import timedelta
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=timedelta(seconds=60))
    from oracle import oracle as O
    import collatz_b200 as cb
    per = size // world
    o = O.range_verify(off + rank * per, per, k, True, 1, 2)
    mine = cb.RangeResult(o.seeds, o.failures, 0, o.max_exc, o.max_exc_seed, o.max_st, o.max_st_seed)
    parts = [None] * world
    dist.all_gather_object(parts, mine)
    if rank == 0:
        c = cb.combine_range_results(parts)
        q.put((c.seeds_checked, c.max_stopping_time, c.max_stopping_time_seed, c.max_excursion,
               c.max_excursion_seed))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2])
def test_two_rank_split_combines(world):
    from oracle import oracle as O
    off, size, k = (1 << 40) + 5, 1 << 22, 24
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, off, size, k, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    w = O.range_verify(off, size, k, True, 1, 4)
    assert got == (w.seeds, w.max_st, w.max_st_seed, w.max_exc, w.max_exc_seed)
