"""Serving mode (collatz_server_*): every request's result in the mix equals
the same request run alone (collatz_verify_range / collatz_trajectory, which
the range and trajectory tests pin to the oracle), bit for bit."""
import random
import threading

import pytest

pytestmark = pytest.mark.gpu


def _range_key(r):
    return (r.seeds_checked, r.failures, r.widened, r.max_excursion, r.max_excursion_seed,
            r.max_stopping_time, r.max_stopping_time_seed, r.errors)


def _mix(rng, n_range, n_traj):
    reqs = []
    for _ in range(n_range):
        k = rng.choice([16, 20, 24, 24, 24])
        off = rng.randrange(1 << 40, 1 << 64)
        if rng.random() < 0.5:
            off -= off % (1 << k)  # aligned to the sieve modulus
        size = int(2 ** rng.uniform(10, 24))
        reqs.append(("range", (off, size, k)))
    for _ in range(n_traj):
        n = rng.choice([1, 3, 100, 1000])
        reqs.append(("traj", [rng.getrandbits(rng.randint(64, 256)) | 1 for _ in range(n)]))
    reqs.append(("range", (5, 1 << 16, 24)))        # starts below 2^k (unsieved part)
    reqs.append(("range", (2, 1 << 14, 16, True, True)))          # negative integers (cycle minima)
    reqs.append(("range", ((1 << 45) + 3, 1 << 18, 24, True, True)))
    reqs.append(("range", (1 << 40, 0, 24)))        # empty
    reqs.append(("traj", [0, 1, 2, 27, (1 << 256) - 1]))
    rng.shuffle(reqs)
    return reqs


def _submit(srv, kind, arg):
    if kind != "range":
        return srv.submit_trajectory(arg)
    return srv.submit_range(*arg[:4], negative=len(arg) > 4 and arg[4])


def _check(verifier, kind, arg, resp):
    assert resp.status == 0, resp
    if kind == "range":
        alone = verifier.verify_range(*arg[:4], negative=len(arg) > 4 and arg[4])
        assert _range_key(resp.range) == _range_key(alone), (arg, resp.range, alone)
    else:
        assert resp.trajectory() == verifier.trajectory(arg)


def test_served_equals_alone(verifier):
    import collatz_b200 as cb
    rng = random.Random(2026)
    reqs = _mix(rng, 40, 12)
    v = verifier(26)
    # small slices and few slots: requests are cut across many slices, wait
    # for slots, and share slices with requests of other sizes
    with cb.Server(26, slice_items=1 << 10, max_active=8) as srv:
        tickets = [_submit(srv, kind, arg) for kind, arg in reqs]
        resps = [srv.wait(t, timeout=300) for t in tickets]
        info = srv.info()
    for (kind, arg), resp in zip(reqs, resps):
        _check(v, kind, arg, resp)
    assert info["completed"] == len(reqs)
    assert info["range_slices"] > 1
    assert all(r.admit_s >= r.submit_s and r.done_s >= r.admit_s for r in resps)


def test_concurrent_submitters(verifier):
    import collatz_b200 as cb
    v = verifier(26)
    out, errors = {}, []

    def client(i, srv):
        try:
            rng = random.Random(100 + i)
            mine = _mix(rng, 6, 3)
            tickets = [_submit(srv, kind, arg) for kind, arg in mine]
            out[i] = list(zip(mine, [srv.wait(t, timeout=300) for t in tickets]))
        except Exception as e:  # noqa: BLE001
            errors.append(e)

    with cb.Server(26, slice_items=1 << 14) as srv:
        th = [threading.Thread(target=client, args=(i, srv)) for i in range(4)]
        for t in th:
            t.start()
        for t in th:
            t.join()
    assert not errors, errors
    for i in range(4):
        for (kind, arg), resp in out[i]:
            _check(v, kind, arg, resp)


def test_admission_refused_when_memory_reserve_exceeds_device():
    import collatz_b200 as cb
    with cb.Server(26, hbm_reserve=1 << 62) as srv:
        t1 = srv.submit_range(1 << 40, 1 << 20)
        t2 = srv.submit_trajectory([27, 97])
        assert srv.wait(t1, timeout=60).status == cb.E_ADMISSION
        assert srv.wait(t2, timeout=60).status == cb.E_ADMISSION
        assert srv.info()["refused"] == 2


def test_submit_validation():
    import collatz_b200 as cb
    with cb.Server(26, traj_batch_seeds=1 << 10) as srv:
        with pytest.raises(cb.CollatzError) as e:
            srv.submit_range(1 << 40, 1 << 20, k=40)
        assert e.value.status == cb.E_ARG
        with pytest.raises(cb.CollatzError) as e:
            srv.submit_range(1 << 40, (1 << 48) + 1)
        assert e.value.status == cb.E_LIMIT
        with pytest.raises(cb.CollatzError) as e:
            srv.submit_trajectory(list(range(3, 3 + (1 << 10) + 1)))
        assert e.value.status == cb.E_LIMIT
        with pytest.raises(cb.CollatzError):
            srv.wait(12345, timeout=0.1)


def test_queries_wait_for_memory_and_complete(verifier):
    """An hbm_reserve that leaves room for a fraction of the queued queries:
    admission runs out of budget, waits for the budget thread's next read of
    free memory (batches that finished have given their memory back), and
    every query completes with the results of the query run alone."""
    import numpy as np
    import collatz_b200 as cb
    v = verifier(26)
    with cb.Server(26) as probe:
        free = probe.info()["hbm_free"]
    rng = np.random.default_rng(7)
    qs = []
    for _ in range(400):  # 2.1 MB of admission budget each, 840 MB in all
        s = rng.integers(0, 1 << 32, size=(1 << 14, 8), dtype=np.uint64).astype(np.uint32)
        s[:, 4:] = 0
        s[:, 3] |= np.uint32(1 << 31)
        qs.append(s)
    with cb.Server(26, hbm_reserve=free - (100 << 20)) as srv:
        tickets = [srv.submit_trajectory_array(s) for s in qs]
        resps = [srv.wait(t, timeout=120) for t in tickets]
        info = srv.info()
    assert info["refused"] == 0
    for s, r in zip(qs[::20], resps[::20]):
        assert r.status == 0
        status, st, exc = v.trajectory_array(s)
        assert (status == r.traj_status).all()
        assert (st == r.traj_stopping_time).all()
        assert (exc == r.traj_excursion).all()
    assert all(r.status == 0 for r in resps)
