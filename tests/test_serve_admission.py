"""The serving loop's HBM-budget admission, on CPU with a fake budget (no
GPU): requests wait while their workspace would not fit next to what is
admitted, are admitted as memory frees up, never push the accounted memory
past the budget, and the accounting returns to its reserve when all finish
(also with releases from several threads)."""

import threading

import numpy as np
import pytest

from fastprox_b200.serve import Admission, Request, _ws_bytes, make_requests


def test_admission_waits_and_admits_under_a_fake_budget():
    adm = Admission(budget_bytes=100, reserved=20)
    assert adm.try_admit(50)
    assert not adm.try_admit(40)  # 20 + 50 + 40 > 100: waits
    assert adm.try_admit(30)
    assert adm.used == 100 and adm.peak == 100
    adm.release(50)
    assert adm.try_admit(40)
    adm.release(30)
    adm.release(40)
    assert adm.used == 20
    with pytest.raises(RuntimeError):
        adm.release(30)


def test_stream_of_requests_stays_under_budget():
    """A simulated stream: each request holds its workspace for a service time,
    the loop admits in arrival order as memory frees; the budget is never
    exceeded and every request is served."""
    reqs = make_requests(5.0, rate=200.0, seed=3)
    budget = 2e9
    adm = Admission(budget, reserved=0)
    rng = np.random.default_rng(4)
    service = {r.i: rng.uniform(0.005, 0.05) for r in reqs}
    t, running, waiting, served = 0.0, [], [], 0
    nxt = 0
    while served < len(reqs):
        while nxt < len(reqs) and reqs[nxt].t <= t:
            waiting.append(reqs[nxt])
            nxt += 1
        still = []
        for r in waiting:
            b = _ws_bytes(r)
            assert b <= budget  # every request fits an empty budget
            if adm.try_admit(b):
                running.append((t + service[r.i], b))
            else:
                still.append(r)
        waiting = still
        assert adm.used <= budget
        t += 0.001
        fin = [x for x in running if x[0] <= t]
        running = [x for x in running if x[0] > t]
        for _, b in fin:
            adm.release(b)
            served += 1
    assert adm.used == 0 and adm.peak <= budget


def test_release_from_threads():
    adm = Admission(1e6)
    sizes = [1000 + i for i in range(200)]
    for b in sizes:
        assert adm.try_admit(b)
    ts = [threading.Thread(target=adm.release, args=(b,)) for b in sizes]
    for th in ts:
        th.start()
    for th in ts:
        th.join()
    assert abs(adm.used) < 1e-6


def test_workspace_bytes_by_kind():
    r2 = Request(0, 0.0, "iso2d", 100, 0.1)
    r3 = Request(1, 0.0, "iso3d", 128, 0.1)
    assert _ws_bytes(r3) > _ws_bytes(r2) > 0
