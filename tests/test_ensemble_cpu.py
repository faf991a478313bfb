"""Host side of the batched ensemble (td1c_b200/ensemble.py): seeded job draws, the cost
model, the partition over ranks and the gather of observables over two gloo ranks."""
import math
import os
import socket

import numpy as np
import pytest

from td1c_b200 import ensemble as E


def test_job_list_is_seeded_and_in_range():
    a, b, c = E.job_list(7), E.job_list(7), E.job_list(8)
    assert a == b and a != c and len(a) == 64
    for j in a:
        assert 15 <= j["lmax1"] <= 63 and j["lmax2"] == 2 * j["lmax1"]
        assert 30 <= j["nfe"] <= 80 and j["ndvr"] == 20 and j["rmax"] == 2.0 * j["nfe"]
        assert 1e13 <= j["fint"] <= 5e14 and 400.0 <= j["wlen"] <= 1600.0 and 0.0 <= j["cep"] < 2 * math.pi
        nact = sum(1 for o in j["orbitals"] if o[3] == 1)
        nfc = sum(1 for o in j["orbitals"] if o[3] == -1)
        if nact == 0:  # He TDHF: one dynamic-core orbital
            assert j["orbitals"] == [(1, 0, 0, 0)] and j["znuc"] == 2.0
        else:
            assert 2 <= nact <= 9 and nfc == 1
            assert j["nela"] + j["nelb"] == 2 + min(8, 2 * nact) == j["znuc"]
        assert sum(o[2] for o in j["orbitals"] if o[3] == 1) == 0 or nact in (2, 3, 6, 7)
    sizes = {(j["lmax1"], j["nfe"], len(j["orbitals"])) for j in a}
    assert len(sizes) > 50  # uneven sizes


def test_every_job_has_determinants():
    """Every drawn job has a non-empty CI space in its M sector (a fully occupied active space
    takes M = 2 sum m); checked with the oracle's string tables on a reduced grid."""
    from oracle.oracle import Oracle
    seen = set()
    for small in (False, True):
        for j in E.job_list(7, small=small):
            key = (len(j["orbitals"]), j["mtot"])
            if key in seen:
                continue
            seen.add(key)
            d = Oracle(dict(j, lmax1=5, lmax2=10, nfe=4, rmax=8.0, rmask=6.0)).dims
            assert d["lcic"] >= 1, (j["name"], j["mtot"], d["lcic"])
    assert len(seen) >= 8
    for j in E.job_list(7, small=True):
        assert 5 <= j["lmax1"] <= 15 and 8 <= j["nfe"] <= 24


def test_cost_model_and_partition():
    jobs = E.job_list(7)
    cost = [E.cost(j) for j in jobs]
    assert all(c > 0 for c in cost)
    small = E.job(15, 30, 4, 1e14, 800.0, 0.0)
    big = E.job(63, 80, 4, 1e14, 800.0, 0.0)
    assert E.cost(big) > 10 * E.cost(small)
    for world in (1, 2, 3, 8):
        lists, load = E.partition(cost, world)
        flat = sorted(j for lst in lists for j in lst)
        assert flat == list(range(len(jobs)))
        assert all(lst == sorted(lst) for lst in lists)
        for r in range(world):
            assert abs(load[r] - sum(cost[j] for j in lists[r])) < 1e-9 * sum(cost)
        # longest-processing-time bound: makespan <= 4/3 of a lower bound on the optimum
        assert max(load) <= 4.0 / 3.0 * max(sum(cost) / world, max(cost))


def test_a_drawn_job_is_a_workload_the_oracle_accepts():
    from oracle.oracle import Oracle
    wl = E.job(15, 30, 2, 3e13, 1000.0, 1.0)
    o = Oracle(dict(wl, split_type=1))
    assert o.dims["nrad"] == E.dims(wl)["nrad"]
    assert o.dims["nfcore"] == 1 and o.dims["nact"] == 2


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        jobs = E.job_list(11, n=20)
        lists, _ = E.partition([E.cost(j) for j in jobs], world)
        mine = {j: {"dipole_end": float(j) ** 2, "rank": rank} for j in lists[rank]}
        q.put((rank, E.gather(mine, dist)))
    finally:
        dist.destroy_process_group()


def test_gather_over_two_gloo_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res[1] is None
    merged = res[0]
    assert list(merged) == list(range(20))
    assert all(merged[j]["dipole_end"] == float(j) ** 2 for j in merged)
    assert {merged[j]["rank"] for j in merged} == {0, 1}


def test_gather_without_a_group():
    assert E.gather({3: "c", 1: "a"}) == {1: "a", 3: "c"}
