"""The batched ensemble on one GPU: independent jobs of uneven size stepped by one captured graph.

Eight small jobs (He TDHF, Ne CAS, a frozen + dynamic core + active case in
both gauges, an open shell; different grids, lmax and pulses), each in a
context of its own, advance together through td1c_gpu_ensemble_split2: one
CUDA graph per step holds one split2 step of every job on the job's own
streams.  Every job must match the oracle's split2 of the same job to 1e-10
and equal the same steps run job after job.  Then the bounded wait of the
staged kernels is made to run out in one job's context (ST_TIMEOUT, no copy
or MMA in flight) and the ensemble, with the autotuner's launch shapes,
still matches.
"""
import numpy as np
import pytest

from td1c_b200 import workloads as W

from .helpers import oracle_tables, oracle_state, rel_err

JOBS = [
    dict(W.HE_SMALL, fint=1e14, wlen=800.0, cep=0.0),
    dict(W.HE_SMALL, nfe=10, rmax=20.0, rmask=15.0, lmax1=7, lmax2=14, fint=3e14, wlen=600.0, cep=40.0),
    dict(W.NE_SMALL, fint=5e14, wlen=800.0),
    dict(W.NE_SMALL, lmax1=4, lmax2=8, fint=1e14, wlen=1000.0, cep=90.0),
    dict(W.MIXED_SMALL),
    dict(W.MIXED_SMALL, fint=2e14, wlen=700.0, cep=10.0),
    dict(W.LENGTH_SMALL),
    dict(W.OPEN_SMALL),
]


def _state_factory(oracles):
    def state(h, wl):
        from oracle.oracle import Oracle
        o = Oracle(wl)
        o.set_split(1)
        orb, cic = oracle_state(o)
        o.set_wfn0(orb, cic)
        orb, cic = o.orth(orb, cic)
        oracles.append((o, orb, cic))
        return orb, cic
    return state


def _t0(wl):
    freq = 1239.84190 / (wl["wlen"] * 27.2113845)
    return 0.4 * wl["numcyc"] * 2 * np.pi / freq


@pytest.mark.gpu
def test_ensemble_matches_oracle_and_sequential(cuda_ok):
    import torch
    from oracle.oracle import Oracle
    from td1c_b200 import autotune
    from td1c_b200.ensemble import DeviceEnsemble
    jobs = [dict(wl, split_type=1, dt=0.002) for wl in JOBS]
    oracles = []
    ens = DeviceEnsemble(jobs, tables=lambda wl: oracle_tables(Oracle(wl)), state=_state_factory(oracles))
    try:
        nstep = 4
        t0 = [_t0(wl) for wl in jobs]
        start = [(x.clone(), y.clone()) for x, y in zip(ens.orb, ens.cic)]
        seq = [(x.clone(), y.clone()) for x, y in start]
        ms = ens.run(nstep, t0=t0)
        ms_seq = ens.run_sequential(nstep, t0=t0, orb=[s[0] for s in seq], cic=[s[1] for s in seq])
        assert ms > 0 and ms_seq > 0
        for j, (o, orb, cic) in enumerate(oracles):
            w, c, _ = o.split2(orb, cic, t0[j], jobs[j]["dt"], nstep)
            got_o = ens.orb[j].cpu().numpy()
            got_c = ens.cic[j].cpu().numpy()
            assert rel_err(got_o, w.reshape(-1)) < 1e-10, (j, rel_err(got_o, w.reshape(-1)))
            assert rel_err(got_c, c) < 1e-10, (j, rel_err(got_c, c))
            assert torch.equal(ens.orb[j], seq[j][0]) or rel_err(got_o, seq[j][0].cpu().numpy()) < 1e-13
            assert ens.h[j].last_status() == 0
        # a bounded wait that runs out in one job's context; the context stays usable
        assert ens.h[3].wait_selftest() == 32
        # the autotuner's shapes (searched on copies of the states), then the ensemble again
        choice = autotune.tune(ens, nstep=1, caps=(0.0, 1.0), splits=(0, 32))
        assert len(choice["mt"]) == len(jobs) and set(choice["mt"]) <= {3, 6}
        for j, (x, y) in enumerate(start):
            ens.orb[j].copy_(x)
            ens.cic[j].copy_(y)
        ens.run(nstep, t0=t0)
        for j, (o, orb, cic) in enumerate(oracles):
            w, c, _ = o.split2(orb, cic, t0[j], jobs[j]["dt"], nstep)
            assert rel_err(ens.orb[j].cpu().numpy(), w.reshape(-1)) < 1e-10, j
            assert ens.h[j].last_status() == 0
    finally:
        ens.final()
