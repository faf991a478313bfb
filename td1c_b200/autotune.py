"""Autotuner of an ensemble's launch shapes, searched on the device.

Each job's context has three launch shapes (td1c_gpu_set_tuning): the FP64
Legendre GEMM's m-tiles per CTA (48 or 96 rows), the cap of the persistent
mean-field action grid, and the K split of int2e.  Alone on the GPU a job
takes every SM for its persistent kernels; side by side in the ensemble graph
the jobs compete for them.  The tuner therefore
  1. times one RHS of every job alone (td1c_gpu_profile) with each m-tile and
     keeps the faster;
  2. times whole ensemble steps (on copies of the states, so the jobs do not
     advance) for grid caps proportional to each job's share of the work
     (factor f of the SM count times the job's share; f = 0 is no cap) and
     for int2e splits (-1: int2e on the job's main stream after the mean-field
     action instead of beside it), and keeps the fastest.
The choice is returned (and written as JSON when a path is given) with the
times it was based on.
"""
import json

import numpy as np

from .ensemble import cost


def tune(ens, nstep=2, nsm=148, caps=(0.0, 2.0, 1.0, 0.5), splits=(0, 64, 32, -1), path=None):
    torch = ens.torch
    lf = np.zeros(9)
    choice = {"mt": [], "mf_cap_factor": None, "i2_split": None, "times_ms": {}}
    # 1. the Legendre m-tile of every job, alone
    for j, h in enumerate(ens.h):
        hw, hc = torch.empty_like(ens.orb[j]), torch.empty_like(ens.cic[j])
        best = None
        for mt in (3, 6):
            h.set_tuning(mt, 0, 0)
            h.profile(1, lf, ens.orb[j].data_ptr(), ens.cic[j].data_ptr(), hw.data_ptr(), hc.data_ptr())
            t = sum(h.profile(3, lf, ens.orb[j].data_ptr(), ens.cic[j].data_ptr(), hw.data_ptr(), hc.data_ptr()).values())
            choice["times_ms"]["job%d_mt%d" % (j, mt)] = t
            if best is None or t < best[1]:
                best = (mt, t)
        choice["mt"].append(best[0])
    # 2. grid caps and int2e splits of the ensemble step, on copies of the states
    share = np.array([cost(wl) for wl in ens.jobs])
    share = share / share.sum()
    orb = [x.clone() for x in ens.orb]
    cic = [x.clone() for x in ens.cic]

    def apply(f, split):
        for j, h in enumerate(ens.h):
            cap = 0 if f == 0.0 else max(4, int(round(f * nsm * share[j])))
            h.set_tuning(choice["mt"][j], cap, split)

    def timed():
        for j in range(len(ens.h)):
            orb[j].copy_(ens.orb[j])
            cic[j].copy_(ens.cic[j])
        ens.run(1, orb=orb, cic=cic)  # warm-up: one-body factors and graph set-up
        return ens.run(nstep, orb=orb, cic=cic) / nstep

    best = None
    for f in caps:
        apply(f, 0)
        t = timed()
        choice["times_ms"]["cap%g" % f] = t
        if best is None or t < best[1]:
            best = (f, t)
    choice["mf_cap_factor"] = best[0]
    best_s = None
    for sp in splits:
        apply(choice["mf_cap_factor"], sp)
        t = timed()
        choice["times_ms"]["split%d" % sp] = t
        if best_s is None or t < best_s[1]:
            best_s = (sp, t)
    choice["i2_split"] = best_s[0]
    apply(choice["mf_cap_factor"], choice["i2_split"])
    choice["step_ms"] = best_s[1]
    if path:
        with open(path, "w") as fh:
            json.dump(choice, fh, indent=1)
    return choice
