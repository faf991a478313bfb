"""A small, fixed workload for profiler captures: a few RHS evaluations of the full-size Ne
TD-CASSCF configuration on the seeded state, through the C-ABI.

    python -m td1c_b200.profile_case [--mode 0|1|2] [--reps N] [--prop]

mode 0 plain FP64, 1 mixed (persistent split TF32), 2 mixed on the per-tile kernel; --prop runs
--reps split2 steps (from the committed relaxed start state, at --t0, default the pulse onset)
instead of bare RHS evaluations.  Prints the status word; exits non-zero when it is not 0.
"""
import argparse
import os
import sys

import numpy as np


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--mode", type=int, default=1)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--prop", action="store_true")
    ap.add_argument("--t0", type=float, default=0.0, help="start time of the --prop steps (au)")
    a = ap.parse_args()
    import torch
    from td1c_b200 import basis, workloads as W
    from td1c_b200.hprod import HProd
    from td1c_b200.wfn import seeded_orbitals, seeded_cic
    wl = dict(W.NE_CAS, split_type=1)
    rad, ang = basis.build(wl)
    h = HProd(wl, rad, ang)
    tb = h.ci_tables()
    orb = seeded_orbitals(wl, rad["xrad"], rad["wrad"], rad["mask"])
    cic = seeded_cic(wl, h.dims["lcic"], tb["stra"], tb["strb"], tb["detoff"], tb["afirst"], tb["acount"])
    h.set_wfn0(orb, cic)
    d_orb = torch.from_numpy(orb.reshape(-1).copy()).cuda()
    d_cic = torch.from_numpy(cic.copy()).cuda()
    d_hw, d_hc = torch.empty_like(d_orb), torch.empty_like(d_cic)
    h.set_mixed(a.mode)
    if a.prop:
        from td1c_b200.data.make_relaxed_state import load
        orb, cic, _ = load()
        h.set_wfn0(orb, cic)
        d_orb = torch.from_numpy(orb.reshape(-1).copy()).cuda()
        d_cic = torch.from_numpy(cic.copy()).cuda()
        h.split2_dev(d_orb.data_ptr(), d_cic.data_ptr(), a.t0, wl["dt"], a.reps)
    else:
        for _ in range(a.reps):
            h.htot_dev(1.0, np.zeros(9), d_orb.data_ptr(), d_cic.data_ptr(), d_hw.data_ptr(), d_hc.data_ptr())
    h.sync()
    st = h.last_status()
    print("status", st)
    h.final()
    return 0 if st == 0 else 1


if __name__ == "__main__":
    sys.exit(main())
