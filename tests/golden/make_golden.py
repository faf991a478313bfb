"""Generate the oracle fixtures in this directory.

The td1c reference ships no tests or golden outputs and cannot be built in
this environment, so these fixtures are outputs of the CPU oracle (the
restatement of the reference path) on seeded inputs.  They pin the oracle
against regressions and give the GPU tests a fixed target; they are not
reference-binary outputs.  Regenerate with:  python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle.oracle import Oracle  # noqa: E402
from td1c_b200 import workloads as W  # noqa: E402
from tests.helpers import oracle_state  # noqa: E402

CASES = [W.NE_SMALL, W.MIXED_SMALL, W.LENGTH_SMALL, W.OPEN_SMALL, W.HE_SMALL]
TIMES = [0.0, 40.0]


def main():
    for wl in CASES:
        o = Oracle(wl)
        orb, cic = oracle_state(o)
        o.set_wfn0(orb, cic)
        out = dict(orb=orb, cic=cic)
        for k, t in enumerate(TIMES):
            lf = o.field(t)
            hw, hc = o.htot(1.0, lf, orb, cic)
            e = o.energies()
            out["lfield%d" % k] = lf
            out["hwfn%d" % k] = hw
            out["hcic%d" % k] = hc
            out["ene%d" % k] = np.array([e["ene_fcore"], e["ene_dcore"], e["ene_core"], e["ene_act"], e["ene_tot"]])
        np.savez_compressed(os.path.join(HERE, wl["name"] + ".npz"), **out)
        print("wrote", wl["name"])


if __name__ == "__main__":
    main()
