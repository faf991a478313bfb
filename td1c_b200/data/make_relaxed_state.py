"""Make the relaxed start states of the benchmark workloads (runs on a GPU).

The seeded orbitals and CI vector of a workload (Philox, td1c_b200.wfn; Ne
TD-CASSCF or He TDHF)
are orthonormalised and relaxed in imaginary time with ETD-RK2 steps
(init_prop12 with cletdrk2: 300 cycles of dt = 0.01 au) on the GPU, then
stored compactly: float32 real and imaginary parts, components below 1e-9 of
the orbital's largest dropped (sparse index list), CI in float64.  Both arms of
the benchmark load this file (through the reference's .orb/.cic text format),
so the CPU reference and the GPU start from the same numbers.

    python td1c_b200/data/make_relaxed_state.py [ne|he] [out.npz]
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

CYCLES, DT, DROP = 300, 0.01, 1e-9
PATH = os.path.join(HERE, "ne_tdcasscf_relaxed.npz")
PATHS = {"ne": PATH, "he": os.path.join(HERE, "he_tdhf_relaxed.npz")}


def path_for(workload_name):
    """The committed state file of a workload (by its td1c_b200.workloads name), or None."""
    from td1c_b200 import workloads as W
    for key, wl in (("ne", W.NE_CAS), ("he", W.HE_TDHF)):
        if wl["name"] == workload_name:
            return PATHS[key]
    return None


def main(which="ne", out=None):
    import torch
    from td1c_b200 import basis, workloads as W
    from td1c_b200.hprod import HProd
    from td1c_b200.wfn import seeded_orbitals, seeded_cic
    out = out or PATHS[which]
    wl = dict({"ne": W.NE_CAS, "he": W.HE_TDHF}[which], split_type=1)
    rad, ang = basis.build(wl)
    h = HProd(wl, rad, ang)
    d = h.dims
    tb = h.ci_tables()
    orb = seeded_orbitals(wl, rad["xrad"], rad["wrad"], rad["mask"])
    cic = seeded_cic(wl, d["lcic"], tb["stra"], tb["strb"], tb["detoff"], tb["afirst"], tb["acount"])
    h.set_wfn0(orb, cic)
    y = torch.from_numpy(orb.reshape(-1).copy()).cuda()
    yc = torch.from_numpy(cic.copy()).cuda()
    h.set_time_kind(0)
    h.orth_dev(y.data_ptr(), yc.data_ptr())
    h.set_split(1)
    ene = h.relax_etdrk2_dev(y.data_ptr(), yc.data_ptr(), DT, CYCLES)
    torch.cuda.synchronize()
    o = y.cpu().numpy().reshape(len(wl["orbitals"]), -1)
    keep = np.abs(o) >= DROP * np.abs(o).max(axis=1, keepdims=True)
    idx = np.flatnonzero(keep.reshape(-1)).astype(np.int32)
    flat = o.reshape(-1)[idx]
    np.savez_compressed(out, workload=wl["name"], shape=np.array(o.shape), idx=idx, re=flat.real.astype(np.float32),
                        im=flat.imag.astype(np.float32), cic=yc.cpu().numpy(), energy=float(ene[-1]), cycles=CYCLES, dt=DT)
    h.final()
    print("wrote %s: %d of %d components, energy %.10f" % (out, idx.size, o.size, ene[-1]))


def load(path=PATH):
    """(orbitals [nfun x nbas] complex128, CI complex128, info) of a stored state."""
    z = np.load(path)
    shape = tuple(int(x) for x in z["shape"])
    o = np.zeros(int(np.prod(shape)), dtype=np.complex128)
    o[z["idx"]] = z["re"].astype(np.float64) + 1j * z["im"].astype(np.float64)
    return o.reshape(shape), np.array(z["cic"], dtype=np.complex128), {
        "workload": str(z["workload"]), "energy": float(z["energy"]), "cycles": int(z["cycles"]), "dt": float(z["dt"])}


if __name__ == "__main__":
    main(*sys.argv[1:3])
