"""Host side of the batched ensemble: many independent atoms, one job list per GPU.

The ensemble's jobs are independent propagations of uneven size and field, so
the multi-GPU form is replicas of job lists: the jobs are drawn once from a
seeded Philox stream, partitioned over the ranks by their estimated cost, run
by each rank on its own GPU, and their observables are gathered to rank 0 in
job order.  No data-path collective is involved; the gather is one host
exchange at the end.

Job draws (one per job, in this order, from numpy's Philox generator):
  lmax1 ~ U{15..63} (lmax2 = 2 lmax1), FEDVR elements nfe ~ U{30..80} of 21
  points over 2 au each, active orbitals nact ~ U{1..9}, intensity
  log-uniform in [1e13, 5e14] W/cm^2, wavelength ~ U[400, 1600] nm, CEP ~ U[0, 2 pi).
nact = 1 is He TDHF (two electrons in one orbital).  nact >= 2 keeps a frozen
1s and puts min(8, 2 nact) electrons in the first nact orbitals of the
sequence 2s 2p-1 2p0 2p1 3s 3p-1 3p0 3p1 3d0, on the neutral atom's nucleus.
Every job uses the velocity gauge, a 3-cycle sin^2 pulse and dt = 0.004 au.
"""
import math

import numpy as np

from .workmodel import rhs_work

ACTIVE_SHELLS = [(2, 0, 0), (2, 1, -1), (2, 1, 0), (2, 1, 1), (3, 0, 0), (3, 1, -1), (3, 1, 0), (3, 1, 1), (3, 2, 0)]
NDVR = 20  # 21 Gauss-Lobatto points per element
ELEMENT_AU = 2.0


def job(lmax1, nfe, nact, fint, wlen, cep, jid=0):
    """The workload of one ensemble job (same keys as td1c_b200.workloads)."""
    rmax = ELEMENT_AU * nfe
    mtot = 0
    if nact == 1:
        orbitals, znuc, nel = [(1, 0, 0, 0)], 2.0, 2
    else:
        orbitals = [(1, 0, 0, -1)] + [s + (1,) for s in ACTIVE_SHELLS[:nact]]
        nel = 2 + min(8, 2 * nact)
        znuc = float(nel)
        if 2 * nact <= 8:
            # every active orbital doubly occupied: the one determinant has M = 2 sum(m)
            mtot = 2 * sum(s[2] for s in ACTIVE_SHELLS[:nact])
    return dict(name="ensemble_job%03d_lmax%d_nfe%d_nact%d" % (jid, lmax1, nfe, nact), znuc=znuc, rmin=0.0, rmax=rmax,
                ndvr=NDVR, nfe=nfe, lmax1=lmax1, lmax2=2 * lmax1, nlat=0, orbitals=orbitals, nela=nel // 2,
                nelb=nel // 2, mtot=mtot, smul=1, igauge=1, icomp=1, rmask=0.8 * rmax, mask_cos_order=4.0, fint=fint,
                wlen=wlen, numcyc=3.0, cep=cep, dt=0.004, seed=1000 + jid)


def job_list(seed, n=64, small=False):
    """The ensemble's n jobs, drawn from a seeded Philox stream: lmax1 in [15, 63] and 30 to 80
    elements, or (small) lmax1 in [5, 15] and 8 to 24 elements."""
    rng = np.random.Generator(np.random.Philox(seed))
    jobs = []
    lrange, frange = ((5, 16), (8, 25)) if small else ((15, 64), (30, 81))
    for j in range(n):
        lmax1 = int(rng.integers(*lrange))
        nfe = int(rng.integers(*frange))
        nact = int(rng.integers(1, 10))
        fint = float(10.0 ** rng.uniform(13.0, math.log10(5e14)))
        wlen = float(rng.uniform(400.0, 1600.0))
        cep = float(rng.uniform(0.0, 2.0 * math.pi))
        jobs.append(job(lmax1, nfe, nact, fint, wlen, cep, jid=j))
    return jobs


def dims(wl):
    """The grid dimensions the work model needs, from the workload alone."""
    nrad = wl["ndvr"] * wl["nfe"]  # clfedvr: ndvr points per element (the last shared), Nr = nrad - 1
    return {"nrad": nrad, "nlat": wl["nlat"] or wl["lmax2"] + 1}


def steps(wl):
    """Time steps of the whole pulse."""
    freq = 1239.84190 / (wl["wlen"] * 27.2113845)
    return int(math.ceil(wl["numcyc"] * 2.0 * math.pi / freq / wl["dt"]))


def cost(wl, fp64_tflops=35.0, hbm_gbs=6650.0, rhs_per_step=4):
    """Estimated seconds of one job on one GPU: per RHS phase the slower of its FLOPs at the FP64
    tensor rate and its compulsory bytes at the HBM rate, times the RHS evaluations of the pulse."""
    per_rhs = sum(max(f / (fp64_tflops * 1e12), b / (hbm_gbs * 1e9)) for f, b in rhs_work(wl, dims(wl)).values())
    return per_rhs * rhs_per_step * steps(wl)


def partition(costs, world):
    """Job indices per rank: longest job first onto the least loaded rank (ties to the lower rank);
    every job on exactly one rank, each rank's list in job order."""
    load = [0.0] * world
    lists = [[] for _ in range(world)]
    for j in sorted(range(len(costs)), key=lambda k: (-costs[k], k)):
        r = min(range(world), key=lambda q: (load[q], q))
        lists[r].append(j)
        load[r] += costs[j]
    return [sorted(x) for x in lists], load


def gather(results, dist=None, dst=0):
    """Gather every rank's {job id: observables} to rank `dst`; returns the merged dict in job order
    there (None elsewhere).  Without a process group the local dict is returned."""
    if dist is None or not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return dict(sorted(results.items()))
    parts = [None] * dist.get_world_size() if dist.get_rank() == dst else None
    dist.gather_object(results, parts, dst=dst)
    if dist.get_rank() != dst:
        return None
    merged = {}
    for p in parts:
        for k in p:
            if k in merged:
                raise ValueError("job %r ran on two ranks" % (k,))
        merged.update(p)
    return dict(sorted(merged.items()))


# ---------------------------------------------------------------------------
# the ensemble on one GPU: a context per job, one captured graph per step
# ---------------------------------------------------------------------------
class DeviceEnsemble:
    """Independent jobs, each in a context of its own (own tables, buffers and streams), stepped
    together by td1c_gpu_ensemble_split2: one CUDA graph per step holds one split2 step of every job.

    tables(wl) -> (rad, ang) gives the grids and tables of a job (default: the package's builder);
    state(h, wl) -> (orb, cic) its initial state (default: seeded, orthonormalised and relaxed in
    imaginary time for relax_cycles ETD-RK2 cycles of relax_dt)."""

    def __init__(self, jobs, tables=None, state=None, relax_cycles=40, relax_dt=0.01):
        import torch
        from . import basis
        from .hprod import HProd
        from .wfn import seeded_orbitals, seeded_cic
        self.torch = torch
        self.jobs = [dict(wl, split_type=1) for wl in jobs]
        self.h, self.orb, self.cic = [], [], []
        for wl in self.jobs:
            rad, ang = tables(wl) if tables else basis.build(wl)
            h = HProd(wl, rad, ang, new_context=True)
            if state:
                orb, cic = state(h, wl)
                h.set_wfn0(orb, cic)
            else:
                d, tb = h.dims, h.ci_tables()
                orb = seeded_orbitals(wl, rad["xrad"], rad["wrad"], rad["mask"])
                cic = seeded_cic(wl, d["lcic"], tb["stra"], tb["strb"], tb["detoff"], tb["afirst"], tb["acount"])
                h.set_wfn0(orb, cic)
            y = torch.from_numpy(np.ascontiguousarray(orb).reshape(-1).copy()).cuda()
            yc = torch.from_numpy(np.ascontiguousarray(cic).copy()).cuda()
            if not state and relax_cycles:
                h.set_time_kind(0)
                h.orth_dev(y.data_ptr(), yc.data_ptr())
                h.set_split(1)
                h.relax_etdrk2_dev(y.data_ptr(), yc.data_ptr(), relax_dt, relax_cycles)
                h.set_time_kind(1)
            h.set_split(1)
            self.h.append(h)
            self.orb.append(y)
            self.cic.append(yc)
        torch.cuda.synchronize()

    def _arrays(self, t0, orb, cic):
        import ctypes
        n = len(self.jobs)
        ids = (ctypes.c_int * n)(*[h.ctx_id for h in self.h])
        wf = (ctypes.c_void_p * n)(*[x.data_ptr() for x in orb])
        ci = (ctypes.c_void_p * n)(*[x.data_ptr() for x in cic])
        D = ctypes.c_double * n
        t0s = D(*([t0] * n if np.isscalar(t0) else list(t0)))
        dts = D(*[wl["dt"] for wl in self.jobs])
        return ids, wf, ci, t0s, dts, D(*[wl["fint"] for wl in self.jobs]), D(*[wl["wlen"] for wl in self.jobs]), \
            D(*[wl["numcyc"] for wl in self.jobs]), D(*[wl.get("cep", 0.0) for wl in self.jobs])

    def run(self, nstep, t0=0.0, orb=None, cic=None, maxcyc=20, thresh=1e-10):
        """nstep steps of every job together (in place on the job states, or on the given copies);
        returns the device time in ms."""
        import ctypes
        orb = self.orb if orb is None else orb
        cic = self.cic if cic is None else cic
        ids, wf, ci, t0s, dts, fi, wv, nc, cp = self._arrays(t0, orb, cic)
        ms = ctypes.c_double(0.0)
        lib = self.h[0].lib._lib
        self.torch.cuda.synchronize()
        rc = lib.td1c_gpu_ensemble_split2(len(self.jobs), ids, wf, ci, t0s, dts, int(nstep), fi, wv, nc, cp, int(maxcyc),
                                          float(thresh), ctypes.byref(ms))
        if rc:
            raise RuntimeError("td1c_gpu_ensemble_split2 failed (status %d)" % rc)
        return ms.value

    def run_sequential(self, nstep, t0=0.0, orb=None, cic=None, maxcyc=20, thresh=1e-10):
        """The same steps job after job (each job's graph-captured split2 on its own stream); returns
        the summed device time in ms."""
        torch = self.torch
        orb = self.orb if orb is None else orb
        cic = self.cic if cic is None else cic
        total = 0.0
        for j, h in enumerate(self.h):
            s = torch.cuda.ExternalStream(h.stream())
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record(s)
            h.split2_dev(orb[j].data_ptr(), cic[j].data_ptr(), t0 if np.isscalar(t0) else t0[j], self.jobs[j]["dt"], nstep,
                         maxcyc=maxcyc, thresh=thresh)
            e1.record(s)
            torch.cuda.synchronize()
            total += e0.elapsed_time(e1)
        return total

    def simulated_fs(self, nstep):
        """Simulated time of nstep steps of every job, summed over the jobs (fs)."""
        return sum(nstep * wl["dt"] for wl in self.jobs) * 0.02418884254

    def final(self):
        for h in self.h:
            h.final()
        self.h = []
