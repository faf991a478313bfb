#!/usr/bin/env python
"""Benchmark: fs of simulated time per second for the Ne TD-CASSCF propagation
on one B200, learned+mixed against plain FP64, driven through the td1c_b200 C-ABI.

Workload: Ne TD-CASSCF (1s frozen core + CAS(8e, 9o), FEDVR 60 x 21 points,
rmax 120, lmax 47 / 94, velocity gauge, sin^2 800 nm 4-cycle 5e14 W/cm^2
pulse, dt 0.004 au), complex128; `--workload he` runs He TDHF instead.  Start
state: the committed relaxed state of the workload (td1c_b200/data/*.npz,
seeded orbitals and CI relaxed in imaginary time;
td1c_b200/data/make_relaxed_state.py), read through the reference's .orb/.cic
text format by both arms.

A step is td1c's own propagation at this dt: tdse_split2 with clh1itr + clcrk
and split_type 1 (a Crank-Nicolson one-body half step with the laser by
correction cycles, one RK4 step of the two-body part, a second half step, the
absorbing mask).  Three arms over the same window (warm-up steps, then the
timed steps, one trajectory from t0, default the pulse onset):
  fp64           the plain FP64 path;
  mixed          the mean field's pair-density multipoles and pair potentials
                 in split TF32 on tcgen05;
  learned+mixed  mixed, with the stage mean fields predicted from the history
                 of exact step-start mean fields by the network trained on the
                 GPU (200 seeded trajectories), judged every step, windows of 8
                 rolled back and recomputed exactly above the 1e-6 bound.
value  : fs/s of the learned+mixed arm with the state resident in HBM (the
         metric's subject); the fp64 and mixed objects hold the other arms.
e2e    : the learned+mixed arm through the public API with the state copied
         host->device before and device->host after every judged window of
         8 steps (a window is the unit the judge commits).
A second window at the |A(t)| maximum times the three arms where the one-body
correction cycles are the most numerous.  --full-pulse propagates the whole
pulse with every arm and compares dipole, norm and energy with FP64; the
default line carries the last committed full-pulse measurement.
Run with --impl reference for the CPU restatement of the reference path.
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

# the ensemble leg forks one graph into four streams per job: give the device enough hardware
# work queues that the jobs' streams do not share them (read when CUDA starts)
if any(a.startswith("--ensemble") for a in sys.argv[1:]):
    os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from td1c_b200.replicas import AU2FS, job_throughput, max_over_ranks, replica_seed  # noqa: E402


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="ne", choices=["ne", "he"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=0)
    ap.add_argument("--no-mixed", action="store_true", help="skip the mixed and learned+mixed arms")
    ap.add_argument("--no-learned", action="store_true", help="skip the learned+mixed arm")
    ap.add_argument("--mixed-mode", type=int, default=1, choices=[1, 3],
                    help="mixed-precision mode of the mixed and learned arms (3: Poisson interior products "
                         "and int2e in split TF32 as well)")
    ap.add_argument("--no-peak", action="store_true", help="skip the window at the |A| peak")
    ap.add_argument("--train-traj", type=int, default=200, help="trajectories of the learned predictor's training set")
    ap.add_argument("--train-iters", type=int, default=400)
    ap.add_argument("--bound", type=float, default=1e-6, help="the judge's bound (relative mean-field error)")
    ap.add_argument("--prop", default="split2", choices=["split2", "etdrk2", "rk4"])
    # without the committed state file (the He workload): imaginary time tau = 3 au
    # (300 ETD-RK2 cycles of dt 0.01); further relaxation lets the Ne RK4 part of
    # split2 at dt = 0.004 diverge through tiny natural occupations (the oracle too)
    ap.add_argument("--relax-cycles", type=int, default=300)
    ap.add_argument("--relax-dt", type=float, default=0.01)
    ap.add_argument("--t0", type=float, default=0.0, help="start time of the trajectory (au)")
    ap.add_argument("--full-pulse", action="store_true",
                    help="propagate the whole pulse with every arm; write profiles/full_pulse_<workload>.json")
    ap.add_argument("--nprint", type=int, default=100, help="steps between dipole samples of --full-pulse")
    ap.add_argument("--sensitivity", default="",
                    help="--full-pulse: also FP64 trajectories from the start state perturbed by these relative "
                         "sizes (comma-separated, e.g. 1e-12,1e-9), to show how the dynamics amplify a perturbation")
    ap.add_argument("--ensemble", type=int, default=0, help="also step this many seeded jobs as one ensemble")
    ap.add_argument("--ensemble-small", action="store_true",
                    help="the ensemble's jobs from the small range (lmax1 5-15, 8-24 elements)")
    return ap.parse_args()


PROP_NOTE = {
    "split2": "tdse_split2: clh1itr (Crank-Nicolson one-body half steps, laser by correction cycles, "
              "maxcyc 20, thresh 1e-10) + clcrk RK4 on the split_type 1 RHS; mask each step",
    "etdrk2": "tdse_prop12 with cletdrk2 + cldpade (alpha 2, maxcyc 20, thresh 1e-10), split_type 1; mask each step",
    "rk4": "RK4 full H (clcrk), mask each step; every step restarts from the relaxed state (unstable at this dt)",
}
RHS_PER_STEP = {"split2": 4, "etdrk2": 2, "rk4": 4}


def workload(name):
    from td1c_b200 import workloads as W
    return W.NE_CAS if name == "ne" else W.HE_TDHF


def pulse_mid(wl):
    freq = 1239.84190 / (wl["wlen"] * 27.2113845)
    return 0.5 * wl["numcyc"] * 2 * np.pi / freq


def gauge_field(wl, t):
    """lfield(1:3,1:3) of the velocity-gauge sin^2 pulse with only the gauge
    component A(t) filled (what the one-body step reads)."""
    famp = np.sqrt(wl["fint"] / 3.50944506e16)
    freq = 1239.84190 / (wl["wlen"] * 27.2113845)
    period = 2 * np.pi / freq
    lf = np.zeros(9)
    if 0 < t < wl["numcyc"] * period:
        env = np.sin(np.pi * t / (wl["numcyc"] * period)) ** 2
        lf[2] = lf[8] = env * famp / freq * np.sin(freq * t + wl.get("cep", 0.0) * np.pi / 180.0)
    return lf


def a_peak_time(wl):
    """A time near the envelope maximum where |A(t)| = |env A0 sin(w t + cep)| peaks."""
    freq = 1239.84190 / (wl["wlen"] * 27.2113845)
    tc = pulse_mid(wl)
    ph = freq * tc + wl.get("cep", 0.0) * np.pi / 180.0
    k = np.round((ph - 0.5 * np.pi) / np.pi)
    return tc + ((k * np.pi + 0.5 * np.pi) - ph) / freq


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    def __init__(self, gpu):
        self.gpu = gpu
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + q, "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        try:
            for line in open(self.path):
                f = [x.strip() for x in line.split(",")]
                if len(f) < 9:
                    continue
                try:
                    sm.append(float(f[1]))
                    mx = float(f[2])
                except ValueError:
                    continue
                for n, v in zip(names, f[5:9]):
                    if v.lower() == "active":
                        reasons.add(n)
        except OSError:
            pass
        finally:
            try:
                os.unlink(self.path)
            except OSError:
                pass
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get("hbm_gbs", 6650.0), "measured (MEASURED_PEAKS.json hbm_gbs)"
    return 6650.0, "fallback 6.65 TB/s"


def fp64_peak_tflops(torch):
    """cuBLAS DGEMM throughput measured in this run (the FP64 ceiling the
    register-tiled FP64 kernels are compared against)."""
    n = 4096
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    for _ in range(2):
        torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 1e9
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1) / 1e3)
    del a, b
    return 2.0 * n ** 3 / best / 1e12


MIXED_NOTE = {1: "mixed (split TF32 pair-field transforms)",
              3: "mixed mode 3 (split TF32 pair-field transforms, Poisson interior products and int2e)"}


def committed_state(wl, nrad, lmax1, mmax1, nfun, lcic):
    """The committed relaxed start state of the workload, through the reference's .orb/.cic text
    format (written and read back, as a td1c restart would read it), or None when there is none."""
    from td1c_b200 import wfnio
    from td1c_b200.data.make_relaxed_state import load, path_for
    path = path_for(wl["name"])
    if path is None or not os.path.exists(path):
        return None
    orb, cic, info = load(path)
    if info["workload"] != wl["name"]:
        return None
    with tempfile.TemporaryDirectory() as d:
        po, pc = os.path.join(d, "state.orb"), os.path.join(d, "state.cic")
        wfnio.write_wfn(po, pc, orb, cic, nrad, lmax1, mmax1)
        orb2, cic2 = wfnio.read_wfn(po, pc, nrad, lmax1, nfun, lcic)
    src = "committed relaxed state (td1c_b200/data/%s) via .orb/.cic" % os.path.basename(path)
    return np.asarray(orb2).reshape(nfun, -1), np.asarray(cic2), dict(info, source=src)


def oracle_setup(wl, prop):
    """The oracle with the workload's start state bound: the committed relaxed state where there is
    one (the GPU arm starts from the same), else the seeded state, orthonormalised."""
    from oracle.oracle import Oracle
    from td1c_b200.wfn import seeded_orbitals
    wl = dict(wl, split_type=0 if prop == "rk4" else 1)
    o = Oracle(wl)
    o.set_split(wl["split_type"])
    d = o.dims
    mmax1 = max(abs(x[2]) for x in wl["orbitals"])
    st = committed_state(wl, d["nrad"], wl["lmax1"], mmax1, len(wl["orbitals"]), d["lcic"])
    if st is not None:
        orb, cic, info = st
        o.set_wfn0(orb, cic)
        return o, orb, cic, info["source"]
    orb = seeded_orbitals(wl, o.get("xrad"), o.get("wrad"), o.get("mask"))
    cic = np.ones(d["lcic"], dtype=np.complex128) / np.sqrt(d["lcic"]) if d["nact"] else np.ones(1, dtype=np.complex128)
    o.set_wfn0(orb, cic)
    orb, cic = o.orth(orb, cic)
    return o, orb, cic, "seeded state, orthonormalised (unrelaxed)"


def oracle_step(o, prop, orb, cic, t, dt):
    if prop == "split2":
        w, c, _ = o.split2(orb, cic, t, dt, 1)
    elif prop == "etdrk2":
        w, c, _ = o.etdrk2(orb, cic, t, dt, 1)
    else:
        o.rk4(orb, cic, t, dt, 1)
        return orb, cic  # the full-H RK4 arm restarts from the same state
    return w, c


def cpu_baseline(wl, dt, prop, t0, max_seconds=60.0):
    """The oracle (C++/OpenMP restatement of the reference path) on the host cores: a bounded sample
    of whole steps of the same workload from the same start state and time."""
    o, orb, cic, src = oracle_setup(wl, prop)
    t = t0
    n, tot = 0, 0.0
    while True:
        ts = time.perf_counter()
        orb, cic = oracle_step(o, prop, orb, cic, t, dt)
        tot += time.perf_counter() - ts
        n += 1
        t += dt
        if tot > max_seconds * 0.5 or n >= 3:
            break
    sec_per_step = tot / n
    return {"value": dt * AU2FS / sec_per_step, "unit": "fs/s", "cores": o.num_threads(), "kind": "port",
            "sample": "%d %s step(s) (%d RHS) of %s on the oracle from t = %g au, %s; %.2f s/step"
                      % (n, prop, RHS_PER_STEP[prop] * n, wl["name"], t0, src, sec_per_step)}


def run_reference(args):
    """The reference arm: the CPU restatement of the reference path on all host cores, same start
    state, start time and warm-up as the GPU arm, timed steps capped to about two minutes."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    wl = workload(args.workload)
    dt = wl["dt"]
    o, orb, cic, src = oracle_setup(wl, args.prop)
    t = args.t0
    ts = time.perf_counter()
    for _ in range(max(1, args.warmup)):
        orb, cic = oracle_step(o, args.prop, orb, cic, t, dt)
        t += dt
    t_step = (time.perf_counter() - ts) / max(1, args.warmup)
    k = max(1, min(args.steps, int(120.0 / max(t_step, 1e-3))))
    ts = time.perf_counter()
    for _ in range(k):
        orb, cic = oracle_step(o, args.prop, orb, cic, t, dt)
        t += dt
    el = time.perf_counter() - ts
    v = k * dt * AU2FS / el
    line = {"impl": "reference", "metric": metric_name(), "value": v, "unit": "fs/s", "n_gpus": args.gpus,
            "steps": k, "warmup": max(1, args.warmup), "ms_per_step": el / k * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "c128",
            "data": "synthetic: %s; one trajectory from t0" % src,
            "config": {"workload": wl["name"], "dt_au": dt, "precision": "fp64", "prop": PROP_NOTE[args.prop],
                       "t0_au": args.t0, "start_state": src,
                       "note": "CPU restatement of the reference path (the Fortran/MKL reference does not build here)"},
            "cpu_baseline": {"value": v, "unit": "fs/s", "cores": o.num_threads(), "kind": "port",
                             "sample": "%d %s steps of %s after %d warm-up steps (steps capped to bound the run time)"
                                       % (k, args.prop, wl["name"], max(1, args.warmup))},
            "e2e": {"value": v, "unit": "fs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def profiled_traffic(phase):
    """DRAM bytes per launch of the phase's main kernel from the committed ncu summary, or None."""
    path = os.path.join(ROOT, "profiles", "dram_traffic_per_launch.md")
    if not os.path.exists(path):
        return None
    for line in open(path):
        cells = [c.strip() for c in line.strip().strip("|").split("|")]
        if len(cells) == 3 and cells[0] == phase and cells[2].isdigit():
            return int(cells[2])
    return None


# the benchmark's metric: simulated time per second of the learned+mixed propagation, with the plain
# FP64 path measured beside it (td1c publishes no numbers for it)
METRIC = "fs simulated/s on 1 B200, learned+mixed vs plain FP64, at dipole err \u22641e-5 au"


def metric_name():
    return METRIC


def seeded_fields(n, seed=5):
    """The learned predictor's training pulses: intensity log-uniform in [1e13, 5e14] W/cm^2,
    wavelength uniform in [600, 1200] nm, start time uniform over the middle of the pulse."""
    rng = np.random.Generator(np.random.Philox(seed))
    return [(float(10.0 ** rng.uniform(13.0, np.log10(5e14))), float(rng.uniform(600.0, 1200.0)),
             float(rng.uniform(0.2, 0.8))) for _ in range(n)]


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    import torch
    import torch.distributed as dist
    from td1c_b200 import basis
    from td1c_b200.hprod import HProd
    from td1c_b200.wfn import seeded_orbitals, seeded_cic, velocity_gauge_phase
    from td1c_b200.workmodel import rhs_work

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    torch.cuda.set_device(local)
    wl = dict(workload(args.workload), split_type=0 if args.prop == "rk4" else 1)
    dt = wl["dt"]
    rad, ang = basis.build(wl)
    h = HProd(wl, rad, ang)
    d = h.dims
    nfun = len(wl["orbitals"])
    tb = h.ci_tables()
    dev = torch.device("cuda", local)
    ext = torch.cuda.ExternalStream(h.stream())

    # ---- start state: the committed relaxed state (both arms), else seeded and relaxed on the GPU
    st = committed_state(wl, d["nrad"], wl["lmax1"], ang["mmax1"], nfun, d["lcic"]) if world == 1 else None
    if st is not None:
        orb, cic, info = st
        h.set_wfn0(orb, cic)
        d_orb = torch.from_numpy(np.ascontiguousarray(orb).reshape(-1).copy()).to(dev)
        d_cic = torch.from_numpy(np.ascontiguousarray(cic).copy()).to(dev)
        relax = {"source": info["source"], "cycles": info["cycles"], "dt_au": info["dt"], "energy": info["energy"]}
    else:
        orb = seeded_orbitals(wl, rad["xrad"], rad["wrad"], rad["mask"], seed=replica_seed(wl.get("seed", 0), rank))
        cic = seeded_cic(wl, d["lcic"], tb["stra"], tb["strb"], tb["detoff"], tb["afirst"], tb["acount"])
        h.set_wfn0(orb, cic)
        d_orb = torch.from_numpy(orb.reshape(-1).copy()).to(dev)
        d_cic = torch.from_numpy(cic.copy()).to(dev)
        torch.cuda.synchronize()
        h.set_time_kind(0)
        h.orth_dev(d_orb.data_ptr(), d_cic.data_ptr())
        h.set_split(1)
        ene = h.relax_etdrk2_dev(d_orb.data_ptr(), d_cic.data_ptr(), args.relax_dt, args.relax_cycles)
        h.set_split(wl["split_type"])
        h.set_time_kind(1)
        relax = {"source": "seeded (Philox) and relaxed on the GPU", "cycles": args.relax_cycles, "dt_au": args.relax_dt,
                 "energy": float(ene[-1])}
    torch.cuda.synchronize()
    d_relaxed, c_relaxed = d_orb.clone(), d_cic.clone()

    def placed(t):
        """The start state placed at time t: the velocity-gauge phase of A(t) on the non-frozen orbitals."""
        A = gauge_field(wl, t)[2]
        if wl["igauge"] != 1 or A == 0.0:
            return d_relaxed.clone(), c_relaxed.clone()
        wv = velocity_gauge_phase(wl, d_relaxed.cpu().numpy().reshape(nfun, wl["lmax1"] + 1, -1), rad, ang, A)
        return torch.from_numpy(wv.reshape(-1)).to(dev), c_relaxed.clone()

    t0 = args.t0
    o0, c0 = placed(t0)

    def steps(arm, yo, yc, t, n, use_graph=True):
        """n steps of an arm in place; returns the learned arm's judge statistics (None otherwise)."""
        if arm == "learned":
            return h.split2_learned_dev(yo.data_ptr(), yc.data_ptr(), t, dt, n)
        if args.prop == "split2":
            h.split2_dev(yo.data_ptr(), yc.data_ptr(), t, dt, n, use_graph=use_graph)
        elif args.prop == "etdrk2":
            h.etdrk2_dev(yo.data_ptr(), yc.data_ptr(), t, dt, n, use_graph=use_graph)
        else:
            h.rk4_dev(yo.data_ptr(), yc.data_ptr(), t, dt, n, use_graph=use_graph)
        return None

    def set_arm(arm):
        h.set_mixed(args.mixed_mode if arm in ("mixed", "learned") else 0)

    def window(arm, t_start, n, warm, o_start=None, c_start=None):
        """warm + n steps of an arm from the given start (default the window start state); returns
        (seconds of the n timed steps on the device, end state, judge statistics, launches)."""
        set_arm(arm)
        h.rk4_reset(None, None)
        yo = (o0 if o_start is None else o_start).clone()
        yc = (c0 if c_start is None else c_start).clone()
        steps(arm, yo, yc, t_start, warm)
        h.sync()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(ext)
        jst = steps(arm, yo, yc, t_start + warm * dt, n)
        e1.record(ext)
        torch.cuda.synchronize()
        launches = h.launch_count()
        h.sync()
        return e0.elapsed_time(e1) / 1e3, yo, yc, jst, launches

    def deviations(yo, yc, ro, rc):
        dip = abs(h.dipole_dev(yo.data_ptr(), yc.data_ptr()) - h.dipole_dev(ro.data_ptr(), rc.data_ptr()))
        n1 = np.linalg.norm(yo.cpu().numpy().reshape(nfun, -1), axis=1)
        n2 = np.linalg.norm(ro.cpu().numpy().reshape(nfun, -1), axis=1)
        cn = abs(float(torch.linalg.vector_norm(yc)) - float(torch.linalg.vector_norm(rc)))
        return {"dipole_dev_au": dip, "orbital_norm_dev": float(np.abs(n1 - n2).max()), "ci_norm_dev": cn,
                "state_rel_dev": float((yo - ro).abs().max() / ro.abs().max())}

    # ---- the learned predictor's network, trained on the GPU from seeded trajectories
    net, training = None, None
    if not args.no_mixed and not args.no_learned and args.prop == "split2":
        from td1c_b200 import learned as L
        h.set_mixed(False)
        tt = time.perf_counter()
        R = L.Records(h, 12)
        period = wl["numcyc"] * 2 * np.pi / (1239.84190 / (wl["wlen"] * 27.2113845))
        fields = seeded_fields(args.train_traj)
        for fint, wlen, frac in fields:
            ts = frac * period
            yo, yc = placed(ts)
            buf = R.new_buffer()
            h.learned_record_dev(yo.data_ptr(), yc.data_ptr(), ts, dt, 12, buf.data_ptr(), fint=fint, wlen=wlen)
            h.sync()
            R.add(buf)
        rec = R.all()
        ntrain = (rec.shape[0] // R.nu * 9 // 10) * R.nu
        t_rec = time.perf_counter() - tt
        net = L.new_predictor_net(seed=3)
        tt = time.perf_counter()
        curve = L.train(net, rec[:ntrain], R.nu, R.nfe, R.pair_kind, steps=args.train_iters, batch=8192, lr=1e-5)
        torch.cuda.synchronize()
        t_train = time.perf_counter() - tt
        ev = L.evaluate(net, rec[ntrain:].contiguous(), R.nu, R.nfe, R.pair_kind)
        training = {"trajectories": len(fields), "steps_recorded": 8, "records": int(rec.shape[0]),
                    "units": R.nu, "fields": "I log-uniform 1e13-5e14 W/cm^2, wavelength 600-1200 nm, start 0.2-0.8 "
                                              "of the pulse, seeded (Philox)",
                    "record_s": t_rec, "train_s": t_train, "iters": args.train_iters, "objective": "mean log(1 + L / eps) on a fixed batch of training records, L the relative squared "
                                 "error, eps its median for the cubic; the best weights are kept",
                    "objective_start_last_best": [curve[0], curve[-1], min(curve)],
                    "held_out_one_step_rel_err": ev,
                    "network": "MLP 32-256-256-256-8, tanh, FP32 weights (Adam), BF16 inference on tcgen05"}
        h.set_learned(net, use_net=True, bound=args.bound)
        del rec, R

    # ---- the arms over the window from t0
    arms = ["fp64"] + ([] if args.no_mixed else ["mixed"]) + ([] if (args.no_mixed or net is None) else ["learned"])
    res = {}
    with Clocks(local) as clk:
        for arm in arms:
            sec, yo, yc, jst, launches = window(arm, t0, args.steps, args.warmup)
            sec = max_over_ranks(sec, dist if world > 1 else None, dev)
            res[arm] = {"sec": sec, "end": (yo, yc), "judge": jst, "launches": launches}
    set_arm("fp64")
    fp_end = res["fp64"]["end"]
    wn = fp_end[0].cpu().numpy().reshape(nfun, -1)
    traj = {"t_start_au": t0 + args.warmup * dt, "t_end_au": t0 + (args.warmup + args.steps) * dt,
            "orbital_norm_dev": float(np.abs(np.linalg.norm(wn, axis=1) - 1.0).max()), "finite": bool(np.all(np.isfinite(wn)))}

    def arm_line(arm):
        r = res[arm]
        v = job_throughput(world, args.steps, dt, r["sec"])
        out = {"value": v, "unit": "fs/s", "ms_per_step": r["sec"] / args.steps * 1e3,
               "speedup_vs_fp64": v / job_throughput(world, args.steps, dt, res["fp64"]["sec"])}
        if arm != "fp64":
            out["vs_fp64_at_window_end"] = deviations(r["end"][0], r["end"][1], fp_end[0], fp_end[1])
        if r["judge"] is not None:
            out["judge"] = r["judge"]
        return out

    lines = {arm: arm_line(arm) for arm in arms}
    head_arm = "learned" if "learned" in arms else ("mixed" if "mixed" in arms else "fp64")
    value = lines[head_arm]["value"]
    sec = res[head_arm]["sec"]

    # ---- the same arms at the |A| peak (the start state placed there)
    peak = None
    if not args.no_peak and args.prop == "split2":
        tp = a_peak_time(wl) - 0.5 * min(args.steps, 48) * dt
        po, pc = placed(tp)
        peak = {"t_start_au": tp, "steps": min(args.steps, 48)}
        for arm in arms:
            s_, yo, yc, jst, _ = window(arm, tp, min(args.steps, 48), args.warmup, po, pc)
            peak[arm] = {"value": job_throughput(world, min(args.steps, 48), dt, s_), "ms_per_step": s_ / min(args.steps, 48) * 1e3}
            if jst is not None:
                peak[arm]["judge"] = jst
        set_arm("fp64")

    # ---- end to end through the public API: host buffers, one judged window (8 steps) per call
    set_arm(head_arm)
    h.rk4_reset(None, None)
    yo, yc = res[head_arm]["end"][0].clone(), res[head_arm]["end"][1].clone()
    h_orb = torch.from_numpy(yo.cpu().numpy()).pin_memory()
    h_cic = torch.from_numpy(yc.cpu().numpy()).pin_memory()
    per_call = 8 if head_arm == "learned" else 1
    ke = args.e2e_steps or max(16, min(args.steps, 48))
    ke = (ke + per_call - 1) // per_call * per_call
    t2 = traj["t_end_au"]

    def e2e_call(t):
        with torch.cuda.stream(ext):
            yo.copy_(h_orb, non_blocking=True)
            yc.copy_(h_cic, non_blocking=True)
        steps(head_arm, yo, yc, t, per_call)
        with torch.cuda.stream(ext):
            h_orb.copy_(yo, non_blocking=True)
            h_cic.copy_(yc, non_blocking=True)

    for s_ in range(2):
        e2e_call(t2 + s_ * per_call * dt)
    torch.cuda.synchronize()
    t2 += 2 * per_call * dt
    if world > 1:
        dist.barrier()
    e2, e3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    w0 = time.perf_counter()
    e2.record(ext)
    for s_ in range(ke // per_call):
        e2e_call(t2 + s_ * per_call * dt)
    e3.record(ext)
    torch.cuda.synchronize()
    wall = time.perf_counter() - w0
    sec_e = max_over_ranks(max(e2.elapsed_time(e3) / 1e3, wall), dist if world > 1 else None, dev)
    e2e = job_throughput(world, ke, dt, sec_e)
    bytes_call = (h_orb.numel() + h_cic.numel()) * 16
    set_arm("fp64")

    # ---- one-body half step alone (split2's clh1itr) at the |A| peak field
    h1_ms = None
    if args.prop == "split2":
        lf = gauge_field(wl, a_peak_time(wl))
        d_tmp = d_relaxed.clone()
        h.h1itr_dev(d_tmp.data_ptr(), lf, 0.5 * dt)
        reps, ncyc = 20, 0
        w0 = time.perf_counter()
        for _ in range(reps):
            ncyc = h.h1itr_dev(d_tmp.data_ptr(), lf, 0.5 * dt)
        h1_ms = {"ms": (time.perf_counter() - w0) / reps * 1e3, "corrections": ncyc,
                 "note": "one clh1itr half step at the |A| peak, host-timed with its synchronisation"}
        del d_tmp

    # ---- phase profile and roofline of the dominant kernel (plain FP64 RHS)
    d_hw, d_hc = torch.empty_like(d_relaxed), torch.empty_like(c_relaxed)
    phases = h.profile(5, np.zeros(9), d_relaxed.data_ptr(), c_relaxed.data_ptr(), d_hw.data_ptr(), d_hc.data_ptr())
    work = rhs_work(wl, d)
    if max(phases.values()) <= 0:
        raise RuntimeError("phase profile returned no timings: %r" % phases)
    dom = max(phases, key=lambda k: phases[k])
    fl, by = work.get(dom, (0, 0))
    hbm, hbm_src = measured_peaks()
    f64 = fp64_peak_tflops(torch)
    t_dom = phases[dom] / 1e3
    traffic = profiled_traffic(dom)
    if fl / max(by, 1) > f64 * 1e12 / (hbm * 1e9):
        roof = {"bound": "tensor", "achieved": fl / t_dom / 1e12, "peak": f64, "unit": "TFLOP/s",
                "frac": fl / t_dom / 1e12 / f64, "traffic": traffic, "kernel": dom,
                "peak_source": "FP64: cuBLAS DGEMM 4096^3 measured in this run (B200 has no FP64 tcgen05 kind)"}
    else:
        roof = {"bound": "hbm", "achieved": by / t_dom / 1e9, "peak": hbm, "unit": "GB/s",
                "frac": by / t_dom / 1e9 / hbm, "traffic": traffic, "kernel": dom, "peak_source": hbm_src}
    mixed_dev = None
    if not args.no_mixed:
        h.set_mixed(args.mixed_mode)  # the self-test compares the current mixed mode with FP64
        rd = h.mixed_selftest(d_relaxed.data_ptr(), c_relaxed.data_ptr(), gauge_field(wl, t0))
        h.set_mixed(0)
        mixed_dev = {"rho2": float(rd[0]), "W": float(rd[1]), "hwfn": float(rd[2])}

    # ---- the whole pulse (optional here; the default line carries the committed measurement)
    fp_path = os.path.join(ROOT, "profiles", "full_pulse_%s.json" % wl["name"])
    full = None
    if args.full_pulse:
        full = full_pulse(args, h, wl, dt, arms, set_arm, steps, placed, deviations, torch, fp_path)
    elif os.path.exists(fp_path):
        full = dict(json.load(open(fp_path)), source="committed measurement (python bench.py --full-pulse), %s" % fp_path)

    # ---- the ensemble (optional)
    ens = None
    if args.ensemble:
        ens = ensemble_leg(args.ensemble, small=args.ensemble_small)

    h.final()
    if rank != 0:
        if world > 1:
            dist.destroy_process_group()
        return 0
    line = {
        "metric": metric_name(), "value": value, "unit": "fs/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": sec / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "c128",
        "data": "synthetic: %s; one trajectory per arm from t0 (velocity-gauge phase of A(t0))" % relax["source"],
        "config": {"workload": wl["name"], "dt_au": dt, "arm": {"learned": "learned+mixed", "mixed": "mixed",
                                                                "fp64": "fp64"}[head_arm],
                   "precision": {"learned": "%s + learned stage mean fields (judge bound %g)" % (MIXED_NOTE[args.mixed_mode],
                                                                                                 args.bound),
                                 "mixed": MIXED_NOTE[args.mixed_mode], "fp64": "fp64"}[head_arm],
                   "prop": PROP_NOTE[args.prop], "rhs_per_step": RHS_PER_STEP[args.prop],
                   "window": "one trajectory per arm from t0 = %g au: %d warm-up then %d timed steps" % (t0, args.warmup,
                                                                                                       args.steps),
                   "start_state": relax, "trajectory_fp64": traj, "lcic": d["lcic"], "nfun": nfun,
                   "l2": "working set per step > 126 MB L2 (pair fields 3 x 98 MB)",
                   "parallelism": "replicas" if world > 1 else "1 GPU"},
        "fp64": lines["fp64"],
        "mixed": dict(lines["mixed"], rhs_rel_dev=mixed_dev) if "mixed" in lines else None,
        "learned_mixed": dict(lines["learned"], training=training) if "learned" in lines else None,
        "peak_window": peak,
        "full_pulse": full,
        "ensemble": ens,
        "e2e": {"value": e2e, "unit": "fs/s", "h2d_bytes_per_step": bytes_call / per_call,
                "d2h_bytes_per_step": bytes_call / per_call, "steps": ke, "steps_per_call": per_call,
                "note": "host state copied in before and out after every call of %d step(s)%s" % (
                    per_call, " (one judged window)" if per_call > 1 else "")},
        "gpu_launches": res[head_arm]["launches"],
        "roofline": roof,
        "phases_ms_per_rhs": {k: round(v, 4) for k, v in phases.items()},
        "one_body_half_step": h1_ms,
        "clocks": clk.summary(),
    }
    if world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(wl, dt, args.prop, t0)
    print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()
    return 0


def full_pulse(args, h, wl, dt, arms, set_arm, steps, placed, deviations, torch, path):
    """Every arm over the whole pulse from its onset: dipole every nprint steps (as tdse_print samples it),
    pulse-averaged fs/s, per-chunk step times, and the deviations from FP64; written to path."""
    period = wl["numcyc"] * 2 * np.pi / (1239.84190 / (wl["wlen"] * 27.2113845))
    nstep = int(np.ceil(period / dt))
    nprint = max(1, args.nprint)
    out = {"workload": wl["name"], "steps": nstep, "dt_au": dt, "simulated_fs": nstep * dt * AU2FS, "nprint": nprint,
           "bound": args.bound}
    dips, ends = {}, {}
    # FP64 trajectories from perturbed start states: seeded complex noise of relative size eps (of each
    # orbital's largest component) on the nonzero components of the orbitals
    pert = {"fp64_perturbed_%s" % e.strip(): float(e) for e in args.sensitivity.split(",") if e.strip()}
    rng = np.random.default_rng(11)
    for arm in list(arms) + list(pert):
        set_arm("fp64" if arm in pert else arm)
        h.rk4_reset(None, None)
        yo, yc = placed(0.0)
        if arm in pert:
            o = yo.cpu().numpy().reshape(len(wl["orbitals"]), -1)
            big = np.abs(o).max(axis=1, keepdims=True)
            noise = rng.standard_normal(o.shape) + 1j * rng.standard_normal(o.shape)
            o = o + pert[arm] * big * noise * (np.abs(o) > 0)
            yo = torch.from_numpy(o.reshape(-1)).to(yo.device)
        dl, tl, jacc = [h.dipole_dev(yo.data_ptr(), yc.data_ptr())], [], {"accepted": 0, "rejected": 0, "steps_kept": 0}
        s = 0
        tot = 0.0
        while s < nstep:
            n = min(nprint, nstep - s)
            torch.cuda.synchronize()
            w0 = time.perf_counter()
            jst = steps(arm, yo, yc, s * dt, n)
            h.sync()
            el = time.perf_counter() - w0
            tot += el
            tl.append(el / n * 1e3)
            if jst is not None:
                jacc["accepted"] += int(jst["accepted"])
                jacc["rejected"] += int(jst["rejected"])
                jacc["steps_kept"] += int(jst["predicted_steps"])
            dl.append(h.dipole_dev(yo.data_ptr(), yc.data_ptr()))
            s += n
        dips[arm] = np.array(dl)
        ends[arm] = (yo, yc)
        q = len(tl)
        out[arm] = {"fs_per_s": out["simulated_fs"] / tot, "seconds": tot,
                    "ms_per_step_onset_quarter_peak": [tl[0], tl[q // 4], tl[q // 2]],
                    "finite": bool(torch.isfinite(yo).all()), "status": h.last_status()}
        if arm == "learned":
            out[arm]["judge"] = jacc
    set_arm("fp64")
    for arm in list(arms) + list(pert):
        if arm == "fp64":
            continue
        dd = np.abs(dips[arm] - dips["fp64"])
        dv = deviations(ends[arm][0], ends[arm][1], ends["fp64"][0], ends["fp64"][1])
        out[arm]["max_dipole_dev_au"] = float(dd.max())
        over = np.nonzero(dd > 1e-5)[0]
        out[arm]["first_t_au_dipole_dev_over_1e-5"] = float(min(over[0] * nprint, nstep) * dt) if over.size else None
        out[arm]["vs_fp64_at_end"] = dv
        out[arm]["gates"] = {"dipole_le_1e-5": bool(dd.max() <= 1e-5), "norm_le_1e-8": bool(dv["orbital_norm_dev"] <= 1e-8)}
    out["dipole_fp64_range_au"] = [float(dips["fp64"].min()), float(dips["fp64"].max())]
    with open(path, "w") as fh:
        json.dump(out, fh, indent=1)
    return out


def ensemble_leg(njob, seed=7, nstep=16, small=False):
    """The seeded ensemble's jobs stepped together by one graph per step, against the same steps run
    job after job (fs/s summed over the jobs)."""
    from td1c_b200 import autotune
    from td1c_b200.ensemble import DeviceEnsemble, job_list
    jobs = job_list(seed, njob, small=small)
    ens = DeviceEnsemble(jobs, relax_cycles=20)
    try:
        choice = autotune.tune(ens, nstep=2)
        orb = [x.clone() for x in ens.orb]
        cic = [x.clone() for x in ens.cic]
        ens.run(2, orb=orb, cic=cic)
        ms = ens.run(nstep, orb=orb, cic=cic)
        orb = [x.clone() for x in ens.orb]
        cic = [x.clone() for x in ens.cic]
        ens.run_sequential(2, orb=orb, cic=cic)
        ms_seq = ens.run_sequential(nstep, orb=orb, cic=cic)
        fs = ens.simulated_fs(nstep)
        return {"jobs": njob, "seed": seed, "job_range": "small" if small else "full", "steps": nstep,
                "fs_per_s": fs / (ms / 1e3), "ms_per_step": ms / nstep,
                "one_by_one_fs_per_s": fs / (ms_seq / 1e3), "one_by_one_ms_per_step": ms_seq / nstep,
                "speedup": ms_seq / ms, "tuning": choice}
    finally:
        ens.final()


if __name__ == "__main__":
    sys.exit(main())
