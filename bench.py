#!/usr/bin/env python
"""Benchmark: fs of simulated time per second for the Ne TD-CASSCF
propagation on B200, driven through the td1c_b200 C-ABI.

Workload: Ne TD-CASSCF (1s frozen core + CAS(8e, 9o), FEDVR 60 x 21 points,
rmax 120, lmax 47 / 94, velocity gauge, sin^2 800 nm 4-cycle 5e14 W/cm^2
pulse, dt 0.004 au), FP64 complex arithmetic.  The state is seeded (Philox)
and relaxed in imaginary time on the GPU with ETD-RK2 steps (init_prop12
with cletdrk2) before any timing.

A step (default --prop split2) is td1c's RK4 at this dt as the reference
runs it: tdse_split2 with clh1itr + clcrk and split_type 1 -- a Crank-
Nicolson half step of the one-body Hamiltonian (kinetic, nuclear, laser
coupling by correction cycles), one RK4 step (four RHS evaluations) of the
two-body part, a second one-body half step, and the absorbing mask.  The
steps form one real trajectory (each step starts where the last ended),
timed from the pulse onset (t = 0) like td1c's own tdse loop; the one-body
half step is also timed alone at the |A(t)| maximum, where its correction
cycles are the most numerous.  --prop etdrk2 times cletdrk2 instead;
--prop rk4 the full-H RK4, which is unstable at this dt and therefore
restarts every step from the relaxed state.

value  : fs/s with the state resident in HBM (one CUDA graph per step).
e2e    : fs/s through the public API with the state copied host->device
         before and device->host after every step (pinned host buffers),
         the host copy carrying the trajectory.
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
    ap.add_argument("--no-mixed", action="store_true", help="skip the mixed-precision arm")
    ap.add_argument("--prop", default="split2", choices=["split2", "etdrk2", "rk4"])
    # imaginary time tau = 3 au: the energy is within 0.07 au of its limit and
    # the smallest natural occupation stays ~1e-3.  Relaxed further, the 3d0
    # occupation falls to ~3e-4, the 1-RDM inverse of the mean field grows to
    # ~3e3 and the RK4 part of split2 at dt = 0.004 (throcc1 = 1e-15, the
    # reference defaults) diverges after ~75 steps -- the oracle as well.
    ap.add_argument("--relax-cycles", type=int, default=300)
    # imaginary-time Pade steps need 1 - (dt/2) |E_1s| > 0 for the deepest
    # one-body level (Z = 10: E_1s = -50 au), i.e. dt < 0.04
    ap.add_argument("--relax-dt", type=float, default=0.01)
    ap.add_argument("--t0", type=float, default=0.0, help="start time of the trajectory (au)")
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


def oracle_setup(wl, prop):
    """The oracle with the workload's seeded state (orthonormalised) bound."""
    from oracle.oracle import Oracle
    from td1c_b200.wfn import seeded_orbitals
    wl = dict(wl, split_type=0 if prop == "rk4" else 1)
    o = Oracle(wl)
    o.set_split(wl["split_type"])
    d = o.dims
    orb = seeded_orbitals(wl, o.get("xrad"), o.get("wrad"), o.get("mask"))
    cic = np.ones(d["lcic"], dtype=np.complex128) / np.sqrt(d["lcic"]) if d["nact"] else np.ones(1, dtype=np.complex128)
    o.set_wfn0(orb, cic)
    orb, cic = o.orth(orb, cic)
    return o, orb, cic


def oracle_step(o, prop, orb, cic, t, dt):
    if prop == "split2":
        w, c, _ = o.split2(orb, cic, t, dt, 1)
    elif prop == "etdrk2":
        w, c, _ = o.etdrk2(orb, cic, t, dt, 1)
    else:
        o.rk4(orb, cic, t, dt, 1)
        return orb, cic  # the full-H RK4 arm restarts from the same state
    return w, c


def cpu_baseline(wl, dt, prop, max_seconds=60.0):
    """The oracle (C++/OpenMP restatement of the reference path) on the host
    cores: a bounded sample of whole steps of the same workload."""
    o, orb, cic = oracle_setup(wl, prop)
    t = 0.0
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
            "sample": "%d %s step(s) (%d RHS) of %s on the oracle from the seeded state, %.2f s/step"
                      % (n, prop, RHS_PER_STEP[prop] * n, wl["name"], sec_per_step)}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    wl = workload(args.workload)
    dt = wl["dt"]
    o, orb, cic = oracle_setup(wl, args.prop)
    t = 0.0
    ts = time.perf_counter()
    for _ in range(max(1, min(args.warmup, 1))):
        orb, cic = oracle_step(o, args.prop, orb, cic, t, dt)
        t += dt
    t_step = time.perf_counter() - ts
    k = max(1, min(args.steps, int(120.0 / max(t_step, 1e-3))))
    ts = time.perf_counter()
    for _ in range(k):
        orb, cic = oracle_step(o, args.prop, orb, cic, t, dt)
        t += dt
    el = time.perf_counter() - ts
    v = k * dt * AU2FS / el
    line = {"impl": "reference", "metric": metric_name(), "value": v, "unit": "fs/s", "n_gpus": args.gpus,
            "steps": k, "warmup": 1, "ms_per_step": el / k * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "c128",
            "data": "synthetic (seeded orbitals and CI, orthonormalised; a trajectory from the pulse onset)",
            "config": {"workload": wl["name"], "dt_au": dt, "precision": "fp64", "prop": PROP_NOTE[args.prop],
                       "note": "CPU restatement of the reference path (the Fortran/MKL reference does not build here)"},
            "cpu_baseline": {"value": v, "unit": "fs/s", "cores": o.num_threads(), "kind": "port",
                             "sample": "%d %s steps of %s (steps capped to bound the run time)" % (k, args.prop, wl["name"])},
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


# the headline metric of the td1c propagation benchmark, as published with its numbers
METRIC = "fs simulated/s on 1 B200, learned+mixed vs plain FP64, at dipole err \u22641e-5 au"


def metric_name():
    return METRIC


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
    tb = h.ci_tables()
    orb = seeded_orbitals(wl, rad["xrad"], rad["wrad"], rad["mask"], seed=replica_seed(wl.get("seed", 0), rank))
    cic = seeded_cic(wl, d["lcic"], tb["stra"], tb["strb"], tb["detoff"], tb["afirst"], tb["acount"])
    h.set_wfn0(orb, cic)
    dev = torch.device("cuda", local)
    d_orb = torch.from_numpy(orb.reshape(-1).copy()).to(dev)
    d_cic = torch.from_numpy(cic.copy()).to(dev)
    ext = torch.cuda.ExternalStream(h.stream())
    torch.cuda.synchronize()

    # ---- set-up (untimed): imaginary-time relaxation with ETD-RK2 steps
    h.set_time_kind(0)
    h.orth_dev(d_orb.data_ptr(), d_cic.data_ptr())
    h.set_split(1)
    ene = h.relax_etdrk2_dev(d_orb.data_ptr(), d_cic.data_ptr(), args.relax_dt, args.relax_cycles)
    h.set_split(wl["split_type"])
    h.set_time_kind(1)
    relax = {"cycles": args.relax_cycles, "dt_au": args.relax_dt, "energy": float(ene[-1]),
             "last_change": float(ene[-1] - ene[-2]) if len(ene) > 1 else None}
    # the trajectory starts where the reference's does, at the pulse onset
    # (t = 0, A = 0); a state placed at a later time would need the
    # velocity-gauge phase of A(t0) that the frozen core carries
    t0 = args.t0
    A0 = gauge_field(wl, t0)[2]
    if wl["igauge"] == 1 and A0 != 0.0:
        wv = velocity_gauge_phase(wl, d_orb.cpu().numpy().reshape(len(wl["orbitals"]), wl["lmax1"] + 1, -1), rad, ang, A0)
        d_orb.copy_(torch.from_numpy(wv.reshape(-1)))
    d_orb0, d_cic0 = d_orb.clone(), d_cic.clone()
    torch.cuda.synchronize()

    def steps(t, n, use_graph=True):
        if args.prop == "split2":
            h.split2_dev(d_orb.data_ptr(), d_cic.data_ptr(), t, dt, n, use_graph=use_graph)
        elif args.prop == "etdrk2":
            h.etdrk2_dev(d_orb.data_ptr(), d_cic.data_ptr(), t, dt, n, use_graph=use_graph)
        else:
            h.rk4_dev(d_orb.data_ptr(), d_cic.data_ptr(), t, dt, n, use_graph=use_graph)

    # ---- device-resident throughput: one trajectory from t0
    if args.prop == "rk4":
        h.rk4_reset(d_orb0.data_ptr(), d_cic0.data_ptr())
    else:
        h.rk4_reset(None, None)
    steps(t0, args.warmup)
    h.sync()
    t1 = t0 + args.warmup * dt
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    with Clocks(local) as clk:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(ext)
        steps(t1, args.steps)
        e1.record(ext)
        torch.cuda.synchronize()
    launches = h.launch_count()
    h.sync()
    sec = max_over_ranks(e0.elapsed_time(e1) / 1e3, dist if world > 1 else None, dev)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    value = job_throughput(world, args.steps, dt, sec)
    d_orb_end, d_cic_end = d_orb.clone(), d_cic.clone()  # the FP64 state at the end of the window
    wn = d_orb.cpu().numpy().reshape(len(wl["orbitals"]), -1)
    traj = {"t_start_au": t1, "t_end_au": t1 + args.steps * dt,
            "orbital_norm_dev": float(np.abs(np.linalg.norm(wn, axis=1) - 1.0).max()),
            "finite": bool(np.all(np.isfinite(wn)))}

    # ---- end to end through the public API (host buffers every step, the
    # host copy carrying the trajectory)
    h.rk4_reset(None, None)
    h_orb = torch.from_numpy(d_orb.cpu().numpy()).pin_memory()
    h_cic = torch.from_numpy(d_cic.cpu().numpy()).pin_memory()
    ke = args.e2e_steps or max(10, min(args.steps, 50))
    t2 = t1 + args.steps * dt

    def e2e_step(t):
        with torch.cuda.stream(ext):
            d_orb.copy_(h_orb, non_blocking=True)
            d_cic.copy_(h_cic, non_blocking=True)
        steps(t, 1)
        with torch.cuda.stream(ext):
            h_orb.copy_(d_orb, non_blocking=True)
            h_cic.copy_(d_cic, non_blocking=True)

    for s in range(3):
        e2e_step(t2 + s * dt)
    torch.cuda.synchronize()
    t2 += 3 * dt
    if world > 1:
        dist.barrier()
    e2 = torch.cuda.Event(enable_timing=True)
    e3 = torch.cuda.Event(enable_timing=True)
    w0 = time.perf_counter()
    e2.record(ext)
    for s in range(ke):
        e2e_step(t2 + s * dt)
    e3.record(ext)
    torch.cuda.synchronize()
    wall = time.perf_counter() - w0
    sec_e = max_over_ranks(max(e2.elapsed_time(e3) / 1e3, wall), dist if world > 1 else None, dev)
    e2e = job_throughput(world, ke, dt, sec_e)
    bytes_step = (h_orb.numel() + h_cic.numel()) * 16

    # ---- one-body half step alone (split2's clh1itr) at the |A| peak field
    h1_ms = None
    if args.prop == "split2":
        lf = gauge_field(wl, a_peak_time(wl))
        d_tmp = d_orb.clone()
        h.h1itr_dev(d_tmp.data_ptr(), lf, 0.5 * dt)
        reps = 20
        ncyc = 0
        w0 = time.perf_counter()
        for _ in range(reps):
            ncyc = h.h1itr_dev(d_tmp.data_ptr(), lf, 0.5 * dt)
        h1_ms = {"ms": (time.perf_counter() - w0) / reps * 1e3, "corrections": ncyc,
                 "note": "one clh1itr half step at the |A| peak, host-timed with its synchronisation"}
        del d_tmp

    # ---- phase profile and roofline of the dominant kernel
    d_hw = torch.empty_like(d_orb)
    d_hc = torch.empty_like(d_cic)
    d_orb.copy_(d_orb0)
    d_cic.copy_(d_cic0)
    torch.cuda.synchronize()
    lf = np.zeros(9)
    phases = h.profile(5, lf, d_orb.data_ptr(), d_cic.data_ptr(), d_hw.data_ptr(), d_hc.data_ptr())
    work = rhs_work(wl, d)
    if max(phases.values()) <= 0:
        raise RuntimeError("phase profile returned no timings: %r" % phases)
    dom = max(phases, key=lambda k: phases[k])
    fl, by = work.get(dom, (0, 0))
    hbm, hbm_src = measured_peaks()
    f64 = fp64_peak_tflops(torch)
    t_dom = phases[dom] / 1e3
    intensity = fl / max(by, 1)
    ridge = f64 * 1e12 / (hbm * 1e9)
    traffic = profiled_traffic(dom)
    if intensity > ridge:
        roof = {"bound": "tensor", "achieved": fl / t_dom / 1e12, "peak": f64, "unit": "TFLOP/s",
                "frac": fl / t_dom / 1e12 / f64, "traffic": traffic, "kernel": dom,
                "peak_source": "FP64: cuBLAS DGEMM 4096^3 measured in this run (B200 has no FP64 tcgen05 kind)"}
    else:
        roof = {"bound": "hbm", "achieved": by / t_dom / 1e9, "peak": hbm, "unit": "GB/s",
                "frac": by / t_dom / 1e9 / hbm, "traffic": traffic, "kernel": dom, "peak_source": hbm_src}

    # ---- the mixed-precision form (pair-density multipoles and pair potentials in split TF32 on the
    # tensor cores) over the same window: same start state, warm-up and timed steps; its deviation
    # from the FP64 trajectory at the end of the window, and of one RHS at the window's start
    mixed = None
    if not args.no_mixed:
        d_orb.copy_(d_orb0)
        d_cic.copy_(d_cic0)
        torch.cuda.synchronize()
        rhs_dev = h.mixed_selftest(d_orb.data_ptr(), d_cic.data_ptr(), gauge_field(wl, t0))
        h.set_mixed(True)
        if args.prop == "rk4":
            h.rk4_reset(d_orb0.data_ptr(), d_cic0.data_ptr())
        else:
            h.rk4_reset(None, None)
        steps(t0, args.warmup)
        h.sync()
        torch.cuda.synchronize()
        e4, e5 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e4.record(ext)
        steps(t1, args.steps)
        e5.record(ext)
        torch.cuda.synchronize()
        h.sync()
        sec_m = max_over_ranks(e4.elapsed_time(e5) / 1e3, dist if world > 1 else None, dev)
        h.set_mixed(False)
        dip_m = h.dipole_dev(d_orb.data_ptr(), d_cic.data_ptr())
        dip_p = h.dipole_dev(d_orb_end.data_ptr(), d_cic_end.data_ptr())
        nf = len(wl["orbitals"])
        nm = np.linalg.norm(d_orb.cpu().numpy().reshape(nf, -1), axis=1)
        npl = np.linalg.norm(d_orb_end.cpu().numpy().reshape(nf, -1), axis=1)
        vm = job_throughput(world, args.steps, dt, sec_m)
        mixed = {"value": vm, "unit": "fs/s", "ms_per_step": sec_m / args.steps * 1e3, "speedup_vs_fp64": vm / value,
                 "precision": "pair-density multipoles and pair potentials in split TF32 (tcgen05, FP32 accumulation); "
                              "all else FP64",
                 "dipole_dev_end_au": abs(dip_m - dip_p), "orbital_norm_dev_end": float(np.abs(nm - npl).max()),
                 "rhs_rel_dev": {"rho2": float(rhs_dev[0]), "W": float(rhs_dev[1]), "hwfn": float(rhs_dev[2])},
                 "window": "t0 + warm-up, then the timed steps (as the FP64 value); deviations at the window's end "
                           "against the FP64 trajectory"}

    h.final()
    if rank != 0:
        if world > 1:
            dist.destroy_process_group()
        return 0
    line = {
        "metric": metric_name(), "value": value, "unit": "fs/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": sec / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "c128",
        "data": ("synthetic: seeded orbitals/CI (Philox) relaxed in imaginary time, gauge phase of A(t0); one trajectory"
                 if args.prop != "rk4" else "synthetic: seeded orbitals/CI (Philox) relaxed; every step restarts"),
        "config": {"workload": wl["name"], "dt_au": dt, "precision": "fp64 (plain path)",
                   "prop": PROP_NOTE[args.prop], "rhs_per_step": RHS_PER_STEP[args.prop],
                   "window": "one trajectory from t0 (default the pulse onset, as tdse starts); warm-up steps first",
                   "relax": relax, "trajectory": traj, "lcic": d["lcic"], "nfun": len(wl["orbitals"]),
                   "l2": "working set per step > 126 MB L2 (pair fields 3 x 98 MB)", "parallelism": "replicas" if world > 1 else "1 GPU"},
        "e2e": {"value": e2e, "unit": "fs/s", "h2d_bytes_per_step": bytes_step, "d2h_bytes_per_step": bytes_step,
                "steps": ke},
        "gpu_launches": launches,
        "roofline": roof,
        "phases_ms_per_rhs": {k: round(v, 4) for k, v in phases.items()},
        "one_body_half_step": h1_ms,
        "clocks": clk.summary(),
        "mixed": mixed,
    }
    if world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(wl, dt, args.prop)
    print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
