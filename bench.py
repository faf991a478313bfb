#!/usr/bin/env python
"""Benchmark: fs of simulated time per second for the Ne TD-CASSCF RK4
propagation on B200, driven through the td1c_b200 C-ABI.

A step is one full RK4 step (clcrk, four RHS evaluations hprod_htot plus the
stage combinations and the absorbing mask) of the Ne TD-CASSCF workload
(1s frozen core + CAS(8e, 9o), FEDVR 60 x 21 points, rmax 120, lmax 47 /
94, velocity gauge, dt 0.004 au), FP64 complex arithmetic.  Full-H RK4 at
dt = 0.004 au lies outside RK4's stability region on this grid (the FEDVR
one-body spectrum reaches ~4e6 au), so every step restarts from the seeded
synthetic state (a device-to-device copy inside the timed region) and
performs the complete four-stage update on it; the field still advances with
the step time.

value  : fs/s with the state resident in HBM (one CUDA graph per step).
e2e    : fs/s through the public API with the state copied host->device
         before and device->host after every step (pinned host buffers).
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

AU2FS = 0.02418884254  # fs per atomic time unit (mod_const.F90:21)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="ne", choices=["ne", "he"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=0)
    return ap.parse_args()


def workload(name):
    from td1c_b200 import workloads as W
    return W.NE_CAS if name == "ne" else W.HE_TDHF


def pulse_mid(wl):
    freq = 1239.84190 / (wl["wlen"] * 27.2113845)
    return 0.5 * wl["numcyc"] * 2 * np.pi / freq


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


def cpu_baseline(wl, dt, max_seconds=60.0):
    """The oracle (C++/OpenMP restatement of the reference path) on the host
    cores: a bounded sample of whole RK4 steps of the same workload."""
    from oracle.oracle import Oracle
    from td1c_b200.wfn import seeded_orbitals, seeded_cic
    o = Oracle(wl)
    d = o.dims
    orb = seeded_orbitals(wl, o.get("xrad"), o.get("wrad"), o.get("mask"))
    cic = np.ones(d["lcic"], dtype=np.complex128) / np.sqrt(d["lcic"]) if d["nact"] else np.ones(1, dtype=np.complex128)
    o.set_wfn0(orb, cic)
    t0 = pulse_mid(wl)
    n, tot = 0, 0.0
    while True:
        ts = time.perf_counter()
        o.rk4(orb, cic, t0, dt, 1)
        tot += time.perf_counter() - ts
        n += 1
        if tot > max_seconds * 0.5 or n >= 3:
            break
    sec_per_step = tot / n
    return {"value": dt * AU2FS / sec_per_step, "unit": "fs/s", "cores": o.num_threads(), "kind": "port",
            "sample": "%d RK4 step(s) (%d RHS) of %s on the oracle, %.2f s/step" % (n, 4 * n, wl["name"], sec_per_step)}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from oracle.oracle import Oracle
    from td1c_b200.wfn import seeded_orbitals
    wl = workload(args.workload)
    dt = wl["dt"]
    o = Oracle(wl)
    d = o.dims
    orb = seeded_orbitals(wl, o.get("xrad"), o.get("wrad"), o.get("mask"))
    cic = np.ones(d["lcic"], dtype=np.complex128) / np.sqrt(d["lcic"]) if d["nact"] else np.ones(1, dtype=np.complex128)
    o.set_wfn0(orb, cic)
    t0 = pulse_mid(wl)
    ts = time.perf_counter()
    for _ in range(max(1, min(args.warmup, 1))):
        o.rk4(orb, cic, t0, dt, 1)
    t_step = time.perf_counter() - ts
    k = max(1, min(args.steps, int(120.0 / max(t_step, 1e-3))))
    ts = time.perf_counter()
    for _ in range(k):
        o.rk4(orb, cic, t0, dt, 1)
    el = time.perf_counter() - ts
    v = k * dt * AU2FS / el
    line = {"impl": "reference", "metric": metric_name(), "value": v, "unit": "fs/s", "n_gpus": args.gpus,
            "steps": k, "warmup": 1, "ms_per_step": el / k * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "c128", "data": "synthetic (seeded orbitals, every step from the seeded state)",
            "config": {"workload": wl["name"], "dt_au": dt, "precision": "fp64",
                       "note": "CPU restatement of the reference path (the Fortran/MKL reference does not build here)"},
            "cpu_baseline": {"value": v, "unit": "fs/s", "cores": o.num_threads(), "kind": "port",
                             "sample": "%d RK4 steps of %s (steps capped to bound the run time)" % (k, wl["name"])},
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


def metric_name():
    try:
        return json.load(open(os.path.join(ROOT, "BASELINE.json")))["metric"]
    except Exception:
        return "fs simulated/s"


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    import torch
    import torch.distributed as dist
    from td1c_b200 import basis
    from td1c_b200.hprod import HProd
    from td1c_b200.wfn import seeded_orbitals, seeded_cic
    from td1c_b200.workmodel import rhs_work

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    torch.cuda.set_device(local)
    wl = workload(args.workload)
    dt = wl["dt"]
    rad, ang = basis.build(wl)
    h = HProd(wl, rad, ang)
    d = h.dims
    tb = h.ci_tables()
    orb = seeded_orbitals(wl, rad["xrad"], rad["wrad"], rad["mask"], seed=wl.get("seed", 0) + rank)
    cic = seeded_cic(wl, d["lcic"], tb["stra"], tb["strb"], tb["detoff"], tb["afirst"], tb["acount"])
    h.set_wfn0(orb, cic)
    dev = torch.device("cuda", local)
    d_orb = torch.from_numpy(orb.reshape(-1).copy()).to(dev)
    d_cic = torch.from_numpy(cic.copy()).to(dev)
    d_orb0, d_cic0 = d_orb.clone(), d_cic.clone()
    t0 = pulse_mid(wl)
    ext = torch.cuda.ExternalStream(h.stream())
    torch.cuda.synchronize()

    # ---- device-resident throughput
    h.rk4_reset(d_orb0.data_ptr(), d_cic0.data_ptr())
    h.rk4_dev(d_orb.data_ptr(), d_cic.data_ptr(), t0, dt, args.warmup)
    h.sync()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    with Clocks(local) as clk:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(ext)
        h.rk4_dev(d_orb.data_ptr(), d_cic.data_ptr(), t0, dt, args.steps)
        e1.record(ext)
        torch.cuda.synchronize()
    launches = h.launch_count()
    h.sync()
    sec = e0.elapsed_time(e1) / 1e3
    if world > 1:
        t = torch.tensor([sec], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        sec = float(t.item())
        dist.barrier()
    torch.cuda.synchronize()
    value = world * args.steps * dt * AU2FS / sec

    # ---- end to end through the public API (host buffers every step)
    h.rk4_reset(None, None)
    h_orb = torch.from_numpy(orb.reshape(-1).copy()).pin_memory()
    h_cic = torch.from_numpy(cic.copy()).pin_memory()
    o_orb = torch.empty_like(h_orb).pin_memory()
    o_cic = torch.empty_like(h_cic).pin_memory()
    ke = args.e2e_steps or max(10, min(args.steps, 50))

    def e2e_step(s):
        with torch.cuda.stream(ext):
            d_orb.copy_(h_orb, non_blocking=True)
            d_cic.copy_(h_cic, non_blocking=True)
        h.rk4_dev(d_orb.data_ptr(), d_cic.data_ptr(), t0 + s * dt, dt, 1)
        with torch.cuda.stream(ext):
            o_orb.copy_(d_orb, non_blocking=True)
            o_cic.copy_(d_cic, non_blocking=True)

    for s in range(3):
        e2e_step(s)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    e2 = torch.cuda.Event(enable_timing=True)
    e3 = torch.cuda.Event(enable_timing=True)
    w0 = time.perf_counter()
    e2.record(ext)
    for s in range(ke):
        e2e_step(s)
    e3.record(ext)
    torch.cuda.synchronize()
    wall = time.perf_counter() - w0
    sec_e = max(e2.elapsed_time(e3) / 1e3, wall)
    if world > 1:
        t = torch.tensor([sec_e], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        sec_e = float(t.item())
    e2e = world * ke * dt * AU2FS / sec_e
    bytes_step = (h_orb.numel() + h_cic.numel()) * 16

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

    h.final()
    if rank != 0:
        if world > 1:
            dist.destroy_process_group()
        return 0
    line = {
        "metric": metric_name(), "value": value, "unit": "fs/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": sec / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "c128",
        "data": "synthetic: seeded orbitals/CI (Philox), every step restarts from the seeded state",
        "config": {"workload": wl["name"], "dt_au": dt, "precision": "fp64 (plain path)",
                   "rk": "RK4 full H (clcrk), mask each step", "lcic": d["lcic"], "nfun": len(wl["orbitals"]),
                   "l2": "working set per step > 126 MB L2 (pair fields 3 x 98 MB)", "parallelism": "replicas" if world > 1 else "1 GPU"},
        "e2e": {"value": e2e, "unit": "fs/s", "h2d_bytes_per_step": bytes_step, "d2h_bytes_per_step": bytes_step,
                "steps": ke},
        "gpu_launches": launches,
        "roofline": roof,
        "phases_ms_per_rhs": {k: round(v, 4) for k, v in phases.items()},
        "clocks": clk.summary(),
    }
    if world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(wl, dt)
    print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
