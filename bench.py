"""Benchmark: qasMHD per-step update in Mcell-updates/s (FP64) on B200.

Default workload (N=1): 3D low-Mach Kelvin-Helmholtz 256^3 (M = 0.01, beta = 100),
MLAU flux + characteristic WCNS4 + CUCT-weighted CT + SSP-RK3, CFL 0.4, dt refreshed
every 2nd step as in exec_ -- the largest single-GPU configuration of the benchmark set
and the one the throughput target of the plain FP64 path is stated on.  One "step" = one
full RK3 time step of the whole grid.
The timed region is K steps; it is timed `--windows` times and the median window is
the reported value.  Under torchrun (N>1) every rank advances its own independent
replica (the plain path is a single domain; replicas only), so per-GPU work is
fixed: weak scaling.

--impl reference runs the reference's own OpenMP code, compiled from its sources
(oracle/_ref), on the host's physical cores for the same workload and config.

Prints one JSON line (rank 0).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

ALG_BYTES_PER_CELL_UPDATE = 512  # 8 FP64 fields: stage 1 reads u^n, writes; stages 2-3 read stage input + u^n, write

# Algorithmic FP64 arrays per cell and launch of the kernels that can dominate a step
# (reads + writes, each array streamed once):
#   k_lr     reads ro,vn,vt,vu,bt,bu,pr, the centre normal field and the face normal field (9);
#            writes the 7+7 face states and the CUCT induction states (2 in 2D, 4 in 3D)
#   k_flux   reads the 7+7 face states, the face normal field, the induction states (2/4), vn
#            and the shock detector (MLAU/LHLLD: 1 in 2D, 2 in 3D); writes 8 fluxes and the
#            central induction fluxes (1 in 2D, 2 in 3D)
#   k_sweep  (face states + flux of one axis in one kernel, the 3D default) reads the 7 stencil
#            fields, the centre and face normal fields and the shock detector (1 in 2D, 2 in 3D,
#            MLAU/LHLLD); writes 7 fluxes and the central induction fluxes (1 in 2D, 2 in 3D):
#            the face states never leave the SM
KERNEL_ARRAYS = {
    "k_lr": {1: 8 + 14, 2: 9 + 16, 3: 9 + 18},
    "k_flux": {1: 15 + 8, 2: 14 + 1 + 2 + 2 + 8 + 1, 3: 14 + 1 + 4 + 3 + 8 + 2},
    "k_sweep": {1: 8 + 7, 2: 9 + 1 + 7 + 1, 3: 9 + 2 + 7 + 2},
}
# FP64 work per cell, counted by ncu (dadd + dmul + dfma instructions, and flops with a dfma
# counted 2): k_lr on the 2D Orszag-Tang 1024^2 workload (ODR=4; profiles/k_lr_ot2d_1024.md),
# k_sweep (MLAU) on KH 128^3 (profiles/k_sweep_kh3d_256.md: 1588-1604 per direction)
FP64_INSTR_PER_CELL = {"k_lr": 1054.0, "k_sweep": 1600.0}
FP64_FLOPS_PER_CELL = {"k_lr": 1262.0, "k_sweep": 1923.0}
# ncu dram__bytes_read.sum + dram__bytes_write.sum of one launch of the dominant kernel, per
# workload: k_lr (y faces) of OT 1024^2 (profiles/k_lr_ot2d_1024.md); for KH 3D the KH 128^3
# captures (136^3 padded cells: k_lr x faces 200.12 + 314.29 MB; k_sweep the mean of its x, y, z
# launches, 378.0 + 405.8 + 405.0 MB / 3) scaled by padded cells to 264^3 (traffic per cell is
# size-independent: every array is streamed once, the 126 MB L2 holds no full array)
KERNEL_TRAFFIC_PER_LAUNCH = {("k_lr", "ot2d_1024"): 76.70e6 + 92.25e6,
                             ("k_lr", "kh3d_256"): (200.12e6 + 314.29e6) * (264 / 136) ** 3,
                             ("k_sweep", "kh3d_256"): (378.0e6 + 405.8e6 + 405.0e6) / 3 * (264 / 136) ** 3}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--windows", type=int, default=5, help="timed windows of --steps steps; the median is reported")
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["kh3d_256", "ot2d_1024", "kh3d_128", "bw1d_1024"], default="kh3d_256")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-steps", type=int, default=None,
                    help="full RK3 steps of the reference's OpenMP build in cpu_baseline (default: 10 in 3D, 3 else)")
    ap.add_argument("--lr-staging", type=int, choices=[0, 1], default=None,
                    help="reconstruction stencils: 1 = TMA-staged in shared memory, 0 = global loads "
                         "(default: the library's default for the grid)")
    ap.add_argument("--fused-sweep", type=int, choices=[0, 1], default=None,
                    help="face states + flux of an axis in one kernel (1) or two (0); default: the library's")
    ap.add_argument("--e2e-steps", type=int, default=10)
    ap.add_argument("--no-ensemble", action="store_true")
    ap.add_argument("--ensemble-steps", type=int, default=200)
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--no-decomposed", action="store_true",
                    help="skip the slab-decomposition leg (KH 256^3 in 4 z-slabs on this GPU vs one domain)")
    ap.add_argument("--no-second", action="store_true",
                    help="skip the second plain workload (2D Orszag-Tang 1024^2 beside the 3D default)")
    ap.add_argument("--adjoint-only", action="store_true",
                    help="print only the adjoint comparison over --steps steps (profiling aid)")
    ap.add_argument("--ensemble-only", action="store_true",
                    help="print only the batched-ensemble comparison over --steps steps (profiling aid)")
    ap.add_argument("--lr-forms-case", action="store_true",
                    help="profiling aid: one eager exec_ step of Orszag-Tang 512^2 with the global-load "
                         "reconstruction, then one with the TMA-staged reconstruction; prints nothing timed")
    return ap.parse_args()


def lr_forms_case():
    from qasmhd_b200 import lib as L
    from qasmhd_b200 import problems as P
    p = P.orszag_tang(512)
    for st in (0, 1):
        with L.Context.from_problem(p) as ctx:
            ctx.set_option(L.QAS_OPT_LR_STAGING, st)
            ctx.upload(p.state)
            ctx.run(max_steps=1, flg=1, stop_rule=0, cfl=p.cfl, use_graph=False)
            ctx.download(p.state.shape)
    print(json.dumps({"lr_forms_case": "ok"}))


def make_problem(name, world=1):
    """The workload's problem and its config dict; both arms print the same dict."""
    from qasmhd_b200 import problems as P
    if name == "ot2d_1024":
        p = P.orszag_tang(1024)
        cfg = {"workload": "orszag_tang_2d_1024x1024", "grid": [1024, 1024], "solver": "HLLD", "order": "WCNS4",
               "rk": 3, "ct": "CUCT", "bc": "periodic", "gamma": "5/3"}
    elif name == "kh3d_128":  # a smaller case of the same workload, for profiler captures
        p = P.kelvin_helmholtz(3, 128)
        cfg = {"workload": "kelvin_helmholtz_3d_128^3", "grid": [128, 128, 128], "solver": "MLAU",
               "order": "WCNS4", "rk": 3, "ct": "CUCT", "bc": "periodic x,z / open y", "mach": 0.01, "beta": 100}
    elif name == "kh3d_256":
        p = P.kelvin_helmholtz(3, 256)
        cfg = {"workload": "kelvin_helmholtz_3d_256^3", "grid": [256, 256, 256], "solver": "MLAU",
               "order": "WCNS4", "rk": 3, "ct": "CUCT", "bc": "periodic x,z / open y", "mach": 0.01, "beta": 100}
    else:
        p = P.brio_wu(1024)
        cfg = {"workload": "brio_wu_1d_1024", "grid": [1024], "solver": "HLLD", "order": "WCNS4", "rk": 3}
    # working set of the plain path per step: 77 FP64 arrays of nd cells (state, ut, primitives,
    # face states, fluxes, EMFs), well above the 126 MB L2 for the 2D and 3D workloads
    cfg["parallelism"] = f"replicas{world}"
    cfg["l2"] = "no flush: working set per step ~%.2f GB > 126 MB L2" % (77 * p.nd * 8 / 1e9)
    return p, cfg


class ClockSampler:
    """SM clocks and clock-event (throttle) reasons sampled through NVML every few
    milliseconds during the timed region (read-only queries)."""

    def __init__(self, device_index: int, period_s: float = 0.005):
        self.dev = device_index
        self.period = period_s
        self.samples = []
        self.max_mhz = None
        self._stop = threading.Event()
        self.thread = None
        self.ok = False

    def start(self):
        try:
            import pynvml
            pynvml.nvmlInit()
            h = pynvml.nvmlDeviceGetHandleByIndex(self.dev)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM)
            self.ok = True
        except Exception:
            return

        def loop():
            while not self._stop.is_set():
                try:
                    sm = pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM)
                    rs = pynvml.nvmlDeviceGetCurrentClocksEventReasons(h)
                    self.samples.append((sm, rs))
                except Exception:
                    pass
                time.sleep(self.period)

        self.thread = threading.Thread(target=loop, daemon=True)
        self.thread.start()

    def stop(self):
        if not self.ok:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        self._stop.set()
        self.thread.join(timeout=2)
        import pynvml
        names = {"hw_slowdown": pynvml.nvmlClocksEventReasonHwSlowdown,
                 "hw_thermal_slowdown": pynvml.nvmlClocksEventReasonHwThermalSlowdown,
                 "sw_thermal_slowdown": pynvml.nvmlClocksEventReasonSwThermalSlowdown,
                 "sw_power_cap": pynvml.nvmlClocksEventReasonSwPowerCap}
        reasons = sorted({nm for _, rs in self.samples for nm, bit in names.items() if rs & bit})
        sm = [s for s, _ in self.samples]
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": self.max_mhz,
                "reasons": reasons, "samples": len(sm)}


def host_cpu() -> str:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def host_cores():
    """(logical CPUs this process may run on, distinct physical cores among them).  Physical
    cores are told apart by (package id, core id) from sysfs; without sysfs every logical CPU
    counts as a core."""
    try:
        cpus = sorted(os.sched_getaffinity(0))
    except (AttributeError, OSError):
        cpus = list(range(os.cpu_count() or 1))
    cores = set()
    for c in cpus:
        base = f"/sys/devices/system/cpu/cpu{c}/topology/"
        try:
            with open(base + "physical_package_id") as f:
                pk = f.read().strip()
            with open(base + "core_id") as f:
                co = f.read().strip()
            cores.add((pk, co))
        except OSError:
            cores.add(("cpu", str(c)))
    return len(cpus), len(cores)


def _cpu_run(prob, steps, exe=None):
    """Time `steps` full RK3 steps of the reference's OpenMP build on the host's physical
    cores (OMP_PROC_BIND=close, OMP_PLACES=cores); returns (median step s, threads, logical)."""
    from oracle import refcase as R
    logical, physical = host_cores()
    r = R.run_reference(prob, R.MODE_RUN, nsteps=steps, nthreads=physical, exe=exe, bind=True)
    st = r["step_times"]
    per = float(np.median(st)) if len(st) else r["elapsed"] / max(steps, 1)
    return per, physical, logical


def cpu_baseline(prob, steps):
    """The reference's own OpenMP code (oracle/_ref, -O2 -fopenmp) on a bounded sample of the
    workload: `steps` full RK3 steps, median step time."""
    from oracle import refcase as R
    if not R.reference_available(prob.dim, prob.ctw):
        return None
    per, threads, logical = _cpu_run(prob, steps)
    return {"value": prob.interior_cells / per / 1e6, "unit": "Mcell-updates/s", "cores": threads,
            "logical_cpus": logical, "kind": "reference", "cpu": host_cpu(),
            "sample": f"{prob.name}: {steps} full RK3 steps, median step time {per:.3f} s, reference -O2 "
                      f"-fopenmp, OMP_NUM_THREADS={threads} (physical cores) OMP_PROC_BIND=close OMP_PLACES=cores"}


def cpu_baseline_o3(prob, steps):
    """The same bounded sample through the reference built with its alternative flags
    (Makefile.inc:3, -O3 -march=native: here the host's x86-64 ISA level).  Timing only: FMA
    contraction changes its last bits."""
    from oracle import refcase as R
    exe = R.o3_binary(prob.dim)
    if exe is None:
        return None
    per, threads, logical = _cpu_run(prob, steps, exe=exe)
    return {"value": prob.interior_cells / per / 1e6, "unit": "Mcell-updates/s", "cores": threads,
            "logical_cpus": logical, "kind": "reference", "cpu": host_cpu(),
            "sample": f"{prob.name}: {steps} full RK3 steps, median step time {per:.3f} s, reference "
                      f"-O3 -march=x86-64-{R.host_isa_level()} -fopenmp, OMP_NUM_THREADS={threads} "
                      "OMP_PROC_BIND=close"}


def ensemble_compare(steps):
    """Batched ensemble (512 seeded 2D instances, log-uniform sides 64..512, half
    Orszag-Tang/HLLD, half Kelvin-Helmholtz/MLAU) in one launch sequence per step, against
    the same instances run one after another through the plain path: each with its own
    graph-captured exec_ loop for the same `steps` steps, and with eager launches over
    min(steps, 20) steps (per-step rate).  Device time by CUDA events."""
    import torch

    from qasmhd_b200 import lib as L
    from qasmhd_b200 import problems as P
    probs = P.ensemble(512)
    cells = sum(p.interior_cells for p in probs)
    b = L.Batch(probs)
    for q, p in enumerate(probs):
        b.upload(q, p.state)
    b.autotune(1)
    b.run(max_steps=2, flg=1, stop_rule=0, cfl=0.4)
    ext = torch.cuda.ExternalStream(b.stream())
    s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    l0 = b.kernel_launches()
    s0.record(ext)
    b.run(max_steps=steps, flg=1, stop_rule=0, cfl=0.4)
    s1.record(ext)
    s1.synchronize()
    ms_b = s0.elapsed_time(s1)
    launches_b = b.kernel_launches() - l0
    b.close()
    eager_steps = min(steps, 20)
    ms_p = {True: 0.0, False: 0.0}
    launches_p = 0
    for p in probs:
        with L.Context.from_problem(p) as c:
            for graph in (True, False):
                n = steps if graph else eager_steps
                c.upload(p.state)
                c.run_reset()
                c.run(max_steps=2, flg=1, stop_rule=0, cfl=0.4, use_graph=graph)
                ext = torch.cuda.ExternalStream(c.stream())
                s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                l0 = c.kernel_launches()
                s0.record(ext)
                c.run(max_steps=n, flg=1, stop_rule=0, cfl=0.4, use_graph=graph)
                s1.record(ext)
                s1.synchronize()
                ms_p[graph] += s0.elapsed_time(s1) / n
                if graph:
                    launches_p += c.kernel_launches() - l0
    ms_b_step = ms_b / steps
    return {"workload": "ensemble_512_2d_64-512_OT-HLLD_KH-MLAU", "instances": len(probs), "cells": cells,
            "steps": steps, "batched_mcells": cells / ms_b_step / 1e3,
            "per_instance_mcells": cells / ms_p[True] / 1e3, "ratio": ms_p[True] / ms_b_step,
            "per_instance_eager_mcells": cells / ms_p[False] / 1e3, "ratio_vs_eager": ms_p[False] / ms_b_step,
            "eager_steps": eager_steps, "batched_launches": launches_b, "per_instance_launches": launches_p,
            "basis": "ratio: per-instance runs each with its own graph-captured exec_ loop over the same steps (the "
                     "strict baseline); ratio_vs_eager: per-instance plain (eager) kernel launches, per-step rate"}


def second_workload(name, steps=20, warmup=3, windows=5, cpu_steps=3):
    """Another plain workload timed like the headline (graph-captured exec_ loop, median of
    `windows` windows of `steps` steps) beside the reference's OpenMP build on the host's
    physical cores, with its host round trip (qas_step_host, and the serial composition)."""
    import torch

    from qasmhd_b200 import lib as L
    prob, cfg = make_problem(name)
    with L.Context.from_problem(prob) as ctx:
        ctx.upload(prob.state)
        ctx.run(max_steps=warmup, flg=1, stop_rule=0, cfl=prob.cfl, use_graph=True)
        ext = torch.cuda.ExternalStream(ctx.stream())
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        wins = []
        for _ in range(windows):
            a.record(ext)
            ctx.run(max_steps=steps, flg=1, stop_rule=0, cfl=prob.cfl, use_graph=True)
            b.record(ext)
            b.synchronize()
            wins.append(a.elapsed_time(b) / steps)
        ms = statistics.median(wins)
        prof = ctx.profile(min(steps, 10), flg=1, cfl=prob.cfl)
        host = torch.empty((8, prob.nd), dtype=torch.float64, pin_memory=True)
        ctx.download_into(host.numpy())
        hptr = host.numpy()

        def e2e_ms(fn, n):
            for _ in range(3):
                fn()
            torch.cuda.synchronize()
            a.record(ext)
            for _ in range(n):
                fn()
            b.record(ext)
            b.synchronize()
            return a.elapsed_time(b) / n

        def serial_step():
            ctx.upload(hptr)
            ctx.run(max_steps=1, flg=1, stop_rule=0, cfl=prob.cfl, use_graph=False)
            ctx.download_into(hptr)

        ms_serial = e2e_ms(serial_step, 5)
        ms_host = e2e_ms(lambda: ctx.step_host(hptr, hptr, flg=1, stop_rule=0, cfl=prob.cfl), 5)
        del host
    gpu = prob.interior_cells / (ms * 1e-3) / 1e6
    cpu = cpu_baseline(prob, cpu_steps) if cpu_steps > 0 else None
    cpu3 = cpu_baseline_o3(prob, cpu_steps) if cpu_steps > 0 else None
    out = {"workload": cfg["workload"], "config": cfg, "value": gpu, "unit": "Mcell-updates/s",
           "ms_per_step": ms, "steps": steps, "windows_ms_per_step": wins,
           "kernels_ms_per_launch": {k: round(v[1] / v[0], 4) for k, v in prof.items()},
           "cpu_baseline": cpu, "cpu_baseline_o3": cpu3,
           "e2e": {"value": prob.interior_cells / (ms_host * 1e-3) / 1e6, "unit": "Mcell-updates/s",
                   "ms_per_step": ms_host, "h2d_bytes_per_step": 64 * prob.nd, "d2h_bytes_per_step": 64 * prob.nd,
                   "api": "qas_step_host"},
           "e2e_serial": {"value": prob.interior_cells / (ms_serial * 1e-3) / 1e6, "unit": "Mcell-updates/s",
                          "ms_per_step": ms_serial},
           "step_roofline": {"achieved": ALG_BYTES_PER_CELL_UPDATE * prob.interior_cells / (ms * 1e-3) / 1e9,
                             "unit": "GB/s", "basis": "512 algorithmic B per cell-update"}}
    if cpu:
        out["ratio_vs_cpu"] = gpu / cpu["value"]
    if cpu3:
        out["ratio_vs_cpu_o3"] = gpu / cpu3["value"]
    return out


def decomposed_compare(nparts=4, steps=6):
    """KH 256^3 split into z-slabs (qas_dd_*: ghost-plane copies after each fill, primitive pass
    and shock detector; gathered CFL maximum) on this one GPU, against the single domain, both
    eager (no graph), wall time around the run call with a device synchronise on both sides:
    the cost of the exchanges themselves, which on several GPUs become NVLink peer copies."""
    import torch

    from qasmhd_b200 import lib as L
    from qasmhd_b200 import problems as P
    prob = P.kelvin_helmholtz(3, 256)
    out = {"workload": "kelvin_helmholtz_3d_256^3", "nparts": nparts, "steps": steps, "timing": "host wall, synced"}
    with L.Context.from_problem(prob) as ctx:
        ctx.upload(prob.state)
        ctx.run(max_steps=2, flg=1, stop_rule=0, cfl=prob.cfl, use_graph=False)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ctx.run(max_steps=steps, flg=1, stop_rule=0, cfl=prob.cfl, use_graph=False)
        torch.cuda.synchronize()
        single = (time.perf_counter() - t0) / steps
    with L.Decomposition(prob, nparts) as dd:
        dd.upload(prob.state)
        dd.run(max_steps=2, flg=1, stop_rule=0, cfl=prob.cfl)
        torch.cuda.synchronize()
        k0, c0 = dd.kernel_launches()
        t0 = time.perf_counter()
        dd.run(max_steps=steps, flg=1, stop_rule=0, cfl=prob.cfl)
        torch.cuda.synchronize()
        split = (time.perf_counter() - t0) / steps
        k1, c1 = dd.kernel_launches()
    out.update({"single_ms_per_step": 1e3 * single, "split_ms_per_step": 1e3 * split,
                "overhead": split / single - 1.0, "copies_per_step": (c1 - c0) / steps,
                "split_mcells": prob.interior_cells / split / 1e6})
    return out


def adjoint_compare(nsteps=400, every=20, eta=0.5e-4):
    """Discrete adjoint of the 2D Kelvin-Helmholtz step (256^2, M = 0.1, Roe + WCNS4 + CT,
    RK3, uniform eta, checkpoints every `every` steps) against the plain forward path over
    the same steps (graph-captured exec_ loop with the same resistive sub-cycles).  Device
    time by CUDA events on the context's stream; dt sequence frozen from a first run."""
    import torch

    from qasmhd_b200 import lib as L
    from qasmhd_b200.adjoint import cfl_dts
    from qasmhd_b200.problems import RMN_ROE, kelvin_helmholtz
    prob = kelvin_helmholtz(dim=2, n=256, mach=0.1, rmn=RMN_ROE, odr=4, rk=3, ctw=1)
    u0 = prob.state.reshape(8, -1).copy()
    with L.Context.from_problem(prob) as ctx:
        dts = cfl_dts(ctx, u0, nsteps, prob.cfl, eta)
        ext = torch.cuda.ExternalStream(ctx.stream())

        def timed(f):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(ext)
            f()
            e1.record(ext)
            e1.synchronize()
            return e0.elapsed_time(e1)

        g = np.random.default_rng(1).standard_normal(u0.shape) * 1e-3
        for rep in range(2):  # first pass warms graphs and allocations
            ctx.upload(u0)
            ctx.run_reset()
            ms_f = timed(lambda: ctx.run(max_steps=nsteps, flg=1, stop_rule=0, cfl=prob.cfl, use_graph=True,
                                         eta0=eta))
            ctx.upload(u0)
            ms_af = timed(lambda: ctx.adjoint_forward(dts, eta, every))
            ms_b = timed(lambda: ctx.adjoint_backward(g))
    return {"workload": "kh2d_256_M0.1_roe_wcns4_ct_rk3_eta5e-5", "steps": nsteps, "ckpt_every": every,
            "forward_ms_per_step": ms_f / nsteps, "adjoint_forward_ms_per_step": ms_af / nsteps,
            "backward_ms_per_step": ms_b / nsteps, "ratio": ms_b / ms_f,
            "ratio_with_checkpointed_forward": (ms_af + ms_b) / ms_f,
            "basis": f"ratio = backward (segment recompute with tape + reverse sweep) / plain forward of the "
                     f"same {nsteps} steps; gradients checked against the reference's dual-number derivative"}


def run_reference_arm(args):
    """The reference's own OpenMP build (oracle/_ref, -O2 -fopenmp, its default flags) on the
    host's physical cores, W + K full steps of the same workload; rank 0 only."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    prob, cfg = make_problem(args.workload, world)
    if rank != 0:
        return
    from oracle import refcase as R
    if not R.reference_available(prob.dim, prob.ctw):
        print(json.dumps({"impl": "reference", "unavailable": "reference oracle binaries (oracle/_ref) not built"}))
        return
    logical, threads = host_cores()
    r = R.run_reference(prob, R.MODE_RUN, nsteps=args.warmup + args.steps, nthreads=threads, bind=True)
    st = r["step_times"][args.warmup:]
    total = float(np.sum(st))
    value = prob.interior_cells * len(st) / total / 1e6
    line = {"metric": "Mcell-updates/s/GPU FP64 (per-step update)", "value": value, "unit": "Mcell-updates/s",
            "impl": "reference", "n_gpus": args.gpus, "steps": len(st), "warmup": args.warmup,
            "ms_per_step": 1e3 * total / len(st), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded initial state of the named problem)",
            "config": cfg,
            "cpu_baseline": {"value": value, "unit": "Mcell-updates/s", "cores": threads, "logical_cpus": logical,
                             "kind": "reference", "cpu": host_cpu(),
                             "sample": f"{prob.name}: {args.warmup}+{len(st)} full RK3 steps, reference -O2 -fopenmp, "
                                       f"OMP_NUM_THREADS={threads} (physical cores) OMP_PROC_BIND=close"},
            "e2e": {"value": value, "unit": "Mcell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    exe = R.o3_binary(prob.dim)
    if exe:  # a few steps through the reference's alternative -O3 -march=native flags
        n3 = min(args.steps, 3)
        r3 = R.run_reference(prob, R.MODE_RUN, nsteps=1 + n3, nthreads=threads, exe=exe, bind=True)
        st3 = r3["step_times"][1:]
        line["o3_native"] = {"value": prob.interior_cells * len(st3) / float(np.sum(st3)) / 1e6,
                             "unit": "Mcell-updates/s", "cores": threads, "steps": len(st3),
                             "build": f"-O3 -march=x86-64-{R.host_isa_level()} -fopenmp (timing only)"}
    print(json.dumps(line))


def main():
    args = parse()
    if args.impl == "reference":
        run_reference_arm(args)
        return
    import torch
    import torch.distributed as dist

    from qasmhd_b200 import lib as L

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if args.lr_forms_case:
        if rank == 0:
            lr_forms_case()
        return
    if args.adjoint_only or args.ensemble_only:
        if rank == 0:
            out = {}
            if args.adjoint_only:
                out["adjoint"] = adjoint_compare(nsteps=args.steps)
            if args.ensemble_only:
                out["batched"] = ensemble_compare(args.steps)
            print(json.dumps(out))
        return
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))

    prob, cfg = make_problem(args.workload, world)
    cells = prob.interior_cells
    ctx = L.Context.from_problem(prob, device=local)
    if args.lr_staging is not None:
        ctx.set_option(L.QAS_OPT_LR_STAGING, args.lr_staging)
    if args.fused_sweep is not None:
        ctx.set_option(L.QAS_OPT_FUSED_SWEEP, args.fused_sweep)
    ctx.upload(prob.state)
    ext = torch.cuda.ExternalStream(ctx.stream(), device=torch.device("cuda", local))

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    # warm-up (includes setdt(1) and the graph capture)
    ctx.run(max_steps=args.warmup, flg=1, stop_rule=0, cfl=prob.cfl, use_graph=True)
    barrier()
    clocks = ClockSampler(local)
    clocks.start()
    windows = []
    launches = 0
    for _ in range(max(1, args.windows)):
        barrier()
        l0 = ctx.kernel_launches()
        start = torch.cuda.Event(enable_timing=True)
        end = torch.cuda.Event(enable_timing=True)
        start.record(ext)
        ctx.run(max_steps=args.steps, flg=1, stop_rule=0, cfl=prob.cfl, use_graph=True)
        end.record(ext)
        end.synchronize()
        barrier()
        launches = ctx.kernel_launches() - l0
        t = torch.tensor([start.elapsed_time(end)], device="cuda")
        if world > 1:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        windows.append(float(t.item()))
    clk = clocks.stop()
    ms_max = statistics.median(windows)
    ms_step = ms_max / args.steps
    value = cells * args.steps * world / (ms_max * 1e-3) / 1e6

    # end-to-end through the public API with pinned host buffers: every step uploads the
    # state, advances one exec_ step and downloads the state (the drop-in for ideal() on
    # host arrays).  qas_step_host overlaps the copies with the kernels; the serial
    # composition (qas_upload_block + qas_run + qas_download_block) is timed beside it.
    host = torch.empty((8, prob.nd), dtype=torch.float64, pin_memory=True)
    host.copy_(torch.from_numpy(np.ascontiguousarray(prob.state).reshape(8, -1)))
    hptr = host.numpy()
    nb = hptr.nbytes

    def e2e_time(step_fn):
        for _ in range(3):  # warm-up: the first calls capture the step's graphs
            step_fn()
        torch.cuda.synchronize()
        barrier()
        e_start = torch.cuda.Event(enable_timing=True)
        e_end = torch.cuda.Event(enable_timing=True)
        e_start.record(ext)
        for _ in range(args.e2e_steps):
            step_fn()
        e_end.record(ext)
        e_end.synchronize()
        barrier()
        te = torch.tensor([e_start.elapsed_time(e_end)], device="cuda")
        if world > 1:
            dist.all_reduce(te, op=dist.ReduceOp.MAX)
        return cells * args.e2e_steps * world / (float(te.item()) * 1e-3) / 1e6

    def serial_step():
        ctx.upload(hptr)
        ctx.run(max_steps=1, flg=1, stop_rule=0, cfl=prob.cfl, use_graph=False)
        ctx.download_into(hptr)

    e_serial = e2e_time(serial_step)
    e_value = e2e_time(lambda: ctx.step_host(hptr, hptr, flg=1, stop_rule=0, cfl=prob.cfl))

    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    hbm_peak = peaks.get("hbm_gbs", 6650.0)
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
    step_gbs = ALG_BYTES_PER_CELL_UPDATE * cells / (ms_step * 1e-3) / 1e9

    # dominant kernel, timed live with CUDA events on the context's stream over
    # min(K, 10) eager steps after the timed region
    prof = ctx.profile(min(args.steps, 10), flg=1, cfl=prob.cfl)
    dom = max(prof, key=lambda k: prof[k][1])
    dom_launches, dom_ms = prof[dom]
    dom_ms_launch = dom_ms / dom_launches
    step_prof_ms = sum(v[1] for v in prof.values())
    dom_cells = prob.nd  # the face kernels cover every cell but two ghost layers per side along their axis
    arrays = KERNEL_ARRAYS.get(dom, {}).get(prob.dim)
    achieved = arrays * 8.0 * dom_cells / (dom_ms_launch * 1e-3) / 1e9 if arrays else None
    line = {
        "metric": "Mcell-updates/s/GPU FP64 (per-step update)", "value": value, "unit": "Mcell-updates/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
        "windows": len(windows), "windows_ms": windows, "timing": "median of the timed windows of K steps",
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded initial state of the named problem)",
        "config": cfg,
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                     "frac": (achieved / hbm_peak) if achieved else None,
                     "traffic": KERNEL_TRAFFIC_PER_LAUNCH.get((dom, args.workload)),
                     "launch_ms": dom_ms_launch, "share_of_step": dom_ms / step_prof_ms,
                     "basis": f"algorithmic {arrays} FP64 arrays per cell per launch x {dom_cells} cells / live "
                              f"CUDA-event launch time; peak of {peak_src}; traffic = ncu dram read+write "
                              "per launch"},
        "step_roofline": {"achieved": step_gbs, "peak": hbm_peak, "unit": "GB/s", "frac": step_gbs / hbm_peak,
                          "basis": "whole step, 512 algorithmic B per cell-update"},
        "kernels_ms_per_launch": {k: round(v[1] / v[0], 4) for k, v in prof.items()},
        "e2e": {"value": e_value, "unit": "Mcell-updates/s", "h2d_bytes_per_step": nb, "d2h_bytes_per_step": nb,
                "api": "qas_step_host (copies overlapped with the kernels by items of planes)"},
        "e2e_serial": {"value": e_serial, "unit": "Mcell-updates/s",
                       "api": "qas_upload_block + qas_run(1 step) + qas_download_block"},
        "gpu_launches": launches,
        "gpu_launches_basis": "kernel launches of one timed window of K steps",
        "clocks": clk,
    }
    if dom in FP64_INSTR_PER_CELL:
        # the dominant kernel is FP64-bound: its FP64 rate against the measured DFMA peak
        fp64_peak = L.fp64_peak_tflops()
        tflops = FP64_FLOPS_PER_CELL[dom] * prob.nd / (dom_ms_launch * 1e-3) / 1e12
        pipe = FP64_INSTR_PER_CELL[dom] * prob.nd / (dom_ms_launch * 1e-3) / (fp64_peak * 1e12 / 2.0)
        line["fp64"] = {"kernel": dom, "achieved_tflops": tflops, "peak_tflops": fp64_peak,
                        "frac": tflops / fp64_peak, "pipe_frac": pipe,
                        "basis": "ncu-counted FP64 flops per cell x cells / live launch time; peak = measured DFMA "
                                 "throughput (qas_fp64_peak); pipe_frac = FP64 instructions vs the DFMA issue rate"}
    if rank == 0 and not args.no_cpu_baseline and world == 1:
        steps_cpu = args.cpu_steps if args.cpu_steps is not None else (10 if prob.dim == 3 else 3)
        line["cpu_baseline"] = cpu_baseline(prob, steps_cpu)
        line["cpu_baseline_o3"] = cpu_baseline_o3(prob, max(2, steps_cpu // 2))
        if line["cpu_baseline"]:
            line["ratio_vs_cpu"] = value / line["cpu_baseline"]["value"]
            line["e2e"]["ratio_vs_cpu"] = e_value / line["cpu_baseline"]["value"]
    ctx.close()
    if rank == 0 and not args.no_second and world == 1:
        other = "ot2d_1024" if args.workload != "ot2d_1024" else "kh3d_256"
        line["second"] = second_workload(other, cpu_steps=0 if args.no_cpu_baseline else 3)
    if rank == 0 and not args.no_ensemble and world == 1:
        line["batched"] = ensemble_compare(args.ensemble_steps)
    if rank == 0 and not args.no_adjoint and world == 1:
        line["adjoint"] = adjoint_compare()
    if rank == 0 and not args.no_decomposed and world == 1:
        line["decomposed"] = decomposed_compare()
    if world > 1:
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line))


if __name__ == "__main__":
    main()
