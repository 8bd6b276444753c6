"""Benchmark: arrested-Newton-flow relaxation throughput of a 4096^2 chiral magnet.

Workload (one "step" = one full RK4 arrested-Newton-flow step of the whole lattice):
chiral magnet, 4096 x 4096 sites over a 128 x 128 reduced domain (lsx = 128/4095),
J = 40e-12, K = 0.8e6, D = 4e-3, M = 580e3, B = 0.2 T, Heusler DMI, demag on (psi
relaxed as the 4th field), unit magnetisation, arrested Newton flow (killkinen on), FP32
fields with FP64 energy reductions.  (Without the arrest the demag saddle's dynamics is
unstable: longitudinal magnetisation and psi modes grow at ~sqrt(coup_mu)/2 per unit time,
and the energy of this lattice runs from 1.0e3 to -2.0e7 within 2000 steps; the step's
cost does not depend on the arrest.)  Initial field: 64 anti-skyrmions at
seeded jittered 8 x 8 lattice positions plus N(0, 1e-3) noise (synthetic; the
reference has no dataset).

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]

Under torchrun each rank relaxes its own lattice (independent replicas, no
data-path collective: weak scaling); the step time is the max over ranks.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import json
import math
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

XLEN = YLEN = 4096
XSIZE = 128.0
METRIC = "Mpoint-updates/s per flow step at dE/E<=1e-6 vs plain FP64; achieved HBM GB/s"
UNIT = "Mpoint-updates/s"
# words of nf components moved per site and step: S1 2 (phi in, l1 out), S2 3, S3 7
# (phi, V, l1, l2 in; T4, cV, cP out), S4 5 (T4, cP, cV in; phi', V' out) as four
# kernels; S1 2, S2+S3 fused 6, S4 5 when stages 2 and 3 run as one kernel
WORDS_SEPARATE, WORDS_FUSED = 17, 13
# end to end: one host->device load of the field and velocity, E2E_CALLS one-step
# Simulation.step calls (each returns E and err to the host), one device->host read-back
E2E_CALLS = 100


def chiral_params(xlen=None, ylen=None, xsize=None):
    from soliton_solver_b200.theories import load_theory
    xlen, ylen, xsize = xlen or XLEN, ylen or YLEN, xsize or XSIZE
    th = load_theory("Chiral magnet")
    p = th.params.default_params(xlen=xlen, ylen=ylen, xsize=xsize, ysize=xsize * (ylen - 1) / (xlen - 1) if xlen > 1
                                 else xsize, J=40e-12, K=0.8e6, D=4e-3, M=580e3, B=0.2, dmi_term="Heusler",
                                 demag=True, unit_magnetization=True, killkinen=True)
    return th, p


def config(extra=None):
    c = {"workload": "chiral magnet 4096x4096, Heusler DMI, demag on, B=0.2 T, 64-skyrmion lattice, arrested RK4 Newton flow",
         "theory": "Chiral magnet", "xlen": XLEN, "ylen": YLEN, "nf": 4, "fields": "fp32", "reductions": "fp64",
         "l2": "no flush: working set 1.6 GB per step >> 126 MB L2"}
    if extra:
        c.update(extra)
    return c


# ---------------------------------------------------------------------------
# clocks sampled during the timed region
# ---------------------------------------------------------------------------
class Clocks:
    """SM clock, power and clock-event reasons of this rank's GPU, sampled while the
    benchmark runs; summary() keeps the samples between the first and last mark() (the
    timed region).  NVML is polled every millisecond from a thread (the timed region of a
    short run lasts ~15 ms); without NVML, nvidia-smi samples every 20 ms.  Raw samples go
    to SS_BENCH_CLOCKS_DIR when set."""

    Q = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.thread = None
        self.samples = []  # (time, sm MHz, max sm MHz, power W, set of reasons)
        self.marks = []
        out = os.environ.get("SS_BENCH_CLOCKS_DIR") or tempfile.gettempdir()
        self.path = os.path.join(out, f"clocks_gpu{index}.csv")

    def _nvml_handle(self, nv):
        """NVML handle of the CUDA device `index` (matched by UUID: CUDA_VISIBLE_DEVICES
        may renumber), else NVML's device `index`."""
        try:
            import torch
            want = str(torch.cuda.get_device_properties(self.index).uuid).lower()
            for i in range(nv.nvmlDeviceGetCount()):
                h = nv.nvmlDeviceGetHandleByIndex(i)
                u = nv.nvmlDeviceGetUUID(h)
                u = (u.decode() if isinstance(u, bytes) else u).lower()
                if want and want in u:
                    return h
        except Exception:
            pass
        return nv.nvmlDeviceGetHandleByIndex(self.index)

    def _poll(self, nv, h, stop):
        bits = [nv.nvmlClocksEventReasonHwSlowdown, nv.nvmlClocksEventReasonHwThermalSlowdown,
                nv.nvmlClocksEventReasonSwThermalSlowdown, nv.nvmlClocksEventReasonSwPowerCap]
        smax = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
        while not stop.is_set():
            try:
                t = time.time()
                sm = float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM))
                pw = nv.nvmlDeviceGetPowerUsage(h) / 1000.0
                rs = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                self.samples.append((t, sm, smax, pw, {n for n, b in zip(self.NAMES, bits) if rs & b}))
            except Exception:
                break
            stop.wait(0.001)

    def __enter__(self):
        import threading
        try:
            import pynvml as nv
            nv.nvmlInit()
            h = self._nvml_handle(nv)
            self._stop = threading.Event()
            self.thread = threading.Thread(target=self._poll, args=(nv, h, self._stop), daemon=True)
            self.thread.start()
            return self
        except Exception:
            self.thread = None
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "20"], stdout=self.fh,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def mark(self):
        """Record the wall time of a timed-region boundary."""
        self.marks.append(time.time())

    def __exit__(self, *a):
        if self.thread is not None:
            self._stop.set()
            self.thread.join(timeout=5)
            if os.environ.get("SS_BENCH_CLOCKS_DIR"):
                os.makedirs(os.path.dirname(self.path), exist_ok=True)
                with open(self.path, "w") as fh:
                    for t, sm, smax, pw, rs in self.samples:
                        fh.write(f"{t:.6f},{sm:.0f},{smax:.0f},{pw:.1f},{'|'.join(sorted(rs))}\n")
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.fh.close()

    def _smi_samples(self):
        import datetime
        out = []
        for line in open(self.path).read().strip().splitlines():
            r = [x.strip() for x in line.split(",")]
            if len(r) < 10:
                continue
            try:
                t = datetime.datetime.strptime(r[0], "%Y/%m/%d %H:%M:%S.%f").timestamp()
                out.append((t, float(r[2]), float(r[3]), float(r[4]),
                            {n for n, v in zip(self.NAMES, r[6:10]) if v.lower() == "active"}))
            except ValueError:
                continue
        return out

    def summary(self):
        if self.thread is not None:
            samples, source = self.samples, "nvml, 1 ms"
        elif self.proc is not None and os.path.exists(self.path):
            samples, source = self._smi_samples(), "nvidia-smi, 20 ms"
        else:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["clock sampling unavailable"]}
        lo, hi = (self.marks[0], self.marks[-1]) if len(self.marks) >= 2 else (-math.inf, math.inf)
        sel = [x for x in samples if lo <= x[0] <= hi]
        reasons = set().union(*[x[4] for x in sel]) if sel else set()
        return {"sm_mhz": float(np.median([x[1] for x in sel])) if sel else None,
                "sm_max_mhz": max(x[2] for x in sel) if sel else None,
                "power_w_max": max(x[3] for x in sel) if sel else None, "reasons": sorted(reasons),
                "samples": len(sel), "source": source}


# ---------------------------------------------------------------------------
# CPU leg: the FP64 oracle on bounded stripes, one thread per stripe
# ---------------------------------------------------------------------------
def cpu_sample(steps, warmup, threads=None, rows=128):
    """Time the oracle's flow step on ``threads`` independent rows x 4096 stripes of the
    workload (each a Dirichlet sub-lattice with the workload's spacing); returns
    point-updates/s and a description."""
    from oracle import flow64 as ref
    from soliton_solver_b200.initial_conditions import skyrmion_lattice
    threads = threads or min(os.cpu_count() or 1, 16)
    th, p = chiral_params(rows, YLEN, XSIZE * (rows - 1) / (XLEN - 1))
    p = p.with_(ysize=XSIZE)
    rp = p.resolved()
    p_i, p_f = th.params.pack_device_params(rp)
    F0 = skyrmion_lattice(rp, n=1, R=1.0, seed=0).numpy().reshape(4, rows, YLEN)
    V0 = np.zeros_like(F0)

    def run(n):
        F, V = F0.copy(), V0.copy()
        ref.relax("chiral_magnet", F, V, 1e300, p_i, p_f, n)

    with cf.ThreadPoolExecutor(threads) as ex:
        for _ in range(warmup):
            list(ex.map(run, [1] * threads))
        t = time.perf_counter()
        for _ in range(steps):
            list(ex.map(run, [1] * threads))
        dt = (time.perf_counter() - t) / max(steps, 1)
    value = threads * rows * YLEN / dt / 1e6
    sample = (f"{threads} independent {rows}x{YLEN} stripes of the workload (FP64 numpy oracle restating the "
              f"reference kernels), 1 flow step each per timed step")
    return value, threads, sample, dt


def reference_sample(steps, warmup, n=16):
    """The reference's own flow step (baseline/_ref under Numba's CUDA simulator) on
    independent n x n sub-lattices of the workload, one process per core; falls back
    to the oracle port when the reference is not installed.  Returns (value, cores,
    kind, sample, seconds per step)."""
    sys.path.insert(0, os.path.join(ROOT, "baseline"))
    import reference_runner as rr
    why = rr.available()
    if why is None:
        pts, procs, dt, _ = rr.time_flow_steps(n=n, spacing=XSIZE / (XLEN - 1), steps=steps, warmup=warmup)
        value = pts / 1e6  # point-updates/s -> the metric's Mpoint-updates/s
        sample = (f"{procs} independent processes (one core each), each the reference's Simulation.step (FP64 "
                  f"Numba kernels under NUMBA_ENABLE_CUDASIM=1, soliton_solver 1.1.1 from baseline/_ref) on a "
                  f"{n}x{n} sub-lattice of the workload (same couplings and spacing, Heusler, demag on, B=0.2 T; "
                  f"the reference's ground state + N(0,1e-3) noise); {steps} timed steps after {warmup} warm-up")
        return value, procs, "reference", sample, dt
    value, threads, sample, dt = cpu_sample(steps, warmup)
    return value, threads, "port", f"{sample} (reference unavailable: {why})", dt


def reference_arm(args, rank, world):
    if rank != 0:
        return 0
    # each step of the simulator costs ~5 s per 16x16 sample: a bounded number of them
    steps, warmup = min(max(args.steps, 1), 4), min(max(args.warmup, 0), 1)
    value, cores, kind, sample, dt = reference_sample(steps, warmup)
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": steps,
            "warmup": warmup, "ms_per_step": dt * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
            "config": config({"sample": sample}),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": kind, "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------
def gpu_arm(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist
    from soliton_solver_b200.core.simulation import Simulation
    from soliton_solver_b200.initial_conditions import skyrmion_lattice

    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    th, p = chiral_params()
    sim = Simulation(p, th, precision="fp32", device=dev)
    F0 = skyrmion_lattice(sim.rp, n=8, R=1.0, seed=1000 + rank, device=dev)
    sim.load_field(F0)
    s = sim.solver
    stream = torch.cuda.current_stream(dev)
    N = XLEN * YLEN
    K, W = args.steps, args.warmup

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(x):
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    E_traj = torch.empty(K, dtype=torch.float64, device=dev)
    err_traj = torch.empty(K, dtype=torch.float64, device=dev)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    tuning = s.autotune(5)
    if args.variants:
        # pinned staging variants (S1..S4), e.g. to profile the set a normal run picks
        for m, v in enumerate(args.variants.split(","), start=1):
            s.set_variant(m, int(v))
        tuning = {m: (a, b, s._lib.ss_get_variant(s._h, m)) for m, (a, b, _) in tuning.items()}
    with Clocks(local_rank) as clk:
        # warm-up (untimed); also gives the clock sampler time to start
        s.step(max(W, 1), 1e300)
        time.sleep(0.5)
        barrier()
        torch.cuda.synchronize(dev)
        clk.mark()
        ev0.record(stream)
        s.step_async(K, math.nan, E_traj, err_traj)
        ev1.record(stream)
        torch.cuda.synchronize(dev)
        clk.mark()
    s.check_status()
    barrier()
    ms = max_over_ranks(ev0.elapsed_time(ev1))
    ms_step = ms / K
    value = world * N * K / (ms / 1e3) / 1e6
    # stage launches per step, then the call's trailing energy pass and finish kernel
    launches = (3 if (s.tma_enabled and s._lib.ss_get_variant(s._h, 6) == 1) else 4) * K + 2

    # roofline of the stage kernels (3 launches per step with stages 2 and 3 fused, else 4)
    from soliton_solver_b200._native import load as _load  # noqa: F401 (library loaded)
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    peak = float(peaks.get("hbm_gbs", 6650.0))
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
    fused = s.tma_enabled and s._lib.ss_get_variant(s._h, 6) == 1
    words = WORDS_FUSED if fused else WORDS_SEPARATE
    bytes_step = words * 4 * 4 * N
    achieved = bytes_step / (ms_step / 1e3) / 1e9
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "flow_kernel_traffic.json")
    if os.path.exists(tpath):
        try:
            traffic = json.load(open(tpath)).get("bytes_per_launch_at_4096")
        except Exception:
            traffic = None

    # end to end through the reference-facing API: host field in (pinned), one
    # Simulation.step(E) per step returning (E, err) to the host, host field out.
    host_F = F0.to(torch.float32).cpu().pin_memory()
    host_V = torch.zeros_like(host_F).pin_memory()
    out_F = torch.empty_like(host_F).pin_memory()
    # a fixed number of one-step calls, so the figure does not depend on the timed K
    Ke = E2E_CALLS
    barrier()
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    sim.Field.copy_(host_F, non_blocking=True)
    sim.Velocity.copy_(host_V, non_blocking=True)
    E = 1e300
    for _ in range(Ke):
        E, err = sim.step(E)
    out_F.copy_(sim.Field, non_blocking=True)
    torch.cuda.synchronize(dev)
    e2e_s = max_over_ranks(time.perf_counter() - t0)
    e2e_value = world * N * Ke / e2e_s / 1e6
    h2d = (host_F.numel() + host_V.numel()) * 4 / Ke
    d2h = out_F.numel() * 4 / Ke + 16

    extra = {}
    if rank == 0 and not args.no_compare:
        extra = compare_fp64_and_plain(args, dev, F0)
    cpu = cpu_port = None
    if rank == 0 and world == 1 and not args.no_cpu:
        v, cores, kind, sample, _ = reference_sample(1, 1)
        cpu = {"value": v, "unit": UNIT, "cores": cores, "kind": kind, "sample": sample}
        v, threads, sample, _ = cpu_sample(1, 0)
        cpu_port = {"value": v, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample}
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
                "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32 fields / f64 reductions", "data": "synthetic",
                "config": config({"parallelism": f"replicas x{world}" if world > 1 else "single lattice",
                                  "global_sites": world * N}),
                "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                             "frac": achieved / peak, "traffic": traffic, "peak_source": peak_src,
                             "kernel": "flow_kernel<ChiralMagnet,float> stage launches (S1, S2+S3 fused, S4)"
                                       if fused else "flow_kernel<ChiralMagnet,float> (4 stage launches per step)",
                             "launches_per_step": 3 if fused else 4,
                             "algorithmic_bytes_per_step": bytes_step},
                "cpu_baseline": cpu, "cpu_baseline_port": cpu_port,
                "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                        "steps": Ke, "api": "Simulation.step(prev_energy) per step",
                        "note": f"pinned host field+velocity in once, {Ke} one-step calls each returning (E, err), "
                                "field out once; wall clock, max over ranks"},
                "gpu_launches": launches, "clocks": clk.summary(),
                "autotune": {**{f"S{m}": {"tile_per_cta_ms": a, "pipelined_ms": b, "chosen": "pipelined" if c else
                                          "tile_per_cta"} for m, (a, b, c) in tuning.items() if m != 6},
                             "S2+S3": {"two_kernels_ms": tuning[6][0], "fused_ms": tuning[6][1],
                                       "chosen": "fused" if tuning[6][2] else "two kernels"}}}
        line.update(extra)
        print(json.dumps(line), flush=True)
    return 0


def c2_params():
    from soliton_solver_b200.theories import load_theory
    th = load_theory("Chiral magnet")
    p = th.params.default_params(xlen=320, ylen=320, xsize=10.0, ysize=10.0, J=40e-12, K=0.8e6, D=4e-3, M=580e3,
                                 B=0.0, dmi_term="Heusler", demag=False, unit_magnetization=True, killkinen=True)
    return th, p


def relaxed_accuracy(dev, tol=1e-6, plain_steps=20_000):
    """Time to a relaxed state of the 320^2 chiral magnet (10 x 10 reduced domain, Heusler
    DMI, demag off, B = 0, arrested Newton flow from an anti-skyrmion), through the
    product API Simulation.minimize(tol): max|dE/dphi| < tol.

    fp64:      FP64 fields throughout (its converged energy is the FP64 minimum E*).
    fp32+fp64: the default schedule: FP32 flow to its energy plateau, then FP64 on the
               projected state to tol.
    For each: wall seconds (host clock around the call, which synchronises), steps per
    phase, final energy vs E*, and the first step at which the energy is within 1e-6 of
    E* (FP64 stored energies; for the FP32 phase the FP64 energy of the projected state
    at chunk ends, a separate recorded run).  The plain FP64 form follows the fused FP64
    trajectory to rounding (the largest relative energy difference over plain_steps steps
    is reported), so its time to solution is the FP64 step count times its own measured
    step time."""
    import torch
    from soliton_solver_b200.core.simulation import Simulation
    from soliton_solver_b200.initial_conditions import anti_skyrmion
    th, p = c2_params()
    out = {"config": "chiral magnet 320x320 over 10x10 J/D, Heusler, demag off, B=0, anti-skyrmion R=1 + "
                     "N(0,1e-3), arrested Newton flow, Simulation.minimize(tol=1e-6)"}

    def run(prec, schedule, record):
        sim = Simulation(p, th, precision=prec, device=dev)
        sim.load_field(anti_skyrmion(sim.rp, R=1.0, sigma=1e-3, seed=0, device=dev))
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        res = sim.minimize(tol=tol, schedule=schedule, record=record)
        res["wall_s"] = time.perf_counter() - t0
        res["skyrmion_number"] = sim.observables()["skyrmion_number"]
        res.pop("field64", None)
        del sim
        torch.cuda.empty_cache()
        return res

    r64 = run("fp64", "fp64", True)
    E_star = r64["energy"]
    tr = r64.pop("trajectory")
    rel = np.abs(tr["energy"] - E_star) / abs(E_star)
    r64["first_step_within_1e-6"] = int(np.argmax(rel <= 1e-6)) + 1
    mixed = run("fp32", "fp32+fp64", False)
    rec = run("fp32", "fp32+fp64", True)
    tr = rec.pop("trajectory")
    proj = tr["projected"]
    relp = np.abs(proj[:, 1] - E_star) / abs(E_star)
    mixed["first_chunk_end_within_1e-6_projected"] = int(proj[np.argmax(relp <= 1e-6), 0]) if (relp <= 1e-6).any() \
        else None
    mixed["projected_rel_at_switch"] = float(relp[-1]) if len(relp) else None
    mixed["rel_diff_vs_fp64"] = abs(mixed["energy"] - E_star) / abs(E_star)
    # plain FP64 (the reference's structure on the GPU): the fused FP64 trajectory up to rounding
    p20 = Simulation(p, th, precision="plain_fp64", device=dev)
    f20 = Simulation(p, th, precision="fp64", device=dev)
    for sim in (p20, f20):
        sim.load_field(anti_skyrmion(sim.rp, R=1.0, sigma=1e-3, seed=0, device=dev))
    E0 = f20.observables()["energy"]
    torch.cuda.synchronize(dev)
    t = time.perf_counter()
    Ep, _ = p20.relax(plain_steps, E0)
    torch.cuda.synchronize(dev)
    plain_step_s = (time.perf_counter() - t) / plain_steps
    Ef, _ = f20.relax(plain_steps, E0)
    out["plain_fp64_vs_fused_fp64"] = {"steps": plain_steps, "bitwise_equal_energies": bool(np.array_equal(Ep, Ef)),
                                       "max_rel_energy_diff": float(np.max(np.abs(Ep - Ef) / np.abs(Ef))),
                                       "plain_s_per_step": plain_step_s}
    out["plain_fp64_time_to_solution_s"] = plain_step_s * r64["steps"]
    out["fp64"] = r64
    out["fp32+fp64"] = mixed
    out["speedup_vs_fp64"] = r64["wall_s"] / mixed["wall_s"]
    out["speedup_vs_plain_fp64"] = out["plain_fp64_time_to_solution_s"] / mixed["wall_s"]
    del p20, f20
    torch.cuda.empty_cache()
    return out


def c5_workflow(dev, tol=1e-5, max_steps=300_000, rel_delta=1e-2, fd_steps=200_000, adjoint_iters=20000,
                log_path=None):
    """The large chiral magnet end to end: the workload's 4096^2 lattice (64 anti-skyrmions,
    B = 0.2 T, Heusler, demag on) relaxed by Simulation.minimize(tol) (FP32 arrested flow
    to its energy plateau, then FP64 on the projected state), its topological charge, and
    dE_min/dB, dE_min/dD from the envelope theorem (and the discretisation-corrected
    relaxed_coupling_gradients) against central differences of relaxed energies at
    c (1 +- rel_delta).  Each shifted lattice relaxes from the relaxed state by the FP32
    flow to its energy plateau and contributes its FP64 projected energy: FP32 resolves
    the energy to ~1e-9 relative, far below the 1e-4 the check needs (the difference is
    ~1e-2 of E).  The undamped RK4 dynamics is unstable for this saddle system (see the
    module docstring), so the first 2000 steps are steps of the arrested flow too.
    Central-difference truncation at rel_delta = 1e-2: ~1e-5 relative.  With log_path,
    the results so far are written there after every phase."""
    import torch
    from soliton_solver_b200.autograd import relaxed_coupling_gradients
    from soliton_solver_b200.core.simulation import Simulation
    from soliton_solver_b200.initial_conditions import skyrmion_lattice

    th, p = chiral_params()
    out = {"config": config({"tol": tol, "rel_delta": rel_delta, "max_steps": max_steps, "fd_steps": fd_steps})}

    def log():
        if log_path:
            with open(log_path, "w") as fh:
                json.dump(out, fh, default=float)

    sim = Simulation(p, th, precision="fp32", device=dev)
    sim.load_field(skyrmion_lattice(sim.rp, n=8, R=1.0, seed=1000, device=dev))
    out["Q0"] = sim.observables()["skyrmion_number"]
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    res = sim.minimize(tol=tol, max_steps=max_steps)
    out["relax_wall_s"] = time.perf_counter() - t0
    out["relax"] = {k: v for k, v in res.items() if k not in ("trajectory",)}
    obs = sim.observables()
    out["Q"] = obs["skyrmion_number"]
    out["Q_dev_from_integer"] = abs(obs["skyrmion_number"] - round(obs["skyrmion_number"]))
    out["energy"] = res["energy"]
    log()
    t0 = time.perf_counter()
    g, info = relaxed_coupling_gradients(sim, names=("B", "D"), max_iter=adjoint_iters)
    out["adjoint_wall_s"] = time.perf_counter() - t0
    out["adjoint"] = g
    out["adjoint_info"] = dict(info)
    log()
    F64 = sim.Field64.clone()
    del sim
    torch.cuda.empty_cache()
    fd = {}
    t0 = time.perf_counter()
    for name in ("B", "D"):
        c = getattr(p, name)
        d = rel_delta * c
        Es = []
        for sgn in (1, -1):
            s2 = Simulation(p.with_(**{name: c + sgn * d}), th, precision="fp32", device=dev)
            s2.load_field(F64)
            r2 = s2.minimize(tol=tol, max_steps=fd_steps, schedule="fp32")
            Es.append((s2.projected_energy(), r2["steps"], r2["phases"][0]["stop"]))
            del s2
            torch.cuda.empty_cache()
        fd[name] = {"fd": (Es[0][0] - Es[1][0]) / (2 * d), "delta": d, "steps": [Es[0][1], Es[1][1]],
                    "stop": [Es[0][2], Es[1][2]], "energies": [Es[0][0], Es[1][0]]}
        fd[name]["rel_err_adjoint"] = abs(g[name] - fd[name]["fd"]) / abs(fd[name]["fd"])
        fd[name]["rel_err_uncorrected"] = abs(info["uncorrected"][name] - fd[name]["fd"]) / abs(fd[name]["fd"])
        out["finite_differences"] = fd
        out["fd_wall_s"] = time.perf_counter() - t0
        log()
    return out


def reference_numba_gpu(n=4096, steps=5, timeout=900):
    """The reference's own Simulation.step on Numba's real CUDA target (its FP64 kernels,
    host-side arrest), on the workload's n x n lattice, in a process of its own."""
    cmd = [sys.executable, os.path.join(ROOT, "baseline", "reference_runner.py"), "gpu", str(n), str(steps)]
    try:
        r = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout)
        lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
        res = json.loads(lines[-1]) if lines else {"ok": False, "error": (r.stderr or "no output")[-300:]}
    except subprocess.TimeoutExpired:
        res = {"ok": False, "error": f"timed out after {timeout} s"}
    res["note"] = ("soliton_solver 1.1.1 from baseline/_ref, numba's built-in CUDA target, FP64, wall clock around "
                   "Simulation.step calls (each synchronises)")
    return res


def batched_sweep(dev, steps=20, seed=4, reps=3):
    """The batched baby Skyrme sweep: 256 lattices with edges from {64, 128, 256, 512},
    kappa, mpi ~ U(0.5, 2), windings B in 1..4, hedgehogs with R ~ U(1, 3), FP32 fields.
    Lattice spacing 0.1 and dt = 0.002: a winding-4 hedgehog with R = 1 and kappa = 2 has
    |grad m| ~ 13, so the Skyrme term's stiffness bounds the explicit step near h/26.
    The autotuner first picks each size class's tile shape (ss_batch_autotune).  Then
    `steps` steps of every lattice are captured as one CUDA graph (ss_batch_graph_create:
    per step one launch per RK stage over all lattices' tiles, per-lattice energies and
    arrest on the device) and replayed `reps` times between CUDA events; the same steps
    issued by ss_batch_step (stream launches plus its per-call host copies) are timed
    beside it.  Roofline: 13 words x 3 components x 4 bytes per point-update."""
    import torch
    from soliton_solver_b200.core.batch import BatchSolver
    from soliton_solver_b200.initial_conditions import hedgehog
    from soliton_solver_b200.theories import load_theory
    th = load_theory("Baby Skyrme")
    rng = np.random.default_rng(seed)
    edges = rng.choice([64, 128, 256, 512], size=256)
    params = [th.params.default_params(xlen=int(e), ylen=int(e), lsx=0.1, lsy=0.1, time_step=0.002,
                                       kappa=float(rng.uniform(0.5, 2)), mpi=float(rng.uniform(0.5, 2)),
                                       unit_magnetization=True) for e in edges]
    b = BatchSolver(th, params, "fp32", device=dev)
    for i, p in enumerate(params):
        b.load(i, hedgehog(p.resolved(), charge=int(rng.integers(1, 5)), R=float(rng.uniform(1, 3)), seed=i,
                           device=dev))
    tuned = b.autotune(3)  # tile shape per size class (16 x 64 or 8 x 32 sites)
    b.step(3, 1e300)
    sites = int(sum(int(e) * int(e) for e in edges))
    torch.cuda.synchronize(dev)
    t = time.perf_counter()
    E, _ = b.step(steps)
    torch.cuda.synchronize(dev)
    dt_stream = time.perf_counter() - t
    b.capture(steps)
    b.replay()
    stream = torch.cuda.current_stream(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize(dev)
    e0.record(stream)
    for _ in range(reps):
        b.replay()
    e1.record(stream)
    torch.cuda.synchronize(dev)
    ms = e0.elapsed_time(e1) / (reps * steps)
    Eg, _ = b.trajectory()
    peak = float(json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))).get("hbm_gbs", 6650.0)) \
        if os.path.exists(os.path.join(ROOT, "MEASURED_PEAKS.json")) else 6650.0
    gbs = sites * WORDS_FUSED * 3 * 4 / (ms / 1e3) / 1e9
    return {"lattices": 256, "sites": sites, "steps_per_graph": steps, "replays": reps,
            "value": sites / (ms / 1e3) / 1e6, "unit": UNIT, "ms_per_step": ms,
            "achieved_gbs": gbs, "frac_of_measured_hbm": gbs / peak, "bytes_per_point_update": WORDS_FUSED * 3 * 4,
            "stream_value": sites * steps / dt_stream / 1e6, "stream_ms_per_step": dt_stream / steps * 1e3,
            "tma": b.tma_enabled, "finite": bool(np.isfinite(E).all() and np.isfinite(Eg).all()),
            "tile_shapes": {f"{k[0]}x{k[1]}": {"ms_16x64": v[0], "ms_8x32": v[1], "chosen": "8x32" if v[2] else "16x64"}
                            for k, v in tuned.items()},
            "note": "one CUDA-graph launch per `steps` steps of all 256 lattices, CUDA events around the replays; "
                    "stream_value: ss_batch_step incl. its host synchronisation"}


def small_lattice_graph(dev, steps=2000, chunk=100):
    """The 320^2 chiral magnet (10 x 10 reduced domain, Heusler, demag off), FP32: the same
    steps issued as stream launches vs replays of a captured `chunk`-step CUDA graph."""
    import torch
    from soliton_solver_b200.core.simulation import Simulation
    from soliton_solver_b200.initial_conditions import anti_skyrmion
    from soliton_solver_b200.theories import load_theory
    th = load_theory("Chiral magnet")
    p = th.params.default_params(xlen=320, ylen=320, xsize=10.0, ysize=10.0, dmi_term="Heusler", demag=False,
                                 unit_magnetization=True)
    out = {}
    for mode in ("stream", "graph"):
        sim = Simulation(p, th, precision="fp32", device=dev)
        sim.load_field(anti_skyrmion(sim.rp, R=1.0, seed=0, device=dev))
        s = sim.solver
        s.step(5, 1e300)
        if mode == "graph":
            s.capture(chunk)
            s.replay()
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        stream = torch.cuda.current_stream(dev)
        e0.record(stream)
        for _ in range(steps // chunk):
            if mode == "graph":
                s.replay()
            else:
                s.step_async(chunk)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        ms = e0.elapsed_time(e1)
        out[mode] = {"value": 320 * 320 * steps / (ms / 1e3) / 1e6, "unit": UNIT, "us_per_step": ms * 1e3 / steps}
        del sim
    return out


def render_rgba(dev, F0, reps=20):
    """Headless magnetisation colormap (ss_render_rgba) of the workload's 4096^2 FP32
    field: 12 B read + 4 B written per pixel; CUDA events around `reps` launches."""
    import torch
    from soliton_solver_b200.core import colormaps as cm
    F = F0.to(device=dev, dtype=torch.float32).contiguous()
    out = torch.empty((YLEN, XLEN, 4), dtype=torch.uint8, device=dev)
    p_i = np.array([XLEN, YLEN], dtype=np.int32)
    for _ in range(3):
        cm.render_magnetization_to_rgba[None, None](out, F, XLEN, YLEN, p_i)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        cm.render_magnetization_to_rgba[None, None](out, F, XLEN, YLEN, p_i)
    e1.record()
    torch.cuda.synchronize(dev)
    us = e0.elapsed_time(e1) / reps * 1e3
    gbs = XLEN * YLEN * 16 / (us * 1e-6) / 1e9
    peak = float(json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))).get("hbm_gbs", 6650.0)) \
        if os.path.exists(os.path.join(ROOT, "MEASURED_PEAKS.json")) else 6650.0
    # beside it: the reference's per-pixel colormap restated on the CPU (the oracle), on a
    # 128 x 128 corner of the same field
    from oracle import colormaps as ocm
    n = 128
    Fs = F.view(-1, XLEN, YLEN)[:, :n, :n].double().cpu().numpy().reshape(-1)
    t = time.perf_counter()
    ocm.render_magnetization(Fs, n, n)
    cpu_pps = n * n / (time.perf_counter() - t)
    return {"kernel": "render_kernel<float, magnetization> (ss_render_rgba)", "pixels": XLEN * YLEN,
            "us_per_image": us, "achieved_gbs": gbs, "frac": gbs / peak, "bytes_per_pixel": 16,
            "cpu_pixels_per_s": cpu_pps, "speedup": XLEN * YLEN / (us * 1e-6) / cpu_pps,
            "cpu_sample": "oracle restatement of the reference's per-pixel colormap, 128x128 corner, 1 core"}


def initial_condition(dev, reps=10):
    """The chiral magnet's skyrmion ansatz (ss_initialize) written into a 4096^2 FP32
    field and velocity: 8 words written per site, FP64 sin/cos/exp/atan2 per site."""
    import torch
    from soliton_solver_b200 import _native as nat
    from soliton_solver_b200.core.simulation import Simulation
    th, p = chiral_params()
    sim = Simulation(p, th, precision="fp32", device=dev)
    s = sim.solver
    for _ in range(2):
        s.initialize(sim.Field, sim.Velocity, nat.SS_INIT_ANSATZ, nat.SS_ANSATZ_ANTI, 0.3)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        s.initialize(sim.Field, sim.Velocity, nat.SS_INIT_ANSATZ, nat.SS_ANSATZ_ANTI, 0.3)
    e1.record()
    torch.cuda.synchronize(dev)
    us = e0.elapsed_time(e1) / reps * 1e3
    del sim
    torch.cuda.empty_cache()
    # beside it: the ansatz restated in numpy on the CPU (the oracle), on a 512^2 lattice
    from oracle import init as oin
    thn, pn = chiral_params(512, 512)
    p_i, p_f = thn.params.pack_device_params(pn.resolved())
    t = time.perf_counter()
    oin.initial("chiral_magnet", p_i, p_f, ansatz=oin.ANSATZ_ANTI, rotation=0.3)
    cpu_sps = 512 * 512 / (time.perf_counter() - t)
    return {"kernel": "init_kernel<chiral, float> (ss_initialize, anti-skyrmion ansatz)", "sites": XLEN * YLEN,
            "us": us, "achieved_gbs": XLEN * YLEN * 32 / (us * 1e-6) / 1e9, "bytes_per_site": 32,
            "cpu_sites_per_s": cpu_sps, "speedup": XLEN * YLEN / (us * 1e-6) / cpu_sps,
            "cpu_sample": "oracle numpy restatement of the ansatz kernel, 512x512 chiral lattice, 1 process"}


def dat_field_dump(dev, F0, reps=3):
    """The .dat text of the workload's 4096^2 x 4 FP32 field at 32 significant digits
    (output_field_dat's bytes) formatted on the GPU (ss_format_text: length pass, scan,
    write pass), device-resident text; against the reference writer's per-value Python
    formatting timed on a 200 000-value sample of the same field."""
    import ctypes
    import torch
    from soliton_solver_b200 import _native as nat
    from oracle import io as oio
    v = F0.to(device=dev, dtype=torch.float32).contiguous().reshape(-1)
    n = v.numel()
    lib = nat.load()
    nb = ctypes.c_size_t()
    nat.check(lib.ss_text_workspace_bytes(n, ctypes.byref(nb)))
    ws = torch.empty(int(nb.value), dtype=torch.uint8, device=dev)
    length = ctypes.c_longlong()
    stream = torch.cuda.current_stream(dev).cuda_stream
    args = (v.data_ptr(), nat.SS_FP32, n, 32, YLEN, XLEN * YLEN)
    nat.check(lib.ss_format_text(*args, None, 0, ctypes.byref(length), ws.data_ptr(), ws.numel(), stream))
    out = torch.empty(int(length.value), dtype=torch.uint8, device=dev)
    ts = []
    for _ in range(reps):
        torch.cuda.synchronize(dev)
        t = time.perf_counter()
        nat.check(lib.ss_format_text(*args, out.data_ptr(), out.numel(), ctypes.byref(length), ws.data_ptr(),
                                     ws.numel(), stream))
        torch.cuda.synchronize(dev)
        ts.append(time.perf_counter() - t)
    dt = min(ts)
    sample = v[:200000].cpu().numpy()
    t = time.perf_counter()
    oio.field_text(sample, 1, 200000, 1, 32)
    py = 200000 / (time.perf_counter() - t)
    del out, ws
    torch.cuda.empty_cache()
    return {"values": n, "text_bytes": int(length.value), "s": dt, "values_per_s": n / dt,
            "text_gbs": length.value / dt / 1e9, "python_format_values_per_s": py, "speedup": n / dt / py,
            "note": "ss_format_text incl. its length pass, scan and one stream sync; wall clock"}


def fused_fp64(dev, F0, steps=50):
    """The same lattice with FP64 fields through the fused stage kernels (autotuned):
    the precision-matched comparison with the plain FP64 form."""
    import torch
    from soliton_solver_b200.core.simulation import Simulation
    th, p = chiral_params()
    sim = Simulation(p, th, precision="fp64", device=dev)
    sim.load_field(F0)
    s = sim.solver
    s.autotune(3)
    s.step(3, 1e300)
    E = torch.empty(steps, dtype=torch.float64, device=dev)
    err = torch.empty(steps, dtype=torch.float64, device=dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize(dev)
    e0.record()
    s.step_async(steps, math.nan, E, err)
    e1.record()
    torch.cuda.synchronize(dev)
    ms = e0.elapsed_time(e1) / steps
    words = WORDS_FUSED if (s.tma_enabled and s._lib.ss_get_variant(s._h, 6) == 1) else WORDS_SEPARATE
    gbs = words * 4 * 8 * XLEN * YLEN / (ms / 1e3) / 1e9
    out = {"value": XLEN * YLEN / (ms / 1e3) / 1e6, "unit": UNIT, "ms_per_step": ms, "steps": steps,
           "achieved_gbs": gbs, "bytes_per_point_update": words * 4 * 8, "finite": bool(torch.isfinite(E).all()),
           "note": "FP64 fields, fused stage kernels, same lattice; CUDA events"}
    del sim
    torch.cuda.empty_cache()
    return out


def compare_fp64_and_plain(args, dev, F0):
    """Relaxed-state accuracy (320^2), and the plain-FP64 form's speed on this lattice."""
    import torch
    from soliton_solver_b200.core.simulation import Simulation
    th, p = chiral_params()
    out = {}
    for key, fn in (("accuracy", relaxed_accuracy), ("batched_sweep", batched_sweep),
                    ("graph_320", small_lattice_graph), ("render_rgba", lambda d: render_rgba(d, F0)),
                    ("initial_condition", initial_condition), ("dat_field_dump", lambda d: dat_field_dump(d, F0))):
        try:
            out[key] = fn(dev)
        except Exception as exc:  # reported, not fatal: the headline line must still print
            out[key] = {"error": f"{type(exc).__name__}: {exc}"}
    try:
        out["fused_fp64"] = fused_fp64(dev, F0)
    except Exception as exc:
        out["fused_fp64"] = {"error": f"{type(exc).__name__}: {exc}"}
    if not args.no_reference_gpu:
        out["reference_numba_gpu"] = reference_numba_gpu()
    sim = Simulation(p, th, precision="plain_fp64", device=dev)
    sim.load_field(F0)
    sim.relax(1, 1e300)
    torch.cuda.synchronize(dev)
    t = time.perf_counter()
    kp = 3
    sim.relax(kp, math.nan)
    torch.cuda.synchronize(dev)
    dt = (time.perf_counter() - t) / kp
    out["plain_fp64"] = {"value": XLEN * YLEN / dt / 1e6, "unit": UNIT, "ms_per_step": dt * 1e3,
                         "note": "reference-structured FP64 CUDA form (derivative buffers, per-stage launches, "
                                 "host-side arrest), same lattice"}
    del sim
    torch.cuda.empty_cache()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU-baseline leg")
    ap.add_argument("--no-compare", action="store_true", help="skip the FP64 / plain-FP64 comparison")
    ap.add_argument("--no-reference-gpu", action="store_true",
                    help="skip the reference's own kernels on Numba's CUDA target")
    ap.add_argument("--variants", default="", help="pin the staging variant of stages 1-4 after autotuning "
                                                    "(comma-separated, 0 one tile per CTA, 1 pipelined)")
    ap.add_argument("--size", type=int, default=4096, help="lattice edge (4096 is the workload; smaller sizes "
                                                             "are for profiler captures)")
    ap.add_argument("--section", default="", choices=["", "accuracy", "batched_sweep", "graph_320", "render_rgba",
                                                       "initial_condition", "dat_field_dump", "fused_fp64",
                                                       "reference_numba_gpu"],
                    help="run only this block of the comparison and print it as one JSON line (profiling)")
    ap.add_argument("--workflow-log", default="", help="with --workflow: write the results so far to this file "
                                                       "after every phase")
    ap.add_argument("--workflow", default="", choices=["", "c5"],
                    help="c5: relax the workload's lattice to tol and check dE/dB, dE/dD against finite "
                         "differences (minutes of GPU time; prints one JSON line)")
    args = ap.parse_args()
    global XLEN, YLEN, XSIZE
    if args.size != 4096:
        XLEN = YLEN = args.size
        XSIZE = 128.0 * (args.size - 1) / 4095
    args.warmup = max(args.warmup, 3)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return reference_arm(args, rank, world)
    if args.section:
        import torch
        dev = torch.device("cuda", local_rank)
        torch.cuda.set_device(dev)
        fn = {"accuracy": relaxed_accuracy, "batched_sweep": batched_sweep, "graph_320": small_lattice_graph,
              "initial_condition": initial_condition, "reference_numba_gpu": lambda d: reference_numba_gpu()}.get(
            args.section)
        if fn is None:  # the blocks that work on the workload's field
            from soliton_solver_b200.initial_conditions import skyrmion_lattice
            th, p = chiral_params()
            F0 = skyrmion_lattice(p.resolved(), n=8, R=1.0, seed=1000, device=dev)
            fn = {"render_rgba": lambda d: render_rgba(d, F0), "dat_field_dump": lambda d: dat_field_dump(d, F0),
                  "fused_fp64": lambda d: fused_fp64(d, F0)}[args.section]
        print(json.dumps({"section": args.section, **fn(dev)}, default=float), flush=True)
        return 0
    if args.workflow == "c5":
        import torch
        dev = torch.device("cuda", local_rank)
        torch.cuda.set_device(dev)
        print(json.dumps(c5_workflow(dev, log_path=args.workflow_log or None), default=float), flush=True)
        return 0
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local_rank))
    try:
        return gpu_arm(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    sys.exit(main())
