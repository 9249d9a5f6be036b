"""Benchmark of the RK3 time-step loop on one or more B200s.

Workload (one "step" = one Shu-Osher RK3 step = 3 RHS evaluations + stage
updates + the CFL reduction): decaying isotropic turbulence at 256^3, turbulent
Mach 0.5, Re 1000, Ma 0.5, Pr 0.72, gamma 1.4, Steger-Warming + WENO5, C8th
viscous terms, CFL 0.5, seeded random-phase solenoidal field with
E(k) ~ k^4 exp(-2 (k/4)^2) (synthetic; the reference publishes no dataset).

Headline `value`: RK3 steps/s of the FP32-stencil / FP64-accumulation form,
device-timed with CUDA events on the library's stream (max over ranks).
Also reported: the plain FP64 form's steps/s, Gcell/s, errors of the FP32 form
against the FP64 form after a fixed-dt run, the per-kernel roofline, clocks,
an end-to-end number through the public API with host buffers, and the
reference CPU path timed on this host's cores.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
Multi-GPU: launched under torchrun; every rank runs an independent replica
(the path does not shard: replicas only), scaling "weak".
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_DEFAULT = 256
WORKLOAD = dict(gamma=1.4, Pr=0.72, Ma=0.5, Re=1000.0, cfl=0.5, mach_t=0.5, k0=4.0, seed=12345,
                fvs="stagerwarming", recon="weno5", vis="c8th")
METRIC = "RK3 steps/s & Gcell/s at 256^3 FP32 vs FP64 at stated err; adjoint/fwd cost"
STEP_BYTES_PER_CELL = 360.0   # 3 stages x (read U 40 + read U0 40 + write U 40)
CPU_SAMPLE_N = 64


def env_rank():
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# ----------------------------------------------------------------------------
# multi-rank plumbing
# ----------------------------------------------------------------------------

def dist_init(world: int, use_cuda: bool):
    if world <= 1:
        return None
    import datetime
    import torch.distributed as dist
    dist.init_process_group("nccl" if use_cuda else "gloo",
                            timeout=datetime.timedelta(seconds=300))
    return dist


def dist_max(dist, value: float, use_cuda: bool) -> float:
    """Max of a float over ranks (every rank calls it)."""
    if dist is None:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device="cuda" if use_cuda else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def dist_barrier(dist, use_cuda: bool):
    if dist is None:
        return
    import torch
    if use_cuda:
        t = torch.zeros(1, device="cuda")
        dist.all_reduce(t)
        torch.cuda.synchronize()
    else:
        dist.barrier()


# ----------------------------------------------------------------------------
# clocks during the timed region
# ----------------------------------------------------------------------------

class ClockSampler:
    """SM clock and clock-event reasons sampled during the timed region: NVML
    polled from a thread every 5 ms (so even a 0.1 s region gets ~20
    samples), or nvidia-smi -lms 20 where NVML is unavailable."""
    PERIOD_S = 0.005
    NAMES = (("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40),
             ("sw_thermal_slowdown", 0x20), ("sw_power_cap", 0x4))
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.rows = []          # (sm_mhz, max_mhz, reason bits)
        self.source = None
        self._stop = None
        self._thread = None
        self.proc = None
        self.path = None

    def _nvml_handle(self):
        import pynvml
        pynvml.nvmlInit()
        try:
            import torch
            uuid = str(torch.cuda.get_device_properties(self.device).uuid)
            return pynvml.nvmlDeviceGetHandleByUUID(("GPU-" + uuid).encode())
        except Exception:
            return pynvml.nvmlDeviceGetHandleByIndex(self.device)

    def __enter__(self):
        import threading
        try:
            import pynvml
            h = self._nvml_handle()
            mx = pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM)
            self._stop = threading.Event()

            def poll():
                while not self._stop.is_set():
                    try:
                        sm = pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM)
                        rs = pynvml.nvmlDeviceGetCurrentClocksEventReasons(h)
                        self.rows.append((float(sm), float(mx), int(rs)))
                    except Exception:
                        pass
                    self._stop.wait(self.PERIOD_S)
            self._thread = threading.Thread(target=poll, daemon=True)
            self._thread.start()
            self.source = "nvml 5 ms"
            return self
        except Exception:
            self._thread = None
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "20"], stdout=self.fh,
                stderr=subprocess.DEVNULL)
            self.source = "nvidia-smi 20 ms"
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self._thread is not None:
            self._stop.set()
            self._thread.join(timeout=2)
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.fh.close()
            with open(self.path) as f:
                for line in f:
                    parts = [x.strip() for x in line.split(",")]
                    if len(parts) >= 9 and parts[1].replace(".", "").isdigit():
                        bits = sum(b for (_, b), v in zip(self.NAMES, parts[5:9])
                                   if v.lower() == "active")
                        mx = float(parts[2]) if parts[2].replace(".", "").isdigit() else 0.0
                        self.rows.append((float(parts[1]), mx, bits))
            os.unlink(self.path)

    def summary(self):
        out = {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": len(self.rows),
               "source": self.source}
        if not self.rows:
            return out
        reasons = sorted({name for _, _, bits in self.rows for name, b in self.NAMES if bits & b})
        out.update(sm_mhz=statistics.median(r[0] for r in self.rows),
                   sm_max_mhz=max(r[1] for r in self.rows), reasons=reasons)
        return out


# ----------------------------------------------------------------------------
# our arm
# ----------------------------------------------------------------------------

def make_params(ns, n, precision, dt_fixed=-1.0):
    w = WORKLOAD
    two_pi = 2 * math.pi
    return ns.SolverParams.default().replace(
        n=n, gamma=w["gamma"], Pr=w["Pr"], Ma=w["Ma"], Re=w["Re"], cfl=w["cfl"],
        dt_fixed=dt_fixed, fvs_type=w["fvs"], recon=w["recon"], vis_scheme=w["vis"],
        Lx=two_pi, Ly=two_pi, Lz=two_pi, precision=precision,
        char_recon=1 if w.get("char") else 0)


def workload_name(n):
    w = WORKLOAD
    scheme = "SW+WENO5, C8th" + (", characteristic-wise reconstruction" if w.get("char") else "")
    return f"isotropic turbulence {n}^3, Mach_t 0.5, Re 1000, {scheme}"


def workload_input(n):
    from ns3d_cpp_b200 import initial
    w = WORKLOAD
    return initial.isotropic(n, mach_t=w["mach_t"], Ma=w["Ma"], gamma=w["gamma"], k0=w["k0"],
                             seed=w["seed"])


def kernel_bytes_per_cell(cls: str, rsize: int) -> float:
    """Algorithmic (compulsory) HBM bytes per cell of one launch of a kernel class."""
    w = 5 * 8          # rho,u,v,w,p read once
    if cls == "sweep_x":
        return w + 5 * rsize
    if cls in ("sweep_y", "sweep_z"):
        return w + 10 * rsize
    # viscous flux values per cell: 9 in the FP64 form; 12 in the FP32 form
    # (three float4 blocks, one per differentiated direction)
    fv = 12 if rsize == 4 else 9
    if cls == "visc_flux":
        return 4 * 8 + fv * rsize
    if cls in ("update", "sweep_z_update"):
        # current + recorded state (stage 1 reads only the recorded one: the
        # mean over the three stages is 5/3 state reads), T_acc, the viscous
        # flux values, 6 doubles written; the fused z sweep reads the current
        # state for its splits and the same cell's values again for the stage
        # (cache hits), so the same bytes
        return (5.0 / 3.0) * w + 5 * rsize + fv * rsize + 6 * 8
    return 0.0


def timed_steps(torch, s, steps: int, warmup: int, dist, use_cuda, profile=True):
    """W untimed steps, then K steps bracketed by barrier + synchronize, timed
    with CUDA events recorded on the library's own stream."""
    stream = torch.cuda.ExternalStream(s.stream_handle())
    for _ in range(warmup):
        s.step(1)
    s.synchronize()
    dist_barrier(dist, use_cuda)
    torch.cuda.synchronize()
    if profile:
        s.profile(True)
    l0 = s.launch_count()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    s.step(steps)
    e1.record(stream)
    e1.synchronize()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    launches = s.launch_count() - l0
    prof = s.profile_read() if profile else {}
    if profile:
        s.profile(False)
    dist_barrier(dist, use_cuda)
    return ms, launches, prof


def error_run(ns, n, W, steps, device):
    """FP32-stencil vs FP64 after `steps` steps at the same fixed dt."""
    with ns.Solver(make_params(ns, n, "fp64"), device=device) as s:
        s.upload_primitive(W)
        dt0 = s.compute_timestep()
    res = {}
    for prec in ("fp64", "fp32acc64"):
        with ns.Solver(make_params(ns, n, prec, dt_fixed=dt0), device=device) as s:
            s.upload_primitive(W)
            s.step(steps)
            st = s.compute_turbulence_statistics()
            Ek = s.compute_energy_spectrum()
            res[prec] = (st, Ek)
    (a, Ea), (b, Eb) = res["fp64"], res["fp32acc64"]
    big = Ea > 1e-6 * Ea.max()

    def rel(x, y):
        return abs(x - y) / abs(y)
    return {"steps": steps, "dt": dt0,
            "total_energy": rel(b["total_energy"], a["total_energy"]),
            "kinetic_energy": rel(b["kinetic_energy"], a["kinetic_energy"]),
            "dissipation": rel(b["dissipation"], a["dissipation"]),
            "spectrum_max": float(np.max(np.abs(Eb[big] - Ea[big]) / Ea[big])),
            "reference": "FP64 form of this code (itself 1e-12 parity with the oracle)"}


def e2e_run(torch, ns, n, W, steps, device, prefetch=True, dist=None, use_cuda=True, world=1):
    """Same metric through the public API with host buffers: every step uploads
    its inputs (the state) from pinned host memory, steps, and reads the total
    energy back. With `prefetch`, step k+1's upload is started (on the
    library's copy stream) before step k runs, so the PCIe transfer overlaps
    the step; all `steps` copies lie inside the timed region (the first one
    unprefetched, none started after the last step)."""
    pinned = torch.empty((5,) + W.shape[1:], dtype=torch.float64, pin_memory=True)
    pinned.numpy()[...] = W
    host = pinned.numpy()
    with ns.Solver(make_params(ns, n, "fp32acc64"), device=device) as s:
        stream = torch.cuda.ExternalStream(s.stream_handle())
        for _ in range(2):  # warm-up, staging buffer allocated
            s.prefetch_primitive(host)
            s.upload_primitive(host)
            s.step(1)
            s.compute_total_energy()
        s.synchronize()
        torch.cuda.synchronize()
        dist_barrier(dist, use_cuda)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        t0 = time.perf_counter()
        e0.record(stream)
        for k in range(steps):
            s.upload_primitive(host)
            if prefetch and k + 1 < steps:
                s.prefetch_primitive(host)
            s.step(1)
            s.compute_total_energy()
        e1.record(stream)
        e1.synchronize()
        wall = time.perf_counter() - t0
        ms = e0.elapsed_time(e1)
    dist_barrier(dist, use_cuda)
    ms = dist_max(dist, ms, use_cuda)
    wall = dist_max(dist, wall, use_cuda)
    h2d = 5 * W[0].size * 8
    d2h = 12 * 8
    path = ("Solver.upload_primitive(pinned host; the next step's prefetch_primitive overlapping "
            "this step) + step(1) + compute_total_energy" if prefetch else
            "Solver.upload_primitive(pinned host) + step(1) + compute_total_energy")
    # whole job: every rank runs its own replica; the slowest rank's time
    return {"value": world * steps / (ms / 1e3), "unit": "steps/s", "h2d_bytes_per_step": h2d,
            "d2h_bytes_per_step": d2h, "wall_steps_per_s": world * steps / wall, "path": path}


def adjoint_cost(torch, ns, device, nsteps=200, K=20, n=64, fd_dirs=2):
    """Adjoint workload: Taylor-Green 64^3 + seeded 1e-3 solenoidal perturbation,
    Re 400, Ma 0.2, SW (entropy fix 1e-3) + WENO5, C8th, 200 RK3 steps,
    checkpoint every 20. Cost = (checkpointed forward + reverse sweep with
    recompute) / plain forward, both on the library's stream, FP64."""
    from ns3d_cpp_b200 import initial
    two_pi = 2 * math.pi
    p = ns.SolverParams.default().replace(
        n=n, gamma=1.4, Pr=0.72, Ma=0.2, Re=400.0, cfl=0.5, fvs_type="stagerwarming",
        recon="weno5", vis_scheme="c8th", Lx=two_pi, Ly=two_pi, Lz=two_pi,
        sw_entropy_eps=1e-3, sutherland_s_over_tref=110.4 / 273.15, precision="fp64")
    W = initial.taylor_green(n, Ma=0.2, perturb=1e-3, seed=2024)
    with ns.Solver(p, device=device) as s:
        stream = torch.cuda.ExternalStream(s.stream_handle())
        s.upload_primitive(W)
        s.adjoint(nsteps, K)                 # warm-up: modules, the context's checkpoint arrays
        s.upload_primitive(W)
        s.step(3)

        def timed(fn):
            s.upload_primitive(W)
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            t0 = time.perf_counter()
            e0.record(stream)
            out = fn()
            e1.record(stream)
            e1.synchronize()
            return e0.elapsed_time(e1) / 1e3, time.perf_counter() - t0, out
        fwd_dev, fwd_wall, _ = timed(lambda: s.step(nsteps))
        adj_dev, adj_wall, (grad, J, dts) = timed(lambda: s.adjoint(nsteps, K))

        # accuracy, measured here: the gradient along random solenoidal
        # directions against the 4-point central difference of the forward
        # with the recorded dt sequence (h = 1e-6 per unit-rms direction)
        def J_of(Wx):
            s.upload_primitive(Wx)
            s.step_dts(dts)
            return s.compute_total_energy()
        h = 1e-6
        gnorm = math.sqrt(float(np.sum(grad[1:4] ** 2)))
        fd = []
        for k in range(fd_dirs):
            d = np.zeros_like(W)
            d[1:4] = initial.solenoidal_field(n, k0=4.0, seed=100 + k)
            d[1:4] /= math.sqrt(float(np.mean(d[1:4] ** 2)))
            Jd = (-J_of(W + 2 * h * d) + 8 * J_of(W + h * d) - 8 * J_of(W - h * d)
                  + J_of(W - 2 * h * d)) / (12 * h)
            ad = float(np.sum(grad[1:4] * d[1:4]))
            fd.append({"rel": abs(Jd - ad) / abs(ad),
                       "rel_to_norm": abs(Jd - ad) / (gnorm * math.sqrt(float(np.sum(d[1:4] ** 2))))})
        J_replay = J_of(W)
    return {"workload": f"Taylor-Green {n}^3 + 1e-3 solenoidal perturbation, Re 400, Ma 0.2, "
                        f"SW(eps 1e-3)+WENO5, C8th, {nsteps} RK3 steps, checkpoint every {K}",
            "forward_s": fwd_dev, "adjoint_s": adj_dev, "ratio": adj_dev / fwd_dev,
            "ratio_wall": adj_wall / fwd_wall, "J": J,
            "J_replay_rel": abs(J_replay - J) / abs(J),
            "fd_directions": fd,
            "fd": "4-point central difference at h = 1e-6 per unit-rms solenoidal direction "
                  "(k0 4, seeds 100..), forward replayed with the adjoint's dt sequence"}


def ncu_traffic():
    """DRAM bytes per cell per kernel class, from the ncu capture recorded in
    profiles/ncu_traffic.json (dram__bytes_read.sum + dram__bytes_write.sum of
    one launch of each class, on a smaller box; `cells` names its size)."""
    path = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    try:
        with open(path) as f:
            return json.load(f)
    except Exception:
        return {}


def oracle_rhs_errors(ns, n, W, device):
    """The GPU's RHS of the benchmark field in both forms against the FP64
    oracle's (the C restatement, bit-exact against the reference), max|a-b| /
    max|b| per conserved variable. Part of the CPU leg: the oracle runs on the
    host's cores."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    w = WORKLOAD
    two_pi = "6.283185307179586"
    cfg = dict(gamma=w["gamma"], Pr=w["Pr"], Ma=w["Ma"], Re=w["Re"], cfl=w["cfl"], dt_fixed=-1,
               fvs_type="StagerWarming", recon="WENO5", vis_scheme="C8th",
               global_nx=n, global_ny=n, global_nz=n, Lx=two_pi, Ly=two_pi, Lz=two_pi,
               char_recon="true" if w.get("char") else "false")
    t0 = time.perf_counter()
    ref = oracle.Oracle(cfg).rhs(W)
    t_orc = time.perf_counter() - t0
    den = np.max(np.abs(ref), axis=(1, 2, 3))
    out = {"oracle_s": t_orc, "threads": os.environ.get("OMP_NUM_THREADS", str(os.cpu_count()))}
    for prec in ("fp64", "fp32acc64"):
        with ns.Solver(make_params(ns, n, prec), device=device) as s:
            s.upload_primitive(W)
            r = s.compute_rhs()
        out[prec] = float(np.max(np.max(np.abs(r - ref), axis=(1, 2, 3)) / den))
    return out


def our_arm(args, rank, world, local):
    import torch
    use_cuda = torch.cuda.is_available()
    if not use_cuda:
        raise SystemExit("bench.py: no CUDA device")
    torch.cuda.set_device(local)
    dist = dist_init(world, use_cuda)
    import ns3d_cpp_b200 as ns
    n = args.n
    W = workload_input(n)
    ncell = n ** 3
    peak, peak_kind = measured_peaks()

    if args.only_fp64:
        # diagnostic mode (kernel captures of the FP64 form): its steps alone
        with ns.Solver(make_params(ns, n, "fp64"), device=local) as s:
            s.upload_primitive(W)
            ms64, _, prof64 = timed_steps(torch, s, args.steps, args.warmup, dist, use_cuda)
        ms64 = dist_max(dist, ms64, use_cuda)
        if rank == 0:
            print(json.dumps({"form": "fp64", "n": n, "steps": args.steps,
                              "steps_per_s": world * args.steps / (ms64 / 1e3),
                              "kernels_ms_per_launch": {c: (v[0] / v[1] if v[1] else None)
                                                        for c, v in prof64.items()}}), flush=True)
        if dist is not None:
            dist.destroy_process_group()
        return

    # --- the headline form: FP32 stencils, FP64 accumulation ---
    with ns.Solver(make_params(ns, n, "fp32acc64"), device=local) as s:
        s.upload_primitive(W)
        with ClockSampler(local) as clk:
            ms, launches, prof = timed_steps(torch, s, args.steps, args.warmup, dist, use_cuda)
        clocks = clk.summary()
    ms_max = dist_max(dist, ms, use_cuda)
    value = world * args.steps / (ms_max / 1e3)

    # --- the plain FP64 form on the same workload ---
    k64 = max(3, args.steps // 3)
    fp64_sps, ms64_max, prof64 = None, None, {}
    if not args.skip_fp64:
        with ns.Solver(make_params(ns, n, "fp64"), device=local) as s:
            s.upload_primitive(W)
            ms64, _, prof64 = timed_steps(torch, s, k64, max(3, args.warmup // 2), dist, use_cuda)
        ms64_max = dist_max(dist, ms64, use_cuda)
        fp64_sps = world * k64 / (ms64_max / 1e3)

    # --- end to end through the public API, host buffers, on every rank ---
    e2e = None
    if args.e2e_steps > 0:
        e2e = e2e_run(torch, ns, n, W, args.e2e_steps, local, dist=dist, use_cuda=use_cuda,
                      world=world)
        # the same loop with each upload issued only after the previous step
        # has returned (no transfer/compute overlap), for comparison
        e2e["serial_steps_per_s"] = e2e_run(torch, ns, n, W, args.e2e_steps, local, prefetch=False,
                                            dist=dist, use_cuda=use_cuda, world=world)["value"]

    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return

    errors = error_run(ns, n, W, args.err_steps, local) if args.err_steps > 0 else None
    adjoint = None if args.skip_adjoint else adjoint_cost(torch, ns, local)

    # dominant kernel roofline (per launch, CUDA-event timed in the timed region)
    rsize = 4
    kern = {}
    for cls, (kms, cnt) in prof.items():
        if cnt:
            b = kernel_bytes_per_cell(cls, rsize) * ncell
            kern[cls] = {"launches": cnt, "ms_total": kms, "ms_per_launch": kms / cnt,
                         "share": kms / max(1e-9, sum(v[0] for v in prof.values())),
                         "alg_bytes_per_launch": b,
                         "achieved_gbs": b / (kms / cnt / 1e3) / 1e9 if b else None}
    dom = max((c for c in kern if c != "other"), key=lambda c: kern[c]["ms_total"])
    tr = ncu_traffic()
    # captured traffic belongs to the component-wise kernels: bytes per cell of
    # the captured launch, times this run's cells
    cap = None if WORKLOAD.get("char") else (tr.get("fp32acc64") or {}).get(dom)
    traffic = None if cap is None else cap["dram_bytes_per_cell"] * ncell
    ach = kern[dom]["achieved_gbs"]
    roofline = {"bound": "hbm", "kernel": dom, "achieved": ach, "peak": peak, "unit": "GB/s",
                "frac": ach / peak, "traffic": traffic, "peak_source": peak_kind,
                "alg_bytes_per_cell": kernel_bytes_per_cell(dom, rsize),
                "alg_bytes_per_launch": kern[dom]["alg_bytes_per_launch"],
                "traffic_capture": None if cap is None else {
                    "metric": "dram__bytes_read.sum + dram__bytes_write.sum, one launch",
                    "cells": tr.get("cells"), "stage": cap.get("stage"),
                    "scaled": f"per cell of the captured box, times {ncell} cells",
                    "alg_bytes_per_cell_of_capture": cap.get("alg_bytes_per_cell")}}
    step_ach = STEP_BYTES_PER_CELL * ncell * (value / world) / 1e9
    roofline_step = {"bound": "hbm", "achieved": step_ach, "peak": peak, "unit": "GB/s",
                     "frac": step_ach / peak, "alg_bytes_per_cell_step": STEP_BYTES_PER_CELL}

    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(args.cpu_sample_steps, n)
        try:
            cpu["oracle_rhs_errors"] = oracle_rhs_errors(ns, n, W, local)
        except Exception as e:  # reported, never fatal for the GPU line
            cpu["oracle_rhs_errors"] = {"error": str(e)}
    orc = (cpu or {}).get("oracle_rhs_errors") or {}

    line = {
        "metric": METRIC,
        "value": value, "unit": "steps/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "fp32 stencils / fp64 accumulate",
        "data": "synthetic: seeded isotropic turbulence (numpy), inputs resident in HBM",
        "config": {"workload": workload_name(n),
                   "n": n, "cells": ncell, "precision": "fp32acc64",
                   "l2": f"inputs larger than L2: {6 * ncell * 8 / 1e6:.0f} MB per state buffer",
                   "parallelism": f"replicas x{world}"},
        "gcell_per_s": value * ncell / 1e9,
        "fp64_steps_per_s": fp64_sps,
        "fp32_over_fp64": None if fp64_sps is None else value / fp64_sps,
        "ke_err_fp32_vs_fp64": None if errors is None else errors["kinetic_energy"],
        "dissipation_err_fp32_vs_fp64": None if errors is None else errors["dissipation"],
        "spectrum_err_fp32_vs_fp64": None if errors is None else errors["spectrum_max"],
        "rhs_err_fp32_vs_oracle": orc.get("fp32acc64"),
        "rhs_err_fp64_vs_oracle": orc.get("fp64"),
        "adjoint_over_forward_cost": None if adjoint is None else adjoint["ratio"],
        "fp64": None if fp64_sps is None else {
            "steps_per_s": fp64_sps, "gcell_per_s": fp64_sps * ncell / 1e9,
            "steps": k64, "ms_per_step": ms64_max / k64,
            "kernels_ms_per_launch": {c: (v[0] / v[1] if v[1] else None)
                                      for c, v in prof64.items()}},
        "errors_fp32_vs_fp64": errors,
        "adjoint_over_forward": adjoint,
        "roofline": roofline, "roofline_step": roofline_step, "kernels": kern,
        "clocks": clocks, "e2e": e2e, "gpu_launches": launches,
        "cpu_baseline": cpu,
    }
    print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


# ----------------------------------------------------------------------------
# the reference CPU path
# ----------------------------------------------------------------------------

def _cpu_worker(args):
    """One replica: the reference (or the oracle port) on a periodic sub-box.
    Runs in a spawned process; returns seconds per RK3 step."""
    kind, n, steps, warm, char = args
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    from ns3d_cpp_b200 import initial
    w = WORKLOAD
    two_pi = "6.283185307179586"
    cfg = dict(gamma=w["gamma"], Pr=w["Pr"], Ma=w["Ma"], Re=w["Re"], cfl=w["cfl"], dt_fixed=-1,
               fvs_type="StagerWarming", recon="WENO5", vis_scheme="C8th",
               global_nx=n, global_ny=n, global_nz=n, Lx=two_pi, Ly=two_pi, Lz=two_pi,
               Post_BasicField="False", IsotropicAnalyse="False", monitor_Res="False",
               monitor_Energy="False", char_recon="true" if char else "false")
    W = initial.isotropic(n, mach_t=w["mach_t"], Ma=w["Ma"], gamma=w["gamma"], k0=w["k0"],
                          seed=w["seed"])
    if kind == "reference":
        r = oracle.Ref(cfg)
        r.set_primitive(W)
        for _ in range(warm):
            r.cfl_step()
        t0 = time.perf_counter()
        for _ in range(steps):
            r.cfl_step()
        return (time.perf_counter() - t0) / steps
    os.environ["OMP_NUM_THREADS"] = "1"
    o = oracle.Oracle(cfg)
    for _ in range(warm):
        W, _, _ = o.cfl_step(W)
    t0 = time.perf_counter()
    for _ in range(steps):
        W, _, _ = o.cfl_step(W)
    return (time.perf_counter() - t0) / steps


def run_cpu(steps: int, warm: int, n_equiv: int):
    """Reference path on all host cores as independent single-rank replicas
    (the reference's one-rank build; no MPI on this host). Returns a dict."""
    import multiprocessing as mp
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    kind = "reference" if oracle.have_ref() else "port"
    cores = os.cpu_count() or 1
    ctx = mp.get_context("spawn")
    t0 = time.perf_counter()
    with ctx.Pool(cores) as pool:
        per_step = pool.map(_cpu_worker,
                            [(kind, CPU_SAMPLE_N, steps, warm, bool(WORKLOAD.get("char")))] * cores)
    wall = time.perf_counter() - t0
    cells = CPU_SAMPLE_N ** 3
    cell_rate = sum(cells / t for t in per_step)
    return {"value": cell_rate / n_equiv ** 3, "unit": "steps/s", "cores": cores, "kind": kind,
            "cell_updates_per_s": cell_rate, "s_per_step_one_core": statistics.mean(per_step),
            "sample": (f"{cores} concurrent single-rank replicas (one per host core, replicas, "
                       f"not one domain), each {steps} RK3 step(s) of the same scheme on a "
                       f"{CPU_SAMPLE_N}^3 periodic isotropic box after {warm} warm-up; "
                       f"steps/s scaled to {n_equiv}^3 by cell count; wall {wall:.1f} s")}


def run_direct(n: int, steps: int = 1):
    """One single-rank replica of the reference on the benchmark's own box
    (n^3, one host core): the figure the 64^3 replicas are scaled to n^3
    from. Returns seconds per step."""
    import multiprocessing as mp
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    kind = "reference" if oracle.have_ref() else "port"
    ctx = mp.get_context("spawn")
    t0 = time.perf_counter()
    with ctx.Pool(1) as pool:
        s_step = pool.map(_cpu_worker, [(kind, n, steps, 0, bool(WORKLOAD.get("char")))])[0]
    return {"n": n, "steps": steps, "s_per_step_one_core": s_step, "kind": kind,
            "wall_s": time.perf_counter() - t0}


def cpu_baseline(steps: int, n: int):
    try:
        return run_cpu(steps, 0, n)
    except Exception as e:  # reported, never fatal for the GPU line
        return {"value": None, "error": str(e)}


def reference_arm(args, rank, world):
    if rank != 0:
        return
    res = run_cpu(args.steps, args.warmup, args.n)
    direct = None
    if getattr(args, "direct_steps", 1) > 0:
        try:
            direct = run_direct(args.n, getattr(args, "direct_steps", 1))
            per_cell_direct = direct["s_per_step_one_core"] / args.n ** 3
            per_cell_replica = res["s_per_step_one_core"] / CPU_SAMPLE_N ** 3
            # 1.0: scaling the replicas' rate to n^3 by cell count holds
            direct["per_cell_vs_replica"] = per_cell_direct / per_cell_replica
            direct["steps_per_s_one_core"] = 1.0 / direct["s_per_step_one_core"]
        except Exception as e:  # reported, never fatal for the line
            direct = {"error": str(e)}
    line = {"impl": "reference", "metric": METRIC, "value": res["value"], "unit": "steps/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic: seeded isotropic turbulence (numpy)",
            "config": {"workload": workload_name(args.n), "n": args.n},
            "cpu_baseline": {"value": res["value"], "unit": "steps/s", "cores": res["cores"],
                             "kind": res["kind"], "sample": res["sample"]},
            "e2e": {"value": res["value"], "unit": "steps/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
            "cell_updates_per_s": res["cell_updates_per_s"],
            "direct_full_size": direct}
    print(json.dumps(line), flush=True)


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=150)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=N_DEFAULT)
    ap.add_argument("--err-steps", type=int, default=500)
    ap.add_argument("--e2e-steps", type=int, default=20)
    ap.add_argument("--cpu-sample-steps", type=int, default=1)
    ap.add_argument("--direct-steps", type=int, default=1,
                    help="reference arm: steps of one single-core replica at the full size")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--skip-fp64", action="store_true", help="only the headline form")
    ap.add_argument("--only-fp64", action="store_true",
                    help="diagnostic: time the plain FP64 form alone (for kernel captures)")
    ap.add_argument("--skip-adjoint", action="store_true", help="no adjoint cost measurement")
    ap.add_argument("--char-recon", action="store_true",
                    help="characteristic-wise reconstruction in both arms (char_recon)")
    args = ap.parse_args(argv)
    args.warmup = max(3, args.warmup)
    if args.char_recon:
        WORKLOAD["char"] = True
        args.skip_adjoint = True   # the adjoint is component-wise only
    rank, world, local = env_rank()
    if args.impl == "reference":
        reference_arm(args, rank, world)
        return
    our_arm(args, rank, world, local)


if __name__ == "__main__":
    main()
