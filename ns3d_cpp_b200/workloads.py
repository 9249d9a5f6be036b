"""The benchmark workloads of the RK3 loop as runnable configurations.

    python -m ns3d_cpp_b200.workloads <name> [--device D] [--steps K]

Each run uploads its initial field, advances it on the GPU in chunks of the
monitor interval (no host round trip per step), and at every monitor step
evaluates what maincycle.cpp:62-92 monitors: the total kinetic energy
(compute_total_energy) and, for isotropic turbulence, the shell spectrum and
the KE / dissipation statistics (isotropic_post_process). Device time per
kernel class comes from the library's event profiling. Prints one JSON line.

Workloads (periodic [0, 2 pi)^3, gamma 1.4, Pr 0.72, CFL 0.5, C8th viscous):
  tgv32    Taylor-Green 32^3, Ma 0.1, Re 1600, SW + WENO5, FP64, 100 steps
  iso128   isotropic 128^3, Mach_t 0.3, Re 500, LF + MDCD, FP64, 200 steps,
           spectrum every 50
  iso256   isotropic 256^3, Mach_t 0.5, Re 1000, SW + WENO5, 500 steps, FP64
           and FP32-stencil forms, errors of the latter against the former
  iso512   isotropic 512^3, Mach_t 0.4, Re 2000, k0 4, FP32-stencil form,
           UPWIND_7TH and WENO5, 100 steps, per-kernel HBM roofline
  iso128char  the iso128 field with characteristic-wise reconstruction
           (char_recon), SW + WENO5, FP64 and FP32-stencil forms, 200 steps
(the adjoint workload, Taylor-Green 64^3, runs through bench.py / the tests).
The isotropic Ma is solver.in's 0.5; Sutherland S/Tref is 110.4/273.15 for the
Taylor-Green workloads, the reference's 110.4/288.15 otherwise.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import time

import numpy as np

from . import initial
from .solver import Solver, SolverParams

TWO_PI = 2.0 * math.pi

WORKLOADS = {
    "tgv32": dict(kind="tgv", n=32, Ma=0.1, Re=1600.0, fvs="stagerwarming", recons=("weno5",),
                  steps=100, monitor=10, precisions=("fp64",), sutherland=110.4 / 273.15),
    "iso128": dict(kind="iso", n=128, Ma=0.5, mach_t=0.3, Re=500.0, fvs="laxfriedrichs",
                   recons=("mdcd",), steps=200, monitor=50, precisions=("fp64",)),
    "iso256": dict(kind="iso", n=256, Ma=0.5, mach_t=0.5, Re=1000.0, fvs="stagerwarming",
                   recons=("weno5",), steps=500, monitor=100, precisions=("fp64", "fp32acc64")),
    "iso128char": dict(kind="iso", n=128, Ma=0.5, mach_t=0.3, Re=500.0, fvs="stagerwarming",
                       recons=("weno5",), steps=200, monitor=50, precisions=("fp64", "fp32acc64"),
                       char_recon=True),
    "iso512": dict(kind="iso", n=512, Ma=0.5, mach_t=0.4, Re=2000.0, fvs="stagerwarming",
                   recons=("upwind_7th", "weno5"), steps=100, monitor=50,
                   precisions=("fp32acc64",)),
}

# compulsory HBM bytes per cell of one launch (R = bytes of the compute type),
# the same accounting as bench.py
def _kernel_bytes(cls: str, rsize: int) -> float:
    w = 40.0
    fv = 12 if rsize == 4 else 9   # viscous flux values per cell (FP32: three float4 blocks)
    return {"sweep_x": w + 5 * rsize, "sweep_y": w + 10 * rsize, "sweep_z": w + 10 * rsize,
            "visc_flux": 32 + fv * rsize,
            "update": (5.0 / 3.0) * w + (5 + fv) * rsize + 48,  # stage 1 reads one state
            "sweep_z_update": (5.0 / 3.0) * w + (5 + fv) * rsize + 48}.get(cls, 0.0)


def params_for(w: dict, recon: str, precision: str, dt_fixed: float = -1.0) -> SolverParams:
    kw = dict(n=w["n"], gamma=1.4, Pr=0.72, Ma=w["Ma"], Re=w["Re"], cfl=0.5, dt_fixed=dt_fixed,
              fvs_type=w["fvs"], recon=recon, vis_scheme="c8th", Lx=TWO_PI, Ly=TWO_PI, Lz=TWO_PI,
              precision=precision)
    if "sutherland" in w:
        kw["sutherland_s_over_tref"] = w["sutherland"]
    if w.get("char_recon"):
        kw["char_recon"] = 1
    p = SolverParams.default().replace(**kw)
    if recon == "ud7l":
        p.ud7l_alpha = 1.0
    return p


def initial_for(w: dict) -> np.ndarray:
    if w["kind"] == "tgv":
        return initial.taylor_green(w["n"], Ma=w["Ma"])
    return initial.isotropic(w["n"], mach_t=w["mach_t"], Ma=w["Ma"], k0=4.0, seed=12345)


def _peak_gbs() -> float:
    here = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    try:
        with open(os.path.join(here, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"])
    except Exception:
        return 6650.0


def run_one(w: dict, W: np.ndarray, recon: str, precision: str, steps: int, device: int,
            dt_fixed: float = -1.0) -> dict:
    """Advance `steps` steps in monitor chunks; returns timings and monitors."""
    p = params_for(w, recon, precision, dt_fixed)
    ncell = w["n"] ** 3
    rsize = 8 if precision == "fp64" else 4
    out = {"recon": recon, "precision": precision, "monitors": []}
    with Solver(p, device=device) as s:
        s.upload_primitive(W)
        s.step(2)                          # warm-up
        s.upload_primitive(W)
        s.synchronize()
        s.profile(True)
        done, device_s = 0, 0.0
        t_wall = 0.0
        while done < steps:
            k = min(w["monitor"], steps - done)
            t0 = time.perf_counter()
            s.step(k)
            s.synchronize()
            t_wall += time.perf_counter() - t0
            done += k
            mon = {"step": done, "total_energy": s.compute_total_energy()}
            if w["kind"] == "iso":
                st = s.compute_turbulence_statistics()
                mon.update(kinetic_energy=st["kinetic_energy"], dissipation=st["dissipation"],
                           mach_t=st["mach_t"], u_rms=st["u_rms"])
                mon["spectrum_head"] = [float(x) for x in s.compute_energy_spectrum(12)]
            out["monitors"].append(mon)
        prof = s.profile_read()
        s.profile(False)
        out["final_spectrum"] = [float(x) for x in s.compute_energy_spectrum()]
    peak = _peak_gbs()
    kern = {}
    for cls, (ms, cnt) in prof.items():
        if not cnt:
            continue
        device_s += ms / 1e3
        b = _kernel_bytes(cls, rsize) * ncell
        per = ms / cnt
        kern[cls] = {"launches": cnt, "ms_per_launch": per,
                     "hbm_frac": (b / (per / 1e3) / 1e9) / peak if b else None}
    out.update(steps=steps, device_s=device_s, wall_s=t_wall, steps_per_s=steps / device_s,
               gcell_per_s=steps * ncell / device_s / 1e9, kernels=kern,
               step_hbm_frac=360.0 * ncell * (steps / device_s) / 1e9 / peak)
    return out


def run(name: str, device: int = 0, steps: int | None = None) -> dict:
    w = WORKLOADS[name]
    n_steps = steps or w["steps"]
    W = initial_for(w)
    res = {"workload": name, "n": w["n"], "steps": n_steps, "runs": []}
    for recon in w["recons"]:
        for prec in w["precisions"]:
            res["runs"].append(run_one(w, W, recon, prec, n_steps, device))
    if "fp64" in w["precisions"] and "fp32acc64" in w["precisions"]:
        # FP32-stencil vs FP64 at one fixed dt: end-time KE, dissipation, E(k)
        rc = w["recons"][0]
        with Solver(params_for(w, rc, "fp64"), device=device) as s:
            s.upload_primitive(W)
            dt0 = s.compute_timestep()
        a = run_one(w, W, rc, "fp64", n_steps, device, dt_fixed=dt0)
        b = run_one(w, W, rc, "fp32acc64", n_steps, device, dt_fixed=dt0)
        ma, mb = a["monitors"][-1], b["monitors"][-1]
        Ea, Eb = np.array(a["final_spectrum"]), np.array(b["final_spectrum"])
        big = Ea > 1e-6 * Ea.max()
        res["fp32_vs_fp64"] = {
            "dt": dt0,
            "total_energy": abs(mb["total_energy"] - ma["total_energy"]) / ma["total_energy"],
            "kinetic_energy": abs(mb["kinetic_energy"] - ma["kinetic_energy"]) / ma["kinetic_energy"],
            "dissipation": abs(mb["dissipation"] - ma["dissipation"]) / ma["dissipation"],
            "spectrum_max": float(np.max(np.abs(Eb[big] - Ea[big]) / Ea[big]))}
    return res


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawTextHelpFormatter)
    ap.add_argument("workload", choices=sorted(WORKLOADS))
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--steps", type=int, default=None)
    a = ap.parse_args(argv)
    res = run(a.workload, a.device, a.steps)
    for r in res["runs"]:
        r.pop("final_spectrum", None)
    print(json.dumps(res))


if __name__ == "__main__":
    main()
