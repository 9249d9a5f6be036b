"""Alternative kernel schedules give the same bits as the plain ones.

Two schedules of one Shu-Osher stage are built (range_kutta.cpp:11-163): the
sweeps, the viscous flux and k_update as separate launches, and the z sweep
fused with the update (NS3D_FUSE=1, read from the environment when a context
is created). Both perform the same floating-point operations per cell in the
same order, so the states, the CFL dt and the time loop's step counts must
agree exactly.

The FP32 form's sweeps with the split software-pipelined beside the
reconstruction (k_sweep_x_pipe, k_sweep_pipe; NS3D_PIPE=0 selects
k_sweep_x_warp_f32 and k_sweep_ring) evaluate the same formulas, but the
compiler contracts their double split into FMAs in its own way, so the two
agree to float rounding of the split-flux deviations rather than bit for bit;
both sit within the FP32 form's bounds against the FP64 oracle (the 256^3 RHS
in test_size_parity takes the pipelined sweeps).
"""
import os

import numpy as np
import pytest

import ns3d_cpp_b200 as ns
from ns3d_cpp_b200 import initial
from conftest import SCHEMES, ref_cfg, relerr, scheme_id
from test_gpu_parity import params_from_cfg

pytestmark = pytest.mark.gpu

SCHEDULES = {"plain": {}, "fuse_z": {"NS3D_FUSE": "1"}}
PIPE_SCHEDULES = {"plain": {"NS3D_PIPE": "0"}, "pipelined": {"NS3D_PIPE": "3"}}


def _solver(params, env):
    old = {k: os.environ.get(k) for k in ("NS3D_FUSE", "NS3D_PIPE")}
    try:
        for k in old:
            os.environ.pop(k, None)
        os.environ.update(env)
        return ns.Solver(params)
    finally:
        for k, v in old.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v


def _run_steps(params, env, W, nsteps, chunks):
    with _solver(params, env) as s:
        s.upload_primitive(W)
        for c in chunks:
            s.step(c)
        assert sum(chunks) == nsteps
        return s.download_primitive(), s.last_dt()


@pytest.mark.parametrize("precision", ["fp64", "fp32acc64"])
@pytest.mark.parametrize("kw", SCHEMES, ids=scheme_id)
def test_schedules_bit_identical(kw, precision):
    """Five CFL steps of a 64 x 32 x 48 Taylor-Green field (split as 3 + 2
    calls) in each schedule."""
    nx, ny, nz = 64, 32, 48
    cfg = ref_cfg(nx, **kw)
    cfg.update(global_ny=ny, global_nz=nz, Ly=2 * np.pi * ny / nx, Lz=2 * np.pi * nz / nx)
    p = params_from_cfg(cfg, precision=precision)
    W = initial.taylor_green(nx, Ma=0.3, perturb=0.05, seed=5)[:, :nz, :ny, :]
    W = np.ascontiguousarray(W)
    out = {name: _run_steps(p, env, W, 5, (3, 2)) for name, env in SCHEDULES.items()}
    W0, dt0 = out["plain"]
    Wf, dtf = out["fuse_z"]
    assert dtf == dt0
    for q in range(W0.shape[0]):
        assert np.array_equal(Wf[q], W0[q]), q


def test_fused_time_loop_stops_identically():
    """time_advance with output clipping and TotalTime reached mid-call."""
    n = 32
    cfg = ref_cfg(n, Ma=0.3, TotalTime=0.06, output_Timefreq=0.0173)
    p = params_from_cfg(cfg, precision="fp32acc64")
    W = initial.taylor_green(n, Ma=0.3, perturb=0.05, seed=9)
    res = {}
    for name, env in SCHEDULES.items():
        with _solver(p, env) as s:
            s.upload_primitive(W)
            segs = [s.time_advance_segment(40) for _ in range(3)]
            t, k = s.time_advance(400)
            res[name] = (segs, t, k, s.download_primitive())
    segs0, t0, k0, W0 = res["plain"]
    assert k0 > 0
    segs, t, k, Wf = res["fuse_z"]
    assert segs == segs0 and t == t0 and k == k0
    assert np.array_equal(Wf, W0)


@pytest.mark.parametrize("kw", SCHEMES + [dict(sw_entropy_eps=1e-3)], ids=scheme_id)
def test_pipelined_sweeps_match_plain(kw, oracle_mod):
    """FP32 form, 128 x 32 x 40 Taylor-Green box at Ma 0.3 (rows of four 32-cell
    chunks, the pipelined x sweep's smallest case): the RHS with and without the
    pipelined split within 1e-6 (the rounding of one float split-flux deviation
    moves a face flux by ~1e-7 of the RHS scale), as close to the FP64 oracle
    as the plain sweep's (and within the FP32 form's 5e-5 for SW + WENO5), and
    after five CFL steps within the FP32 form's 1e-5."""
    nx, ny, nz = 128, 32, 40
    cfg = ref_cfg(nx, Ma=0.3, **kw)
    cfg.update(global_ny=ny, global_nz=nz, Ly=2 * np.pi * ny / nx, Lz=2 * np.pi * nz / nx)
    p = params_from_cfg(cfg, precision="fp32acc64")
    W = initial.taylor_green(nx, Ma=0.3, perturb=0.05, seed=7)[:, :nz, :ny, :]
    W = np.ascontiguousarray(W)
    out = {}
    for name, env in PIPE_SCHEDULES.items():
        with _solver(p, env) as s:
            s.upload_primitive(W)
            rhs = s.compute_rhs()
            s.step(5)
            out[name] = (rhs, s.download_primitive(), s.last_dt())
    (r0, W0, dt0), (r1, W1, dt1) = out["plain"], out["pipelined"]
    ref = oracle_mod.Oracle(cfg).rhs(W)
    e_pipe, e0, e1 = relerr(r1, r0), relerr(r0, ref), relerr(r1, ref)
    print(f"rhs pipelined vs plain {e_pipe.max():.2e}, vs oracle {e0.max():.2e} / {e1.max():.2e}")
    assert np.all(e_pipe <= 1e-6), e_pipe
    assert np.all(e1 <= e0 + 2e-6), (e0, e1)
    if not kw:
        assert np.all(e1 <= 5e-5), e1
    assert abs(dt1 - dt0) <= 1e-8 * dt0
    # over the steps the two differ by the FP32 form's own rounding noise
    # (measured up to 3e-6 norm-wise, in w, whose maximum is the 0.05
    # perturbation), inside the 1e-5 of the FP32 form's state bound
    assert np.all(relerr(W1, W0) <= 1e-5), relerr(W1, W0)
