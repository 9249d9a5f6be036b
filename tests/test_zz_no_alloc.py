"""ns3d_compute_rhs_noalloc, the entry point for callers that may not allocate
device memory (their GPU memory belongs to another allocator or budget): it
must give the same RHS as the context-based ns3d_compute_rhs, call after call,
and match the oracle, while the test (not the entry point) owns every buffer
it touches. Two boxes: 24x20x16 (the per-thread x sweep and the per-cell
viscous kernel) and 64x32x32, the largest box the fixed scratch holds (65536
cells), which takes the warp-per-row x sweep and the tiled viscous kernel
(whose FP32 form reads the viscous fluxes inside the scratch as float4)."""
import ctypes

import numpy as np
import pytest

import ns3d_cpp_b200 as ns
from ns3d_cpp_b200 import _lib, initial
from conftest import ref_cfg, relerr

pytestmark = pytest.mark.gpu

TOL = 1e-12  # both sides run the same kernels; the parity tests' FP64 bound
# against the FP64 oracle: the FP64 form's parity bound, the FP32 form's RHS bound
TOL_ORACLE = {"fp64": 1e-12, "fp32acc64": 5e-5}
BOXES = [(16, 20, 24), (32, 32, 64)]  # (nz, ny, nx)


def params(precision, nz=16, ny=20, nx=24):
    p = ns.SolverParams.default().replace(
        gamma=1.4, Pr=0.72, Ma=0.1, Re=1600.0, cfl=0.5, fvs_type="stagerwarming", recon="weno5",
        vis_scheme="c8th", Lx=2 * np.pi, Ly=2 * np.pi, Lz=2 * np.pi, precision=precision)
    p.global_nx, p.global_ny, p.global_nz = nx, ny, nz
    return p.derive()


def box_input(p, seed):
    W = initial.taylor_green(p.global_nx, Ma=0.1, perturb=0.05, seed=seed)
    # crop the cube to the (nz, ny, nx) box: still periodic-smooth enough for a check
    return np.ascontiguousarray(W[:, :p.global_nz, :p.global_ny, :p.global_nx])


def oracle_cfg(p):
    cfg = ref_cfg(p.global_nx)
    cfg.update(global_ny=p.global_ny, global_nz=p.global_nz)
    return cfg


@pytest.mark.parametrize("box", BOXES, ids=lambda b: "x".join(map(str, b[::-1])))
@pytest.mark.parametrize("precision", ["fp64", "fp32acc64"])
def test_noalloc_rhs_matches_compute_rhs_two_calls(oracle_mod, precision, box):
    import torch
    lib = _lib.load()
    nz, ny, nx = box
    p = params(precision, nz=nz, ny=ny, nx=nx)
    assert nx * ny * nz <= 65536
    orc = oracle_mod.Oracle(oracle_cfg(p))
    stream = torch.cuda.current_stream().cuda_stream
    for seed in (1, 2):  # two calls in a row, different inputs
        W = box_input(p, seed)
        with ns.Solver(p) as s:
            s.upload_primitive(W)
            want = s.compute_rhs()
        d_in = [torch.from_numpy(W[q].copy()).cuda() for q in range(5)]
        d_out = torch.full((5,) + W.shape[1:], float("nan"), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        st = lib.ns3d_compute_rhs_noalloc(ctypes.byref(p), *[t.data_ptr() for t in d_in],
                                          d_out.data_ptr(), stream)
        torch.cuda.synchronize()
        assert st == 0
        got = d_out.cpu().numpy()
        assert np.all(relerr(got, want) <= TOL), relerr(got, want)
        ref = orc.rhs(W)
        assert np.all(relerr(got, ref) <= TOL_ORACLE[precision]), relerr(got, ref)


def test_noalloc_rejects_boxes_above_its_scratch():
    lib = _lib.load()
    p = params("fp64", nz=48, ny=48, nx=48)  # 110592 > NS3D_NOALLOC_MAX_CELLS
    dummy = ctypes.c_void_p(1)
    st = lib.ns3d_compute_rhs_noalloc(ctypes.byref(p), dummy, dummy, dummy, dummy, dummy, dummy,
                                      None)
    assert st == 1
