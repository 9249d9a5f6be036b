"""Residual monitor: compute_diagnostics (postprocess.cpp:7-98) and its
table writer write_residuals_tecplot (output.cpp:92-128).

The oracle's restatement is pinned bit-exact against the reference's own
diagnostics; the library's row writer is byte-identical to the reference's
file; the device reduction (ns3d_residuals) matches the oracle on the same
states within the tolerance of a reordered FP64 sum."""
import ctypes
import os
import tempfile

import numpy as np
import pytest

import ns3d_cpp_b200 as ns
from ns3d_cpp_b200 import _lib, initial
from conftest import ref_cfg

needs_ref = pytest.mark.skipif(
    not os.path.exists(os.path.join(os.path.dirname(__file__), "..", "oracle", "_ref",
                                    "libns3d_ref.so")),
    reason="reference build (oracle/_ref) not present")

# device sums run in a different order than the reference's single running total
RTOL_DEVICE = 1e-12


def params_for(cfg):
    with tempfile.NamedTemporaryFile("w", suffix=".in", delete=False) as f:
        f.write("".join(f"{k} = {v}\n" for k, v in cfg.items()))
        path = f.name
    try:
        return ns.read_solver_params_from_file(path)
    finally:
        os.unlink(path)


def box(nx, ny, nz, seed=3, **kw):
    cfg = ref_cfg(nx, Ma=0.3, **kw)
    cfg.update(global_ny=ny, global_nz=nz, Ly=2 * np.pi * ny / nx, Lz=2 * np.pi * nz / nx)
    W = initial.taylor_green(max(nx, ny, nz), Ma=0.3, perturb=0.05, seed=seed)[:, :nz, :ny, :nx]
    return cfg, np.ascontiguousarray(W)


def write_row(path, step, res, etot):
    r = np.ascontiguousarray(res, dtype=np.float64)
    return _lib.load().ns3d_residuals_write(path.encode(), int(step),
                                            r.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                            float(etot))


@needs_ref
@pytest.mark.parametrize("dims", [(12, 10, 8), (16, 16, 16)])
def test_oracle_residuals_match_reference(oracle_mod, dims):
    cfg, W = box(*dims)
    r = oracle_mod.Ref(cfg)
    r.set_primitive(W)
    dx = r.params()["dx"]
    for _ in range(2):
        U0 = r.U()
        assert r.cfl_step() > 0
        got = oracle_mod.residuals(r.U(), U0, dx)
        want = r.diagnostics()
        assert np.array_equal(got, want), (got, want)
        assert np.all(want > 0)


@needs_ref
def test_residual_table_is_byte_identical_to_reference(oracle_mod):
    """Rows for steps 1, 2 and 5 (step 1 starts the file with its header), then
    a second step 1 that truncates it again, as time_advance does on a restart."""
    cfg, W = box(12, 10, 8, seed=4)
    r = oracle_mod.Ref(cfg)
    r.set_primitive(W)
    with tempfile.TemporaryDirectory() as d:
        ours = os.path.join(d, "ours.dat")
        for step in (1, 2, 5, 1, 2):
            r.cfl_step()
            res = r.diagnostics()
            ref_path = r.write_residuals(d, step, energy=True)
            assert write_row(ours, step, res, r.total_energy()) == 0
        with open(ref_path, "rb") as f:
            a = f.read()
        with open(ours, "rb") as f:
            b = f.read()
    lines = b.decode().splitlines()
    assert lines[0] == 'TITLE = "Residuals vs Step"' and len(lines) == 4
    assert lines[2].split()[0] == "1" and lines[3].split()[0] == "2"
    assert oracle_mod.residuals_row(2, [float(x) for x in lines[3].split()[1:6]],
                                    float(lines[3].split()[6])) == lines[3] + "\n"
    assert a == b


def test_residual_writer_errors():
    with tempfile.TemporaryDirectory() as d:
        assert write_row(os.path.join(d, "no", "such", "dir.dat"), 1, np.zeros(5), 0.0) == 5
        lib = _lib.load()
        assert lib.ns3d_residuals_write(None, 1, None, 0.0) == 1


@pytest.mark.gpu
@pytest.mark.parametrize("scheme", [dict(), dict(recon="MDCD", fvs_type="LaxFriedrichs")])
def test_device_residuals_match_oracle(oracle_mod, scheme):
    cfg, W = box(32, 24, 16, seed=6, **scheme)
    p = params_for(cfg)
    dx = p.dx
    with ns.Solver(p) as s:
        s.upload_primitive(W)
        # upload records U0 from the state itself: nothing has changed yet
        assert np.all(s.residuals() == 0.0)
        for _ in range(3):
            U0 = s.download_conserved()
            s.step(1)
            U = s.download_conserved()
            got = s.residuals()
            want = oracle_mod.residuals(U, U0, dx)
            assert np.all(np.abs(got - want) <= RTOL_DEVICE * np.abs(want)), (got, want)


@pytest.mark.gpu
def test_device_residuals_after_multistep_calls(oracle_mod):
    """A call of several steps (step, time_advance) leaves U0 at the start of its
    last step, as the reference's loop does."""
    cfg, W = box(24, 24, 24, seed=7)
    p = params_for(cfg)
    with ns.Solver(p) as a, ns.Solver(p) as b:
        a.upload_primitive(W)
        b.upload_primitive(W)
        a.step(2)
        U0 = a.download_conserved()
        a.step(1)
        b.step(3)
        ra, rb = a.residuals(), b.residuals()
        assert np.array_equal(ra, rb)
        want = oracle_mod.residuals(a.download_conserved(), U0, p.dx)
        assert np.all(np.abs(ra - want) <= RTOL_DEVICE * np.abs(want))
        t, k = b.time_advance(2)
        assert k == 2 and np.all(b.residuals() > 0)


@needs_ref
@pytest.mark.gpu
def test_device_residuals_match_reference_fp64(oracle_mod):
    """The FP64 form's step equals the reference's step, so the device residuals
    equal the reference's diagnostics within the reordered-sum tolerance (and the
    last bits of pow(T, 1.5) in the viscosity)."""
    cfg, W = box(16, 16, 16, seed=8)
    p = params_for(cfg)
    r = oracle_mod.Ref(cfg)
    r.set_primitive(W)
    with ns.Solver(p) as s:
        s.upload_primitive(W)
        for _ in range(2):
            r.cfl_step()
            s.step(1)
            want, got = r.diagnostics(), s.residuals()
            assert np.all(np.abs(got - want) <= 1e-9 * np.abs(want)), (got, want)
