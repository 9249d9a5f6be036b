"""Binary checkpoint of a context (ns3d_checkpoint_write / _read): a run
continued from it repeats the uninterrupted run bit for bit (state, T, the
time_advance clock with its output-time clipping, the CFL minimum), in both
precision forms, and ns3d_run continued from it writes the uninterrupted run's
files; damaged, foreign and mismatched files (another grid, another gas) are
refused."""
import ctypes
import os
import struct
import tempfile

import numpy as np
import pytest

import ns3d_cpp_b200 as ns
from ns3d_cpp_b200 import initial
from conftest import ref_cfg

HEADER = 152  # bytes before the six state arrays


def params_for(cfg):
    with tempfile.NamedTemporaryFile("w", suffix=".in", delete=False) as f:
        f.write("".join(f"{k} = {v}\n" for k, v in cfg.items()))
        path = f.name
    try:
        return ns.read_solver_params_from_file(path)
    finally:
        os.unlink(path)


def setup(nx, ny, nz, seed=3, **kw):
    cfg = ref_cfg(nx, Ma=0.3, **kw)
    cfg.update(global_ny=ny, global_nz=nz, Ly=2 * np.pi * ny / nx, Lz=2 * np.pi * nz / nx,
               TotalTime=10.0, output_Timefreq=0.02)
    W = initial.taylor_green(max(nx, ny, nz), Ma=0.3, perturb=0.05, seed=seed)[:, :nz, :ny, :nx]
    return params_for(cfg), np.ascontiguousarray(W)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "fp32acc64"])
def test_continued_run_repeats_uninterrupted_run(precision):
    p, W = setup(32, 24, 16)
    p.precision = ns.solver.PRECISION[precision]
    with tempfile.TemporaryDirectory() as d, ns.Solver(p) as a, ns.Solver(p) as b:
        path = os.path.join(d, "state.ckpt")
        a.upload_primitive(W)
        t_a, k = a.time_advance(3)
        assert k == 3
        a.checkpoint_write(path)
        assert os.path.getsize(path) == HEADER + 6 * 8 * 32 * 24 * 16
        b.checkpoint_read(path)
        # the read state is the recorded one: no residual before the next step
        assert np.all(b.residuals() == 0.0)
        assert np.array_equal(a.download_primitive(with_T_c=True), b.download_primitive(with_T_c=True))
        for _ in range(2):
            ta, ka = a.time_advance(4)
            tb, kb = b.time_advance(4)
            assert (ta, ka) == (tb, kb) and ta > t_a
            assert a.last_dt() == b.last_dt()
            assert np.array_equal(a.download_primitive(with_T_c=True),
                                  b.download_primitive(with_T_c=True))
            assert np.array_equal(a.residuals(), b.residuals())


@pytest.mark.gpu
def test_checkpoint_of_a_fresh_upload():
    """No step yet: the CFL minimum is not stored and is recomputed on the next
    step; the clock starts at zero."""
    p, W = setup(16, 16, 16, seed=4)
    with tempfile.TemporaryDirectory() as d, ns.Solver(p) as a, ns.Solver(p) as b:
        path = os.path.join(d, "fresh.ckpt")
        a.upload_primitive(W)
        a.checkpoint_write(path)
        b.checkpoint_read(path)
        assert a.time_advance(2) == b.time_advance(2)
        assert np.array_equal(a.download_primitive(), b.download_primitive())


@pytest.mark.gpu
def test_damaged_and_foreign_files_are_refused():
    p, W = setup(16, 12, 8, seed=5)
    q, _ = setup(16, 12, 12, seed=5)
    with tempfile.TemporaryDirectory() as d, ns.Solver(p) as a, ns.Solver(q) as other:
        good = os.path.join(d, "good.ckpt")
        a.upload_primitive(W)
        a.step(1)
        a.checkpoint_write(good)
        blob = open(good, "rb").read()
        before = a.download_primitive()

        def refused(data, status, ctx=a):
            path = os.path.join(d, "bad.ckpt")
            with open(path, "wb") as f:
                f.write(data)
            with pytest.raises(ns.NS3DError) as e:
                ctx.checkpoint_read(path)
            assert e.value.status == status

        flipped = bytearray(blob)
        flipped[HEADER + 8 * 1000 + 3] ^= 0x10      # one bit of the payload
        refused(bytes(flipped), 5)
        refused(blob[:-8], 5)                       # truncated
        refused(b"not a checkpoint" * 8, 5)
        refused(blob[:8] + b"\x01" + blob[9:], 5)   # another version
        refused(blob, 1, ctx=other)                 # another grid
        with pytest.raises(ns.NS3DError) as e:
            a.checkpoint_read(os.path.join(d, "missing.ckpt"))
        assert e.value.status == 5
        with pytest.raises(ns.NS3DError) as e:
            a.checkpoint_write(os.path.join(d, "no", "such", "dir.ckpt"))
        assert e.value.status == 5
        # a refused read leaves the state as it was
        assert np.array_equal(a.download_primitive(), before)
        a.checkpoint_read(good)
        assert np.array_equal(a.download_primitive(), before)


def _header(p, **over):
    """A version 2 checkpoint header for params `p` (the layout the library writes)."""
    f = dict(magic=b"NS3DCKPT", version=2, nbytes=HEADER, nx=p.global_nx, ny=p.global_ny,
             nz=p.global_nz, precision=p.precision, time=0.5, out_next=0.6, dtmin_bits=0,
             dtmin_valid=0, reserved=0, dx=p.dx, dy=p.dy, dz=p.dz, gamma=p.gamma, Rgas=p.Rgas,
             mu=p.mu, Pr=p.Pr, Cp=p.Cp, S=p.sutherland_s_over_tref, steps=7, hash=0)
    f.update(over)
    h = struct.pack("<8sII4i2dQII3d6dqQ", f["magic"], f["version"], f["nbytes"], f["nx"], f["ny"],
                    f["nz"], f["precision"], f["time"], f["out_next"], f["dtmin_bits"],
                    f["dtmin_valid"], f["reserved"], f["dx"], f["dy"], f["dz"], f["gamma"],
                    f["Rgas"], f["mu"], f["Pr"], f["Cp"], f["S"], f["steps"], f["hash"])
    assert len(h) == HEADER
    return h


def test_checkpoint_header_check_on_the_host():
    """ns3d_checkpoint_check (no context, no GPU): the header must name the
    context's grid and gas; a file written under another gamma, Rgas (Ma), mu
    (Re), Pr or Sutherland constant is refused with NS3D_ERR_INVALID, so a
    stored T = p/(rho Rgas) or CFL minimum never enters a context of another
    gas; wrong magic or version is NS3D_ERR_FILE."""
    from ns3d_cpp_b200 import _lib
    lib = _lib.load()
    p, _ = setup(16, 12, 8)
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "h.ckpt")

        def status(**over):
            with open(path, "wb") as f:
                f.write(_header(p, **over))
            return lib.ns3d_checkpoint_check(path.encode(), ctypes.byref(p))

        assert status() == 0
        for k, v in (("gamma", 1.3), ("Rgas", p.Rgas * 1.01), ("mu", p.mu / 2), ("Pr", 0.7),
                     ("Cp", p.Cp + 1e-9), ("S", 110.4 / 273.15), ("nz", 12), ("dx", p.dx * 2)):
            assert status(**{k: v}) == 1, k
        assert status(magic=b"NS3DCKPX") == 5
        assert status(version=1) == 5
        assert status(nbytes=96) == 5
        assert lib.ns3d_checkpoint_check(os.path.join(d, "missing").encode(), ctypes.byref(p)) == 5


@pytest.mark.gpu
def test_checkpoint_of_another_gas_is_refused():
    p, W = setup(16, 12, 8, seed=6)
    q, _ = setup(16, 12, 8, seed=6)
    q = q.replace(Re=q.Re * 2)
    with tempfile.TemporaryDirectory() as d, ns.Solver(p) as a, ns.Solver(q) as b:
        path = os.path.join(d, "a.ckpt")
        a.upload_primitive(W)
        a.step(1)
        a.checkpoint_write(path)
        with pytest.raises(ns.NS3DError) as e:
            b.checkpoint_read(path)
        assert e.value.status == 1


def _files(root):
    out = {}
    for dirpath, _, files in os.walk(root):
        for f in files:
            full = os.path.join(dirpath, f)
            with open(full, "rb") as fh:
                out[os.path.relpath(full, root)] = fh.read()
    return out


@pytest.mark.gpu
def test_run_continued_from_a_checkpoint_writes_the_uninterrupted_files():
    """ns3d_run to step 4, checkpoint, a new context reads it and runs to step
    9: the step numbers, the residual table (not truncated again), the
    spectrum and statistics files and the Tecplot fields equal those of one
    ns3d_run to step 9, byte for byte."""
    cfg = dict(Post_BasicField="True", IsotropicAnalyse="True", monitor_Res="True",
               monitor_Energy="True", monitor_Stepfreq=2, max_steps=9)
    p, W = setup(16, 16, 16, seed=7, **cfg)
    with tempfile.TemporaryDirectory() as d:
        one, split = os.path.join(d, "one"), os.path.join(d, "split")
        with ns.Solver(p) as a:
            a.upload_primitive(W)
            t1, k1 = a.run(one, max_steps=9, verbose=False)
        with ns.Solver(p) as a:
            a.upload_primitive(W)
            _, k = a.run(split, max_steps=4, verbose=False)
            assert k == 4
            a.checkpoint_write(os.path.join(d, "s.ckpt"))
        with ns.Solver(p) as b:
            b.checkpoint_read(os.path.join(d, "s.ckpt"))
            t2, k2 = b.run(split, max_steps=9, verbose=False)
        assert (k1, k2) == (9, 5) and t1 == t2
        A, B = _files(os.path.join(one, "output")), _files(os.path.join(split, "output"))
        assert sorted(A) == sorted(B)
        rows = A["output_residuals.dat"].decode().splitlines()
        assert [int(r.split()[0]) for r in rows[2:]] == [1, 2, 4, 6, 8]
        for name in A:
            assert A[name] == B[name], name
