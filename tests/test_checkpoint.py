"""Binary checkpoint of a context (ns3d_checkpoint_write / _read): a run
continued from it repeats the uninterrupted run bit for bit (state, T, the
time_advance clock with its output-time clipping, the CFL minimum), in both
precision forms; damaged, foreign and mismatched files are refused."""
import os
import tempfile

import numpy as np
import pytest

import ns3d_cpp_b200 as ns
from ns3d_cpp_b200 import initial
from conftest import ref_cfg


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
        assert os.path.getsize(path) == 96 + 6 * 8 * 32 * 24 * 16
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
        flipped[96 + 8 * 1000 + 3] ^= 0x10          # one bit of the payload
        refused(bytes(flipped), 5)
        refused(blob[:-8], 5)                       # truncated
        refused(b"not a checkpoint" * 8, 5)
        refused(blob[:8] + b"\x02" + blob[9:], 5)   # another version
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
