"""Field I/O in the reference's Tecplot format (host code of the library):
the writer is byte-identical to write_tecplot_field, the readers give the
state of initialize_from_tecplot[_downsample] + primitiveToConserved."""
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


def params_for(cfg):
    text = "".join(f"{k} = {v}\n" for k, v in cfg.items())
    with tempfile.NamedTemporaryFile("w", suffix=".in", delete=False) as f:
        f.write(text)
        path = f.name
    try:
        return ns.read_solver_params_from_file(path)
    finally:
        os.unlink(path)


def dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def write(p, W, path, time, rank=0):
    W = np.ascontiguousarray(W, dtype=np.float64)
    return _lib.load().ns3d_tecplot_write(ctypes.byref(p), *[dp(W[q]) for q in range(5)],
                                          path.encode(), float(time), int(rank))


def read(p, path, src=None):
    shape = (5, p.global_nz, p.global_ny, p.global_nx)
    W = np.zeros(shape)
    lib = _lib.load()
    if src is None:
        st = lib.ns3d_tecplot_read(ctypes.byref(p), path.encode(), *[dp(W[q]) for q in range(5)])
    else:
        st = lib.ns3d_tecplot_read_downsample(ctypes.byref(p), path.encode(), *src,
                                              *[dp(W[q]) for q in range(5)])
    return st, W


def box_cfg(nx, ny, nz, **kw):
    cfg = ref_cfg(nx, Ma=0.3, **kw)
    cfg.update(global_ny=ny, global_nz=nz, Ly=2 * np.pi * ny / nx, Lz=2 * np.pi * nz / nx,
               x0=0.25, y0=-0.5, z0=1.0)
    return cfg


def state(nx, ny, nz, seed=3):
    W = initial.taylor_green(max(nx, ny, nz), Ma=0.3, perturb=0.05, seed=seed)[:, :nz, :ny, :nx]
    return np.ascontiguousarray(W)


@needs_ref
@pytest.mark.parametrize("time", [0.0, 0.0123456789])
def test_writer_is_byte_identical_to_reference(oracle_mod, time):
    nx, ny, nz = 12, 10, 8
    cfg = box_cfg(nx, ny, nz)
    W = state(nx, ny, nz)
    r = oracle_mod.Ref(cfg)
    r.set_primitive(W)
    with tempfile.TemporaryDirectory() as d:
        ref_path = r.write_tecplot(d, time)
        ours = os.path.join(d, "ours.dat")
        assert write(params_for(cfg), W, ours, time) == 0
        with open(ref_path, "rb") as f:
            a = f.read()
        with open(ours, "rb") as f:
            b = f.read()
    assert a == b


@needs_ref
def test_reader_matches_reference(oracle_mod):
    """A reference-written file read back: the state equals the reference's after
    initialize_from_tecplot + apply_boundary + primitiveToConserved."""
    nx, ny, nz = 12, 10, 8
    cfg = box_cfg(nx, ny, nz)
    r = oracle_mod.Ref(cfg)
    r.set_primitive(state(nx, ny, nz, seed=5))
    with tempfile.TemporaryDirectory() as d:
        path = r.write_tecplot(d, 0.5)
        st, W = read(params_for(cfg), path)
        r2 = oracle_mod.Ref(cfg)
        assert r2.read_tecplot(path) == 0
    assert st == 0
    assert np.array_equal(W, r2.W())


@needs_ref
@pytest.mark.parametrize("target", [(8, 8, 8), (12, 10, 6), (5, 7, 9)])
def test_downsample_matches_reference(oracle_mod, target):
    sx, sy, sz = 16, 14, 12
    src_cfg = box_cfg(sx, sy, sz)
    rs = oracle_mod.Ref(src_cfg)
    rs.set_primitive(state(sx, sy, sz, seed=8))
    nx, ny, nz = target
    cfg = box_cfg(nx, ny, nz)
    with tempfile.TemporaryDirectory() as d:
        path = rs.write_tecplot(d, 0.0)
        st, W = read(params_for(cfg), path, src=(sx, sy, sz))
        r = oracle_mod.Ref(cfg)
        assert r.read_tecplot(path, src=(sx, sy, sz)) == 0
    assert st == 0
    assert np.array_equal(W, r.W())


def test_missing_and_truncated_files():
    cfg = box_cfg(8, 8, 8)
    p = params_for(cfg)
    st, _ = read(p, "/nonexistent/field.dat")
    assert st == 5
    W = state(8, 8, 8)
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "f.dat")
        assert write(p, W, path, 0.0) == 0
        with open(path) as f:
            lines = f.readlines()
        with open(path, "w") as f:
            f.writelines(lines[:-3])       # three records short
        st, _ = read(p, path)
        assert st == 5
        assert write(p, W, os.path.join(d, "no", "such", "dir.dat"), 0.0) == 5


def test_round_trip_through_the_text_format():
    """Write then read (9 significant digits): the state back within the
    format's rounding; a larger box exercises the threaded formatter/parser."""
    nx, ny, nz = 64, 48, 40
    cfg = box_cfg(nx, ny, nz)
    p = params_for(cfg)
    W = state(nx, ny, nz, seed=9)
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "f.dat")
        assert write(p, W, path, 1.0) == 0
        st, W2 = read(p, path)
        with open(path) as f:
            head = [next(f) for _ in range(4)]
    assert st == 0
    assert head[2].startswith(f"ZONE T=\"rank_0 time=1.00000000e+00\" I={nx} J={ny} K={nz}")
    assert np.all(np.abs(W2 - W) <= 5e-9 * np.abs(W) + 1e-300)
    # the first record: x0, y0, z0 and the first cell
    x, y, z = (float(t) for t in head[3].split()[:3])
    assert (x, y, z) == (0.25, -0.5, 1.0)


@pytest.mark.gpu
def test_context_write_and_read():
    """ns3d_write_tecplot / ns3d_read_tecplot: the file of the state equals the
    array writer's; reading it back equals the array reader's result."""
    nx, ny, nz = 32, 24, 16
    cfg = box_cfg(nx, ny, nz)
    p = params_for(cfg)
    W = state(nx, ny, nz, seed=2)
    with tempfile.TemporaryDirectory() as d:
        a, b = os.path.join(d, "ctx.dat"), os.path.join(d, "arr.dat")
        with ns.Solver(p) as s:
            s.upload_primitive(W)
            s.step(2)
            Wg = s.download_primitive()
            s.write_tecplot(a, 0.75)
            assert write(p, Wg, b, 0.75) == 0
            with open(a, "rb") as f1, open(b, "rb") as f2:
                assert f1.read() == f2.read()
            s.read_tecplot(a)
            Wr = s.download_primitive()
        st, Wa = read(p, a)
    assert st == 0
    assert np.array_equal(Wr, Wa)
