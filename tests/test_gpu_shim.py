"""Drop-in check: the reference's own time_advance / runge_kutta_3 call sites,
compiled from its sources with range_kutta.cpp, timestep.cpp, postprocess.cpp
and output.cpp replaced by the C++ shim over the C ABI
(oracle/_ref/libns3d_ref_gpu.so), against the unmodified reference
(oracle/_ref/libns3d_ref.so). The shim keeps the state on the GPU between
calls; the driver syncs Field3D before reading it (ns3d_shim_sync)."""
import os
import tempfile
import time

import numpy as np
import pytest

from conftest import ref_cfg, relerr

pytestmark = pytest.mark.gpu

ORACLE_DIR = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle")
HAVE = all(os.path.exists(os.path.join(ORACLE_DIR, "_ref", f))
           for f in ("libns3d_ref.so", "libns3d_ref_gpu.so"))
needs_builds = pytest.mark.skipif(not HAVE, reason="reference builds (oracle/_ref) not present")

FIELDS = ("rho", "u", "v", "w", "p", "T", "c", "rhou", "rhov", "rhow", "E")


def full(r, name):
    g = r.ng
    out = np.empty((r.nz + 2 * g, r.ny + 2 * g, r.nx + 2 * g))
    assert r.lib.ref_get_full(r.h, name.encode(), out.ctypes.data_as(
        __import__("ctypes").POINTER(__import__("ctypes").c_double))) == 0
    return out


@needs_builds
@pytest.mark.parametrize("kw", [dict(), dict(fvs_type="LaxFriedrichs", recon="MDCD",
                                             vis_scheme="C6th")],
                         ids=["sw-weno5-c8", "lf-mdcd-c6"])
def test_reference_time_advance_through_shim(oracle_mod, kw):
    from ns3d_cpp_b200 import initial
    n = 12
    cfg = ref_cfg(n, TotalTime=0.03, output_Timefreq=0.011, max_steps=50, **kw)
    W = initial.taylor_green(n, Ma=0.1, perturb=0.05, seed=4)
    a = oracle_mod.Ref(cfg)
    b = oracle_mod.Ref(cfg, library=oracle_mod.REF_GPU_SO)
    a.set_primitive(W)
    b.set_primitive(W)
    with tempfile.TemporaryDirectory() as d:
        a.time_advance(d)
        b.time_advance(d)
    g = a.ng
    inner = (slice(g, -g), slice(g, -g))
    for name in FIELDS:
        fa, fb = full(a, name), full(b, name)
        # interior and ghost faces (what the reference reads); edges/corners too
        assert np.all(relerr(fb[None], fa[None]) <= 1e-12), name
        assert np.array_equal(fb[:, inner[0], inner[1]] == 0, fa[:, inner[0], inner[1]] == 0)


@needs_builds
def test_shim_compute_rhs_and_timestep(oracle_mod):
    from ns3d_cpp_b200 import initial
    n = 12
    cfg = ref_cfg(n)
    W = initial.taylor_green(n, Ma=0.1, perturb=0.05, seed=8)
    a = oracle_mod.Ref(cfg)
    b = oracle_mod.Ref(cfg, library=oracle_mod.REF_GPU_SO)
    a.set_primitive(W)
    b.set_primitive(W)
    assert a.timestep() == b.timestep()
    assert np.all(relerr(b.rhs(), a.rhs()) <= 1e-12)


def _tree(root):
    out = []
    for dirpath, _, files in os.walk(root):
        out += [os.path.relpath(os.path.join(dirpath, f), root) for f in files]
    return sorted(out)


def _table(path, skip):
    with open(path) as f:
        rows = f.read().splitlines()[skip:]
    return np.array([[float(x) for x in r.split()] for r in rows])


@needs_builds
def test_reference_monitored_time_advance_through_shim(oracle_mod):
    """time_advance with every monitor and output switched on: the residual
    table, energies, spectrum files, statistics rows and Tecplot fields the
    shim's postprocess/output functions write from the resident device state
    match the reference's files to the digits printed, and the final Field3D
    (synced once at the end) matches the reference's."""
    from ns3d_cpp_b200 import initial
    n = 16
    cfg = ref_cfg(n, Ma=0.3, Post_BasicField="True", IsotropicAnalyse="True",
                  monitor_Res="True", monitor_Energy="True", monitor_Stepfreq=2, max_steps=9,
                  TotalTime=10.0, output_Timefreq=0.1)
    W = initial.taylor_green(n, Ma=0.3, perturb=0.05, seed=5)
    a = oracle_mod.Ref(cfg)
    b = oracle_mod.Ref(cfg, library=oracle_mod.REF_GPU_SO)
    a.set_primitive(W)
    b.set_primitive(W)
    with tempfile.TemporaryDirectory() as d:
        da, db = os.path.join(d, "ref"), os.path.join(d, "shim")
        os.makedirs(da)
        os.makedirs(db)
        a.time_advance(da)
        b.time_advance(db)
        files = _tree(os.path.join(da, "output"))
        assert files == _tree(os.path.join(db, "output"))
        assert "output_residuals.dat" in files and "turbulence_stats.dat" in files
        assert sum(f.startswith("time_") for f in files) >= 1
        for f in files:
            x, y = os.path.join(da, "output", f), os.path.join(db, "output", f)
            if f == "output_residuals.dat":
                A, B = _table(x, 2), _table(y, 2)
                assert np.array_equal(A[:, 0], B[:, 0])
                assert np.allclose(B, A, rtol=1e-6, atol=0)
            elif f == "turbulence_stats.dat":
                A, B = _table(x, 1), _table(y, 1)
                assert np.array_equal(A[:, 0], B[:, 0])
                assert np.allclose(B, A, rtol=1e-5, atol=0)
            elif f.endswith("_spectrum.dat"):
                A, B = _table(x, 0), _table(y, 0)
                assert np.array_equal(A[:, 0], B[:, 0])
                assert np.all(np.abs(B[:, 1] - A[:, 1]) <= 2e-5 * np.abs(A[:, 1])
                              + 1e-12 * np.max(np.abs(A[:, 1])))
            else:
                A, B = _table(x, 3), _table(y, 3)
                assert np.allclose(B, A, rtol=1e-7, atol=1e-12)
    for name in FIELDS:
        assert np.all(relerr(full(b, name)[None], full(a, name)[None]) <= 1e-12), name


@needs_builds
def test_shim_resident_equals_eager_and_rates(oracle_mod):
    """The resident state gives the same bits as uploading before and
    downloading after every call (NS3D_SHIM_SYNC=eager), and costs less:
    the reference's time_advance through the shim at 128^3, steps/s of both
    modes printed (the reference's own recordConservedTo0 host copies stay in
    both)."""
    from ns3d_cpp_b200 import initial
    n, steps = 128, 6
    cfg = ref_cfg(n, Ma=0.5, Re=1000, max_steps=steps, TotalTime=100.0, output_Timefreq=100.0)
    W = initial.isotropic(n, mach_t=0.5, Ma=0.5, seed=7)
    out, rate = {}, {}
    for mode in ("resident", "eager"):
        if mode == "eager":
            os.environ["NS3D_SHIM_SYNC"] = "eager"
        try:
            b = oracle_mod.Ref(cfg, library=oracle_mod.REF_GPU_SO)
            b.set_primitive(W)
            with tempfile.TemporaryDirectory() as d:
                b.time_advance(d)   # warm-up: context, module load
                b.set_primitive(W)
                t0 = time.perf_counter()
                b.time_advance(d)
                rate[mode] = steps / (time.perf_counter() - t0)
            out[mode] = {name: full(b, name) for name in ("rho", "u", "p", "E")}
        finally:
            os.environ.pop("NS3D_SHIM_SYNC", None)
    print(f"\nreference time_advance through the shim, {n}^3: resident {rate['resident']:.2f} "
          f"steps/s, eager {rate['eager']:.2f} steps/s")
    for name in out["resident"]:
        assert np.array_equal(out["resident"][name], out["eager"][name]), name
    assert rate["resident"] > rate["eager"]
