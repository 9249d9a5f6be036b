"""Drop-in check: the reference's own time_advance / runge_kutta_3 call sites,
compiled from its sources with range_kutta.cpp and timestep.cpp replaced by the
C++ shim over the C ABI (oracle/_ref/libns3d_ref_gpu.so), against the
unmodified reference (oracle/_ref/libns3d_ref.so)."""
import os
import tempfile

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
