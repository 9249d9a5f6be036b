"""The C ABI library: loads, exports what include/ns3d_gpu.h declares, and its
solver.in parser agrees with the reference's read_solver_params_from_file."""
import ctypes
import os
import tempfile

import numpy as np
import pytest

import ns3d_cpp_b200 as ns
from ns3d_cpp_b200 import _lib
from ns3d_cpp_b200.solver import NS3DError, SolverParams, TurbStats


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    declared = _lib.header_functions()
    assert len(declared) >= 20
    for name in declared:
        assert hasattr(lib, name), name
    assert set(declared) == set(_lib._SIGS)


def test_struct_layouts_match():
    lib = _lib.load()
    assert lib.ns3d_params_size() == ctypes.sizeof(SolverParams)
    assert lib.ns3d_turb_stats_size() == ctypes.sizeof(TurbStats)


def test_defaults_are_solverparams_defaults():
    p = SolverParams.default()
    # field_structures.h:86-165 and the parser's grid defaults
    assert (p.gamma, p.Pr, p.Ma, p.Re, p.cfl, p.dt_fixed) == (1.4, 0.71, 0.4, 500.0, 0.1, -1.0)
    assert (p.fvs_type, p.recon, p.vis_scheme, p.char_recon) == (0, 0, 1, 0)
    assert (p.mdcd_diss, p.mdcd_disp, p.ud7l_alpha) == (0.01, 0.0463783, 0.4)
    assert (p.global_nx, p.stencil, p.ghost_layers) == (16, 6, 3)
    assert p.sutherland_s_over_tref == 110.4 / 288.15 and p.sw_entropy_eps == 0.0


SOLVER_IN = """# ============================
# Solver Parameter File
Length_ref      = 1.0
Re          = 1600
Ma          = 0.1
gamma       = 1.4
Pr          = 0.72
cfl         = 0.5
dt_fixed    = -0.0005
fvs_type    = {fvs}
recon       = {recon}
vis_scheme  = {vis}
char_recon  = False
mdcd_disp = 0.05
mdcd_diss = 0.02
ud7l_alpha = 0.7
global_nx   = 24
global_ny   = 20
global_nz   = 16
bc_xmin = Periodic
bc_xmax = Periodic
x0 = 0.5
Lx = 6.283185307179586
Ly = 3.0
Lz = 2.5
max_steps = 123
monitor_Stepfreq = 7
output_Timefreq = 0.25
TotalTime = 1.5
Post_BasicField       = False
IsotropicAnalyse      = True
monitor_Res           = False
monitor_Energy        = True
unknown_key = 3
"""


@pytest.mark.parametrize("fvs,recon,vis", [("StagerWarming", "WENO5", "C8th"),
                                           ("LaxFriedrichs", "MDCD", "C4th"),
                                           ("stagerwarming", "ud7l", "c6th"),
                                           ("LaxFriedrichs", "UPWIND_7TH", "C4th"),
                                           ("StagerWarming", "LINEAR", "C4th")])
def test_parser_matches_reference(oracle_mod, fvs, recon, vis):
    text = SOLVER_IN.format(fvs=fvs, recon=recon, vis=vis)
    with tempfile.NamedTemporaryFile("w", suffix=".in", delete=False) as f:
        f.write(text)
        path = f.name
    try:
        p = ns.read_solver_params_from_file(path)
    finally:
        os.unlink(path)
    assert p.global_nx == 24 and p.global_ny == 20 and p.global_nz == 16
    assert p.max_steps == 123 and p.monitor_Stepfreq == 7
    assert p.post_basicfield == 0 and p.isotropic_analyse == 1 and p.monitor_res == 0
    assert p.x0 == 0.5 and p.periods[0] == 1
    if not oracle_mod.have_ref():
        pytest.skip("reference build not present")
    # the same text through the reference's own parser
    lines = dict(l.split("=", 1) for l in text.splitlines() if "=" in l and not l.startswith("#"))
    r = oracle_mod.Ref({k.strip(): v.strip() for k, v in lines.items()})
    rp = r.params()
    for name in ("gamma", "Pr", "Ma", "Re", "cfl", "dt_fixed", "Cv", "Cp", "Rgas", "mu", "dx",
                 "dy", "dz", "mdcd_diss", "mdcd_disp", "ud7l_alpha", "TotalTime",
                 "output_Timefreq"):
        assert getattr(p, name) == rp[name], name
    dims = (ctypes.c_int * 9)()
    r.lib.ref_dims(r.h, dims)
    assert (p.ghost_layers, p.stencil, p.fvs_type, p.recon, p.vis_scheme) == tuple(dims[3:8])


def test_parser_errors():
    with pytest.raises(NS3DError) as e:
        ns.read_solver_params_from_file("/nonexistent/solver.in")
    assert e.value.status == 5
    with tempfile.NamedTemporaryFile("w", suffix=".in", delete=False) as f:
        f.write("Re = abc\n")
        path = f.name
    try:
        with pytest.raises(NS3DError) as e:
            ns.read_solver_params_from_file(path)
        assert e.value.status == 1
    finally:
        os.unlink(path)


def test_extension_keys():
    with tempfile.NamedTemporaryFile("w", suffix=".in", delete=False) as f:
        f.write("sw_entropy_eps = 1e-3\nsutherland_s_over_tref = 0.404\nprecision = fp32acc64\n")
        path = f.name
    try:
        p = ns.read_solver_params_from_file(path)
    finally:
        os.unlink(path)
    assert p.sw_entropy_eps == 1e-3 and p.sutherland_s_over_tref == 0.404 and p.precision == 1


def test_replace_and_derive():
    p = SolverParams.default().replace(n=32, recon="UD7L", vis_scheme="C8th", Ma=0.2,
                                       Lx=2 * np.pi, Ly=2 * np.pi, Lz=2 * np.pi)
    assert p.ghost_layers == 4 and p.stencil == 8
    assert p.Rgas == 1.0 / (0.2 * 0.2 * 1.4)
    assert p.dx == 2 * np.pi / 32


def test_create_rejects_out_of_scope_configs():
    """Configurations the product does not build are refused before any GPU use."""
    base = SolverParams.default().replace(n=16)
    lib = _lib.load()
    for kw in (dict(recon=1),):
        p = base.replace(**kw)
        ctx = ctypes.c_void_p()
        assert lib.ns3d_create(ctypes.byref(p), 0, ctypes.byref(ctx)) == 2
    p = base.copy()
    p.bc[0] = 1
    p.derive()
    ctx = ctypes.c_void_p()
    assert lib.ns3d_create(ctypes.byref(p), 0, ctypes.byref(ctx)) == 2
    p = base.replace(n=4)
    assert lib.ns3d_create(ctypes.byref(p), 0, ctypes.byref(ctx)) == 1
