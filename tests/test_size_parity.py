"""Parity at the sizes the benchmark configurations run, through the C ABI.

The oracle (OpenMP-parallel C restatement, bit-exact against the reference's
own sources) follows the GPU at full size here:

* 256^3 decaying isotropic turbulence, Steger-Warming + WENO5, C8th, Mach_t
  0.5, Re 1000: the field the benchmark times. FP64 form: RHS and two CFL
  steps (range_kutta.cpp:11-163) to 1e-12 norm-wise. FP32-stencil form: RHS
  and two steps against the FP64 oracle at the FP32 tolerances.
* the 512^3 configuration's UPWIND_7TH scheme (reconstruction.cpp:227-232),
  Mach_t 0.4, Re 2000, k0 4, run the same way on a 256^3 field.
* 128^3 isotropic, Lax-Friedrichs + MDCD, Mach_t 0.3, Re 500: ten CFL steps
  and the spectrum / statistics of the result.
* 512^3 itself (too large for the oracle at test cost): exact periodic
  translation invariance and mass telescoping of the RHS, both schemes.

Tolerances are norm-wise relative (max|a-b|/max|b| per variable).
"""
import numpy as np
import pytest

import ns3d_cpp_b200 as ns
from ns3d_cpp_b200 import initial, workloads
from conftest import ref_cfg, relerr

pytestmark = pytest.mark.gpu

TOL64 = 1e-12
# FP32-stencil form against the FP64 oracle on Mach_t 0.4-0.5 turbulence: the
# mass equation's RHS is the divergence of split fluxes whose float deviations
# (from each 64-cell segment's first cell) are O(1), so it carries ~1e-4 of its
# maximum (measured at 256^3: WENO5 5.4e-5, UPWIND_7TH 1.2e-4; the momentum and
# energy equations 1e-5..3e-5); two steps later the state agrees to ~2e-7
TOL32_RHS = 3e-4
TOL32_STATE = 1e-5


def _params(cfg, precision):
    w = dict(kind="iso", n=cfg["global_nx"], Ma=cfg["Ma"], Re=float(cfg["Re"]),
             fvs=cfg["fvs_type"].lower())
    return workloads.params_for(w, cfg["recon"].lower(), precision)


def _gpu_rhs_and_steps(cfg, W, precision, nsteps):
    with ns.Solver(_params(cfg, precision)) as s:
        s.upload_primitive(W)
        rhs = s.compute_rhs()
        s.step(nsteps)
        return rhs, s.download_primitive(), s.last_dt()


def _check_size(oracle_mod, cfg, W, nsteps=2):
    o = oracle_mod.Oracle(cfg)
    ref_rhs = o.rhs(W)
    Wo, dts = W, []
    for _ in range(nsteps):
        Wo, dt, st = o.cfl_step(Wo)
        assert st == 0
        dts.append(dt)
    rhs64, W64, dt64 = _gpu_rhs_and_steps(cfg, W, "fp64", nsteps)
    e_rhs64, e_st64 = relerr(rhs64, ref_rhs), relerr(W64, Wo)
    assert abs(dt64 - dts[-1]) <= 1e-14 * dts[-1]
    rhs32, W32, _ = _gpu_rhs_and_steps(cfg, W, "fp32acc64", nsteps)
    e_rhs32, e_st32 = relerr(rhs32, ref_rhs), relerr(W32, Wo)
    print(f"\n{cfg['global_nx']}^3 {cfg['fvs_type']}+{cfg['recon']}: FP64 rhs {e_rhs64.max():.2e} "
          f"state {e_st64.max():.2e}; FP32 rhs {e_rhs32.max():.2e} state {e_st32.max():.2e}")
    assert np.all(e_rhs64 <= TOL64), e_rhs64
    assert np.all(e_st64 <= TOL64), e_st64
    assert np.all(e_rhs32 <= TOL32_RHS), e_rhs32
    assert np.all(e_st32 <= TOL32_STATE), e_st32


def test_benchmark_field_256_weno5(oracle_mod):
    """The benchmark's own workload: isotropic 256^3, Mach_t 0.5, Re 1000,
    SW + WENO5, C8th, the seeded field bench.py times."""
    n = 256
    cfg = ref_cfg(n, Ma=0.5, Re=1000)
    W = initial.isotropic(n, mach_t=0.5, Ma=0.5, k0=4.0, seed=12345)
    _check_size(oracle_mod, cfg, W)


def test_upwind7_scheme_256(oracle_mod):
    """The 512^3 configuration's scheme (UPWIND_7TH, Mach_t 0.4, Re 2000, k0 4)
    on a 256^3 field, where the oracle can follow."""
    n = 256
    cfg = ref_cfg(n, Ma=0.5, Re=2000, recon="UPWIND_7TH")
    W = initial.isotropic(n, mach_t=0.4, Ma=0.5, k0=4.0, seed=4096)
    _check_size(oracle_mod, cfg, W)


def test_iso128_lf_mdcd_ten_steps(oracle_mod):
    """The 128^3 configuration (LF + MDCD, Mach_t 0.3, Re 500) for ten CFL
    steps, then the monitors the configuration asks for at that state."""
    w = workloads.WORKLOADS["iso128"]
    W = workloads.initial_for(w)
    cfg = ref_cfg(128, Ma=0.5, Re=500, fvs_type="LaxFriedrichs", recon="MDCD")
    o = oracle_mod.Oracle(cfg)
    Wo = W
    for _ in range(10):
        Wo, dt, st = o.cfl_step(Wo)
        assert st == 0
    with ns.Solver(workloads.params_for(w, "mdcd", "fp64")) as s:
        s.upload_primitive(W)
        s.step(10)
        assert abs(s.last_dt() - dt) <= 1e-14 * dt
        Wg = s.download_primitive()
        ke = s.compute_total_energy()
        Ek = s.compute_energy_spectrum()
        stats = s.compute_turbulence_statistics()
    err = relerr(Wg, Wo)
    print(f"\n128^3 LF+MDCD 10 steps: {err.max():.2e}")
    assert np.all(err <= TOL64), err
    assert abs(ke - o.total_energy(Wo)) <= 1e-12 * ke
    Eo = oracle_mod.spectrum(Wo[1], Wo[2], Wo[3])
    big = Eo > 1e-12 * Eo.max()
    np.testing.assert_allclose(Ek[big], Eo[big], rtol=1e-10)
    so = oracle_mod.turbulence_stats(o.turb_sums(Wo), Eo, 128 ** 3, o.d["gamma"], o.d["Rgas"])
    for k in ("kinetic_energy", "dissipation", "u_rms"):
        assert abs(stats[k] - so[k]) <= 1e-10 * abs(so[k]), k


@pytest.mark.parametrize("recon", ["upwind_7th", "weno5"])
@pytest.mark.parametrize("precision", ["fp64", "fp32acc64"])
def test_512_translation_and_mass(recon, precision):
    """512^3, Mach_t 0.4, Re 2000, k0 4: every cell runs the same operations,
    so shifting the periodic field shifts the RHS exactly (the FP32 form takes
    its split-flux offset per x row and per 64-cell y / z segment, so it is
    shifted by whole segments and not along x), and the mass equation's
    divergence telescopes to zero."""
    n = 512
    w = workloads.WORKLOADS["iso512"]
    p = workloads.params_for(w, recon, precision)
    shift = (3, -5, 7) if precision == "fp64" else (128, -64, 0)
    with ns.Solver(p) as s:
        s.init_isotropic(k0=4, mach_t=0.4)
        W = s.download_primitive()
        r1 = s.compute_rhs()
        s.upload_primitive(np.roll(W, shift, axis=(1, 2, 3)))
        del W
        r2 = s.compute_rhs()
    for q in range(5):
        assert np.array_equal(np.roll(r1[q], shift, axis=(0, 1, 2)), r2[q]), q
    mass = abs(r1[0].sum()) / np.abs(r1[0]).sum()
    assert mass < (1e-12 if precision == "fp64" else 1e-5)
