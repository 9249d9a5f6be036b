"""The oracle (C restatement) pinned against the reference: golden fixtures made
by the reference itself, the live reference build where present, and
known-answer tests the reference never had."""
import math
import os
import tempfile

import numpy as np
import pytest
from numpy.polynomial import polynomial as Pn

from conftest import CHAR_SCHEMES, SCHEMES, ref_cfg, relerr, scheme_id

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def golden_input(n):
    from golden.make_golden import golden_input as gi
    return gi(n)


@pytest.mark.parametrize("kw", SCHEMES + CHAR_SCHEMES, ids=scheme_id)
def test_oracle_matches_reference_golden(oracle_mod, kw):
    """RHS and two CFL steps of the oracle equal the reference's outputs."""
    g = np.load(os.path.join(GOLD, "rhs_steps_8.npz"))
    key = scheme_id(kw)
    o = oracle_mod.Oracle(ref_cfg(8, **kw))
    W = golden_input(8)
    rhs = o.rhs(W)
    assert np.all(relerr(rhs, g[f"{key}/rhs"]) <= 1e-13)
    dts = []
    for _ in range(2):
        W, dt, st = o.cfl_step(W)
        assert st == 0
        dts.append(dt)
    np.testing.assert_allclose(dts, g[f"{key}/dts"], rtol=1e-14, atol=0)
    assert np.all(relerr(W, g[f"{key}/W2"]) <= 1e-13)


def test_oracle_matches_reference_golden_16(oracle_mod):
    g = np.load(os.path.join(GOLD, "tgv_weno5_16.npz"))
    o = oracle_mod.Oracle(ref_cfg(16))
    W = golden_input(16)
    assert np.all(relerr(o.rhs(W), g["rhs"]) <= 1e-13)
    for k in range(2):
        W, dt, st = o.cfl_step(W)
        assert abs(dt - g["dts"][k]) <= 1e-15 * dt
    assert np.all(relerr(W, g["W2"]) <= 1e-13)
    # compute_total_energy after the two steps
    assert abs(o.total_energy(W) - float(g["ke"])) <= 1e-13 * abs(float(g["ke"]))


needs_ref = pytest.mark.skipif(
    not os.path.exists(os.path.join(os.path.dirname(__file__), "..", "oracle", "_ref",
                                    "libns3d_ref.so")),
    reason="reference build (oracle/_ref) not present")


@needs_ref
@pytest.mark.parametrize("kw", SCHEMES, ids=scheme_id)
def test_oracle_bit_exact_vs_live_reference(oracle_mod, kw):
    """Seeded random input, non-power-of-two box: bit-exact RHS and 3 steps."""
    from ns3d_cpp_b200 import initial
    n = 12
    cfg = ref_cfg(n, **kw)
    W = initial.taylor_green(n, Ma=0.1, perturb=0.05, seed=7)
    r = oracle_mod.Ref(cfg)
    r.set_primitive(W)
    o = oracle_mod.Oracle(cfg)
    assert np.array_equal(o.rhs(W), r.rhs())
    Wo = W
    for _ in range(3):
        dtr = r.cfl_step()
        Wo, dto, st = o.cfl_step(Wo)
        assert dtr == dto and st == 0
    assert np.array_equal(Wo, r.W())


@needs_ref
@pytest.mark.parametrize("kw", CHAR_SCHEMES, ids=scheme_id)
def test_oracle_char_recon_bit_exact_vs_live_reference(oracle_mod, kw):
    """Characteristic-wise reconstruction (du_inviscous_character): bit-exact
    RHS and 3 CFL steps against the reference on a non-power-of-two box."""
    from ns3d_cpp_b200 import initial
    n = 12
    cfg = ref_cfg(n, **kw)
    W = initial.taylor_green(n, Ma=0.1, perturb=0.05, seed=7)
    r = oracle_mod.Ref(cfg)
    r.set_primitive(W)
    o = oracle_mod.Oracle(cfg)
    rhs = o.rhs(W)
    assert np.array_equal(rhs, r.rhs())
    # the characteristic path differs from the component-wise one
    assert not np.array_equal(rhs, oracle_mod.Oracle(ref_cfg(n, **{k: v for k, v in kw.items()
                                                                  if k != "char_recon"})).rhs(W))
    Wo = W
    for _ in range(3):
        dtr = r.cfl_step()
        Wo, dto, st = o.cfl_step(Wo)
        assert dtr == dto and st == 0
    assert np.array_equal(Wo, r.W())


@needs_ref
def test_oracle_conserved_upload_matches_reference(oracle_mod):
    """upload of a conserved state: conservedToPrimitive + halo + prim2cons."""
    from ns3d_cpp_b200 import initial
    n = 8
    cfg = ref_cfg(n)
    W = initial.taylor_green(n, Ma=0.1, perturb=0.02, seed=1)
    o = oracle_mod.Oracle(cfg)
    U = o.prim2cons(W)[0]
    r = oracle_mod.Ref(cfg)
    r.set_conserved(U)
    assert np.array_equal(o.cons2prim(U), r.W())
    assert np.array_equal(o.prim2cons(o.cons2prim(U))[0], r.U())


@needs_ref
def test_time_advance_loop_matches_reference(oracle_mod):
    """dt clipping to TotalTime and the output schedule (maincycle.cpp:12-50)."""
    from ns3d_cpp_b200 import initial
    n = 8
    cfg = ref_cfg(n, TotalTime=0.05, output_Timefreq=0.0123, max_steps=40)
    W = initial.taylor_green(n, Ma=0.1)
    r = oracle_mod.Ref(cfg)
    r.set_primitive(W)
    with tempfile.TemporaryDirectory() as d:
        r.time_advance(d)
    o = oracle_mod.Oracle(cfg)
    W2, t, steps, dts = o.time_advance(W, 40, 0.05, 0.0123)
    assert abs(t - 0.05) < 1e-12
    assert np.array_equal(W2, r.W())


# ---------------------------------------------------------------------------
# Known-answer tests (the reference ships none)
# ---------------------------------------------------------------------------

@pytest.mark.parametrize("kw", SCHEMES, ids=scheme_id)
def test_freestream_preserved_exactly(oracle_mod, kw):
    o = oracle_mod.Oracle(ref_cfg(8, **kw))
    W = np.empty((5, 8, 8, 8))
    W[0], W[1], W[2], W[3], W[4] = 1.3, 0.7, -0.2, 0.4, 71.0
    r = o.rhs(W)
    if kw.get("vis_scheme") in ("C4th", "C6th"):
        # the C4/C6 sums (-f2 + 8 f1 - 8 f-1 + f-2 ...) of a constant round to
        # O(ulp^2) (as in the reference); C8 uses pairwise differences: exact 0
        assert np.max(np.abs(r)) < 1e-28
    else:
        assert np.all(r == 0.0)


@pytest.mark.parametrize("fvs", ["StagerWarming", "LaxFriedrichs"])
def test_split_sums_to_physical_flux(oracle_mod, fvs):
    o = oracle_mod.Oracle(ref_cfg(8, fvs_type=fvs))
    g = 1.4
    rng = np.random.default_rng(0)
    for _ in range(50):
        rho, u, v, w = rng.uniform(0.5, 2), *rng.uniform(-2, 2, 3)
        p = rng.uniform(0.5, 3)
        E = p / (g - 1) + 0.5 * rho * (u * u + v * v + w * w)
        for d, un in enumerate((u, v, w)):
            fp, fm = o.split([rho, u, v, w, p], d)
            n = np.eye(3)[d]
            F = np.array([rho * un, rho * u * un + p * n[0], rho * v * un + p * n[1],
                          rho * w * un + p * n[2], (E + p) * un])
            np.testing.assert_allclose(fp + fm, F, rtol=1e-13, atol=1e-13)


def test_sw_entropy_fix_zero_is_reference(oracle_mod):
    a = oracle_mod.Oracle(ref_cfg(8))
    b = oracle_mod.Oracle(dict(ref_cfg(8), sw_entropy_eps=0.0))
    W = golden_input(8)
    assert np.array_equal(a.rhs(W), b.rhs(W))
    c = oracle_mod.Oracle(dict(ref_cfg(8), sw_entropy_eps=1e-3))
    d = relerr(c.rhs(W), a.rhs(W))
    assert np.all(d > 0) and np.all(d < 1e-2)


def test_ud7l_alpha1_is_upwind7_bit_exact(oracle_mod):
    a = oracle_mod.Oracle(ref_cfg(8, recon="UD7L", ud7l_alpha=1.0))
    b = oracle_mod.Oracle(ref_cfg(8, recon="UPWIND_7TH"))
    rng = np.random.default_rng(3)
    for _ in range(200):
        win = rng.standard_normal(8)
        for flag in (1.0, -1.0):
            assert a.recon_scalar(win, flag) == b.recon_scalar(win, flag)
    W = golden_input(8)
    assert np.array_equal(a.rhs(W), b.rhs(W))


def _cell_avg(coef, i):
    ic = Pn.polyint(coef)
    return Pn.polyval(i + 0.5, ic) - Pn.polyval(i - 0.5, ic)


@pytest.mark.parametrize("recon,S,deg", [("WENO5", 6, 2), ("MDCD", 6, 3), ("MDCD_HYBRID", 6, 2),
                                         ("UPWIND_7TH", 8, 6), ("UD7L", 8, 6), ("LINEAR", 2, 0)])
def test_reconstruction_polynomial_exactness(oracle_mod, recon, S, deg):
    """Face value of cell averages of a polynomial of degree <= deg is exact."""
    o = oracle_mod.Oracle(ref_cfg(8, recon=recon, ud7l_alpha=0.4))
    mid = (S - 1) // 2
    rng = np.random.default_rng(deg)
    for d in range(deg + 1):
        coef = rng.standard_normal(d + 1)
        win = np.array([_cell_avg(coef, m - mid) for m in range(S)])
        face = Pn.polyval(0.5, coef)
        assert abs(o.recon_scalar(win, 1.0) - face) <= 1e-13 * max(1.0, abs(face))
        # the minus side sees the mirrored window: cells i+1+mid .. , face i+1/2
        winm = np.array([_cell_avg(coef, 1 + mid - m) for m in range(S)])[::-1]
        assert abs(o.recon_scalar(winm, -1.0) - face) <= 1e-13 * max(1.0, abs(face))


@pytest.mark.parametrize("vis,order", [("C4th", 4), ("C6th", 6), ("C8th", 8)])
def test_central_derivative_order(oracle_mod, vis, order):
    errs = []
    for n in (16, 32):
        o = oracle_mod.Oracle(ref_cfg(n, vis_scheme=vis))
        x = np.arange(n) * (2 * np.pi / n)
        Z, Y, X = np.meshgrid(x, x, x, indexing="ij")
        W = np.empty((5, n, n, n))
        W[0], W[1], W[2], W[3], W[4] = 1.0, np.sin(X), 0.0, 0.0, 71.4
        _, g = o.viscous_flux(W)
        errs.append(np.max(np.abs(g[0] - np.cos(X))))
    rate = math.log2(errs[0] / errs[1])
    assert rate > order - 0.3


def test_tgv_kinetic_energy_at_t0(oracle_mod):
    from ns3d_cpp_b200 import initial
    o = oracle_mod.Oracle(ref_cfg(32))
    W = initial.taylor_green(32)
    assert abs(o.total_energy(W) - (2 * np.pi) ** 3 / 8) < 1e-10


def test_spectrum_parseval(oracle_mod):
    from ns3d_cpp_b200 import initial
    W = initial.isotropic(32, mach_t=0.3, Ma=0.5, seed=5)
    Ek = oracle_mod.spectrum(W[1], W[2], W[3])
    ke = 0.5 * np.mean(W[1] ** 2 + W[2] ** 2 + W[3] ** 2)
    assert abs(Ek.sum() - ke) < 1e-12 * ke
    assert len(Ek) == 65


def test_spectrum_and_stats_match_reference_golden(oracle_mod):
    """Spectrum binning/normalisation and the KE/dissipation statistics against
    the reference's isotropic_post_process output (its spectrum file holds 6
    significant digits, which its dissipation then uses)."""
    from golden.make_golden import isotropic_input
    g = np.load(os.path.join(GOLD, "isotropic_post_16.npz"))
    cfg = ref_cfg(16, Ma=0.5, Re=500, fvs_type="LaxFriedrichs", recon="MDCD")
    W = isotropic_input(16)
    Ek = oracle_mod.spectrum(W[1], W[2], W[3])
    np.testing.assert_array_equal(g["k"], np.arange(33))
    big = g["Ek"] > 1e-30
    np.testing.assert_allclose(Ek[big], g["Ek"][big], rtol=6e-6)
    assert np.all(Ek[~big] < 1e-25)
    o = oracle_mod.Oracle(cfg)
    d = o.d
    stats = dict(zip([str(s) for s in g["stat_names"]], g["stats"]))
    # the reference's dissipation uses the 6-digit spectrum it re-reads from disk
    Ek6 = np.array([float(f"{e:.6g}") for e in Ek])
    s6 = oracle_mod.turbulence_stats(o.turb_sums(W), Ek6, 16 ** 3, d["gamma"], d["Rgas"])
    s = oracle_mod.turbulence_stats(o.turb_sums(W), Ek, 16 ** 3, d["gamma"], d["Rgas"])
    for name in ("kinetic_energy", "tke", "u_rms", "Mach_t", "taylor_Li"):
        assert abs(s[name] - stats[name]) <= 1e-7 * abs(stats[name]), name
    assert abs(s6["dissipation"] - stats["dissipation"]) <= 1e-7 * stats["dissipation"]
    # Re_lambda needs no spectrum; the Kolmogorov and Taylor scales use the
    # dissipation of the 6-digit spectrum (the stats row holds 8 digits)
    for name in ("Re_lambda", "eta", "u_eta", "tau_eta", "taylor"):
        assert abs(s6[name] - stats[name]) <= 1e-7 * abs(stats[name]), name
    assert abs(s["dissipation"] - stats["dissipation"]) <= 1e-5 * stats["dissipation"]
    assert abs(o.total_energy(W) - float(g["ke"])) <= 1e-13 * float(g["ke"])


def test_mdcd_hybrid_switch_is_discontinuous(oracle_mod):
    """mdcd_hybrid_reconstruction (reconstruction.cpp:151-225) switches between
    its linear and nonlinear stencils at min(sai1, sai2) = 0.4, so the
    reference's own FP64 RHS jumps when a perturbation carries a face across
    the threshold: on the 16^3 Taylor-Green box at Ma 0.1 a 1e-7 relative
    perturbation of every variable moves the MDCD_HYBRID RHS by more than 1e-2
    (max norm), against under 1e-3 for WENO5, while a 1e-9 perturbation of the
    velocities moves both alike. This is why the FP32-stencil form, whose
    split-flux deviations are rounded to float, is held to the FP32 bounds for
    every scheme but this one."""
    from ns3d_cpp_b200 import initial
    n = 16
    W = initial.taylor_green(n, Ma=0.1, perturb=0.05, seed=9)
    moved = {}
    for name, kw in (("hybrid", dict(vis_scheme="C6th", recon="MDCD_HYBRID")), ("weno5", {})):
        o = oracle_mod.Oracle(ref_cfg(n, **kw))
        r = o.rhs(W)
        rng = np.random.default_rng(0)
        Wa = W * (1 + 1e-7 * rng.standard_normal(W.shape))
        Wv = W.copy()
        Wv[1:4] *= 1 + 1e-9 * rng.standard_normal(Wv[1:4].shape)
        moved[name] = (relerr(o.rhs(Wa), r).max(), relerr(o.rhs(Wv), r).max())
    assert moved["hybrid"][0] > 1e-2 and moved["weno5"][0] < 1e-3, moved
    assert moved["hybrid"][1] < 1e-6 and moved["weno5"][1] < 1e-6, moved
