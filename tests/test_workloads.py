"""The benchmark workloads end to end on the GPU (FP64 parity where the oracle
can follow at test cost; conservation/monotonicity properties otherwise)."""
import numpy as np
import pytest

import ns3d_cpp_b200 as ns
from ns3d_cpp_b200 import workloads
from conftest import ref_cfg, relerr

pytestmark = pytest.mark.gpu


def test_tgv32_fp64_100_steps_match_oracle(oracle_mod):
    """Taylor-Green 32^3, SW + WENO5, C8th, CFL 0.5, Sutherland 110.4/273.15.

    Every kernel reproduces the reference's arithmetic except pow(T, 1.5) in
    Sutherland's law: CUDA's pow and glibc's differ by 1 ulp for ~7% of
    arguments (and glibc's is itself not correctly rounded for ~5%), so no
    device code can match it bit for bit. WENO5's weights amplify such 1-ulp
    differences over many steps. The control is the oracle against itself
    with pow(T,1.5) replaced by T*sqrt(T): the GPU must stay within 1e-12 for
    10 steps and, after 100, within 10x of the reference's own drift under
    that 1-ulp change."""
    w = workloads.WORKLOADS["tgv32"]
    W = workloads.initial_for(w)
    with ns.Solver(workloads.params_for(w, "weno5", "fp64")) as s:
        s.upload_primitive(W)
        s.step(10)
        Wg10 = s.download_primitive()
        s.step(90)
        Wg = s.download_primitive()
        ke = s.compute_total_energy()
    cfg = ref_cfg(32, Ma=0.1, Re=1600, sutherland_s_over_tref=110.4 / 273.15)
    o = oracle_mod.Oracle(cfg)
    c = oracle_mod.Oracle(dict(cfg, mu_variant=1))
    Wo = Wc = W
    for k in range(100):
        Wo, _, st = o.cfl_step(Wo)
        Wc, _, _ = c.cfl_step(Wc)
        assert st == 0
        if k == 9:
            assert np.all(relerr(Wg10, Wo) <= 1e-12), relerr(Wg10, Wo)
    drift_gpu = float(relerr(Wg, Wo).max())
    drift_ctl = float(relerr(Wc, Wo).max())
    print(f"100 steps: GPU vs oracle {drift_gpu:.2e}, oracle 1-ulp control {drift_ctl:.2e}")
    assert drift_gpu <= max(1e-12, 10 * drift_ctl)
    assert abs(ke - o.total_energy(Wo)) <= 1e-12 * ke
    # viscous decay of the kinetic energy from (2 pi)^3 / 8
    assert ke < (2 * np.pi) ** 3 / 8


def test_iso128_monitors_and_first_steps(oracle_mod):
    """Isotropic 128^3, LF + MDCD, 200 steps with the spectrum every 50:
    decaying energy, positive dissipation, Parseval at every monitor; the first
    two steps against the oracle."""
    w = workloads.WORKLOADS["iso128"]
    res = workloads.run("iso128")
    mons = res["runs"][0]["monitors"]
    assert [m["step"] for m in mons] == [50, 100, 150, 200]
    e = [m["total_energy"] for m in mons]
    assert all(b < a for a, b in zip(e, e[1:]))
    assert all(m["dissipation"] > 0 for m in mons)
    W = workloads.initial_for(w)
    with ns.Solver(workloads.params_for(w, "mdcd", "fp64")) as s:
        s.upload_primitive(W)
        st = s.compute_turbulence_statistics()
        Ek = s.compute_energy_spectrum()
        assert abs(Ek.sum() - st["kinetic_energy"]) <= 1e-12 * st["kinetic_energy"]
        assert abs(st["mach_t"] - 0.3) < 1e-12
        s.step(2)
        Wg = s.download_primitive()
    cfg = ref_cfg(128, Ma=0.5, Re=500, fvs_type="LaxFriedrichs", recon="MDCD")
    o = oracle_mod.Oracle(cfg)
    Wo = W
    for _ in range(2):
        Wo, _, _ = o.cfl_step(Wo)
    assert np.all(relerr(Wg, Wo) <= 1e-12)
