"""Hand-written discrete adjoint (FP64), through the C ABI.

References: central finite differences of the GPU forward with the recorded dt
sequence, and autograd of an independent FP64 PyTorch restatement of the same
discretisation (oracle/torch_ref.py, pinned against the C oracle here).
"""
import math

import numpy as np
import pytest
import torch

import ns3d_cpp_b200 as ns
from ns3d_cpp_b200 import initial
from conftest import SCHEMES, ref_cfg, relerr, scheme_id

ADJ_SCHEMES = [dict(sw_entropy_eps=1e-3), dict(fvs_type="LaxFriedrichs", recon="MDCD"),
               dict(recon="UPWIND_7TH", vis_scheme="C6th"), dict(fvs_type="LaxFriedrichs",
                                                                 vis_scheme="C4th")]


def params_from_cfg(cfg, **extra):
    from test_gpu_parity import params_from_cfg as pfc
    return pfc(cfg, **extra)


@pytest.mark.parametrize("kw", [k for k in SCHEMES if k.get("recon") != "MDCD_HYBRID"] +
                         [dict(sw_entropy_eps=1e-3)], ids=scheme_id)
def test_torch_reference_matches_oracle(oracle_mod, kw):
    """The autograd reference restates the same discretisation as the oracle."""
    from torch_ref import TorchRef
    cfg = ref_cfg(12, **kw)
    o = oracle_mod.Oracle(cfg)
    W = initial.taylor_green(12, Ma=0.1, perturb=0.05, seed=2)
    t = TorchRef(o.d)
    assert np.all(relerr(t.rhs(torch.tensor(W)).numpy(), o.rhs(W)) <= 1e-12)
    W1, _ = o.rk3(W, 1e-3)
    assert np.all(relerr(t.rk3(torch.tensor(W), 1e-3).numpy(), W1) <= 1e-14)


@pytest.mark.gpu
@pytest.mark.parametrize("kw", ADJ_SCHEMES, ids=scheme_id)
def test_rhs_vjp_dot_product(kw):
    """<lam, dR[v]> by central differences equals <R^T lam, v>."""
    n = 16
    cfg = ref_cfg(n, **kw)
    W = initial.taylor_green(n, Ma=0.1, perturb=0.05, seed=3)
    rng = np.random.default_rng(1)
    lam = rng.standard_normal(W.shape)
    v = np.stack([initial.solenoidal_field(n, seed=7)[0], *initial.solenoidal_field(n, seed=8),
                  initial.solenoidal_field(n, seed=9)[0]])
    v[0] *= 0.01 / np.abs(v[0]).max()
    v[1:4] /= np.abs(v[1:4]).max()
    v[4] *= 0.5 / np.abs(v[4]).max()
    # 4-point central difference: WENO5's weights make the RHS strongly
    # nonlinear, so the 2-point form at this h is truncation-bound (~3e-7)
    h = 1e-5
    with ns.Solver(params_from_cfg(cfg)) as s:
        r = {}
        for k in (-2, -1, 1, 2):
            s.upload_primitive(W + k * h * v)
            r[k] = s.compute_rhs()
        s.upload_primitive(W)
        g = s.rhs_vjp(lam)
    fd = float(np.sum(lam * (-r[2] + 8 * r[1] - 8 * r[-1] + r[-2])) / (12 * h))
    ad = float(np.sum(g * v))
    assert abs(fd - ad) <= 1e-7 * abs(ad), (fd, ad)


@pytest.mark.gpu
@pytest.mark.parametrize("kw", ADJ_SCHEMES, ids=scheme_id)
def test_adjoint_matches_torch_autograd(oracle_mod, kw):
    """Gradient of end-time KE after 3 steps (checkpoint every 2) against
    autograd of the FP64 PyTorch restatement, same dt sequence."""
    from torch_ref import TorchRef
    n = 12
    cfg = ref_cfg(n, **kw)
    W = initial.taylor_green(n, Ma=0.1, perturb=0.05, seed=5)
    with ns.Solver(params_from_cfg(cfg)) as s:
        s.upload_primitive(W)
        grad, J, dts = s.adjoint(3, 2)
    t = TorchRef(oracle_mod.Oracle(cfg).d)
    Wt = torch.tensor(W, requires_grad=True)
    Y = Wt
    for dt in dts:
        Y = t.rk3(Y, float(dt))
    Jt = t.kinetic_energy(Y)
    Jt.backward()
    assert abs(J - Jt.item()) <= 1e-12 * abs(J)
    assert np.all(relerr(grad, Wt.grad.numpy()) <= 1e-9), relerr(grad, Wt.grad.numpy())


def c4_setup(n=64):
    """BASELINE adjoint workload: Taylor-Green at 64^3 with a seeded 1e-3
    solenoidal perturbation, Re 400, Ma 0.2, SW (entropy fix 1e-3) + WENO5."""
    cfg = ref_cfg(n, Re=400, Ma=0.2, sw_entropy_eps=1e-3, sutherland_s_over_tref=110.4 / 273.15)
    W = initial.taylor_green(n, Ma=0.2, perturb=1e-3, seed=2024)
    return cfg, W


@pytest.mark.gpu
def test_adjoint_vs_central_fd_on_16_directions():
    """Gradient of end-time kinetic energy w.r.t. the initial velocity field,
    200 RK3 steps, checkpoint every 20, against central differences of the
    forward with the recorded dt sequence: 1e-6 relative per direction.
    Over 200 steps the map is strongly nonlinear (the entropy fix's
    sqrt(l^2 + 1e-6) near l = 0 limits its Taylor radius to h ~ 1e-5), so the
    difference is the 4-point central one, J'(d) ~ (-J(2h) + 8J(h) - 8J(-h)
    + J(-2h)) / 12h, at h = 1e-6 per unit-rms direction. What remains at that
    h is the forward's rounding (~2e-13 of J) over h: ~3e-6..1e-5 absolute in
    J'(d). So the bound is relative to |J'||d| for every direction (1e-7),
    and per direction the median must be within 1e-6 of |J'(d)|; directions
    nearly orthogonal to J' (|J'(d)| < 0.3% of |J'||d|) sit on the floor."""
    cfg, W = c4_setup()
    p = params_from_cfg(cfg)
    with ns.Solver(p) as s:
        s.upload_primitive(W)
        grad, J, dts = s.adjoint(200, 20)

        def J_of(Wx):
            s.upload_primitive(Wx)
            s.step_dts(dts)
            return s.compute_total_energy()

        assert abs(J_of(W) - J) <= 1e-14 * J
        h = 1e-6
        gnorm = math.sqrt(float(np.sum(grad[1:4] ** 2)))
        rel, rel_norm = [], []
        for k in range(16):
            d = np.zeros_like(W)
            d[1:4] = initial.solenoidal_field(W.shape[1], k0=4.0, seed=100 + k)
            d[1:4] /= math.sqrt(float(np.mean(d[1:4] ** 2)))
            fd = (-J_of(W + 2 * h * d) + 8 * J_of(W + h * d) - 8 * J_of(W - h * d) +
                  J_of(W - 2 * h * d)) / (12 * h)
            ad = float(np.sum(grad[1:4] * d[1:4]))
            rel.append(abs(fd - ad) / abs(ad))
            rel_norm.append(abs(fd - ad) / (gnorm * math.sqrt(float(np.sum(d[1:4] ** 2)))))
    print("FD vs adjoint, per direction:", ["%.1e" % r for r in rel])
    assert max(rel_norm) <= 1e-7, rel_norm
    assert float(np.median(rel)) <= 1e-6, rel


@pytest.mark.gpu
def test_adjoint_matches_fp64_reference_gradient_at_c4():
    """The same 200-step, 64^3 gradient against autograd of the FP64 PyTorch
    restatement (on the GPU, one checkpoint per step), same dt sequence."""
    from torch.utils.checkpoint import checkpoint
    import oracle
    from torch_ref import TorchRef
    cfg, W = c4_setup()
    with ns.Solver(params_from_cfg(cfg)) as s:
        s.upload_primitive(W)
        grad, J, dts = s.adjoint(200, 20)
    t = TorchRef(oracle.derived(cfg))
    Wt = torch.tensor(W, device="cuda", requires_grad=True)
    Y = Wt
    for dt in dts:
        Y = checkpoint(t.rk3, Y, float(dt), use_reentrant=False)
    Jt = t.kinetic_energy(Y)
    Jt.backward()
    gt = Wt.grad.cpu().numpy()
    assert abs(J - Jt.item()) <= 1e-12 * J
    # norm-wise over the velocity components the gradient is taken for
    err = np.sqrt(np.sum((grad[1:4] - gt[1:4]) ** 2) / np.sum(gt[1:4] ** 2))
    assert err <= 1e-9, err


class KineticEnergyAfterSteps(torch.autograd.Function):
    """J(u0, v0, w0) = kinetic energy after `nsteps` RK3 steps, forward on the
    GPU through the C ABI, backward through the hand-written adjoint
    (test-harness wrapper, not part of the library)."""

    @staticmethod
    def forward(ctx, vel, solver, W_base, nsteps, K):
        W = W_base.copy()
        W[1:4] = vel.detach().cpu().numpy()
        solver.upload_primitive(W)
        dts = []
        for _ in range(nsteps):
            solver.step(1)
            dts.append(solver.last_dt())
        J = solver.compute_total_energy()
        ctx.save_for_backward(vel)
        ctx.solver, ctx.W, ctx.dts, ctx.K = solver, W, np.array(dts), K
        return torch.tensor(J, dtype=torch.float64)

    @staticmethod
    def backward(ctx, gJ):
        ctx.solver.upload_primitive(ctx.W)
        grad, _, _ = ctx.solver.adjoint(len(ctx.dts), ctx.K, dts=ctx.dts)
        return gJ * torch.tensor(grad[1:4]), None, None, None, None


@pytest.mark.gpu
def test_autograd_function_wrapper(oracle_mod):
    from torch_ref import TorchRef
    n = 12
    cfg = ref_cfg(n, sw_entropy_eps=1e-3)
    W = initial.taylor_green(n, Ma=0.1, perturb=0.05, seed=6)
    vel = torch.tensor(W[1:4].copy(), requires_grad=True)
    with ns.Solver(params_from_cfg(cfg)) as s:
        J = KineticEnergyAfterSteps.apply(vel, s, W, 4, 3)
        J.backward()
    t = TorchRef(oracle_mod.Oracle(cfg).d)
    Wt = torch.tensor(W)
    vt = torch.tensor(W[1:4].copy(), requires_grad=True)
    Y = torch.cat([Wt[:1], vt, Wt[4:]])
    with ns.Solver(params_from_cfg(cfg)) as s:
        s.upload_primitive(W)
        _, _, dts = s.adjoint(4, 3)
    for dt in dts:
        Y = t.rk3(Y, float(dt))
    t.kinetic_energy(Y).backward()
    assert np.all(relerr(vel.grad.numpy(), vt.grad.numpy()) <= 1e-9)
