"""Generate the golden fixtures from the reference itself (oracle/_ref).

Run from the repository root where the reference tree is available:
    python tests/golden/make_golden.py
Each fixture holds the outputs of the reference's own compute_rhs,
compute_timestep + runge_kutta_3 (two CFL steps) and, for the isotropic case,
isotropic_post_process (spectrum file, 6 significant digits, and the stats row,
8 digits) for a deterministic input built by `golden_input` below, so the
inputs need not be stored; isotropic_ic.npz holds the reference's own
init_isotropic_turbulence field (rho, u, v, w, p) for the boxes IC_BOXES.
"""
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests"))

from conftest import CHAR_SCHEMES, SCHEMES, ref_cfg, scheme_id  # noqa: E402


def golden_input(n: int, Ma: float = 0.1, gamma: float = 1.4) -> np.ndarray:
    """Taylor-Green vortex plus a deterministic smooth perturbation (no RNG)."""
    x = np.arange(n) * (2 * np.pi / n)
    Z, Y, X = np.meshgrid(x, x, x, indexing="ij")
    W = np.empty((5, n, n, n))
    W[0] = 1.0 + 0.05 * np.sin(X + 2 * Y) * np.cos(3 * Z)
    W[1] = np.sin(X) * np.cos(Y) * np.cos(Z) + 0.03 * np.cos(2 * Z + Y)
    W[2] = -np.cos(X) * np.sin(Y) * np.cos(Z) + 0.02 * np.sin(3 * X)
    W[3] = 0.04 * np.sin(Y + Z)
    W[4] = 1.0 / (gamma * Ma * Ma) + (np.cos(2 * X) + np.cos(2 * Y)) * (np.cos(2 * Z) + 2.0) / 16.0
    return W


def isotropic_input(n: int, Ma: float = 0.5, gamma: float = 1.4) -> np.ndarray:
    """Deterministic multi-mode velocity field, rho = 1, T = 1."""
    x = np.arange(n) * (2 * np.pi / n)
    Z, Y, X = np.meshgrid(x, x, x, indexing="ij")
    W = np.empty((5, n, n, n))
    W[0] = 1.0
    W[1] = 0.3 * np.sin(X) * np.cos(Y) * np.cos(Z) + 0.1 * np.sin(3 * Y + Z) + 0.05 * np.cos(5 * Z)
    W[2] = -0.3 * np.cos(X) * np.sin(Y) * np.cos(Z) + 0.08 * np.cos(2 * X + 3 * Z)
    W[3] = 0.07 * np.sin(4 * X + Y) + 0.02 * np.cos(6 * Y)
    W[4] = 1.0 / (Ma * Ma * gamma)
    return W


def main():
    import oracle
    if not oracle.have_ref():
        # this script reads the reference's own sources to make the fixtures
        oracle.build(ref=True, ref_dir=os.environ.get("NS3D_REF_DIR") or "/root/reference")
    out = {}
    for kw in SCHEMES + CHAR_SCHEMES:
        n = 8
        cfg = ref_cfg(n, **kw)
        r = oracle.Ref(cfg)
        r.set_primitive(golden_input(n))
        rhs = r.rhs()
        dts = []
        for _ in range(2):
            dts.append(r.cfl_step())
        out[scheme_id(kw)] = dict(rhs=rhs, W2=r.W(), dts=np.array(dts))
    np.savez_compressed(os.path.join(HERE, "rhs_steps_8.npz"),
                        **{f"{k}/{f}": v for k, d in out.items() for f, v in d.items()})
    # one 16^3 WENO5 case
    cfg = ref_cfg(16)
    r = oracle.Ref(cfg)
    r.set_primitive(golden_input(16))
    rhs = r.rhs()
    dts = [r.cfl_step() for _ in range(2)]
    np.savez_compressed(os.path.join(HERE, "tgv_weno5_16.npz"), rhs=rhs, W2=r.W(),
                        dts=np.array(dts), ke=r.total_energy())
    # isotropic post-processing at 16^3: spectrum file + stats row
    cfg = ref_cfg(16, Ma=0.5, Re=500, fvs_type="LaxFriedrichs", recon="MDCD")
    r = oracle.Ref(cfg)
    r.set_primitive(isotropic_input(16))
    with tempfile.TemporaryDirectory() as d:
        k, Ek, stats = r.isotropic_post(d, 0.0)
    np.savez_compressed(os.path.join(HERE, "isotropic_post_16.npz"), k=k, Ek=Ek,
                        stats=np.array([stats[s] for s in sorted(stats)]),
                        stat_names=np.array(sorted(stats)), ke=r.total_energy())
    # the reference's own initial field (init_isotropic_turbulence), one fresh
    # process per box: its generator keeps a static random stream per process
    import subprocess
    ic = {}
    for nx, ny, nz in IC_BOXES:
        with tempfile.TemporaryDirectory() as d:
            out = os.path.join(d, "ic.npy")
            subprocess.run([sys.executable, __file__, "--ic", str(nx), str(ny), str(nz), out],
                           check=True, stdout=subprocess.DEVNULL)
            ic[f"{nx}x{ny}x{nz}"] = np.load(out)
    np.savez_compressed(os.path.join(HERE, "isotropic_ic.npz"), **ic)
    print("golden fixtures written")


# boxes of the initial-field fixture (nx, ny, nz)
IC_BOXES = [(16, 16, 16), (16, 12, 8)]


def ic_cfg(nx, ny, nz):
    return ref_cfg(nx, Ma=0.5, Re=500, global_ny=ny, global_nz=nz)


def _ic_case(nx, ny, nz, out):
    import oracle
    r = oracle.Ref(ic_cfg(nx, ny, nz))
    r.init_isotropic()
    np.save(out, r.W())


if __name__ == "__main__":
    if len(sys.argv) > 1 and sys.argv[1] == "--ic":
        _ic_case(int(sys.argv[2]), int(sys.argv[3]), int(sys.argv[4]), sys.argv[5])
    else:
        main()
