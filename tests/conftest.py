import math
import os
import shutil
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

TWO_PI = "6.283185307179586"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")
    config.addinivalue_line("markers", "slow: larger sizes")


def _have_gpu() -> bool:
    if shutil.which("nvidia-smi") is None:
        return False
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return True


HAVE_GPU = _have_gpu()


def pytest_collection_modifyitems(config, items):
    if HAVE_GPU:
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


def ref_cfg(n, **kw):
    """Reference-format solver.in keys for a periodic [0, 2pi)^3 box."""
    c = dict(gamma=1.4, Pr=0.72, Ma=0.1, Re=1600, cfl=0.5, dt_fixed=-1,
             fvs_type="StagerWarming", recon="WENO5", vis_scheme="C8th",
             global_nx=n, global_ny=n, global_nz=n, Lx=TWO_PI, Ly=TWO_PI, Lz=TWO_PI,
             Post_BasicField="False", IsotropicAnalyse="False", monitor_Res="False",
             monitor_Energy="False")
    c.update(kw)
    return c


# the scheme combinations every parity test walks through
SCHEMES = [
    dict(),
    dict(fvs_type="LaxFriedrichs", recon="MDCD"),
    dict(recon="UPWIND_7TH"),
    dict(recon="UD7L", ud7l_alpha=0.4),
    dict(vis_scheme="C4th"),
    dict(vis_scheme="C6th", recon="MDCD_HYBRID"),
    dict(recon="LINEAR", vis_scheme="C4th"),
    dict(fvs_type="LaxFriedrichs", recon="WENO5", vis_scheme="C6th"),
]


# characteristic-wise reconstruction (du_inviscous_character) over the
# splittings and reconstruction families
CHAR_SCHEMES = [
    dict(char_recon="true"),
    dict(char_recon="true", fvs_type="LaxFriedrichs", recon="MDCD"),
    dict(char_recon="true", recon="UPWIND_7TH", vis_scheme="C4th"),
    dict(char_recon="true", recon="MDCD_HYBRID", vis_scheme="C6th"),
    dict(char_recon="true", fvs_type="LaxFriedrichs", recon="LINEAR"),
]


def scheme_id(kw):
    return "-".join(f"{k}={v}" for k, v in kw.items()) or "default"


def relerr(a, b):
    """Per-variable max|a-b| / max|b| (norm-wise relative error)."""
    a = np.asarray(a)
    b = np.asarray(b)
    ax = tuple(range(1, a.ndim))
    den = np.max(np.abs(b), axis=ax)
    den = np.where(den == 0, 1.0, den)
    return np.max(np.abs(a - b), axis=ax) / den


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle
    oracle.build()
    return oracle
