"""Python bindings for the two CPU oracles. TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's ``cpu_baseline`` leg may
import this module, and only as the checker. The product package never does.

* :class:`Oracle` wraps ``_build/libns3d_oracle.so``, the C restatement
  (``ns3d_oracle.c``) of the reference's RHS + RK3 loop.
* :class:`Ref` wraps ``_ref/libns3d_ref.so``: the reference's own sources,
  compiled from the reference tree by ``oracle/Makefile`` (present only where
  the reference tree was available at build time).
* :func:`spectrum` / :func:`turbulence_stats` restate the shell spectrum and the
  kinetic-energy/dissipation statistics in numpy.

Arrays use the interior-only layout ``(nz, ny, nx)`` (x fastest); a state ``W``
is the primitive tuple (rho, u, v, w, p) stacked as shape ``(5, nz, ny, nx)``.
"""
from __future__ import annotations

import ctypes
import math
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "libns3d_oracle.so")
REF_SO = os.path.join(HERE, "_ref", "libns3d_ref.so")
# the reference's source tree, for building oracle/_ref: the build() argument,
# else $NS3D_REF_DIR; without either only the C restatement is built
REF_DIR = os.environ.get("NS3D_REF_DIR", "")

# reference enum orders, field_structures.h:112-131
FVS = {"stagerwarming": 0, "laxfriedrichs": 1}
RECON = {"weno5": 0, "wcns": 1, "linear": 2, "mdcd": 3, "mdcd_hybrid": 4, "upwind_7th": 5,
         "ud7l": 6}
VIS = {"c8th": 0, "c6th": 1, "c4th": 2}
SUTHERLAND_REF = 110.4 / 288.15          # field_structures.h:100


def build(ref: bool | None = None, ref_dir: str | None = None) -> None:
    """Compile the restatement (always) and the reference build (when the
    reference tree `ref_dir`, or $NS3D_REF_DIR, exists)."""
    ref_dir = ref_dir or REF_DIR
    targets = ["oracle"]
    if ref is None:
        ref = bool(ref_dir) and os.path.isdir(ref_dir)
    args = ["make", "-s", "-C", HERE, "-j8"]
    if ref:
        targets.append("ref")
        gpu_lib = os.path.join(os.path.dirname(HERE), "ns3d_cpp_b200", "libns3d_b200.so")
        if os.path.exists(gpu_lib):
            targets.append("refgpu")
        args.append(f"REF_DIR={ref_dir}")
    subprocess.run(args + targets, check=True)


def have_ref() -> bool:
    return os.path.exists(REF_SO)


# --------------------------------------------------------------------------
# solver.in (reference format, initialization.cpp:199-308)
# --------------------------------------------------------------------------

def solver_in_text(cfg: dict) -> str:
    """Render a solver.in from a dict of reference keys (values as written)."""
    lines = [f"{k} = {v}" for k, v in cfg.items()]
    return "\n".join(lines) + "\n"


def derived(cfg: dict) -> dict:
    """Derived parameters exactly as read_solver_params_from_file computes them
    (initialization.cpp:324-326, 374-377) from reference-format keys."""
    g = float(cfg.get("gamma", 1.4))
    ma = float(cfg.get("Ma", 0.4))
    re = float(cfg.get("Re", 500.0))
    n = [int(cfg.get(f"global_n{a}", 16)) for a in "xyz"]
    L = [float(cfg.get(f"L{a}", 1.0)) for a in "xyz"]
    Cv = 1.0 / (g * (g - 1.0) * ma * ma)
    return dict(gamma=g, Pr=float(cfg.get("Pr", 0.71)), Ma=ma, Re=re, Cv=Cv, Cp=Cv * g,
                Rgas=1.0 / (ma * ma * g), mu=1.0 / re, dx=L[0] / n[0], dy=L[1] / n[1],
                dz=L[2] / n[2], nx=n[0], ny=n[1], nz=n[2],
                fvs=FVS[str(cfg.get("fvs_type", "StagerWarming")).lower()],
                recon=RECON[str(cfg.get("recon", "WENO5")).lower()],
                vis=VIS[str(cfg.get("vis_scheme", "C6th")).lower()],
                mdcd_diss=float(cfg.get("mdcd_diss", 0.01)),
                mdcd_disp=float(cfg.get("mdcd_disp", 0.0463783)),
                ud7l_alpha=float(cfg.get("ud7l_alpha", 0.4)),
                cfl=float(cfg.get("cfl", 0.1)), dt_fixed=float(cfg.get("dt_fixed", -1.0)),
                sw_eps=float(cfg.get("sw_entropy_eps", 0.0)),
                sutherland_s=float(cfg.get("sutherland_s_over_tref", SUTHERLAND_REF)),
                # initialization.cpp:260-261 (values lower-cased before the test)
                char_recon=int(str(cfg.get("char_recon", "false")).lower() in ("yes", "true")))


# --------------------------------------------------------------------------
# C restatement
# --------------------------------------------------------------------------

class OrcParams(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in
                ("gamma", "Pr", "Ma", "Re", "Cv", "Cp", "Rgas", "mu", "dx", "dy", "dz",
                 "mdcd_diss", "mdcd_disp", "ud7l_alpha", "sw_eps", "sutherland_s")] + \
              [(n, ctypes.c_int) for n in ("nx", "ny", "nz", "fvs", "recon", "vis", "mu_variant",
                                           "char_recon")]


def _dp(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


_ORC = None


def _orc_lib():
    global _ORC
    if _ORC is None:
        if not os.path.exists(ORACLE_SO):
            build(ref=False)
        lib = ctypes.CDLL(ORACLE_SO)
        P = ctypes.POINTER(OrcParams)
        D = ctypes.POINTER(ctypes.c_double)
        lib.orc_rhs.argtypes = [P, D, D]
        lib.orc_rk3.argtypes = [P, D, D, ctypes.c_double]
        lib.orc_rk3.restype = ctypes.c_long
        lib.orc_timestep.argtypes = [P, D, ctypes.c_double]
        lib.orc_timestep.restype = ctypes.c_double
        lib.orc_total_energy.argtypes = [P, D]
        lib.orc_total_energy.restype = ctypes.c_double
        lib.orc_prim2cons.argtypes = [P, D, D, D, D]
        lib.orc_cons2prim.argtypes = [P, D, D]
        lib.orc_face_fluxes.argtypes = [P, D, ctypes.c_int, D]
        lib.orc_viscous_flux.argtypes = [P, D, D, D]
        lib.orc_turb_sums.argtypes = [P, D, D]
        lib.orc_recon_scalar.argtypes = [P, D, ctypes.c_int, ctypes.c_double]
        lib.orc_recon_scalar.restype = ctypes.c_double
        lib.orc_split.argtypes = [P, D, ctypes.c_int, D, D]
        _ORC = lib
    return _ORC


class Oracle:
    """The C restatement on an interior-only periodic box of size (nx, ny, nz)."""

    def __init__(self, cfg: dict):
        self.cfg = dict(cfg)
        d = derived(cfg)
        self.d = d
        d.setdefault("mu_variant", int(cfg.get("mu_variant", 0)))
        self.p = OrcParams(**{f: d[f] for f, _ in OrcParams._fields_})
        self.shape = (d["nz"], d["ny"], d["nx"])
        self.lib = _orc_lib()

    def _w(self, W):
        W = np.ascontiguousarray(W, dtype=np.float64)
        assert W.shape == (5,) + self.shape, W.shape
        return W

    def rhs(self, W):
        W = self._w(W)
        out = np.empty_like(W)
        self.lib.orc_rhs(ctypes.byref(self.p), _dp(W), _dp(out))
        return out

    def prim2cons(self, W):
        W = self._w(W)
        U = np.empty_like(W)
        T = np.empty(self.shape)
        c = np.empty(self.shape)
        self.lib.orc_prim2cons(ctypes.byref(self.p), _dp(W), _dp(U), _dp(T), _dp(c))
        return U, T, c

    def cons2prim(self, U):
        U = self._w(U)
        W = np.empty_like(U)
        self.lib.orc_cons2prim(ctypes.byref(self.p), _dp(U), _dp(W))
        return W

    def rk3(self, W, dt, U0=None):
        """One RK3 step (range_kutta.cpp:102). Returns (W_new, status)."""
        W = self._w(W).copy()
        if U0 is None:
            U0 = self.prim2cons(W)[0]
        U0 = self._w(U0)
        st = self.lib.orc_rk3(ctypes.byref(self.p), _dp(W), _dp(U0), float(dt))
        return W, int(st)

    def timestep(self, W, cfl=None):
        return self.lib.orc_timestep(ctypes.byref(self.p), _dp(self._w(W)),
                                     float(self.d["cfl"] if cfl is None else cfl))

    def cfl_step(self, W):
        """recordConservedTo0 + compute_timestep + runge_kutta_3 (maincycle.cpp:14-24)."""
        dt = self.d["dt_fixed"] if self.d["dt_fixed"] >= 0.0 else self.timestep(W)
        W2, st = self.rk3(W, dt)
        return W2, dt, st

    def total_energy(self, W):
        return self.lib.orc_total_energy(ctypes.byref(self.p), _dp(self._w(W)))

    def face_fluxes(self, W, direction):
        W = self._w(W)
        out = np.empty_like(W)
        self.lib.orc_face_fluxes(ctypes.byref(self.p), _dp(W), int(direction), _dp(out))
        return out

    def viscous_flux(self, W):
        W = self._w(W)
        Fv = np.empty((12,) + self.shape)
        g = np.empty((12,) + self.shape)
        self.lib.orc_viscous_flux(ctypes.byref(self.p), _dp(W), _dp(Fv), _dp(g))
        return Fv, g

    def turb_sums(self, W):
        out = np.zeros(12)
        self.lib.orc_turb_sums(ctypes.byref(self.p), _dp(self._w(W)), _dp(out))
        return out

    def split(self, w5, direction):
        """(F+, F-) of one cell state (rho,u,v,w,p) along `direction`."""
        a = np.ascontiguousarray(w5, dtype=np.float64)
        fp = np.empty(5)
        fm = np.empty(5)
        self.lib.orc_split(ctypes.byref(self.p), _dp(a), int(direction), _dp(fp), _dp(fm))
        return fp, fm

    def time_advance(self, W, max_steps, total_time, output_timefreq):
        """The step loop of time_advance (maincycle.cpp:12-50) without monitor
        output: returns (W, current_time, steps_done, dts)."""
        eps = 1e-12
        t = 0.0
        out_next = output_timefreq
        dts = []
        steps = 0
        for _step in range(1, max_steps + 1):
            if abs(total_time - t) <= eps:
                break
            dt = self.d["dt_fixed"]
            if self.d["dt_fixed"] < 0.0:
                dt = self.timestep(W)
            if t >= out_next - eps:
                out_next += output_timefreq
            if t + dt > total_time:
                dt = total_time - t
            if t + dt > out_next:
                dt = out_next - t
                out_next += output_timefreq
            if dt <= eps:
                break
            t += dt
            W, st = self.rk3(W, dt)
            dts.append(dt)
            steps += 1
            if st:
                raise RuntimeError("non-physical state")
            if t >= total_time:
                break
        return W, t, steps, dts

    def recon_scalar(self, window, flag):
        a = np.ascontiguousarray(window, dtype=np.float64)
        return self.lib.orc_recon_scalar(ctypes.byref(self.p), _dp(a), len(a), float(flag))


# --------------------------------------------------------------------------
# The reference itself (compiled from its sources)
# --------------------------------------------------------------------------

_REF = {}
# the reference's sources with range_kutta.cpp / timestep.cpp replaced by the
# product's C++ shim (the drop-in check; needs the GPU library at run time)
REF_GPU_SO = os.path.join(HERE, "_ref", "libns3d_ref_gpu.so")


def _ref_lib(path=REF_SO):
    if path not in _REF:
        lib = ctypes.CDLL(path)
        D = ctypes.POINTER(ctypes.c_double)
        lib.ref_create.restype = ctypes.c_void_p
        lib.ref_create.argtypes = [ctypes.c_char_p]
        lib.ref_destroy.argtypes = [ctypes.c_void_p]
        lib.ref_last_error.restype = ctypes.c_char_p
        lib.ref_last_error.argtypes = [ctypes.c_void_p]
        lib.ref_dims.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int)]
        lib.ref_params.argtypes = [ctypes.c_void_p, D]
        lib.ref_set_primitive.argtypes = [ctypes.c_void_p, D, D, D, D, D]
        lib.ref_set_conserved.argtypes = [ctypes.c_void_p, D, D, D, D, D]
        for f in ("ref_get", "ref_get_full", "ref_get_face"):
            getattr(lib, f).argtypes = [ctypes.c_void_p, ctypes.c_char_p, D]
        lib.ref_record0.argtypes = [ctypes.c_void_p]
        lib.ref_timestep.argtypes = [ctypes.c_void_p]
        lib.ref_timestep.restype = ctypes.c_double
        lib.ref_compute_rhs.argtypes = [ctypes.c_void_p]
        lib.ref_rk3.argtypes = [ctypes.c_void_p, ctypes.c_double]
        lib.ref_cfl_step.argtypes = [ctypes.c_void_p]
        lib.ref_cfl_step.restype = ctypes.c_double
        lib.ref_time_advance.argtypes = [ctypes.c_void_p, ctypes.c_char_p]
        lib.ref_total_energy.argtypes = [ctypes.c_void_p]
        lib.ref_total_energy.restype = ctypes.c_double
        lib.ref_isotropic_post.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_double]
        lib.ref_init_isotropic.argtypes = [ctypes.c_void_p]
        lib.ref_diagnostics.argtypes = [ctypes.c_void_p, D]
        lib.ref_write_residuals.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int,
                                            ctypes.c_int]
        lib.ref_write_tecplot.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_double]
        lib.ref_read_tecplot.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int,
                                         ctypes.c_int, ctypes.c_int]
        _REF[path] = lib
    return _REF[path]


class Ref:
    """One single-rank instance of the reference (Field3D + SolverParams).
    `library` selects the build: the reference itself (default) or the
    reference with the product's shim (REF_GPU_SO)."""

    def __init__(self, cfg: dict, library: str = REF_SO):
        self.lib = _ref_lib(library)
        self.cfg = dict(cfg)
        fd, path = tempfile.mkstemp(suffix=".in")
        with os.fdopen(fd, "w") as f:
            f.write(solver_in_text(cfg))
        self.h = self.lib.ref_create(path.encode())
        os.unlink(path)
        if not self.h:
            raise RuntimeError("reference could not read solver.in")
        dims = (ctypes.c_int * 9)()
        self.lib.ref_dims(self.h, dims)
        self.nx, self.ny, self.nz, self.ng = dims[0], dims[1], dims[2], dims[3]
        self.shape = (self.nz, self.ny, self.nx)

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.ref_destroy(self.h)
            self.h = None

    def params(self) -> dict:
        out = (ctypes.c_double * 21)()
        self.lib.ref_params(self.h, out)
        names = ["gamma", "Pr", "Ma", "Re", "cfl", "dt_fixed", "Cv", "Cp", "Rgas", "mu", "dx",
                 "dy", "dz", "mdcd_diss", "mdcd_disp", "ud7l_alpha", "TotalTime",
                 "output_Timefreq", "max_steps", "monitor_Stepfreq", "mu_at_T1"]
        return dict(zip(names, list(out)))

    def _check(self, rc):
        if rc != 0:
            raise RuntimeError(self.lib.ref_last_error(self.h).decode())

    def set_primitive(self, W):
        W = [np.ascontiguousarray(a, dtype=np.float64) for a in W]
        self._check(self.lib.ref_set_primitive(self.h, *[_dp(a) for a in W]))

    def set_conserved(self, U):
        U = [np.ascontiguousarray(a, dtype=np.float64) for a in U]
        self._check(self.lib.ref_set_conserved(self.h, *[_dp(a) for a in U]))

    def get(self, name):
        out = np.empty(self.shape)
        rc = self.lib.ref_get(self.h, name.encode(), _dp(out))
        if rc:
            raise KeyError(name)
        return out

    def get_face(self, name):
        d = name.split("_")[1][1]
        shp = {"x": (self.nz, self.ny, self.nx + 1), "y": (self.nz, self.ny + 1, self.nx),
               "z": (self.nz + 1, self.ny, self.nx)}[d]
        out = np.empty(shp)
        rc = self.lib.ref_get_face(self.h, name.encode(), _dp(out))
        if rc:
            raise KeyError(name)
        return out

    def W(self):
        return np.stack([self.get(n) for n in ("rho", "u", "v", "w", "p")])

    def U(self):
        return np.stack([self.get(n) for n in ("rho", "rhou", "rhov", "rhow", "E")])

    def rhs(self):
        self._check(self.lib.ref_compute_rhs(self.h))
        return np.stack([self.get("rhs_" + n) for n in ("rho", "rhou", "rhov", "rhow", "E")])

    def record0(self):
        self.lib.ref_record0(self.h)

    def timestep(self):
        return self.lib.ref_timestep(self.h)

    def rk3(self, dt):
        return self.lib.ref_rk3(self.h, float(dt))

    def cfl_step(self):
        return self.lib.ref_cfl_step(self.h)

    def total_energy(self):
        return self.lib.ref_total_energy(self.h)

    def time_advance(self, workdir):
        os.makedirs(os.path.join(workdir, "output"), exist_ok=True)
        self._check(self.lib.ref_time_advance(self.h, workdir.encode()))

    def isotropic_post(self, workdir, t=0.0):
        """Returns (k, Ek) from the spectrum file and the stats row as a dict."""
        os.makedirs(os.path.join(workdir, "output"), exist_ok=True)
        self._check(self.lib.ref_isotropic_post(self.h, workdir.encode(), float(t)))
        spec = np.loadtxt(os.path.join(workdir, "output", f"output_time_{t:.5f}_spectrum.dat"))
        with open(os.path.join(workdir, "output", "turbulence_stats.dat")) as f:
            rows = [r.split() for r in f.read().strip().splitlines()]
        names = ["current_time", "kinetic_energy", "tke", "u_rms", "dissipation", "taylor", "eta",
                 "u_eta", "tau_eta", "taylor_Li", "Re_lambda", "Mach_t"]
        stats = dict(zip(names, [float(x) for x in rows[-1]]))
        return spec[:, 0], spec[:, 1], stats

    def init_isotropic(self):
        self._check(self.lib.ref_init_isotropic(self.h))

    def diagnostics(self) -> np.ndarray:
        """compute_diagnostics: the five residuals of the last step."""
        out = np.zeros(5)
        self._check(self.lib.ref_diagnostics(self.h, _dp(out)))
        return out

    def write_residuals(self, directory: str, step: int, energy: bool = True) -> str:
        """write_residuals_tecplot under `directory`; returns the file's path."""
        self._check(self.lib.ref_write_residuals(self.h, directory.encode(), int(step),
                                                 int(bool(energy))))
        return os.path.join(directory, "output", "output_residuals.dat")

    def write_tecplot(self, directory: str, time: float) -> str:
        """write_tecplot_field under `directory`; returns the file's path."""
        self._check(self.lib.ref_write_tecplot(self.h, directory.encode(), float(time)))
        return os.path.join(directory, "output", f"time_{int(time * 100000)}", "field_rank0.dat")

    def read_tecplot(self, path: str, src=None) -> int:
        """initialize_from_tecplot[_downsample] + boundary + primitiveToConserved;
        returns 0, or 1 when the reference's reader reported failure."""
        sx, sy, sz = src if src else (0, 0, 0)
        r = self.lib.ref_read_tecplot(self.h, path.encode(), sx, sy, sz)
        if r < 0:
            self._check(r)
        return r


# --------------------------------------------------------------------------
# Spectrum and statistics (numpy restatements)
# --------------------------------------------------------------------------

def spectrum(u, v, w):
    """Shell energy spectrum as compute_energy_spectrum_rank0 computes it
    (EnergySpectrum.cpp:62-125): forward transform (e^{-i}), scaled by 1/N,
    E = 0.5(|U|^2+|V|^2+|W|^2), binned by floor(|k|) (the `(int)sqrt(..)+0.5`
    of :120 truncates), 2*NX+1 bins. Inputs are (nz, ny, nx) arrays; for a
    cubic box the reference's transposed indexing (:116-122) bins the same."""
    nz, ny, nx = u.shape
    N = nx * ny * nz
    e = np.zeros(u.shape)
    for a in (u, v, w):
        A = np.fft.fftn(a) * (1.0 / N)
        e += A.real ** 2 + A.imag ** 2
    e *= 0.5
    k1 = np.fft.fftfreq(nx, 1.0 / nx)
    k2 = np.fft.fftfreq(ny, 1.0 / ny)
    k3 = np.fft.fftfreq(nz, 1.0 / nz)
    # the reference maps index i <= N/2 to +i (so N/2 is +N/2): |k| is unchanged
    K3, K2, K1 = np.meshgrid(k3, k2, k1, indexing="ij")
    kk = np.floor(np.sqrt(K1 * K1 + K2 * K2 + K3 * K3)).astype(np.int64)
    Ek = np.bincount(kk.ravel(), weights=e.ravel(), minlength=2 * nx + 1)
    return Ek[: 2 * nx + 1]


def residuals(U, U0, dx: float) -> np.ndarray:
    """compute_diagnostics (postprocess.cpp:7-98) from the conserved state U
    after a step and U0 at its start, both (5, nz, ny, nx): sqrt(sum (U - U0)^2
    dx^3) / max |U| per variable. The sums run in the reference's order (x
    fastest, one running total; np.cumsum is sequential), so single-rank results
    are bit-identical."""
    dx3 = dx * dx * dx
    out = np.empty(5)
    for q in range(5):
        r = (U[q] - U0[q]).ravel()
        s = np.cumsum(r * r * dx3)[-1]
        out[q] = np.sqrt(s) / np.max(np.abs(U[q]))
    return out


def residuals_row(step: int, res, etot: float) -> str:
    """One row of write_residuals_tecplot (output.cpp:124-126)."""
    return f"{step} " + " ".join(f"{x:.8e}" for x in list(res) + [etot]) + "\n"


def turbulence_stats(sums: np.ndarray, Ek: np.ndarray, N: int, gamma: float, Rgas: float):
    """compute_turbulence_statistics (ana_isotropic.cpp:271-313) from the sums of
    :class:`Oracle.turb_sums` and a spectrum. Returns a dict."""
    s = sums
    mean_mu = s[1] / N
    mean_rho = s[2] / N
    nu = mean_mu / mean_rho
    ke = s[0] / N
    u_rms = math.sqrt(s[3] / (3 * N))
    mu_, mv, mw = s[4] / N, s[5] / N, s[6] / N
    tke = 0.5 * ((s[7] / N - mu_ * mu_) + (s[8] / N - mv * mv) + (s[9] / N - mw * mw))
    mach_t = math.sqrt(ke * 2) / (s[10] / N)
    k = np.arange(len(Ek), dtype=np.float64)
    eps = 0.0
    for i in range(len(Ek)):
        eps += 2.0 * nu * k[i] * k[i] * Ek[i]
    # ana_isotropic.cpp:286-303: Taylor length from <(du/dx)^2>, Kolmogorov scales,
    # Taylor microscale
    dudx2 = s[11] / N
    taylor_li = u_rms / math.sqrt(dudx2)
    return dict(kinetic_energy=ke, tke=tke, u_rms=u_rms, dissipation=eps, nu=nu, Mach_t=mach_t,
                mean_mu=mean_mu, mean_rho=mean_rho, dudx2=dudx2, taylor_Li=taylor_li,
                Re_lambda=u_rms * taylor_li / nu, eta=math.pow(nu * nu * nu / eps, 0.25),
                u_eta=math.pow(nu * eps, 0.25), tau_eta=math.pow(nu / eps, 0.5),
                taylor=math.sqrt(15.0 * nu * u_rms * u_rms / eps))
