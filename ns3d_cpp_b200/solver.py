"""Python host mirror of the reference's solver interface over the C ABI.

Names follow the reference: :class:`SolverParams` (field_structures.h:85-166),
:func:`read_solver_params_from_file` (initialization.cpp:199), and on
:class:`Solver` the operations of Field3D / range_kutta / timestep /
maincycle: ``record_conserved0`` (recordConservedTo0), ``compute_rhs``,
``compute_timestep``, ``runge_kutta_3``, ``time_advance``,
``compute_total_energy``, ``compute_energy_spectrum``,
``compute_turbulence_statistics``.

Everything runs in ``libns3d_b200.so`` on the GPU; there is no CPU fallback.
Where the reference aborts (MPI_Abort on a non-physical state) or throws,
these methods raise :class:`NS3DError` carrying the C status code.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import _lib

STATUS = {0: "OK", 1: "ERR_INVALID", 2: "ERR_UNSUPPORTED", 3: "ERR_CUDA", 4: "ERR_NONPHYSICAL",
          5: "ERR_FILE", 6: "ERR_DT", 7: "ERR_NOMEM", 8: "ERR_TIMEOUT"}

FVS = {"stagerwarming": 0, "laxfriedrichs": 1}
RECON = {"weno5": 0, "wcns": 1, "linear": 2, "mdcd": 3, "mdcd_hybrid": 4, "upwind_7th": 5,
         "ud7l": 6}
VIS = {"c8th": 0, "c6th": 1, "c4th": 2}
PRECISION = {"fp64": 0, "fp32acc64": 1}
LAYOUT = {"interior": 0, "ghosted": 1}


class NS3DError(RuntimeError):
    def __init__(self, status: int, message: str = ""):
        self.status = int(status)
        super().__init__(f"{STATUS.get(self.status, self.status)}: {message}")


class SolverParams(ctypes.Structure):
    """``ns3d_params`` of include/ns3d_gpu.h (SolverParams + GridDesc)."""
    _fields_ = [
        ("gamma", ctypes.c_double), ("Pr", ctypes.c_double), ("Ma", ctypes.c_double),
        ("Re", ctypes.c_double), ("cfl", ctypes.c_double), ("dt_fixed", ctypes.c_double),
        ("fvs_type", ctypes.c_int), ("recon", ctypes.c_int), ("vis_scheme", ctypes.c_int),
        ("char_recon", ctypes.c_int),
        ("mdcd_diss", ctypes.c_double), ("mdcd_disp", ctypes.c_double),
        ("ud7l_alpha", ctypes.c_double),
        ("global_nx", ctypes.c_int), ("global_ny", ctypes.c_int), ("global_nz", ctypes.c_int),
        ("x0", ctypes.c_double), ("y0", ctypes.c_double), ("z0", ctypes.c_double),
        ("Lx", ctypes.c_double), ("Ly", ctypes.c_double), ("Lz", ctypes.c_double),
        ("bc", ctypes.c_int * 6),
        ("max_steps", ctypes.c_int), ("monitor_Stepfreq", ctypes.c_int),
        ("output_Timefreq", ctypes.c_double), ("TotalTime", ctypes.c_double),
        ("post_basicfield", ctypes.c_int), ("isotropic_analyse", ctypes.c_int),
        ("monitor_res", ctypes.c_int), ("monitor_energy", ctypes.c_int),
        ("Cv", ctypes.c_double), ("Cp", ctypes.c_double), ("Rgas", ctypes.c_double),
        ("mu", ctypes.c_double), ("dx", ctypes.c_double), ("dy", ctypes.c_double),
        ("dz", ctypes.c_double),
        ("stencil", ctypes.c_int), ("ghost_layers", ctypes.c_int), ("periods", ctypes.c_int * 3),
        ("sw_entropy_eps", ctypes.c_double), ("sutherland_s_over_tref", ctypes.c_double),
        ("precision", ctypes.c_int), ("reserved", ctypes.c_int * 7),
    ]

    @classmethod
    def default(cls) -> "SolverParams":
        p = cls()
        _check(_lib.load().ns3d_params_default(ctypes.byref(p)))
        return p

    def derive(self) -> "SolverParams":
        _check(_lib.load().ns3d_params_derive(ctypes.byref(self)))
        return self

    def copy(self) -> "SolverParams":
        p = SolverParams()
        ctypes.memmove(ctypes.byref(p), ctypes.byref(self), ctypes.sizeof(self))
        return p

    def replace(self, **kw) -> "SolverParams":
        """A derived copy with fields changed; enum fields accept the solver.in
        spellings (e.g. recon="weno5", precision="fp32acc64")."""
        p = self.copy()
        for k, v in kw.items():
            if isinstance(v, str):
                table = {"fvs_type": FVS, "recon": RECON, "vis_scheme": VIS,
                         "precision": PRECISION}[k]
                v = table[v.lower()]
            if k == "n":
                p.global_nx = p.global_ny = p.global_nz = int(v)
                continue
            setattr(p, k, v)
        return p.derive()

    def as_dict(self) -> dict:
        out = {}
        for name, typ in self._fields_:
            v = getattr(self, name)
            out[name] = list(v) if hasattr(v, "__len__") else v
        return out


class TurbStats(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in
                ("kinetic_energy", "tke", "u_rms", "dissipation", "nu", "mean_mu", "mean_rho",
                 "mach_t", "total_energy", "taylor", "eta", "u_eta", "tau_eta", "taylor_li",
                 "re_lambda", "dudx2")]


def _check(status: int, ctx=None) -> None:
    if status != 0:
        msg = ""
        if ctx is not None:
            msg = _lib.load().ns3d_last_error(ctx).decode(errors="replace")
        raise NS3DError(status, msg)


def read_solver_params_from_file(path: str) -> SolverParams:
    """read_solver_params_from_file (initialization.cpp:199-380)."""
    p = SolverParams()
    st = _lib.load().ns3d_params_from_file(os.fsencode(path), ctypes.byref(p))
    if st != 0:
        raise NS3DError(st, f"cannot read {path}")
    return p


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class Solver:
    """One resident periodic domain on one GPU (ns3d_ctx)."""

    def __init__(self, params: SolverParams, device: int = 0):
        self.lib = _lib.load()
        self.params = params.copy().derive()
        self.ctx = ctypes.c_void_p()
        st = self.lib.ns3d_create(ctypes.byref(self.params), int(device), ctypes.byref(self.ctx))
        if st != 0:
            raise NS3DError(st, "ns3d_create failed")
        p = self.params
        self.shape = (p.global_nz, p.global_ny, p.global_nx)
        g = p.ghost_layers
        self.ghosted_shape = (p.global_nz + 2 * g, p.global_ny + 2 * g, p.global_nx + 2 * g)

    # -- lifetime -----------------------------------------------------------
    def close(self) -> None:
        if self.ctx:
            self.lib.ns3d_destroy(self.ctx)
            self.ctx = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _ck(self, st: int) -> None:
        _check(st, self.ctx)

    # -- state --------------------------------------------------------------
    def _prep(self, arrays, layout: str):
        shape = self.shape if layout == "interior" else self.ghosted_shape
        out = []
        for a in arrays:
            a = np.ascontiguousarray(a, dtype=np.float64)
            if a.shape != shape:
                raise ValueError(f"array of shape {a.shape}, expected {shape}")
            out.append(a)
        return out

    def upload_primitive(self, W, layout: str = "interior") -> None:
        """Initial condition path (main.cpp:67-71); also records U0. Uses the
        copy a prefetch_primitive of the same arrays started."""
        arrs = self._prep(W, layout)
        self._ck(self.lib.ns3d_upload_primitive(self.ctx, *[_dptr(a) for a in arrs],
                                                LAYOUT[layout]))
        self._prefetched = None

    def prefetch_primitive(self, W, layout: str = "interior") -> None:
        """Start copying W (float64, C-contiguous; pinned memory for overlap)
        to the device; the next upload_primitive(W) only waits for the copy.
        W must stay unchanged until that upload returns; the solver keeps a
        reference to it until then."""
        arrs = self._prep(W, layout)
        self._ck(self.lib.ns3d_prefetch_primitive(self.ctx, *[_dptr(a) for a in arrs],
                                                  LAYOUT[layout]))
        self._prefetched = arrs

    def upload_conserved(self, U, layout: str = "interior") -> None:
        """conservedToPrimitive + apply_boundary + primitiveToConserved; records U0."""
        arrs = self._prep(U, layout)
        self._ck(self.lib.ns3d_upload_conserved(self.ctx, *[_dptr(a) for a in arrs],
                                                LAYOUT[layout]))

    def download_primitive(self, layout: str = "interior", with_T_c: bool = False):
        shape = self.shape if layout == "interior" else self.ghosted_shape
        out = np.empty((7 if with_T_c else 5,) + shape)
        ptrs = [_dptr(out[q]) for q in range(out.shape[0])]
        if not with_T_c:
            ptrs += [None, None]
        self._ck(self.lib.ns3d_download_primitive(self.ctx, *ptrs, LAYOUT[layout]))
        return out

    def download_conserved(self, layout: str = "interior"):
        shape = self.shape if layout == "interior" else self.ghosted_shape
        out = np.empty((5,) + shape)
        self._ck(self.lib.ns3d_download_conserved(self.ctx, *[_dptr(out[q]) for q in range(5)],
                                                  LAYOUT[layout]))
        return out

    # -- hot path -----------------------------------------------------------
    def record_conserved0(self) -> None:
        self._ck(self.lib.ns3d_record_conserved0(self.ctx))

    def compute_rhs(self, layout: str = "interior"):
        shape = self.shape if layout == "interior" else self.ghosted_shape
        out = np.empty((5,) + shape)
        self._ck(self.lib.ns3d_compute_rhs(self.ctx, *[_dptr(out[q]) for q in range(5)],
                                           LAYOUT[layout]))
        return out

    def compute_timestep(self) -> float:
        dt = ctypes.c_double()
        self._ck(self.lib.ns3d_compute_timestep(self.ctx, ctypes.byref(dt)))
        return dt.value

    def runge_kutta_3(self, dt: float) -> None:
        self._ck(self.lib.ns3d_runge_kutta_3(self.ctx, float(dt)))

    def time_advance(self, max_steps: int):
        """Returns (current_time, steps_done)."""
        t = ctypes.c_double()
        k = ctypes.c_int()
        self._ck(self.lib.ns3d_time_advance(self.ctx, int(max_steps), ctypes.byref(t),
                                            ctypes.byref(k)))
        return t.value, k.value

    def time_advance_segment(self, max_steps: int):
        """time_advance ending early after an output step; returns
        (current_time, steps_done, events) with events a set of "output", "end"."""
        t = ctypes.c_double()
        k = ctypes.c_int()
        ev = ctypes.c_int()
        self._ck(self.lib.ns3d_time_advance_segment(self.ctx, int(max_steps), ctypes.byref(t),
                                                    ctypes.byref(k), ctypes.byref(ev)))
        events = {n for b, n in ((1, "output"), (2, "end")) if ev.value & b}
        return t.value, k.value, events

    def run(self, workdir: str = ".", max_steps: int | None = None, verbose: bool = True):
        """time_advance with the reference's monitor and output files under
        ``workdir``/output (maincycle.cpp:7-112). Returns (current_time, steps)."""
        t = ctypes.c_double()
        k = ctypes.c_int()
        n = self.params.max_steps if max_steps is None else int(max_steps)
        self._ck(self.lib.ns3d_run(self.ctx, workdir.encode(), n, int(bool(verbose)),
                                   ctypes.byref(t), ctypes.byref(k)))
        return t.value, k.value

    def step(self, nsteps: int = 1) -> None:
        self._ck(self.lib.ns3d_step(self.ctx, int(nsteps)))

    def last_dt(self) -> float:
        dt = ctypes.c_double()
        self._ck(self.lib.ns3d_last_dt(self.ctx, ctypes.byref(dt)))
        return dt.value

    def step_times(self) -> np.ndarray:
        """current_time after each step of the last step / time_advance call."""
        n = ctypes.c_int()
        self._ck(self.lib.ns3d_step_times(self.ctx, None, 0, ctypes.byref(n)))
        out = np.zeros(n.value)
        if n.value:
            self._ck(self.lib.ns3d_step_times(
                self.ctx, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), n.value,
                ctypes.byref(n)))
        return out

    def synchronize(self) -> None:
        self._ck(self.lib.ns3d_synchronize(self.ctx))

    def device_bytes(self) -> int:
        b = ctypes.c_size_t()
        self._ck(self.lib.ns3d_device_bytes(self.ctx, ctypes.byref(b)))
        return b.value

    # -- discrete adjoint ---------------------------------------------------
    def rhs_vjp(self, lam_rhs):
        """(d rhs / d W)^T lam_rhs at the current state; both (5, nz, ny, nx)."""
        lr = np.ascontiguousarray(lam_rhs, dtype=np.float64)
        if lr.shape != (5,) + self.shape:
            raise ValueError(f"lam_rhs of shape {lr.shape}")
        out = np.empty_like(lr)
        self._ck(self.lib.ns3d_rhs_vjp(self.ctx, _dptr(lr), _dptr(out)))
        return out

    def step_dts(self, dts) -> None:
        """runge_kutta_3 steps with a prescribed dt sequence."""
        d = np.ascontiguousarray(dts, dtype=np.float64)
        self._ck(self.lib.ns3d_step_dts(self.ctx, len(d), _dptr(d)))

    def adjoint(self, nsteps: int, checkpoint_every: int, dts=None, lam_final=None):
        """Gradient of an end-time objective w.r.t. the current state.
        Returns (grad (5, nz, ny, nx), J, dts); J is the total kinetic energy
        when `lam_final` is None."""
        grad = np.empty((5,) + self.shape)
        J = ctypes.c_double(np.nan)
        dts_out = np.empty(nsteps)
        din = None if dts is None else np.ascontiguousarray(dts, dtype=np.float64)
        lf = None if lam_final is None else np.ascontiguousarray(lam_final, dtype=np.float64)
        self._ck(self.lib.ns3d_adjoint(self.ctx, int(nsteps), int(checkpoint_every),
                                       None if din is None else _dptr(din), _dptr(dts_out),
                                       None if lf is None else _dptr(lf), _dptr(grad),
                                       ctypes.byref(J)))
        return grad, J.value, (dts_out if din is None else din)

    # -- instrumentation ----------------------------------------------------
    KERNEL_CLASSES = ("sweep_x", "sweep_y", "sweep_z", "visc_flux", "update", "other",
                      "sweep_z_update")

    def stream_handle(self) -> int:
        """The cudaStream_t (as an int) all kernels of this context run on."""
        s = ctypes.c_void_p()
        self._ck(self.lib.ns3d_get_stream(self.ctx, ctypes.byref(s)))
        return s.value or 0

    def profile(self, enable: bool) -> None:
        self._ck(self.lib.ns3d_profile(self.ctx, int(bool(enable))))

    def profile_read(self) -> dict:
        ms = (ctypes.c_double * len(self.KERNEL_CLASSES))()
        n = (ctypes.c_longlong * len(self.KERNEL_CLASSES))()
        self._ck(self.lib.ns3d_profile_read(self.ctx, ms, n))
        return {k: (ms[i], n[i]) for i, k in enumerate(self.KERNEL_CLASSES)}

    def launch_count(self) -> int:
        c = ctypes.c_longlong()
        self._ck(self.lib.ns3d_launch_count(self.ctx, ctypes.byref(c)))
        return c.value

    # -- reductions ---------------------------------------------------------
    def compute_total_energy(self) -> float:
        e = ctypes.c_double()
        self._ck(self.lib.ns3d_total_energy(self.ctx, ctypes.byref(e)))
        return e.value

    def compute_energy_spectrum(self, nbins: int | None = None):
        if nbins is None:
            nbins = 2 * self.params.global_nx + 1
        out = np.empty(nbins)
        self._ck(self.lib.ns3d_energy_spectrum(self.ctx, _dptr(out), int(nbins)))
        return out

    def compute_turbulence_statistics(self, spectrum=None) -> dict:
        """The statistics row; from `spectrum` (E(k), k = 0..) when given, else
        from the state's own spectrum at full precision."""
        s = TurbStats()
        if spectrum is None:
            self._ck(self.lib.ns3d_turbulence_stats(self.ctx, ctypes.byref(s)))
        else:
            e = np.ascontiguousarray(spectrum, dtype=np.float64)
            self._ck(self.lib.ns3d_turbulence_stats_spectrum(self.ctx, _dptr(e), len(e),
                                                             ctypes.byref(s)))
        return {n: getattr(s, n) for n, _ in TurbStats._fields_}

    def residuals(self) -> np.ndarray:
        """compute_diagnostics (postprocess.cpp:7-98) after a step: the five
        normalised L2 residuals of rho, rhou, rhov, rhow, E."""
        out = np.zeros(5)
        self._ck(self.lib.ns3d_residuals(self.ctx, _dptr(out)))
        return out

    def checkpoint_write(self, path: str) -> None:
        """The state, clock and CFL minimum, bit for bit (a binary restart file)."""
        self._ck(self.lib.ns3d_checkpoint_write(self.ctx, path.encode()))

    def checkpoint_read(self, path: str) -> None:
        """Continue from a checkpoint_write file of the same grid."""
        self._ck(self.lib.ns3d_checkpoint_read(self.ctx, path.encode()))

    def write_tecplot(self, path: str, time: float = 0.0) -> None:
        """write_tecplot_field (output.cpp:21-87) of the state to `path`."""
        self._ck(self.lib.ns3d_write_tecplot(self.ctx, path.encode(), float(time)))

    def read_tecplot(self, path: str) -> None:
        """initialize_from_tecplot (initialization.cpp:35-100) into the state."""
        self._ck(self.lib.ns3d_read_tecplot(self.ctx, path.encode()))

    def init_isotropic(self, k0: int = 8, A: float = 0.00013, seed: int = 123,
                       mach_t: float = 0.0) -> None:
        """init_isotropic_turbulence (isotropic_ini.cpp:146-193) on the device: the
        defaults reproduce the reference's field; mach_t > 0 scales the velocity
        to that turbulent Mach number instead of the reference's energy Ek0."""
        self._ck(self.lib.ns3d_init_isotropic(self.ctx, int(k0), float(A), int(seed),
                                              float(mach_t)))
