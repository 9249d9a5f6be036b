/*
 * ns3d_gpu.h -- C ABI of the B200 implementation of ns3d_cpp's right-hand side
 * and RK3 time-step loop (3D compressible Navier-Stokes, periodic box).
 *
 * Plain C: opaque handle, POD parameter struct, host pointers and sizes. Every
 * function returns an ns3d_status (0 = success). One context owns one device
 * copy of the state and one CUDA stream; calls on one context must not overlap
 * from several threads.
 *
 * Each entry point names the reference function it replaces (file:line in
 * wylx-2/ns3d_cpp). The reference's C++ signatures (compute_rhs,
 * runge_kutta_3, compute_timestep over Field3D) are provided on top of this
 * ABI by the C++ shim ns3d_cpp_b200/shim/ns3d_shim.cpp.
 *
 * Arrays cross the boundary in one of two layouts (x fastest in both):
 *   NS3D_LAYOUT_INTERIOR  nx*ny*nz, a[(k*ny + j)*nx + i]
 *   NS3D_LAYOUT_GHOSTED   the reference Field3D layout, sx*sy*sz with
 *                         s = n + 2*ghost_layers, idx3 (field_structures.h:63)
 */
#ifndef NS3D_GPU_H
#define NS3D_GPU_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum ns3d_status {
    NS3D_OK = 0,
    NS3D_ERR_INVALID = 1,      /* bad argument or configuration */
    NS3D_ERR_UNSUPPORTED = 2,  /* valid in the reference, not built here: non-periodic
                                  boundaries, WCNS; adjoint of MDCD_HYBRID / char_recon */
    NS3D_ERR_CUDA = 3,         /* CUDA runtime / cuFFT failure */
    NS3D_ERR_NONPHYSICAL = 4,  /* rho, p or T <= 0 after a step (range_kutta.cpp:149-162) */
    NS3D_ERR_FILE = 5,         /* solver.in cannot be opened (initialization.cpp:206-209) */
    NS3D_ERR_DT = 6,           /* dt <= 1e-12: time_advance stops (maincycle.cpp:46-52) */
    NS3D_ERR_NOMEM = 7,        /* device allocation failed */
    NS3D_ERR_TIMEOUT = 8       /* a bounded device-side wait gave up */
} ns3d_status;

/* Enumerations keep the reference's enum order (field_structures.h:112-145). */
enum { NS3D_FVS_STEGER_WARMING = 0, NS3D_FVS_LAX_FRIEDRICHS = 1 };
enum {
    NS3D_RECON_WENO5 = 0, NS3D_RECON_WCNS = 1, NS3D_RECON_LINEAR = 2, NS3D_RECON_MDCD = 3,
    NS3D_RECON_MDCD_HYBRID = 4, NS3D_RECON_UPWIND_7TH = 5, NS3D_RECON_UD7L = 6
};
enum { NS3D_VIS_C8TH = 0, NS3D_VIS_C6TH = 1, NS3D_VIS_C4TH = 2 };
enum { NS3D_BC_PERIODIC = 0, NS3D_BC_WALL = 1, NS3D_BC_SYMMETRY = 2, NS3D_BC_OUTFLOW = 3,
       NS3D_BC_INFLOW = 4 };
/* Precision forms. FP64: every operation in double, operation order of the
 * reference, no FMA contraction (1e-12 parity form). FP32_ACC64: splitting,
 * reconstruction and viscous stencils in float; state, RK3 stage accumulation
 * and all reductions in double. */
enum { NS3D_PREC_FP64 = 0, NS3D_PREC_FP32_ACC64 = 1 };
enum { NS3D_LAYOUT_INTERIOR = 0, NS3D_LAYOUT_GHOSTED = 1 };

/* SolverParams + GridDesc + the periodicity of CartDecomp
 * (field_structures.h:32-37, 85-166). */
typedef struct ns3d_params {
    /* physical (SolverParams) */
    double gamma, Pr, Ma, Re;
    /* time stepping */
    double cfl, dt_fixed;
    /* schemes */
    int fvs_type, recon, vis_scheme, char_recon;
    double mdcd_diss, mdcd_disp, ud7l_alpha;
    /* grid (GridDesc) */
    int global_nx, global_ny, global_nz;
    double x0, y0, z0, Lx, Ly, Lz;
    /* boundary types xmin, xmax, ymin, ymax, zmin, zmax */
    int bc[6];
    /* simulation control */
    int max_steps, monitor_Stepfreq;
    double output_Timefreq, TotalTime;
    int post_basicfield, isotropic_analyse, monitor_res, monitor_energy;
    /* derived by ns3d_params_derive (initialization.cpp:312-377) */
    double Cv, Cp, Rgas, mu, dx, dy, dz;
    int stencil, ghost_layers;
    int periods[3];
    /* extensions; the defaults reproduce the reference */
    double sw_entropy_eps;          /* |l| -> sqrt(l^2+eps^2) in Steger-Warming (README.md:177-180); 0 */
    double sutherland_s_over_tref;  /* S/Tref of get_mu; 110.4/288.15 (field_structures.h:100) */
    int precision;                  /* NS3D_PREC_*; default FP64 */
    int reserved[7];
} ns3d_params;

typedef struct ns3d_ctx ns3d_ctx;

/* Turbulence statistics of compute_turbulence_statistics (ana_isotropic.cpp:196-314),
 * the spectrum taken at full precision (the reference re-reads it from a 6-digit file). */
typedef struct ns3d_turb_stats {
    double kinetic_energy;  /* <0.5|u|^2> */
    double tke;             /* 0.5 (var u + var v + var w) */
    double u_rms;           /* sqrt(<|u|^2>/3) */
    double dissipation;     /* eps = 2 nu sum_k k^2 E(k), nu = <mu(T)>/<rho> */
    double nu, mean_mu, mean_rho;
    double mach_t;          /* sqrt(2 KE) / <c> */
    double total_energy;    /* sum 0.5 rho |u|^2 dV (compute_total_energy, postprocess.cpp:103) */
    double taylor;          /* Taylor microscale sqrt(15 nu u_rms^2 / eps) */
    double eta;             /* Kolmogorov length (nu^3 / eps)^(1/4) */
    double u_eta;           /* Kolmogorov velocity (nu eps)^(1/4) */
    double tau_eta;         /* Kolmogorov time (nu / eps)^(1/2) */
    double taylor_li;       /* u_rms / sqrt(<(du/dx)^2>) */
    double re_lambda;       /* u_rms taylor_li / nu */
    double dudx2;           /* <(du/dx)^2>, du/dx of compute_gradients_dudx (ViscousFlux.cpp:389) */
} ns3d_turb_stats;

/* ---- parameters ---------------------------------------------------------- */

/* SolverParams() defaults plus the parser's grid defaults (16^3, origin 0). */
ns3d_status ns3d_params_default(ns3d_params *p);
/* read_solver_params_from_file (initialization.cpp:199-380): key = value, '#'
 * comments, case-insensitive keys, unknown keys ignored; then derives. Also
 * accepts the extension keys sw_entropy_eps, sutherland_s_over_tref and
 * precision (fp64 | fp32acc64). */
ns3d_status ns3d_params_from_file(const char *path, ns3d_params *p);
/* The derivation step alone (initialization.cpp:312-377). */
ns3d_status ns3d_params_derive(ns3d_params *p);
/* sizeof(ns3d_params) and sizeof(ns3d_turb_stats), for bindings to check
 * their struct layout (no reference counterpart). */
size_t ns3d_params_size(void);
size_t ns3d_turb_stats_size(void);

/* ---- context ------------------------------------------------------------- */

/* Field3D::allocate (field_structures.h:225) on `device`, interior-only and
 * resident in HBM. Rejects non-periodic boundaries and WCNS with
 * NS3D_ERR_UNSUPPORTED. char_recon selects the characteristic-wise sweeps
 * (du_inviscous_character, InviscousFlux_new.cpp:165-437). */
ns3d_status ns3d_create(const ns3d_params *p, int device, ns3d_ctx **out);
ns3d_status ns3d_destroy(ns3d_ctx *ctx);
/* Last error message of this context (static string for ctx == NULL). */
const char *ns3d_last_error(const ns3d_ctx *ctx);
ns3d_status ns3d_get_params(const ns3d_ctx *ctx, ns3d_params *out);
/* Bytes of device memory the context holds. */
ns3d_status ns3d_device_bytes(const ns3d_ctx *ctx, size_t *bytes);
ns3d_status ns3d_synchronize(ns3d_ctx *ctx);

/* ---- state transfer (host pointers) ---------------------------------------- */

/* Initial condition path: interior primitives, then apply_boundary +
 * primitiveToConserved (main.cpp:67-71). Also records U0 (recordConservedTo0). */
ns3d_status ns3d_upload_primitive(ns3d_ctx *ctx, const double *rho, const double *u,
                                  const double *v, const double *w, const double *p,
                                  int layout);
/* Starts copying the primitives that a following ns3d_upload_primitive will be
 * given (same pointers, interior layout) into a device staging buffer on a
 * copy stream, and returns; that upload then only waits for the copy, so a
 * host loop that prefetches step k+1's state before stepping state k overlaps
 * the transfer with the step. The arrays must stay valid and unchanged until
 * that upload returns, and should be pinned (pageable memory copies
 * synchronously). An upload with other pointers or layout ignores the prefetch.
 * The first call allocates the staging buffer (6 n doubles). No reference
 * counterpart (the reference's Field3D lives in host memory). Ghosted layout:
 * accepted, no effect (the upload gathers on the host). */
ns3d_status ns3d_prefetch_primitive(ns3d_ctx *ctx, const double *rho, const double *u,
                                    const double *v, const double *w, const double *p,
                                    int layout);
/* Conserved state: conservedToPrimitive + apply_boundary + primitiveToConserved
 * (range_kutta.cpp:117-119). Also records U0. */
ns3d_status ns3d_upload_conserved(ns3d_ctx *ctx, const double *rho, const double *rhou,
                                  const double *rhov, const double *rhow, const double *E,
                                  int layout);
/* Primitives (rho,u,v,w,p) as Field3D holds them after a step; optional T, c
 * (NULL to skip). Ghost faces hold periodic images; edges/corners hold the
 * values a Field3D keeps there (rho=1, others 0). */
ns3d_status ns3d_download_primitive(ns3d_ctx *ctx, double *rho, double *u, double *v,
                                    double *w, double *p, double *T, double *c, int layout);
/* Conserved (rho, rhou, rhov, rhow, E) = primitiveToConserved of the state. */
ns3d_status ns3d_download_conserved(ns3d_ctx *ctx, double *rho, double *rhou, double *rhov,
                                    double *rhow, double *E, int layout);

/* ---- the hot path ----------------------------------------------------------- */

/* Field3D::recordConservedTo0 (field_structures.h:454). */
ns3d_status ns3d_record_conserved0(ns3d_ctx *ctx);
/* compute_rhs (range_kutta.cpp:11-99) of the current state; copies the five
 * rhs arrays to the host pointers (any may be NULL). */
ns3d_status ns3d_compute_rhs(ns3d_ctx *ctx, double *rhs_rho, double *rhs_rhou,
                             double *rhs_rhov, double *rhs_rhow, double *rhs_E, int layout);
/* compute_timestep (timestep.cpp:5-33): cfl * min over cells. */
ns3d_status ns3d_compute_timestep(ns3d_ctx *ctx, double *dt);
/* runge_kutta_3 (range_kutta.cpp:102-163) with the recorded U0; returns
 * NS3D_ERR_NONPHYSICAL (instead of MPI_Abort) if rho, p or T <= 0 afterwards. */
ns3d_status ns3d_runge_kutta_3(ns3d_ctx *ctx, double dt);
/* time_advance (maincycle.cpp:7-112) without monitor output: up to `max_steps`
 * steps of recordConservedTo0 + dt (CFL or dt_fixed) + the clipping to
 * TotalTime and output times + runge_kutta_3, all on the device with no host
 * round trip per step. `time` is in/out (current_time); `steps_done` receives
 * the number of completed steps. Stops early exactly where time_advance does. */
ns3d_status ns3d_time_advance(ns3d_ctx *ctx, int max_steps, double *time, int *steps_done);
/* `nsteps` RK3 steps with a CFL (or fixed) dt each, no clipping: the bench step. */
ns3d_status ns3d_step(ns3d_ctx *ctx, int nsteps);
/* The same loop as ns3d_time_advance, also ending right after a step whose if_output
 * is set (maincycle.cpp:33-45), so that a monitor can write that step's output; the
 * next call continues the loop. *events: NS3D_EVENT_OUTPUT when the last completed
 * step is an output step, NS3D_EVENT_END when the loop reached TotalTime. */
#define NS3D_EVENT_OUTPUT 1
#define NS3D_EVENT_END 2
ns3d_status ns3d_time_advance_segment(ns3d_ctx *ctx, int max_steps, double *time, int *steps_done,
                                      int *events);
/* dt of the last step taken on the device. */
ns3d_status ns3d_last_dt(ns3d_ctx *ctx, double *dt);
/* current_time after each step the last ns3d_step / ns3d_time_advance /
 * ns3d_time_advance_segment call completed (the value the reference prints in
 * its "Completed step" line, maincycle.cpp:56-58): copies up to `cap` of them
 * to `times` (may be NULL with cap 0) and stores their number in *n. */
ns3d_status ns3d_step_times(ns3d_ctx *ctx, double *times, int cap, int *n);

/* ---- discrete adjoint (no counterpart in the reference) ------------------- */
/* The derivative of exactly the FP64 forward arithmetic (the adjoint of the
 * discretisation, not of the PDE). Supported: FP64 form, Steger-Warming (use
 * sw_entropy_eps > 0 to make |lambda| smooth) or Lax-Friedrichs, WENO5 or the
 * linear reconstructions, component-wise; MDCD_HYBRID and char_recon return
 * NS3D_ERR_UNSUPPORTED. Arrays are host pointers to 5 consecutive interior
 * blocks (rho, u, v, w, p). The checkpoints and scratch arrays stay in the
 * context after a call (ns3d_device_bytes counts them): a later call that
 * needs no more checkpoints, no larger checkpoint_every and no more steps
 * allocates nothing. */

/* lam_w = (d rhs / d w)^T lam_rhs at the current state (vector-Jacobian
 * product of compute_rhs with respect to the primitives). */
ns3d_status ns3d_rhs_vjp(ns3d_ctx *ctx, const double *lam_rhs, double *lam_w);
/* `nsteps` runge_kutta_3 steps with the given dt sequence (each step records
 * U0 first, as time_advance does). */
ns3d_status ns3d_step_dts(ns3d_ctx *ctx, int nsteps, const double *dts);
/* Gradient of an end-time objective with respect to the current state,
 * through `nsteps` RK3 steps. dts: the dt of every step (NULL: the CFL dt of
 * each step, written to dts_out when that is non-NULL); dt is held fixed, not
 * differentiated. lam_final: dJ/dw at the end state, or NULL for J = the total
 * kinetic energy sum 0.5 rho |u|^2 dV of compute_total_energy
 * (postprocess.cpp:103), whose value is returned in *J. grad receives dJ/dw
 * at the start state. The forward run stores the state every
 * `checkpoint_every` steps; the reverse sweep recomputes each segment's stage
 * states from its checkpoint. Afterwards the context holds the end state. */
ns3d_status ns3d_adjoint(ns3d_ctx *ctx, int nsteps, int checkpoint_every, const double *dts,
                         double *dts_out, const double *lam_final, double *grad, double *J);

/* ---- allocation-free RHS (no counterpart in the reference) ----------------- */

/* Largest box (nx*ny*nz) ns3d_compute_rhs_noalloc accepts. */
#define NS3D_NOALLOC_MAX_CELLS 65536

/* compute_rhs for callers that may not allocate device memory: hosts whose
 * GPU memory is owned by another allocator (a framework's caching allocator,
 * a fixed per-job budget) or that must not stall on cudaMalloc mid-run. No
 * context, no cudaMalloc/cudaFree: the caller passes device pointers to the
 * interior primitives (rho,u,v,w,p; nx*ny*nz each, x fastest) and to `rhs`
 * (5 consecutive blocks of nx*ny*nz: rho, rhou, rhov, rhow, E), plus the
 * cudaStream_t to run on (NULL = legacy default stream), on the current
 * device. The work is enqueued, not waited for. Same result as
 * ns3d_compute_rhs for the same params (p->precision selects the form).
 * The intermediates live in one fixed 7.5 MiB array of this library's device
 * memory, held by every GPU that loads the library until exit; boxes above
 * NS3D_NOALLOC_MAX_CELLS cells are rejected with NS3D_ERR_INVALID. All calls
 * share that array and it keeps the last call's contents, so calls that
 * overlap on the GPU race: serialise them. The first call on each device looks
 * up the array's device address; make that first call before any stream
 * capture. */
ns3d_status ns3d_compute_rhs_noalloc(const ns3d_params *p, const double *rho, const double *u,
                                     const double *v, const double *w, const double *pres,
                                     double *rhs, void *stream);

/* ---- instrumentation (no reference counterpart) -------------------------- */

/* Kernel classes timed by ns3d_profile. */
enum {
    NS3D_KERNEL_SWEEP_X = 0, NS3D_KERNEL_SWEEP_Y = 1, NS3D_KERNEL_SWEEP_Z = 2,
    NS3D_KERNEL_VISC_FLUX = 3, NS3D_KERNEL_UPDATE = 4, NS3D_KERNEL_OTHER = 5,
    /* the z sweep fused with the stage update (component-wise schemes) */
    NS3D_KERNEL_SWEEP_Z_UPDATE = 6,
    NS3D_KERNEL_CLASSES = 7
};
/* The cudaStream_t every kernel of this context is launched on. */
ns3d_status ns3d_get_stream(ns3d_ctx *ctx, void **stream);
/* enable != 0: reset and start recording a CUDA event pair around every
 * launch, per kernel class; enable == 0: stop recording. */
ns3d_status ns3d_profile(ns3d_ctx *ctx, int enable);
/* Summed device milliseconds and launch counts per class since the last
 * ns3d_profile(ctx, 1); arrays of NS3D_KERNEL_CLASSES entries. Synchronizes. */
ns3d_status ns3d_profile_read(ns3d_ctx *ctx, double *ms, long long *launches);
/* Kernels this context has launched since creation. */
ns3d_status ns3d_launch_count(const ns3d_ctx *ctx, long long *count);

/* ---- reductions ----------------------------------------------------------- */

/* compute_total_energy (postprocess.cpp:103-128): sum 0.5 rho |u|^2 dx dy dz. */
ns3d_status ns3d_total_energy(ns3d_ctx *ctx, double *etot);
/* compute_energy_spectrum (EnergySpectrum.cpp:62-125): E(k), k = 0..nbins-1,
 * nbins <= 2*global_nx + 1; transform of u,v,w scaled by 1/N, shells by floor(|k|). */
ns3d_status ns3d_energy_spectrum(ns3d_ctx *ctx, double *Ek, int nbins);
/* ---- field I/O in the reference's Tecplot ASCII format (host code) -------- */
/* write_tecplot_field (output.cpp:21-87) of host arrays (interior layout): the
 * TITLE / VARIABLES / ZONE lines and one "X Y Z rho u v w E p T" record per cell,
 * x fastest, %.8e, byte-identical to the reference's file for the same state; E and
 * T as primitiveToConserved computes them. `rank` labels the title and zone as the
 * reference's per-rank files do. NS3D_ERR_FILE when the file cannot be written. */
ns3d_status ns3d_tecplot_write(const ns3d_params *p, const double *rho, const double *u,
                               const double *v, const double *w, const double *pres,
                               const char *path, double time, int rank);
/* initialize_from_tecplot (initialization.cpp:35-100) into host arrays: the records
 * after the first ZONE line as a whitespace-separated stream; E and T are dropped
 * (the reference rebuilds them from the primitives, main.cpp:70-71). NS3D_ERR_FILE
 * when the file cannot be opened or holds fewer records than cells. */
ns3d_status ns3d_tecplot_read(const ns3d_params *p, const char *path, double *rho, double *u,
                              double *v, double *w, double *pres);
/* initialize_from_tecplot_downsample (initialization.cpp:102-198): nearest-neighbour
 * sampling (llround(g * src / n), clamped) of a src_nx x src_ny x src_nz file. */
ns3d_status ns3d_tecplot_read_downsample(const ns3d_params *p, const char *path, int src_nx,
                                         int src_ny, int src_nz, double *rho, double *u,
                                         double *v, double *w, double *pres);
/* write_residuals_tecplot (output.cpp:92-128): `path` is created with its TITLE /
 * VARIABLES header when step == 1 and appended to otherwise; one row
 * "step res_rho res_rhou res_rhov res_rhow res_E Etot" (%.8e). */
ns3d_status ns3d_residuals_write(const char *path, int step, const double *res, double etot);
/* The same for the context's state: download + write, read + upload. */
ns3d_status ns3d_write_tecplot(ns3d_ctx *ctx, const char *path, double time);
ns3d_status ns3d_read_tecplot(ns3d_ctx *ctx, const char *path);

/* Binary checkpoint of the context (no counterpart in the reference, which restarts
 * from its 9-digit Tecplot field, initialization.cpp:35-100): the current state's
 * rho, u, v, w, p, T bit for bit, the clock and step count of ns3d_time_advance, the
 * state's CFL minimum and the gas it belongs to, with a 64-bit checksum. Reading it
 * into a context of the same grid and gas gives a run that repeats the uninterrupted
 * one exactly (U0 recorded from the read state; ns3d_run numbers on from the stored
 * step count). NS3D_ERR_FILE: unreadable, not a (version 2) checkpoint, truncated or
 * checksum mismatch; NS3D_ERR_INVALID: another grid or another gas (gamma, Rgas, mu,
 * Pr, Cp or Sutherland's S/Tref: T = p/(rho Rgas) and the CFL minimum would no longer
 * belong to the context). ns3d_checkpoint_check tests a file's header against
 * parameters on the host, without a context or a GPU. */
ns3d_status ns3d_checkpoint_write(ns3d_ctx *ctx, const char *path);
ns3d_status ns3d_checkpoint_read(ns3d_ctx *ctx, const char *path);
ns3d_status ns3d_checkpoint_check(const char *path, const ns3d_params *p);
/* Steps the time_advance loops of this context have completed (the step number
 * beside ns3d_time_advance's clock; restored by ns3d_checkpoint_read). */
ns3d_status ns3d_completed_steps(ns3d_ctx *ctx, long long *steps);

/* compute_diagnostics (postprocess.cpp:7-98) after a step: res[q] = sqrt(sum (U - U0)^2
 * dx^3) / max |U| for rho, rhou, rhov, rhow, E, with U the current state and U0 the
 * recorded one (recordConservedTo0 of the step's start; stepping keeps it until the
 * next step). */
ns3d_status ns3d_residuals(ns3d_ctx *ctx, double *res);

/* init_isotropic_turbulence (isotropic_ini.cpp:146-193) with generate_full_turbulence
 * (:25-122) into the context's state: a random-phase solenoidal velocity with spectrum
 * ~ kk exp(-2 kk / k0^2), the phases drawn from mt19937_64(seed) + uniform [0, 1) in the
 * reference's order (no draws for k = 0), inverse transforms on the device (cuFFT),
 * rho = 1, T = 1, p = Rgas. mach_t <= 0 normalises the mean 0.5|u|^2 to
 * Ek0 = 3A/64 sqrt(2 pi) k0^5 as the reference does; mach_t > 0 scales the velocity
 * to that turbulent Mach number sqrt(2 KE) / <c> instead. k0 = 8, A = 0.00013,
 * seed = 123, mach_t = 0 reproduce the reference's first call in a process (its
 * generator keeps one static stream per process). Allocates and frees its scratch
 * (72 bytes per cell on the device). */
ns3d_status ns3d_init_isotropic(ns3d_ctx *ctx, int k0, double A, unsigned long long seed,
                                double mach_t);
/* compute_turbulence_statistics (ana_isotropic.cpp:196-314): every quantity of its
 * statistics row, without the rank-0 gather and the spectrum file round trip. */
ns3d_status ns3d_turbulence_stats(ns3d_ctx *ctx, ns3d_turb_stats *out);
/* The same statistics from a caller's spectrum Ek[0..nbins) (the reference computes
 * them from the spectrum re-read from its 6-digit file, ana_isotropic.cpp:210-221). */
ns3d_status ns3d_turbulence_stats_spectrum(ns3d_ctx *ctx, const double *Ek, int nbins,
                                           ns3d_turb_stats *out);

/* compute_energy_spectrum's file (EnergySpectrum.cpp:127-133): one "k E(k)" row per
 * bin, E(k) in the stream's default 6-digit format (%g). */
ns3d_status ns3d_spectrum_write(const char *path, const double *Ek, int nbins);
/* compute_turbulence_statistics' table (ana_isotropic.cpp:317-342): the header line
 * when `path` does not exist yet, then one appended row of 12 values (%.8e). */
ns3d_status ns3d_stats_write(const char *path, double time, const ns3d_turb_stats *s);

/* time_advance (maincycle.cpp:7-112) with its monitor and output, files under
 * `workdir`/output as the reference writes them under its working directory:
 * every monitor_Stepfreq-th step and step 1, the residuals (monitor_res; rows of
 * output_residuals.dat), the total energy (monitor_energy) and the isotropic
 * post-processing (spectrum file + statistics row); after every output step, the
 * Tecplot field time_<100000 t>/field_rank0.dat (post_basicfield) and the isotropic
 * post-processing. verbose: the reference's "[Step n] ..." monitor lines on stdout.
 * Steps are numbered on from the context's completed steps (ns3d_completed_steps: 0
 * for a new context, the stored count after ns3d_checkpoint_read), and `max_steps` is
 * the last step number, as in the reference's loop; a run continued from a checkpoint
 * so writes the files of the uninterrupted run. Between monitor and output steps the
 * loop runs on the device without host synchronisation. NS3D_ERR_INVALID for
 * monitor_Stepfreq <= 0 (a division by zero in the reference). */
ns3d_status ns3d_run(ns3d_ctx *ctx, const char *workdir, int max_steps, int verbose,
                     double *time, int *steps_done);

#ifdef __cplusplus
}
#endif

#endif /* NS3D_GPU_H */
