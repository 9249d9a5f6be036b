// C-ABI driver around the reference's own hot-path functions, compiled together
// with the unmodified reference sources into oracle/_ref/libns3d_ref.so.
//
// TEST INFRASTRUCTURE ONLY. It is the pin for the oracle restatement
// (oracle/ns3d_oracle.c) and the CPU baseline ("kind": "reference"); product
// code never loads it.
//
// Every entry mirrors a reference call sequence:
//   ref_create        -> read_solver_params_from_file (initialization.cpp:199),
//                        build_cart_decomp / compute_local_desc (field_structures.h:858,887),
//                        Field3D::allocate (field_structures.h:225)       [main.cpp:12-59]
//   ref_set_primitive -> interior primitives, apply_boundary, primitiveToConserved [main.cpp:67-71]
//   ref_set_conserved -> conservedToPrimitive, apply_boundary, primitiveToConserved
//                        [range_kutta.cpp:117-119]
//   ref_record0 / ref_timestep / ref_compute_rhs / ref_rk3 / ref_time_advance
//                     -> recordConservedTo0, compute_timestep, compute_rhs,
//                        runge_kutta_3, time_advance
#include <cstdio>
#include <cstring>
#include <exception>
#include <string>
#include <unistd.h>

#include "field_structures.h"
#include "ns3d_func.h"

struct RefCtx {
    SolverParams P;
    GridDesc G;
    CartDecomp C;
    Field3D F;
    HaloRequests reqs;
    std::string last_error;
};

namespace {

std::vector<double> *cell_field(Field3D &F, const std::string &n) {
#define NS3D_F(x) if (n == #x) return &F.x;
    NS3D_F(rho) NS3D_F(rhou) NS3D_F(rhov) NS3D_F(rhow) NS3D_F(E)
    NS3D_F(rho0) NS3D_F(rhou0) NS3D_F(rhov0) NS3D_F(rhow0) NS3D_F(E0)
    NS3D_F(u) NS3D_F(v) NS3D_F(w) NS3D_F(p) NS3D_F(T) NS3D_F(c)
    NS3D_F(rhs_rho) NS3D_F(rhs_rhou) NS3D_F(rhs_rhov) NS3D_F(rhs_rhow) NS3D_F(rhs_E)
    NS3D_F(du_dx) NS3D_F(du_dy) NS3D_F(du_dz) NS3D_F(dv_dx) NS3D_F(dv_dy) NS3D_F(dv_dz)
    NS3D_F(dw_dx) NS3D_F(dw_dy) NS3D_F(dw_dz) NS3D_F(dT_dx) NS3D_F(dT_dy) NS3D_F(dT_dz)
    NS3D_F(Fvflux_momx) NS3D_F(Fvflux_momy) NS3D_F(Fvflux_momz) NS3D_F(Fvflux_E)
    NS3D_F(Hvflux_momx) NS3D_F(Hvflux_momy) NS3D_F(Hvflux_momz) NS3D_F(Hvflux_E)
    NS3D_F(Gvflux_momx) NS3D_F(Gvflux_momy) NS3D_F(Gvflux_momz) NS3D_F(Gvflux_E)
#undef NS3D_F
    return nullptr;
}

std::vector<double> *face_field(Field3D &F, const std::string &n, int *dir) {
#define NS3D_FF(x, d) if (n == #x) { *dir = d; return &F.x; }
    NS3D_FF(flux_fx_mass, 0) NS3D_FF(flux_fx_momx, 0) NS3D_FF(flux_fx_momy, 0)
    NS3D_FF(flux_fx_momz, 0) NS3D_FF(flux_fx_E, 0)
    NS3D_FF(flux_fy_mass, 1) NS3D_FF(flux_fy_momx, 1) NS3D_FF(flux_fy_momy, 1)
    NS3D_FF(flux_fy_momz, 1) NS3D_FF(flux_fy_E, 1)
    NS3D_FF(flux_fz_mass, 2) NS3D_FF(flux_fz_momx, 2) NS3D_FF(flux_fz_momy, 2)
    NS3D_FF(flux_fz_momz, 2) NS3D_FF(flux_fz_E, 2)
#undef NS3D_FF
    return nullptr;
}

template <class Fn>
int guarded(RefCtx *c, Fn fn) {
    try {
        fn();
        return 0;
    } catch (const std::exception &e) {
        c->last_error = e.what();
        return -1;
    }
}

}  // namespace

// The Field3D shim (ns3d_cpp_b200/shim), when this driver is linked into the
// reference build that uses it, keeps the state on the GPU: host reads of
// Field3D sync it first, host writes invalidate the device copy. Weak, so the
// plain reference build (no shim) links without them.
void ns3d_shim_sync(Field3D &F) __attribute__((weak));
void ns3d_shim_invalidate(const Field3D &F) __attribute__((weak));

static void host_reads(Field3D &F) {
    if (ns3d_shim_sync) ns3d_shim_sync(F);
}
static void host_wrote(const Field3D &F) {
    if (ns3d_shim_invalidate) ns3d_shim_invalidate(F);
}

extern "C" {

void *ref_create(const char *solver_in) {
    auto *c = new RefCtx;
    if (!read_solver_params_from_file(solver_in, c->P, c->G, c->C)) {
        delete c;
        return nullptr;
    }
    build_cart_decomp(c->C);
    LocalDesc L;
    int g = c->P.ghost_layers;
    compute_local_desc(c->G, c->C, L, g, g, g);
    c->F.allocate(L);
    return c;
}

void ref_destroy(void *h) {
    auto *c = static_cast<RefCtx *>(h);
    host_wrote(c->F);  // a later Field3D may take the same addresses
    delete c;
}

const char *ref_last_error(void *h) { return static_cast<RefCtx *>(h)->last_error.c_str(); }

// out: nx, ny, nz, ng, stencil, fvs, recon, vis_scheme, char_recon
void ref_dims(void *h, int *out) {
    auto *c = static_cast<RefCtx *>(h);
    const LocalDesc &L = c->F.L;
    out[0] = L.nx; out[1] = L.ny; out[2] = L.nz; out[3] = L.ngx;
    out[4] = c->P.stencil;
    out[5] = (int)c->P.fvs_type;
    out[6] = (int)c->P.recon;
    out[7] = (int)c->P.vis_scheme;
    out[8] = c->P.char_recon ? 1 : 0;
}

// out: gamma Pr Ma Re cfl dt_fixed Cv Cp Rgas mu dx dy dz mdcd_diss mdcd_disp ud7l_alpha
//      TotalTime output_Timefreq max_steps monitor_Stepfreq get_mu(1.0)
void ref_params(void *h, double *out) {
    auto *c = static_cast<RefCtx *>(h);
    const SolverParams &P = c->P;
    const GridDesc &G = c->G;
    double v[] = {P.gamma, P.Pr, P.Ma, P.Re, P.cfl, P.dt_fixed, P.Cv, P.Cp, P.Rgas, P.mu,
                  G.dx, G.dy, G.dz, P.mdcd_diss, P.mdcd_disp, P.ud7l_alpha, P.TotalTime,
                  P.output_Timefreq, (double)P.max_steps, (double)P.monitor_Stepfreq,
                  P.get_mu(1.0)};
    std::memcpy(out, v, sizeof(v));
}

static void put_interior(RefCtx *c, std::vector<double> &dst, const double *src) {
    const LocalDesc &L = c->F.L;
    long q = 0;
    for (int k = 0; k < L.nz; ++k)
        for (int j = 0; j < L.ny; ++j)
            for (int i = 0; i < L.nx; ++i)
                dst[idx3(i + L.ngx, j + L.ngy, k + L.ngz, L)] = src[q++];
}

int ref_set_primitive(void *h, const double *rho, const double *u, const double *v,
                      const double *w, const double *p) {
    auto *c = static_cast<RefCtx *>(h);
    return guarded(c, [&] {
        put_interior(c, c->F.rho, rho);
        put_interior(c, c->F.u, u);
        put_interior(c, c->F.v, v);
        put_interior(c, c->F.w, w);
        put_interior(c, c->F.p, p);
        apply_boundary(c->F, c->G, c->C, c->P);
        c->F.primitiveToConserved(c->P);
        host_wrote(c->F);
    });
}

int ref_set_conserved(void *h, const double *rho, const double *ru, const double *rv,
                      const double *rw, const double *E) {
    auto *c = static_cast<RefCtx *>(h);
    return guarded(c, [&] {
        put_interior(c, c->F.rho, rho);
        put_interior(c, c->F.rhou, ru);
        put_interior(c, c->F.rhov, rv);
        put_interior(c, c->F.rhow, rw);
        put_interior(c, c->F.E, E);
        c->F.conservedToPrimitive(c->P);
        apply_boundary(c->F, c->G, c->C, c->P);
        c->F.primitiveToConserved(c->P);
        host_wrote(c->F);
    });
}

// Interior (nx*ny*nz, x fastest) of a cell-centred array.
int ref_get(void *h, const char *name, double *out) {
    auto *c = static_cast<RefCtx *>(h);
    host_reads(c->F);
    std::vector<double> *a = cell_field(c->F, name);
    if (!a) return -2;
    const LocalDesc &L = c->F.L;
    long q = 0;
    for (int k = 0; k < L.nz; ++k)
        for (int j = 0; j < L.ny; ++j)
            for (int i = 0; i < L.nx; ++i)
                out[q++] = (*a)[idx3(i + L.ngx, j + L.ngy, k + L.ngz, L)];
    return 0;
}

// Whole ghosted array (sx*sy*sz) of a cell-centred field.
int ref_get_full(void *h, const char *name, double *out) {
    auto *c = static_cast<RefCtx *>(h);
    host_reads(c->F);
    std::vector<double> *a = cell_field(c->F, name);
    if (!a) return -2;
    std::memcpy(out, a->data(), a->size() * sizeof(double));
    return 0;
}

// Face fluxes at the faces the sweep writes: x faces i_face in [ng-1, ng+nx-1]
// over interior (j,k), returned as (nz, ny, nx+1); y and z analogously.
int ref_get_face(void *h, const char *name, double *out) {
    auto *c = static_cast<RefCtx *>(h);
    int dir = -1;
    std::vector<double> *a = face_field(c->F, name, &dir);
    if (!a) return -2;
    const LocalDesc &L = c->F.L;
    const int g = L.ngx;
    long q = 0;
    if (dir == 0) {
        for (int k = g; k < g + L.nz; ++k)
            for (int j = g; j < g + L.ny; ++j)
                for (int i = g - 1; i < g + L.nx; ++i) out[q++] = (*a)[idx_fx(i, j, k, L)];
    } else if (dir == 1) {
        for (int k = g; k < g + L.nz; ++k)
            for (int j = g - 1; j < g + L.ny; ++j)
                for (int i = g; i < g + L.nx; ++i) out[q++] = (*a)[idx_fy(i, j, k, L)];
    } else {
        for (int k = g - 1; k < g + L.nz; ++k)
            for (int j = g; j < g + L.ny; ++j)
                for (int i = g; i < g + L.nx; ++i) out[q++] = (*a)[idx_fz(i, j, k, L)];
    }
    return 0;
}

void ref_record0(void *h) { static_cast<RefCtx *>(h)->F.recordConservedTo0(); }

double ref_timestep(void *h) {
    auto *c = static_cast<RefCtx *>(h);
    return compute_timestep(c->F, c->G, c->P);
}

int ref_compute_rhs(void *h) {
    auto *c = static_cast<RefCtx *>(h);
    return guarded(c, [&] { compute_rhs(c->F, c->C, c->G, c->P, c->reqs); });
}

int ref_rk3(void *h, double dt) {
    auto *c = static_cast<RefCtx *>(h);
    return guarded(c, [&] { runge_kutta_3(c->F, c->C, c->G, c->P, c->reqs, dt); });
}

// One time_advance step as maincycle.cpp:14-24 does it when dt comes from CFL:
// recordConservedTo0, compute_timestep, runge_kutta_3. Returns the dt used.
double ref_cfl_step(void *h) {
    auto *c = static_cast<RefCtx *>(h);
    c->F.recordConservedTo0();
    double dt = c->P.dt_fixed;
    if (c->P.dt_fixed < 0.0) dt = compute_timestep(c->F, c->G, c->P);
    if (ref_rk3(h, dt) != 0) return -1.0;
    return dt;
}

// The reference's own driver loop (maincycle.cpp:7), run inside `workdir`
// (it writes output/ files when post-processing is enabled).
int ref_time_advance(void *h, const char *workdir) {
    auto *c = static_cast<RefCtx *>(h);
    char old[4096];
    if (!getcwd(old, sizeof(old))) return -3;
    if (workdir && chdir(workdir) != 0) return -3;
    int rc = guarded(c, [&] { time_advance(c->F, c->C, c->G, c->P); });
    if (chdir(old) != 0) return -3;
    return rc;
}

double ref_total_energy(void *h) {
    auto *c = static_cast<RefCtx *>(h);
    compute_total_energy(c->F, c->G, c->C, c->P);
    return c->F.global_Etot;
}

// isotropic_post_process (postprocess.cpp:133): spectrum file + turbulence_stats.dat,
// written under `workdir`/output/.
int ref_isotropic_post(void *h, const char *workdir, double t) {
    auto *c = static_cast<RefCtx *>(h);
    char old[4096];
    if (!getcwd(old, sizeof(old))) return -3;
    if (chdir(workdir) != 0) return -3;
    int rc = guarded(c, [&] { isotropic_post_process(c->F, c->G, c->C, c->P, t); });
    if (chdir(old) != 0) return -3;
    return rc;
}

// The reference's isotropic generator (isotropic_ini.cpp:132, k0=8, A=1.3e-4,
// mt19937_64 seed 123) followed by main.cpp:70-71.
// write_tecplot_field with `dir` as the working directory (the reference writes
// output/time_<100000 t>/field_rank0.dat under it).
int ref_write_tecplot(void *h, const char *dir, double time) {
    auto *c = static_cast<RefCtx *>(h);
    char old[4096];
    if (!getcwd(old, sizeof old) || chdir(dir) != 0) return -1;
    int r = guarded(c, [&] { write_tecplot_field(c->F, c->G, c->C, c->P, time); });
    if (chdir(old) != 0) return -1;
    return r;
}

// main.cpp:67-71: initialize_from_tecplot (or the downsampling form when
// src_nx > 0), apply_boundary, primitiveToConserved.
int ref_read_tecplot(void *h, const char *path, int src_nx, int src_ny, int src_nz) {
    auto *c = static_cast<RefCtx *>(h);
    int ok = 1;
    int r = guarded(c, [&] {
        ok = src_nx > 0 ? initialize_from_tecplot_downsample(c->F, c->G, c->C, c->P, path, src_nx,
                                                             src_ny, src_nz)
                        : initialize_from_tecplot(c->F, c->G, c->C, c->P, path);
        if (ok) {
            apply_boundary(c->F, c->G, c->C, c->P);
            c->F.primitiveToConserved(c->P);
        }
        host_wrote(c->F);
    });
    return r != 0 ? r : (ok ? 0 : 1);
}

// compute_diagnostics (postprocess.cpp:7-98) on the state left by the last step
// (U0 recorded at its start); out = global_res_rho, _rhou, _rhov, _rhow, _E.
int ref_diagnostics(void *h, double *out) {
    auto *c = static_cast<RefCtx *>(h);
    return guarded(c, [&] {
        compute_diagnostics(c->F, c->P, c->G);
        const double r[5] = {c->F.global_res_rho, c->F.global_res_rhou, c->F.global_res_rhov,
                             c->F.global_res_rhow, c->F.global_res_E};
        for (int q = 0; q < 5; ++q) out[q] = r[q];
    });
}

// write_residuals_tecplot (output.cpp:92-128) with `dir` as the working
// directory: output/output_residuals.dat, the row of the last diagnostics and
// of F.global_Etot (compute_total_energy first when `energy` is set).
int ref_write_residuals(void *h, const char *dir, int step, int energy) {
    auto *c = static_cast<RefCtx *>(h);
    char old[4096];
    if (!getcwd(old, sizeof old) || chdir(dir) != 0) return -1;
    int r = guarded(c, [&] {
        if (energy) compute_total_energy(c->F, c->G, c->C, c->P);
        write_residuals_tecplot(c->F, step, "output_residuals.dat");
    });
    if (chdir(old) != 0) return -1;
    return r;
}

int ref_init_isotropic(void *h) {
    auto *c = static_cast<RefCtx *>(h);
    return guarded(c, [&] {
        init_isotropic_turbulence(c->F, c->G, c->C, c->P);
        apply_boundary(c->F, c->G, c->C, c->P);
        c->F.primitiveToConserved(c->P);
        host_wrote(c->F);
    });
}

}  // extern "C"
