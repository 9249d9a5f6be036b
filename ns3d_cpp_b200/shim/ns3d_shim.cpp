// ns3d_shim.cpp -- the reference's hot-path entry points over Field3D, run on
// the B200 through the C ABI of ns3d_gpu.h.
//
// Replaces, with identical signatures (ns3d_func.h:99-105):
//   compute_rhs      (range_kutta.cpp:11)
//   runge_kutta_3    (range_kutta.cpp:102)
//   compute_timestep (timestep.cpp:5)
// Compile it against the application's field_structures.h / ns3d_func.h in
// place of range_kutta.cpp and timestep.cpp and link libns3d_b200.so; the
// application's time_advance (maincycle.cpp) and main.cpp stay unchanged.
//
// Semantics:
// * The whole domain lives on one GPU: a single rank whose local block is the
//   global grid (the reference's periodic 1x1x1 decomposition). Anything else
//   is rejected with a clear error.
// * Each call uploads Field3D's primitives (rho,u,v,w,p, ghosted layout; only
//   the interior is read) and, for runge_kutta_3, writes back every array the
//   monitor and output code reads: rho..E, u,v,w,p,T,c (ghost faces hold the
//   periodic images, as after apply_boundary). The rhs_* arrays receive the
//   RHS only from compute_rhs; face fluxes, gradients and viscous fluxes are
//   intermediate in the reference and are not written back.
// * runge_kutta_3 uses U0 = recordConservedTo0 of the state it receives, which
//   is what time_advance guarantees (maincycle.cpp:22); rho0..E0 are checked
//   against that and a mismatch is reported instead of silently used.
// * A non-physical state ends in MPI_Abort with the reference's message
//   (range_kutta.cpp:149-162); NaN is reported too.
// * NS3D_PRECISION=fp32acc64 selects the FP32-stencil form; NS3D_DEVICE picks
//   the GPU (default 0).
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <string>

#include "field_structures.h"
#include "ns3d_func.h"
#include "ns3d_gpu.h"

namespace {

struct Shim {
    ns3d_ctx* ctx = nullptr;
    ns3d_params params{};
};
Shim g_shim;

void fail(const std::string& msg) {
    std::fprintf(stderr, "ns3d shim: %s\n", msg.c_str());
    MPI_Abort(MPI_COMM_WORLD, -1);
    throw std::runtime_error(msg);  // only reached where MPI_Abort returns
}

void check(ns3d_status s, const char* what) {
    if (s != NS3D_OK)
        fail(std::string(what) + " failed: " + ns3d_last_error(g_shim.ctx) + " (status " +
             std::to_string((int)s) + ")");
}

// SolverParams + GridDesc -> ns3d_params, field by field.
ns3d_params to_params(const SolverParams& P, const GridDesc& G) {
    ns3d_params q;
    ns3d_params_default(&q);
    q.gamma = P.gamma;
    q.Pr = P.Pr;
    q.Ma = P.Ma;
    q.Re = P.Re;
    q.cfl = P.cfl;
    q.dt_fixed = P.dt_fixed;
    q.fvs_type = (int)P.fvs_type;
    q.recon = (int)P.recon;
    q.vis_scheme = (int)P.vis_scheme;
    q.char_recon = P.char_recon ? 1 : 0;
    q.mdcd_diss = P.mdcd_diss;
    q.mdcd_disp = P.mdcd_disp;
    q.ud7l_alpha = P.ud7l_alpha;
    q.global_nx = G.global_nx;
    q.global_ny = G.global_ny;
    q.global_nz = G.global_nz;
    q.x0 = G.x0; q.y0 = G.y0; q.z0 = G.z0;
    q.Lx = G.Lx; q.Ly = G.Ly; q.Lz = G.Lz;
    const SolverParams::BCType bc[6] = {P.bc_xmin, P.bc_xmax, P.bc_ymin,
                                        P.bc_ymax, P.bc_zmin, P.bc_zmax};
    for (int f = 0; f < 6; ++f) q.bc[f] = (int)bc[f];
    q.max_steps = P.max_steps;
    q.monitor_Stepfreq = P.monitor_Stepfreq;
    q.output_Timefreq = P.output_Timefreq;
    q.TotalTime = P.TotalTime;
    q.post_basicfield = P.post_basicfield;
    q.isotropic_analyse = P.isotropic_analyse;
    q.monitor_res = P.monitor_res;
    q.monitor_energy = P.monitor_energy;
    const char* prec = std::getenv("NS3D_PRECISION");
    if (prec && std::string(prec) == "fp32acc64") q.precision = NS3D_PREC_FP32_ACC64;
    ns3d_params_derive(&q);
    return q;
}

bool same_params(const ns3d_params& a, const ns3d_params& b) {
    return std::memcmp(&a, &b, sizeof(ns3d_params)) == 0;
}

ns3d_ctx* context(const Field3D& F, const SolverParams& P, const GridDesc& G) {
    const LocalDesc& L = F.L;
    if (L.nx != G.global_nx || L.ny != G.global_ny || L.nz != G.global_nz)
        fail("the B200 path holds the whole domain on one GPU: run with one rank");
    ns3d_params q = to_params(P, G);
    if (L.ngx != q.ghost_layers || L.ngy != q.ghost_layers || L.ngz != q.ghost_layers)
        fail("Field3D ghost width differs from the one the schemes derive");
    if (!g_shim.ctx || !same_params(q, g_shim.params)) {
        if (g_shim.ctx) ns3d_destroy(g_shim.ctx);
        g_shim.ctx = nullptr;
        const char* dev = std::getenv("NS3D_DEVICE");
        check(ns3d_create(&q, dev ? std::atoi(dev) : 0, &g_shim.ctx), "ns3d_create");
        g_shim.params = q;
    }
    return g_shim.ctx;
}

void upload(ns3d_ctx* ctx, const Field3D& F) {
    check(ns3d_upload_primitive(ctx, F.rho.data(), F.u.data(), F.v.data(), F.w.data(),
                                F.p.data(), NS3D_LAYOUT_GHOSTED),
          "ns3d_upload_primitive");
}

void download(ns3d_ctx* ctx, Field3D& F) {
    check(ns3d_download_primitive(ctx, F.rho.data(), F.u.data(), F.v.data(), F.w.data(),
                                  F.p.data(), F.T.data(), F.c.data(), NS3D_LAYOUT_GHOSTED),
          "ns3d_download_primitive");
    check(ns3d_download_conserved(ctx, F.rho.data(), F.rhou.data(), F.rhov.data(),
                                  F.rhow.data(), F.E.data(), NS3D_LAYOUT_GHOSTED),
          "ns3d_download_conserved");
}

// rho0..E0 must be recordConservedTo0 of the current conserved state.
void check_u0(const Field3D& F) {
    const LocalDesc& L = F.L;
    for (int k = L.ngz; k < L.ngz + L.nz; ++k)
        for (int j = L.ngy; j < L.ngy + L.ny; ++j)
            for (int i = L.ngx; i < L.ngx + L.nx; ++i) {
                const int id = idx3(i, j, k, L);
                if (F.rho0[id] != F.rho[id] || F.rhou0[id] != F.rhou[id] ||
                    F.rhov0[id] != F.rhov[id] || F.rhow0[id] != F.rhow[id] ||
                    F.E0[id] != F.E[id])
                    fail("runge_kutta_3 needs rho0..E0 == recordConservedTo0() of the state "
                         "(as time_advance calls it)");
            }
}

}  // namespace

void compute_rhs(Field3D& F, CartDecomp& C, GridDesc& G, SolverParams& P, HaloRequests&) {
    (void)C;
    ns3d_ctx* ctx = context(F, P, G);
    upload(ctx, F);
    check(ns3d_compute_rhs(ctx, F.rhs_rho.data(), F.rhs_rhou.data(), F.rhs_rhov.data(),
                           F.rhs_rhow.data(), F.rhs_E.data(), NS3D_LAYOUT_GHOSTED),
          "ns3d_compute_rhs");
}

double compute_timestep(Field3D& F, const GridDesc& G, const SolverParams& P) {
    ns3d_ctx* ctx = context(F, P, G);
    upload(ctx, F);
    double dt = 0.0;
    check(ns3d_compute_timestep(ctx, &dt), "ns3d_compute_timestep");
    return dt;
}

void runge_kutta_3(Field3D& F, CartDecomp& C, GridDesc& G, SolverParams& P, HaloRequests&,
                   double dt) {
    (void)C;
    ns3d_ctx* ctx = context(F, P, G);
    check_u0(F);
    upload(ctx, F);  // records U0 = prim2cons(state) == rho0..E0
    const ns3d_status s = ns3d_runge_kutta_3(ctx, dt);
    download(ctx, F);
    if (s == NS3D_ERR_NONPHYSICAL) {
        std::printf("Error: Non-physical value detected at rank 0: %s\n", ns3d_last_error(ctx));
        MPI_Abort(MPI_COMM_WORLD, -1);
    }
    check(s, "ns3d_runge_kutta_3");
}
