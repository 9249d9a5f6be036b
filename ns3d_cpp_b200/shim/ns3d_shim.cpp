// ns3d_shim.cpp -- the reference's hot-path entry points over Field3D, run on
// the B200 through the C ABI of ns3d_gpu.h.
//
// Replaces, with identical signatures (ns3d_func.h:99-105, 167-186):
//   compute_rhs             (range_kutta.cpp:11)
//   runge_kutta_3           (range_kutta.cpp:102)
//   compute_timestep        (timestep.cpp:5)
//   compute_diagnostics     (postprocess.cpp:7)
//   compute_total_energy    (postprocess.cpp:103)
//   isotropic_post_process  (postprocess.cpp:133)
//   write_tecplot_field     (output.cpp:21)
//   write_residuals_tecplot (output.cpp:93)
// Compile it against the application's field_structures.h / ns3d_func.h in
// place of range_kutta.cpp, timestep.cpp, postprocess.cpp and output.cpp and
// link libns3d_b200.so; the application's time_advance (maincycle.cpp) and
// main.cpp stay unchanged.
//
// Semantics:
// * The whole domain lives on one GPU: a single rank whose local block is the
//   global grid (the reference's periodic 1x1x1 decomposition). Anything else
//   is rejected with a clear error.
// * The state stays resident on the GPU. The first call for a Field3D uploads
//   its primitives (rho,u,v,w,p, ghosted layout; only the interior is read);
//   later calls work on the device state, and runge_kutta_3 writes nothing
//   back. The monitor and output functions above, which are what reads
//   Field3D between steps in time_advance, run on the device too:
//   compute_diagnostics and compute_total_energy set F.global_res_* and
//   F.global_Etot; isotropic_post_process writes the spectrum file and the
//   statistics row; write_tecplot_field first copies the device state into
//   Field3D (rho..E, u,v,w,p,T,c; ghost faces hold the periodic images, as
//   after apply_boundary) and writes the same file. Host code that reads
//   Field3D elsewhere calls ns3d_shim_sync(F) first; host code that changes
//   it between calls calls ns3d_shim_invalidate(F) (both in ns3d_shim.h).
// * runge_kutta_3 takes U0 from the device state it starts from: what
//   time_advance's recordConservedTo0 right before it records (maincycle.cpp:22).
//   While the state is resident, Field3D's rho0..E0 and res_* are not kept
//   (compute_diagnostics reduces U - U0 on the device instead).
// * A non-physical state ends in MPI_Abort with the reference's message
//   (range_kutta.cpp:149-162), after the state is copied into Field3D; NaN
//   is reported too.
// * NS3D_PRECISION=fp32acc64 selects the FP32-stencil form; NS3D_DEVICE picks
//   the GPU (default 0); NS3D_SHIM_SYNC=eager uploads before and downloads
//   after every call (the state is then never resident).
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <filesystem>
#include <iomanip>
#include <iostream>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "field_structures.h"
#include "ns3d_func.h"
#include "ns3d_gpu.h"
#include "ns3d_shim.h"

namespace {

struct Shim {
    ns3d_ctx* ctx = nullptr;
    ns3d_params params{};
    const Field3D* owner = nullptr;  // the Field3D whose state the device holds
    const double* owner_rho = nullptr;
    bool host_stale = false;         // the device state is newer than Field3D's arrays
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

bool eager() {
    const char* e = std::getenv("NS3D_SHIM_SYNC");
    return e && std::strcmp(e, "eager") == 0;
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

void download(ns3d_ctx* ctx, Field3D& F) {
    check(ns3d_download_primitive(ctx, F.rho.data(), F.u.data(), F.v.data(), F.w.data(),
                                  F.p.data(), F.T.data(), F.c.data(), NS3D_LAYOUT_GHOSTED),
          "ns3d_download_primitive");
    check(ns3d_download_conserved(ctx, F.rho.data(), F.rhou.data(), F.rhov.data(),
                                  F.rhow.data(), F.E.data(), NS3D_LAYOUT_GHOSTED),
          "ns3d_download_conserved");
}

bool holds(const Field3D& F) { return g_shim.owner == &F && g_shim.owner_rho == F.rho.data(); }

// The context for (P, G), with F's state on the device: uploaded on the first
// call for this Field3D (or after a parameter change or an invalidation).
ns3d_ctx* resident(const Field3D& F, const SolverParams& P, const GridDesc& G) {
    const LocalDesc& L = F.L;
    if (L.nx != G.global_nx || L.ny != G.global_ny || L.nz != G.global_nz)
        fail("the B200 path holds the whole domain on one GPU: run with one rank");
    ns3d_params q = to_params(P, G);
    if (L.ngx != q.ghost_layers || L.ngy != q.ghost_layers || L.ngz != q.ghost_layers)
        fail("Field3D ghost width differs from the one the schemes derive");
    if (!g_shim.ctx || !same_params(q, g_shim.params)) {
        if (g_shim.ctx) {
            // a parameter change: hand the current state back before dropping it
            if (g_shim.host_stale && holds(F)) download(g_shim.ctx, const_cast<Field3D&>(F));
            else if (g_shim.host_stale && g_shim.owner)
                std::fprintf(stderr, "ns3d shim: new parameters; the GPU state of another Field3D "
                                     "that was never synced is dropped (ns3d_shim_sync keeps it)\n");
            ns3d_destroy(g_shim.ctx);
        }
        g_shim.ctx = nullptr;
        g_shim.owner = nullptr;
        g_shim.host_stale = false;
        const char* dev = std::getenv("NS3D_DEVICE");
        check(ns3d_create(&q, dev ? std::atoi(dev) : 0, &g_shim.ctx), "ns3d_create");
        g_shim.params = q;
    }
    if (!holds(F) || eager()) {
        if (g_shim.host_stale && g_shim.owner && g_shim.owner != &F)
            std::fprintf(stderr, "ns3d shim: a second Field3D; the GPU state of the first one, "
                                 "never synced, is dropped (ns3d_shim_sync keeps it)\n");
        check(ns3d_upload_primitive(g_shim.ctx, F.rho.data(), F.u.data(), F.v.data(), F.w.data(),
                                    F.p.data(), NS3D_LAYOUT_GHOSTED),
              "ns3d_upload_primitive");
        g_shim.owner = &F;
        g_shim.owner_rho = F.rho.data();
        g_shim.host_stale = false;
    }
    return g_shim.ctx;
}

// After a call that changed the device state: hand it back at once in the
// eager mode, else remember that Field3D is behind.
void advanced(Field3D& F) {
    if (eager()) {
        download(g_shim.ctx, F);
        g_shim.host_stale = false;
    } else {
        g_shim.host_stale = true;
    }
}

}  // namespace

// ---- synchronisation for host code outside the shimmed functions ----------

void ns3d_shim_sync(Field3D& F) {
    if (g_shim.ctx && holds(F) && g_shim.host_stale) {
        download(g_shim.ctx, F);
        g_shim.host_stale = false;
    }
}

void ns3d_shim_invalidate(const Field3D& F) {
    if (holds(F)) {
        g_shim.owner = nullptr;
        g_shim.owner_rho = nullptr;
        g_shim.host_stale = false;
    }
}

// ---- range_kutta.cpp / timestep.cpp -------------------------------------------

void compute_rhs(Field3D& F, CartDecomp& C, GridDesc& G, SolverParams& P, HaloRequests&) {
    (void)C;
    ns3d_ctx* ctx = resident(F, P, G);
    check(ns3d_compute_rhs(ctx, F.rhs_rho.data(), F.rhs_rhou.data(), F.rhs_rhov.data(),
                           F.rhs_rhow.data(), F.rhs_E.data(), NS3D_LAYOUT_GHOSTED),
          "ns3d_compute_rhs");
}

double compute_timestep(Field3D& F, const GridDesc& G, const SolverParams& P) {
    ns3d_ctx* ctx = resident(F, P, G);
    double dt = 0.0;
    check(ns3d_compute_timestep(ctx, &dt), "ns3d_compute_timestep");
    return dt;
}

void runge_kutta_3(Field3D& F, CartDecomp& C, GridDesc& G, SolverParams& P, HaloRequests&,
                   double dt) {
    (void)C;
    ns3d_ctx* ctx = resident(F, P, G);
    // U0 = the state this step starts from (time_advance's recordConservedTo0)
    check(ns3d_record_conserved0(ctx), "ns3d_record_conserved0");
    const ns3d_status s = ns3d_runge_kutta_3(ctx, dt);
    advanced(F);
    if (s == NS3D_ERR_NONPHYSICAL) {
        ns3d_shim_sync(F);
        std::printf("Error: Non-physical value detected at rank 0: %s\n", ns3d_last_error(ctx));
        MPI_Abort(MPI_COMM_WORLD, -1);
    }
    check(s, "ns3d_runge_kutta_3");
}

// ---- postprocess.cpp -----------------------------------------------------------

void compute_diagnostics(Field3D& F, const SolverParams& P, const GridDesc& G) {
    ns3d_ctx* ctx = resident(F, P, G);
    double r[5];
    check(ns3d_residuals(ctx, r), "ns3d_residuals");
    F.global_res_rho = r[0];
    F.global_res_rhou = r[1];
    F.global_res_rhov = r[2];
    F.global_res_rhow = r[3];
    F.global_res_E = r[4];
}

void compute_total_energy(Field3D& F, const GridDesc& G, const CartDecomp& C,
                          const SolverParams& P) {
    (void)C;
    ns3d_ctx* ctx = resident(F, P, G);
    check(ns3d_total_energy(ctx, &F.global_Etot), "ns3d_total_energy");
}

void isotropic_post_process(Field3D& F, const GridDesc& G, const CartDecomp& C,
                            const SolverParams& P, const double current_time) {
    (void)C;
    ns3d_ctx* ctx = resident(F, P, G);
    const int nbins = 2 * G.global_nx + 1;
    std::vector<double> Ek(nbins);
    check(ns3d_energy_spectrum(ctx, Ek.data(), nbins), "ns3d_energy_spectrum");
    std::error_code ec;
    std::filesystem::create_directories("output", ec);
    std::stringstream ss;
    ss << "output/output_time_" << std::fixed << std::setprecision(5) << current_time
       << "_spectrum.dat";
    check(ns3d_spectrum_write(ss.str().c_str(), Ek.data(), nbins), "ns3d_spectrum_write");
    // compute_turbulence_statistics reads the spectrum back from that file
    // (ana_isotropic.cpp:210-221): its 6 significant digits
    for (double& e : Ek) {
        char txt[64];
        std::snprintf(txt, sizeof txt, "%g", e);
        e = std::strtod(txt, nullptr);
    }
    ns3d_turb_stats st;
    check(ns3d_turbulence_stats_spectrum(ctx, Ek.data(), nbins, &st),
          "ns3d_turbulence_stats_spectrum");
    check(ns3d_stats_write("output/turbulence_stats.dat", current_time, &st), "ns3d_stats_write");
}

// ---- output.cpp ----------------------------------------------------------------

void write_tecplot_field(const Field3D& F, const GridDesc& G, const CartDecomp& C,
                         const SolverParams& P, double time) {
    ns3d_ctx* ctx = resident(F, P, G);
    ns3d_shim_sync(const_cast<Field3D&>(F));  // output reads Field3D: bring it up to date
    const std::filesystem::path dir =
        std::filesystem::path("output") / ("time_" + std::to_string(static_cast<int>(time * 100000)));
    std::error_code ec;
    std::filesystem::create_directories(dir, ec);
    const std::string path = (dir / ("field_rank" + std::to_string(C.rank) + ".dat")).string();
    const ns3d_status s = ns3d_write_tecplot(ctx, path.c_str(), time);
    if (s == NS3D_ERR_FILE) {  // the reference reports and carries on
        std::cerr << "Failed to open output file " << path << " for writing\n";
        return;
    }
    check(s, "ns3d_write_tecplot");
}

void write_residuals_tecplot(const Field3D& F, int step, const std::string& filename) {
    std::error_code ec;
    std::filesystem::create_directories("output", ec);
    const double r[5] = {F.global_res_rho, F.global_res_rhou, F.global_res_rhov,
                         F.global_res_rhow, F.global_res_E};
    const std::string path = (std::filesystem::path("output") / filename).string();
    const ns3d_status s = ns3d_residuals_write(path.c_str(), step, r, F.global_Etot);
    if (s != NS3D_OK) std::cerr << "Failed to open residuals file " << path << "\n";
}
