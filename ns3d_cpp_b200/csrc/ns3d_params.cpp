// solver.in parsing and parameter derivation, mirroring
// read_solver_params_from_file (initialization.cpp:199-380) and the
// SolverParams / GridDesc defaults (field_structures.h:32-37, 85-166).
#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstring>
#include <fstream>
#include <stdexcept>
#include <string>

#include "ns3d_gpu.h"

namespace {

std::string trim(const std::string& s) {
    const size_t a = s.find_first_not_of(" \t\r\n");
    const size_t b = s.find_last_not_of(" \t\r\n");
    if (a == std::string::npos) return "";
    return s.substr(a, b - a + 1);
}

std::string lower(std::string s) {
    std::transform(s.begin(), s.end(), s.begin(), [](unsigned char c) { return std::tolower(c); });
    return s;
}

bool parse_bool(const std::string& v) {
    const std::string lv = lower(v);
    return lv == "true" || lv == "yes" || lv == "1" || lv == "on";
}

int parse_bc(const std::string& v) {
    if (v == "inflow") return NS3D_BC_INFLOW;
    if (v == "wall") return NS3D_BC_WALL;
    if (v == "symmetry") return NS3D_BC_SYMMETRY;
    if (v == "outflow") return NS3D_BC_OUTFLOW;
    return NS3D_BC_PERIODIC;
}

}  // namespace

extern "C" size_t ns3d_params_size(void) { return sizeof(ns3d_params); }
extern "C" size_t ns3d_turb_stats_size(void) { return sizeof(ns3d_turb_stats); }

extern "C" ns3d_status ns3d_params_default(ns3d_params* p) {
    if (!p) return NS3D_ERR_INVALID;
    std::memset(p, 0, sizeof(*p));
    // SolverParams member initialisers (field_structures.h:86-165)
    p->gamma = 1.4;
    p->Pr = 0.71;
    p->Ma = 0.4;
    p->Re = 500.0;
    p->cfl = 0.1;
    p->dt_fixed = -1.0;
    p->fvs_type = NS3D_FVS_STEGER_WARMING;
    p->recon = NS3D_RECON_WENO5;
    p->vis_scheme = NS3D_VIS_C6TH;
    p->char_recon = 0;
    p->mdcd_diss = 0.01;
    p->mdcd_disp = 0.0463783;
    p->ud7l_alpha = 0.4;
    for (int f = 0; f < 6; ++f) p->bc[f] = NS3D_BC_PERIODIC;
    p->max_steps = 1;
    p->monitor_Stepfreq = 1;
    p->output_Timefreq = 1.0;
    p->TotalTime = 1.0;
    p->post_basicfield = 1;
    p->isotropic_analyse = 1;
    p->monitor_res = 1;
    p->monitor_energy = 1;
    // grid defaults of the parser (initialization.cpp:214-215) and GridDesc
    p->global_nx = p->global_ny = p->global_nz = 16;
    p->Lx = p->Ly = p->Lz = 1.0;
    // extensions
    p->sw_entropy_eps = 0.0;
    p->sutherland_s_over_tref = 110.4 / 288.15;
    p->precision = NS3D_PREC_FP64;
    return ns3d_params_derive(p);
}

extern "C" ns3d_status ns3d_params_derive(ns3d_params* p) {
    if (!p) return NS3D_ERR_INVALID;
    p->periods[0] = p->bc[0] == NS3D_BC_PERIODIC && p->bc[1] == NS3D_BC_PERIODIC;
    p->periods[1] = p->bc[2] == NS3D_BC_PERIODIC && p->bc[3] == NS3D_BC_PERIODIC;
    p->periods[2] = p->bc[4] == NS3D_BC_PERIODIC && p->bc[5] == NS3D_BC_PERIODIC;
    if (p->global_nx <= 0 || p->global_ny <= 0 || p->global_nz <= 0) return NS3D_ERR_INVALID;
    p->dx = p->Lx / (p->global_nx);
    p->dy = p->Ly / (p->global_ny);
    p->dz = p->Lz / (p->global_nz);
    switch (p->recon) {  // initialization.cpp:329-357
    case NS3D_RECON_WENO5: case NS3D_RECON_MDCD: case NS3D_RECON_MDCD_HYBRID:
        p->ghost_layers = 3; p->stencil = 6; break;
    case NS3D_RECON_LINEAR: p->ghost_layers = 2; p->stencil = 2; break;
    case NS3D_RECON_UPWIND_7TH: case NS3D_RECON_UD7L: p->ghost_layers = 4; p->stencil = 8; break;
    default: break;  // WCNS: the reference leaves the defaults
    }
    switch (p->vis_scheme) {  // :358-372
    case NS3D_VIS_C4TH: p->ghost_layers = std::max(p->ghost_layers, 2); break;
    case NS3D_VIS_C6TH: p->ghost_layers = std::max(p->ghost_layers, 3); break;
    case NS3D_VIS_C8TH: p->ghost_layers = std::max(p->ghost_layers, 4); break;
    default: return NS3D_ERR_INVALID;
    }
    p->Cv = 1.0 / (p->gamma * (p->gamma - 1.0) * p->Ma * p->Ma);  // :374-377
    p->Cp = p->Cv * p->gamma;
    p->Rgas = 1.0 / (p->Ma * p->Ma * p->gamma);
    p->mu = 1.0 / p->Re;
    return NS3D_OK;
}

extern "C" ns3d_status ns3d_params_from_file(const char* path, ns3d_params* p) {
    if (!path || !p) return NS3D_ERR_INVALID;
    std::ifstream fin(path);
    if (!fin.is_open()) return NS3D_ERR_FILE;
    ns3d_params_default(p);
    try {
        std::string line;
        while (std::getline(fin, line)) {
            line = trim(line);
            if (line.empty() || line[0] == '#') continue;
            const size_t eq = line.find('=');
            if (eq == std::string::npos) continue;
            const std::string key = trim(line.substr(0, eq));
            const std::string val = trim(line.substr(eq + 1));
            const std::string k = lower(key);
            const std::string v = lower(val);
            if (k == "gamma") p->gamma = std::stod(val);
            else if (k == "pr") p->Pr = std::stod(val);
            else if (k == "ma") p->Ma = std::stod(val);
            else if (k == "re") p->Re = std::stod(val);
            else if (k == "cfl") p->cfl = std::stod(val);
            else if (k == "dt_fixed") p->dt_fixed = std::stod(val);
            else if (k == "fvs_type") {
                if (v == "stagerwarming") p->fvs_type = NS3D_FVS_STEGER_WARMING;
                else if (v == "laxfriedrichs") p->fvs_type = NS3D_FVS_LAX_FRIEDRICHS;
            } else if (k == "recon") {
                if (v == "mdcd") p->recon = NS3D_RECON_MDCD;
                else if (v == "weno5") p->recon = NS3D_RECON_WENO5;
                else if (v == "linear") p->recon = NS3D_RECON_LINEAR;
                else if (v == "mdcd_hybrid") p->recon = NS3D_RECON_MDCD_HYBRID;
                else if (v == "upwind_7th") p->recon = NS3D_RECON_UPWIND_7TH;
                else if (v == "ud7l") p->recon = NS3D_RECON_UD7L;
            } else if (k == "vis_scheme") {
                if (v == "c4th") p->vis_scheme = NS3D_VIS_C4TH;
                else if (v == "c6th") p->vis_scheme = NS3D_VIS_C6TH;
                else if (v == "c8th") p->vis_scheme = NS3D_VIS_C8TH;
            } else if (k == "char_recon") p->char_recon = (v == "yes" || v == "true");
            else if (k == "mdcd_diss") p->mdcd_diss = std::stod(val);
            else if (k == "mdcd_disp") p->mdcd_disp = std::stod(val);
            else if (k == "ud7l_alpha") p->ud7l_alpha = std::stod(val);
            else if (k == "global_nx") p->global_nx = std::stoi(val);
            else if (k == "global_ny") p->global_ny = std::stoi(val);
            else if (k == "global_nz") p->global_nz = std::stoi(val);
            else if (k == "x0") p->x0 = std::stod(val);
            else if (k == "y0") p->y0 = std::stod(val);
            else if (k == "z0") p->z0 = std::stod(val);
            else if (k == "lx") p->Lx = std::stod(val);
            else if (k == "ly") p->Ly = std::stod(val);
            else if (k == "lz") p->Lz = std::stod(val);
            else if (k == "max_steps") p->max_steps = std::stoi(val);
            else if (k == "monitor_stepfreq") p->monitor_Stepfreq = std::stoi(val);
            else if (k == "output_timefreq") p->output_Timefreq = std::stod(val);
            else if (k == "totaltime") p->TotalTime = std::stod(val);
            // extension keys (absent from the reference; defaults reproduce it)
            else if (k == "sw_entropy_eps") p->sw_entropy_eps = std::stod(val);
            else if (k == "sutherland_s_over_tref") p->sutherland_s_over_tref = std::stod(val);
            else if (k == "precision") {
                if (v == "fp64") p->precision = NS3D_PREC_FP64;
                else if (v == "fp32acc64" || v == "fp32") p->precision = NS3D_PREC_FP32_ACC64;
                else return NS3D_ERR_INVALID;
            }
            // boundary conditions: a separate if-chain in the reference (:296-301)
            if (k == "bc_xmin") p->bc[0] = parse_bc(v);
            else if (k == "bc_xmax") p->bc[1] = parse_bc(v);
            else if (k == "bc_ymin") p->bc[2] = parse_bc(v);
            else if (k == "bc_ymax") p->bc[3] = parse_bc(v);
            else if (k == "bc_zmin") p->bc[4] = parse_bc(v);
            else if (k == "bc_zmax") p->bc[5] = parse_bc(v);
            else if (k == "post_basicfield") p->post_basicfield = parse_bool(val);
            else if (k == "isotropicanalyse") p->isotropic_analyse = parse_bool(val);
            else if (k == "monitor_res") p->monitor_res = parse_bool(val);
            else if (k == "monitor_energy") p->monitor_energy = parse_bool(val);
        }
    } catch (const std::exception&) {
        // std::stod / std::stoi on a malformed value: the reference throws
        return NS3D_ERR_INVALID;
    }
    return ns3d_params_derive(p);
}
