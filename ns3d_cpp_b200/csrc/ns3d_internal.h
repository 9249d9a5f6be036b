// Internal declarations shared between the library's translation units.
#pragma once

#include <string>

#include "ns3d_gpu.h"
#include "ns3d_launch.cuh"

namespace ns3d {

// Validate `p` as ns3d_create does and fill the kernels' launch configuration
// (DevParams, scheme selection, segment lengths); the stream is left null.
ns3d_status build_launch_cfg(const ns3d_params* p, LaunchCfg* L, std::string* msg);

// ---- discrete adjoint launchers (ns3d_adjoint.cu), FP64 ----
// Number of n-sized scratch blocks adj_rhs_vjp needs for the face cotangents.
int adj_scratch_blocks(const LaunchCfg& L);
// lamW += (dR/dW)^T lamR at state W; G: adj_scratch_blocks(L) x n, lg: 16 x n.
cudaError_t adj_rhs_vjp(const LaunchCfg& L, StateView W, const double* lamR, double* G,
                        double* lg, double* lamW);
// One stage reversed (see k_adj_stage).
cudaError_t adj_stage(const LaunchCfg& L, int stage, StateView Wk, StateView Wp,
                      const double* lamWk, double* lamU0, double* lamR, double* lamWp, double dt);
cudaError_t adj_finish(const LaunchCfg& L, StateView W0, const double* lamU0, double* lamW0);
cudaError_t adj_seed_ke(const LaunchCfg& L, StateView W, double* lamW, double dV);

}  // namespace ns3d
