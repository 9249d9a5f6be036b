// Internal declarations shared between the library's translation units.
#pragma once

#include <string>

#include "ns3d_gpu.h"
#include "ns3d_launch.cuh"

namespace ns3d {

// Validate `p` as ns3d_create does and fill the kernels' launch configuration
// (DevParams, scheme selection, segment lengths); the stream is left null.
ns3d_status build_launch_cfg(const ns3d_params* p, LaunchCfg* L, std::string* msg);

}  // namespace ns3d
