// FP32-stencil form: reconstruction, viscous stencils and flux differences in
// float; the flux split is evaluated in double and enters the reconstructions
// as a float deviation from the segment's first split flux; the RK3 stage
// accumulation, conservedToPrimitive and the state stay double.
#define NS3D_LAUNCH_IMPL
#include "ns3d_launch.cuh"

namespace ns3d {
NS3D_INSTANTIATE_LAUNCHERS(float)
}
