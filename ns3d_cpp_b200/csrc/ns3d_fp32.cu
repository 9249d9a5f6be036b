// FP32-stencil form: splitting, reconstruction and viscous stencils in float;
// the RK3 stage accumulation, conservedToPrimitive and the state stay double.
#define NS3D_LAUNCH_IMPL
#include "ns3d_launch.cuh"

namespace ns3d {
NS3D_INSTANTIATE_LAUNCHERS(float)
}
