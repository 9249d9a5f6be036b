// FP64 form: every stencil operation in double, compiled with -fmad=false so
// the reference's rounding sequence (x86-64 SSE2, no FMA contraction) is kept.
#define NS3D_LAUNCH_IMPL
#include "ns3d_launch.cuh"

namespace ns3d {
NS3D_INSTANTIATE_LAUNCHERS(double)
}
