// Instantiation of the dynamical-core kernels for FP32 fields, `fast` variant.
// Built with the default --fmad=true: multiply-adds are contracted into FMAs.
#define KVARIANT fast
// contracted-build forms of some expressions (see smagorinsky_from_strain)
#define MGPU_CONTRACTED 1
#include "dycore_kernels.cuh"

namespace mgpu {
namespace fast {
template int launch_fused_subgrid<float>(const Scalars&, DevState<float>&, cudaStream_t);
template int launch_fused_dynamics<float>(const Scalars&, DevState<float>&, cudaStream_t, cudaEvent_t);
template void launch_fused_pressure_source<float>(const Scalars&, DevState<float>&, cudaStream_t);
template void launch_fused_pstep_swap<float>(const Scalars&, DevState<float>&, cudaStream_t);
}  // namespace fast
}  // namespace mgpu
