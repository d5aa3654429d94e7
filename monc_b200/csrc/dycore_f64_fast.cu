// Instantiation of the dynamical-core kernels for FP64 fields, `fast` variant.
// Built with the default --fmad=true: multiply-adds are contracted into FMAs.
#define KVARIANT fast
// contracted-build forms of some expressions (see smagorinsky_from_strain)
#define MGPU_CONTRACTED 1
#include "dycore_kernels.cuh"

namespace mgpu {
namespace fast {
template int launch_fused_subgrid<double>(const Scalars&, DevState<double>&, cudaStream_t);
template int launch_fused_dynamics<double>(const Scalars&, DevState<double>&, cudaStream_t, cudaEvent_t);
template void launch_fused_pressure_source<double>(const Scalars&, DevState<double>&, cudaStream_t);
template void launch_fused_pstep_swap<double>(const Scalars&, DevState<double>&, cudaStream_t);
}  // namespace fast
}  // namespace mgpu
