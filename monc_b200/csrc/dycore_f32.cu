// Instantiation of the dynamical-core kernels for FP32 fields, `exact` variant.
// Built with --fmad=false: every multiply and add is rounded separately, as MONC's x86-64
// gfortran build evaluates them, so these kernels reproduce MONC's arithmetic exactly
// (transcendental library calls in the surface scheme aside).
#define KVARIANT exact
#include "dycore_kernels.cuh"

namespace mgpu {
namespace exact {
template int launch_component<float>(int, const Scalars&, DevState<float>&, cudaStream_t, unsigned long long*, int64_t*);
template int launch_fused_subgrid<float>(const Scalars&, DevState<float>&, cudaStream_t);
template int launch_fused_dynamics<float>(const Scalars&, DevState<float>&, cudaStream_t, cudaEvent_t);
template void launch_fused_pressure_source<float>(const Scalars&, DevState<float>&, cudaStream_t);
template void launch_fused_pstep_swap<float>(const Scalars&, DevState<float>&, cudaStream_t);
}  // namespace exact
}  // namespace mgpu
