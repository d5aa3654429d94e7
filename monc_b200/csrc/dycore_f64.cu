// Instantiation of the dynamical-core kernels for FP64 fields, `exact` variant.
// Built with --fmad=false: every multiply and add is rounded separately, as MONC's x86-64
// gfortran build evaluates them, so these kernels reproduce MONC's arithmetic exactly
// (transcendental library calls in the surface scheme aside).
#define KVARIANT exact
#include "dycore_kernels.cuh"

namespace mgpu {
namespace exact {
template int launch_component<double>(int, const Scalars&, DevState<double>&, cudaStream_t, unsigned long long*, int64_t*);
template int launch_fused_subgrid<double>(const Scalars&, DevState<double>&, cudaStream_t);
template int launch_fused_dynamics<double>(const Scalars&, DevState<double>&, cudaStream_t, cudaEvent_t);
template void launch_fused_pressure_source<double>(const Scalars&, DevState<double>&, cudaStream_t);
template void launch_fused_pstep_swap<double>(const Scalars&, DevState<double>&, cudaStream_t);
}  // namespace exact
}  // namespace mgpu
