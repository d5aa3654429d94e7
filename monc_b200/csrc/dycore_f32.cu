// Instantiation of the dynamical-core kernels for FP32 fields.
// Multiply-adds are fused (default --fmad=true).
#include "dycore_kernels.cuh"

namespace mgpu {
template int launch_component<float>(int, const Scalars&, DevState<float>&, cudaStream_t, unsigned long long*, int64_t*);
template void launch_fused_subgrid<float>(const Scalars&, DevState<float>&, cudaStream_t);
template void launch_fused_dynamics<float>(const Scalars&, DevState<float>&, cudaStream_t);
template void launch_fused_pressure_source<float>(const Scalars&, DevState<float>&, cudaStream_t);
template void launch_fused_pstep_swap<float>(const Scalars&, DevState<float>&, cudaStream_t);
}  // namespace mgpu
