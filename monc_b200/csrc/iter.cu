// BiCGStab pressure solve (iterativesolver.F90): not yet available on this path.
#include "dycore.h"

namespace mgpu {

struct IterSolverDev {
  int dummy;
};

IterSolverDev* iter_create(const Scalars&, const RefState&, const mgpu_config&, bool, int* status) {
  *status = MGPU_ERR_UNSUPPORTED;
  return nullptr;
}
void iter_destroy(IterSolverDev* it) { delete it; }
template <typename T>
int iter_solve(IterSolverDev*, const Scalars&, T*, cudaStream_t, int64_t*, int*, double*) {
  return MGPU_ERR_UNSUPPORTED;
}
template int iter_solve<double>(IterSolverDev*, const Scalars&, double*, cudaStream_t, int64_t*, int*, double*);
template int iter_solve<float>(IterSolverDev*, const Scalars&, float*, cudaStream_t, int64_t*, int*, double*);

}  // namespace mgpu
