// Halo rows of a y-slab.
//
// A slab model holds rows [y0 - halo, y0 + nyl + halo) of a periodic domain as its ny = nyl + 2*halo
// rows.  Before a step the halo rows are refreshed from the neighbouring slabs: the first `depth`
// interior rows go to the slab below (its top halo), the last `depth` interior rows to the slab
// above (its bottom halo).  This is the y part of MONC's halo swap (halocommunication.F90:109-163,
// the periodic copies of :486-498 when one rank spans the domain), with whole x rows: the slabs
// keep every column, so there are no x faces and no corners to exchange.
//
// One kernel moves every row of every field of both sides, so a halo exchange costs one launch to
// pack and one to unpack however many fields it carries.
#include "dycore.h"

namespace mgpu {

constexpr int kMaxRowFields = 8 + 2 * MGPU_MAX_Q;

template <typename T>
struct RowFields {
  T* f[kMaxRowFields];
};

// Element t of a side's buffer [n][nz][depth][nx] is (field, level, row, x); consecutive threads
// take consecutive x, so the field rows and the buffer are both read and written coalesced.
template <typename T>
__global__ void k_halo_rows(RowFields<T> rf, int n, int nx, int ny, int nz, int depth, int r_lo, int r_hi, T* lo, T* hi,
                            int unpack) {
  const long long row_elems = (long long)depth * nx;
  const long long per_side = (long long)n * nz * row_elems;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < 2 * per_side; t += stride) {
    const int side = t >= per_side ? 1 : 0;
    const long long u = t - side * per_side;
    const long long fk = u / row_elems;  // field * nz + level
    const long long e = u - fk * row_elems;
    const int f = (int)(fk / nz), k = (int)(fk - (long long)f * nz);
    T* field = rf.f[f] + ((long long)k * ny + (side ? r_hi : r_lo)) * nx + e;
    T* buf = (side ? hi : lo) + u;
    if (unpack) *field = *buf;
    else *buf = *field;
  }
}

template <typename T>
void launch_halo_rows(const Scalars& s, T* const* f, int n, int depth, int r_lo, int r_hi, T* lo, T* hi, bool unpack,
                      cudaStream_t st) {
  RowFields<T> rf{};
  for (int q = 0; q < n && q < kMaxRowFields; ++q) rf.f[q] = f[q];
  const long long total = 2LL * n * s.nz * depth * s.nx;
  const long long want = (total + 255) / 256;
  const int blocks = (int)(want < 148LL * 16 ? want : 148LL * 16);
  k_halo_rows<T><<<blocks, 256, 0, st>>>(rf, n, s.nx, s.ny, s.nz, depth, r_lo, r_hi, lo, hi, unpack ? 1 : 0);
}

template void launch_halo_rows<double>(const Scalars&, double* const*, int, int, int, int, double*, double*, bool,
                                       cudaStream_t);
template void launch_halo_rows<float>(const Scalars&, float* const*, int, int, int, int, float*, float*, bool,
                                      cudaStream_t);

}  // namespace mgpu
