// Oracle (test infrastructure only): internal declarations of the CPU restatement of MONC's
// dynamical-core timestep.  Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
// leg use this code, as the checker; the GPU library never links it.
#ifndef MONC_ORACLE_INTERNAL_H
#define MONC_ORACLE_INTERNAL_H

#include <cstddef>
#include <vector>

#include "../include/monc_gpu.h"

namespace oracle {

struct FftPlan {
  int n = 0;
  std::vector<double> wa;
  std::vector<int> ifac;
};
void fft_plan_init(FftPlan& plan, int n);
void zfftf(const FftPlan& plan, double* c, double* work);
void zfftb(const FftPlan& plan, double* c, double* work);
void fftn_r2c(const FftPlan& plan, const double* in, double* out_complex, double* data, double* work);
void fftn_c2r(const FftPlan& plan, const double* in_complex, double* out, double* data, double* work);

// A prognostic field in MONC's layout: data(k, j, i), z fastest, 1-based indices,
// 2-deep halo in x and y (prognostics.F90:13-20, simplesetup.F90:60-137).
struct Field {
  int nz = 0, nyh = 0, nxh = 0;
  std::vector<double> d;
  bool active = false;
  void alloc(int nz_, int nyh_, int nxh_) {
    nz = nz_; nyh = nyh_; nxh = nxh_;
    d.assign((size_t)nz * nyh * nxh, 0.0);
    active = true;
  }
  inline double& operator()(int k, int j, int i) {
    return d[(size_t)(k - 1) + (size_t)nz * ((size_t)(j - 1) + (size_t)nyh * (size_t)(i - 1))];
  }
  inline double operator()(int k, int j, int i) const {
    return d[(size_t)(k - 1) + (size_t)nz * ((size_t)(j - 1) + (size_t)nyh * (size_t)(i - 1))];
  }
  inline double* col(int j, int i) { return &d[(size_t)nz * ((size_t)(j - 1) + (size_t)nyh * (size_t)(i - 1))] - 1; }
};

// 1-based vertical profile
struct Prof {
  std::vector<double> v;
  void alloc(int n) { v.assign(n + 2, 0.0); }
  inline double& operator()(int k) { return v[k]; }
  inline double operator()(int k) const { return v[k]; }
};

}  // namespace oracle
#endif
