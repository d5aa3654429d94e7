// Number types for differentiating the dynamical-core device functions, which are templated on
// their arithmetic type:
//   Dual : forward mode (value, tangent); the tangent-linear model.
//   TV   : reverse mode; every operation appends a node (two parents, two partial derivatives)
//          to a per-thread tape in local memory, and a backward sweep over the tape yields the
//          derivative of the seeded outputs with respect to every leaf (an input read).
// Comparisons act on values, so a branch (the TVD limiter's, the Richardson-number regimes,
// max/min) is frozen at the branch the forward evaluation takes.  Derivatives of |x| and
// copysign at x = 0 take the branch that x >= 0 selects; sqrt'(0) is taken as 0.
#pragma once

#include <cmath>

namespace mgpu {
namespace ad {

// ------------------------------------------------------------------------------------------
// forward mode
// ------------------------------------------------------------------------------------------
struct Dual {
  double v, d;
  __device__ __forceinline__ Dual() : v(0.0), d(0.0) {}
  __device__ __forceinline__ Dual(double x) : v(x), d(0.0) {}
  __device__ __forceinline__ Dual(double x, double dx) : v(x), d(dx) {}
  __device__ __forceinline__ explicit operator int() const { return (int)v; }
};
__device__ __forceinline__ Dual operator+(Dual a, Dual b) { return Dual(a.v + b.v, a.d + b.d); }
__device__ __forceinline__ Dual operator-(Dual a, Dual b) { return Dual(a.v - b.v, a.d - b.d); }
__device__ __forceinline__ Dual operator*(Dual a, Dual b) { return Dual(a.v * b.v, a.d * b.v + a.v * b.d); }
__device__ __forceinline__ Dual operator/(Dual a, Dual b) {
  const double q = a.v / b.v;
  return Dual(q, (a.d - q * b.d) / b.v);
}
__device__ __forceinline__ Dual operator-(Dual a) { return Dual(-a.v, -a.d); }
__device__ __forceinline__ bool operator<(Dual a, Dual b) { return a.v < b.v; }
__device__ __forceinline__ bool operator>(Dual a, Dual b) { return a.v > b.v; }
__device__ __forceinline__ bool operator<=(Dual a, Dual b) { return a.v <= b.v; }
__device__ __forceinline__ bool operator>=(Dual a, Dual b) { return a.v >= b.v; }
__device__ __forceinline__ bool operator==(Dual a, Dual b) { return a.v == b.v; }
__device__ __forceinline__ bool operator!=(Dual a, Dual b) { return a.v != b.v; }
__device__ __forceinline__ Dual fabs(Dual a) { return ::signbit(a.v) ? Dual(-a.v, -a.d) : a; }
__device__ __forceinline__ Dual copysign(Dual a, Dual b) {
  const double r = ::copysign(a.v, b.v);
  return Dual(r, ::signbit(a.v) != ::signbit(b.v) ? -a.d : a.d);
}
__device__ __forceinline__ bool signbit(Dual a) { return ::signbit(a.v); }
// at exactly 0 (a wind speed of a flow at rest) the derivative of sqrt is taken as 0, the
// subgradient of |(u, v)| at the origin
__device__ __forceinline__ Dual sqrt(Dual a) {
  const double r = ::sqrt(a.v);
  return Dual(r, r > 0.0 ? a.d / (2.0 * r) : 0.0);
}
__device__ __forceinline__ Dual log(Dual a) { return Dual(::log(a.v), a.d / a.v); }
__device__ __forceinline__ Dual exp(Dual a) {
  const double r = ::exp(a.v);
  return Dual(r, r * a.d);
}
__device__ __forceinline__ Dual cos(Dual a) { return Dual(::cos(a.v), -::sin(a.v) * a.d); }
__device__ __forceinline__ Dual acos(Dual a) { return Dual(::acos(a.v), -a.d / ::sqrt(1.0 - a.v * a.v)); }
__device__ __forceinline__ Dual pow(Dual a, Dual b) {
  const double r = ::pow(a.v, b.v);
  double d = b.v * ::pow(a.v, b.v - 1.0) * a.d;
  if (b.d != 0.0) d += r * ::log(a.v) * b.d;
  return Dual(r, d);
}
__device__ __forceinline__ Dual rcp(Dual a) { return Dual(1.0) / a; }
__device__ __forceinline__ Dual div_rn(Dual a, Dual b) { return a / b; }

// ------------------------------------------------------------------------------------------
// reverse mode
// ------------------------------------------------------------------------------------------
struct Tape {
  static constexpr int CAP = 768;   // nodes per evaluation
  static constexpr int LCAP = 224;  // leaves per evaluation
  double pa[CAP], pb[CAP];
  short ia[CAP], ib[CAP];
  double adj[CAP];
  int lf_node[LCAP], lf_field[LCAP];
  long long lf_off[LCAP];
  int n, nleaf, overflow;
  __device__ __forceinline__ void reset() { n = 0; nleaf = 0; }
  __device__ __forceinline__ int node(int a, double da, int b, double db) {
    if (n >= CAP) { overflow = 1; return -1; }
    const int id = n++;
    ia[id] = (short)a;
    pa[id] = da;
    ib[id] = (short)b;
    pb[id] = db;
    return id;
  }
  // a leaf: an input value whose adjoint goes to (field, offset) after the sweep
  __device__ __forceinline__ int leaf(int field, long long off) {
    if (nleaf >= LCAP) { overflow = 1; return -1; }
    const int id = node(-1, 0.0, -1, 0.0);
    if (id < 0) return -1;
    lf_node[nleaf] = id;
    lf_field[nleaf] = field;
    lf_off[nleaf] = off;
    ++nleaf;
    return id;
  }
  // adjoints of every node from the seeds already placed in adj[]
  __device__ void sweep() {
    for (int q = n - 1; q >= 0; --q) {
      const double g = adj[q];
      if (g == 0.0) continue;
      if (ia[q] >= 0) adj[ia[q]] += pa[q] * g;
      if (ib[q] >= 0) adj[ib[q]] += pb[q] * g;
    }
  }
  __device__ __forceinline__ void clear_adj() {
    for (int q = 0; q < n; ++q) adj[q] = 0.0;
  }
};

struct TV {
  double v;
  int id;   // tape node, -1 for a constant
  Tape* t;
  __device__ __forceinline__ TV() : v(0.0), id(-1), t(nullptr) {}
  __device__ __forceinline__ TV(double x) : v(x), id(-1), t(nullptr) {}
  __device__ __forceinline__ TV(double x, int i, Tape* tp) : v(x), id(i), t(tp) {}
  __device__ __forceinline__ explicit operator int() const { return (int)v; }
};
__device__ __forceinline__ TV mk1(double r, TV a, double da) {
  if (a.id < 0) return TV(r);
  return TV(r, a.t->node(a.id, da, -1, 0.0), a.t);
}
__device__ __forceinline__ TV mk2(double r, TV a, double da, TV b, double db) {
  if (a.id < 0 && b.id < 0) return TV(r);
  Tape* t = a.id >= 0 ? a.t : b.t;
  return TV(r, t->node(a.id, da, b.id, db), t);
}
__device__ __forceinline__ TV operator+(TV a, TV b) { return mk2(a.v + b.v, a, 1.0, b, 1.0); }
__device__ __forceinline__ TV operator-(TV a, TV b) { return mk2(a.v - b.v, a, 1.0, b, -1.0); }
__device__ __forceinline__ TV operator*(TV a, TV b) { return mk2(a.v * b.v, a, b.v, b, a.v); }
__device__ __forceinline__ TV operator/(TV a, TV b) {
  const double q = a.v / b.v;
  return mk2(q, a, 1.0 / b.v, b, -q / b.v);
}
__device__ __forceinline__ TV operator-(TV a) { return mk1(-a.v, a, -1.0); }
__device__ __forceinline__ bool operator<(TV a, TV b) { return a.v < b.v; }
__device__ __forceinline__ bool operator>(TV a, TV b) { return a.v > b.v; }
__device__ __forceinline__ bool operator<=(TV a, TV b) { return a.v <= b.v; }
__device__ __forceinline__ bool operator>=(TV a, TV b) { return a.v >= b.v; }
__device__ __forceinline__ bool operator==(TV a, TV b) { return a.v == b.v; }
__device__ __forceinline__ bool operator!=(TV a, TV b) { return a.v != b.v; }
__device__ __forceinline__ TV fabs(TV a) { return ::signbit(a.v) ? mk1(-a.v, a, -1.0) : a; }
__device__ __forceinline__ TV copysign(TV a, TV b) {
  return mk1(::copysign(a.v, b.v), a, ::signbit(a.v) != ::signbit(b.v) ? -1.0 : 1.0);
}
__device__ __forceinline__ bool signbit(TV a) { return ::signbit(a.v); }
__device__ __forceinline__ TV sqrt(TV a) {
  const double r = ::sqrt(a.v);
  return mk1(r, a, r > 0.0 ? 0.5 / r : 0.0);
}
__device__ __forceinline__ TV log(TV a) { return mk1(::log(a.v), a, 1.0 / a.v); }
__device__ __forceinline__ TV exp(TV a) {
  const double r = ::exp(a.v);
  return mk1(r, a, r);
}
__device__ __forceinline__ TV cos(TV a) { return mk1(::cos(a.v), a, -::sin(a.v)); }
__device__ __forceinline__ TV acos(TV a) { return mk1(::acos(a.v), a, -1.0 / ::sqrt(1.0 - a.v * a.v)); }
__device__ __forceinline__ TV pow(TV a, TV b) {
  const double r = ::pow(a.v, b.v);
  const double da = b.v * ::pow(a.v, b.v - 1.0);
  const double db = b.id >= 0 ? r * ::log(a.v) : 0.0;
  return mk2(r, a, da, b, db);
}
__device__ __forceinline__ TV rcp(TV a) { return TV(1.0) / a; }
__device__ __forceinline__ TV div_rn(TV a, TV b) { return a / b; }

}  // namespace ad
}  // namespace mgpu
