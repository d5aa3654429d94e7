// Oracle (test infrastructure only): C++ restatement of the complex FFTPACK routines that
// MONC vendors for its pressure solve.  Follows, pass by pass and operation by operation:
//   components/fftsolver/src/fftpack/cffti1.f90  (factorisation into 4,2 and twiddle table)
//   components/fftsolver/src/fftpack/cfftf1.f90  (forward driver, ping-pong between c and ch)
//   components/fftsolver/src/fftpack/cfftb1.f90  (backward driver)
//   components/fftsolver/src/fftpack/passf2.f90, passf3.f90, passf4.f90, passf5.f90 and the
//   passb counterparts
// and the wrappers components/fftsolver/src/fftnorth.F90:17-80 (fftn_r2c / fftn_c2r).
// The radix 2, 3, 4 and 5 passes are restated; lengths with another prime factor (FFTPACK's
// general passf.f90) are rejected by fft_plan_init.
#include "oracle_internal.h"

#include <cmath>
#include <stdexcept>

namespace oracle {

// cffti1.f90: factorise n trying 3,4,2,5 (then odd numbers), move a factor 2 to the front,
// and fill the twiddle table wa(2n) with cos/sin of multiples of 2*pi/n.
void fft_plan_init(FftPlan& plan, int n) {
  plan.n = n;
  plan.wa.assign(2 * n + 2, 0.0);
  plan.ifac.assign(64, 0);
  const int ntryh[4] = {3, 4, 2, 5};
  int nl = n, nf = 0, j = 0, ntry = 0;
  std::vector<int>& ifac = plan.ifac;  // 1-based like the Fortran Ifac(*)
  for (;;) {
    j = j + 1;
    if (j <= 4) ntry = ntryh[j - 1]; else ntry = ntry + 2;
    bool next_try = false;
    while (!next_try) {
      int nq = nl / ntry;
      int nr = nl - ntry * nq;
      if (nr != 0) { next_try = true; break; }
      nf = nf + 1;
      ifac[nf + 2] = ntry;
      nl = nq;
      if (ntry == 2 && nf != 1) {
        for (int i = 2; i <= nf; ++i) {
          int ib = nf - i + 2;
          ifac[ib + 2] = ifac[ib + 1];
        }
        ifac[3] = 2;
      }
      if (nl == 1) break;
    }
    if (nl == 1) break;
  }
  ifac[1] = n;
  ifac[2] = nf;
  for (int k1 = 1; k1 <= nf; ++k1) {
    int ip = ifac[k1 + 2];
    if (ip != 2 && ip != 3 && ip != 4 && ip != 5)
      throw std::runtime_error("oracle FFT supports lengths with prime factors 2, 3 and 5 only");
  }
  const double tpi = 2.0 * std::acos(-1.0);
  const double argh = tpi / (double)n;
  double* wa = plan.wa.data() - 1;  // wa[1..2n]
  int i = 2, l1 = 1;
  for (int k1 = 1; k1 <= nf; ++k1) {
    int ip = ifac[k1 + 2];
    int ld = 0;
    int l2 = l1 * ip;
    int ido = n / l2;
    int idot = ido + ido + 2;
    int ipm = ip - 1;
    for (int jj = 1; jj <= ipm; ++jj) {
      int i1 = i;
      wa[i - 1] = 1.0;
      wa[i] = 0.0;
      ld = ld + l1;
      double fi = 0.0;
      double argld = (double)ld * argh;
      for (int ii = 4; ii <= idot; ii += 2) {
        i = i + 2;
        fi = fi + 1.0;
        double arg = fi * argld;
        wa[i - 1] = std::cos(arg);
        wa[i] = std::sin(arg);
      }
      if (ip > 5) { wa[i1 - 1] = wa[i - 1]; wa[i1] = wa[i]; }
    }
    l1 = l2;
  }
}

// passf2.f90 / passb2.f90; sign = -1 forward, +1 backward.
static void pass2(int ido, int l1, const double* cc_, double* ch_, const double* wa1_, int sign) {
#define CC(i, j, k) cc_[((i) - 1) + ido * (((j) - 1) + 2 * ((k) - 1))]
#define CH(i, k, j) ch_[((i) - 1) + ido * (((k) - 1) + l1 * ((j) - 1))]
#define WA1(i) wa1_[(i) - 1]
  if (ido > 2) {
    for (int k = 1; k <= l1; ++k)
      for (int i = 2; i <= ido; i += 2) {
        CH(i - 1, k, 1) = CC(i - 1, 1, k) + CC(i - 1, 2, k);
        double tr2 = CC(i - 1, 1, k) - CC(i - 1, 2, k);
        CH(i, k, 1) = CC(i, 1, k) + CC(i, 2, k);
        double ti2 = CC(i, 1, k) - CC(i, 2, k);
        if (sign < 0) {
          CH(i, k, 2) = WA1(i - 1) * ti2 - WA1(i) * tr2;
          CH(i - 1, k, 2) = WA1(i - 1) * tr2 + WA1(i) * ti2;
        } else {
          CH(i, k, 2) = WA1(i - 1) * ti2 + WA1(i) * tr2;
          CH(i - 1, k, 2) = WA1(i - 1) * tr2 - WA1(i) * ti2;
        }
      }
  } else {
    for (int k = 1; k <= l1; ++k) {
      CH(1, k, 1) = CC(1, 1, k) + CC(1, 2, k);
      CH(1, k, 2) = CC(1, 1, k) - CC(1, 2, k);
      CH(2, k, 1) = CC(2, 1, k) + CC(2, 2, k);
      CH(2, k, 2) = CC(2, 1, k) - CC(2, 2, k);
    }
  }
#undef CC
#undef CH
#undef WA1
}

// passf4.f90 / passb4.f90
static void pass4(int ido, int l1, const double* cc_, double* ch_, const double* wa1_,
                  const double* wa2_, const double* wa3_, int sign) {
#define CC(i, j, k) cc_[((i) - 1) + ido * (((j) - 1) + 4 * ((k) - 1))]
#define CH(i, k, j) ch_[((i) - 1) + ido * (((k) - 1) + l1 * ((j) - 1))]
#define WA1(i) wa1_[(i) - 1]
#define WA2(i) wa2_[(i) - 1]
#define WA3(i) wa3_[(i) - 1]
  if (ido != 2) {
    for (int k = 1; k <= l1; ++k)
      for (int i = 2; i <= ido; i += 2) {
        double ti1 = CC(i, 1, k) - CC(i, 3, k);
        double ti2 = CC(i, 1, k) + CC(i, 3, k);
        double ti3 = CC(i, 2, k) + CC(i, 4, k);
        double tr4 = (sign < 0) ? CC(i, 2, k) - CC(i, 4, k) : CC(i, 4, k) - CC(i, 2, k);
        double tr1 = CC(i - 1, 1, k) - CC(i - 1, 3, k);
        double tr2 = CC(i - 1, 1, k) + CC(i - 1, 3, k);
        double ti4 = (sign < 0) ? CC(i - 1, 4, k) - CC(i - 1, 2, k) : CC(i - 1, 2, k) - CC(i - 1, 4, k);
        double tr3 = CC(i - 1, 2, k) + CC(i - 1, 4, k);
        CH(i - 1, k, 1) = tr2 + tr3;
        double cr3 = tr2 - tr3;
        CH(i, k, 1) = ti2 + ti3;
        double ci3 = ti2 - ti3;
        double cr2 = tr1 + tr4;
        double cr4 = tr1 - tr4;
        double ci2 = ti1 + ti4;
        double ci4 = ti1 - ti4;
        if (sign < 0) {
          CH(i - 1, k, 2) = WA1(i - 1) * cr2 + WA1(i) * ci2;
          CH(i, k, 2) = WA1(i - 1) * ci2 - WA1(i) * cr2;
          CH(i - 1, k, 3) = WA2(i - 1) * cr3 + WA2(i) * ci3;
          CH(i, k, 3) = WA2(i - 1) * ci3 - WA2(i) * cr3;
          CH(i - 1, k, 4) = WA3(i - 1) * cr4 + WA3(i) * ci4;
          CH(i, k, 4) = WA3(i - 1) * ci4 - WA3(i) * cr4;
        } else {
          CH(i - 1, k, 2) = WA1(i - 1) * cr2 - WA1(i) * ci2;
          CH(i, k, 2) = WA1(i - 1) * ci2 + WA1(i) * cr2;
          CH(i - 1, k, 3) = WA2(i - 1) * cr3 - WA2(i) * ci3;
          CH(i, k, 3) = WA2(i - 1) * ci3 + WA2(i) * cr3;
          CH(i - 1, k, 4) = WA3(i - 1) * cr4 - WA3(i) * ci4;
          CH(i, k, 4) = WA3(i - 1) * ci4 + WA3(i) * cr4;
        }
      }
  } else {
    for (int k = 1; k <= l1; ++k) {
      double ti1 = CC(2, 1, k) - CC(2, 3, k);
      double ti2 = CC(2, 1, k) + CC(2, 3, k);
      double tr4 = (sign < 0) ? CC(2, 2, k) - CC(2, 4, k) : CC(2, 4, k) - CC(2, 2, k);
      double ti3 = CC(2, 2, k) + CC(2, 4, k);
      double tr1 = CC(1, 1, k) - CC(1, 3, k);
      double tr2 = CC(1, 1, k) + CC(1, 3, k);
      double ti4 = (sign < 0) ? CC(1, 4, k) - CC(1, 2, k) : CC(1, 2, k) - CC(1, 4, k);
      double tr3 = CC(1, 2, k) + CC(1, 4, k);
      CH(1, k, 1) = tr2 + tr3;
      CH(1, k, 3) = tr2 - tr3;
      CH(2, k, 1) = ti2 + ti3;
      CH(2, k, 3) = ti2 - ti3;
      CH(1, k, 2) = tr1 + tr4;
      CH(1, k, 4) = tr1 - tr4;
      CH(2, k, 2) = ti1 + ti4;
      CH(2, k, 4) = ti1 - ti4;
    }
  }
#undef CC
#undef CH
#undef WA1
#undef WA2
#undef WA3
}

// passf3.f90 / passb3.f90
static void pass3(int ido, int l1, const double* cc_, double* ch_, const double* wa1_, const double* wa2_, int sign) {
#define CC(i, j, k) cc_[((i) - 1) + ido * (((j) - 1) + 3 * ((k) - 1))]
#define CH(i, k, j) ch_[((i) - 1) + ido * (((k) - 1) + l1 * ((j) - 1))]
#define WA1(i) wa1_[(i) - 1]
#define WA2(i) wa2_[(i) - 1]
  const double taur = -0.5;
  const double taui = (sign < 0) ? -std::sqrt(3.0) / 2.0 : std::sqrt(3.0) / 2.0;
  if (ido != 2) {
    for (int k = 1; k <= l1; ++k)
      for (int i = 2; i <= ido; i += 2) {
        double tr2 = CC(i - 1, 2, k) + CC(i - 1, 3, k);
        double cr2 = CC(i - 1, 1, k) + taur * tr2;
        CH(i - 1, k, 1) = CC(i - 1, 1, k) + tr2;
        double ti2 = CC(i, 2, k) + CC(i, 3, k);
        double ci2 = CC(i, 1, k) + taur * ti2;
        CH(i, k, 1) = CC(i, 1, k) + ti2;
        double cr3 = taui * (CC(i - 1, 2, k) - CC(i - 1, 3, k));
        double ci3 = taui * (CC(i, 2, k) - CC(i, 3, k));
        double dr2 = cr2 - ci3;
        double dr3 = cr2 + ci3;
        double di2 = ci2 + cr3;
        double di3 = ci2 - cr3;
        if (sign < 0) {
          CH(i, k, 2) = WA1(i - 1) * di2 - WA1(i) * dr2;
          CH(i - 1, k, 2) = WA1(i - 1) * dr2 + WA1(i) * di2;
          CH(i, k, 3) = WA2(i - 1) * di3 - WA2(i) * dr3;
          CH(i - 1, k, 3) = WA2(i - 1) * dr3 + WA2(i) * di3;
        } else {
          CH(i, k, 2) = WA1(i - 1) * di2 + WA1(i) * dr2;
          CH(i - 1, k, 2) = WA1(i - 1) * dr2 - WA1(i) * di2;
          CH(i, k, 3) = WA2(i - 1) * di3 + WA2(i) * dr3;
          CH(i - 1, k, 3) = WA2(i - 1) * dr3 - WA2(i) * di3;
        }
      }
  } else {
    for (int k = 1; k <= l1; ++k) {
      double tr2 = CC(1, 2, k) + CC(1, 3, k);
      double cr2 = CC(1, 1, k) + taur * tr2;
      CH(1, k, 1) = CC(1, 1, k) + tr2;
      double ti2 = CC(2, 2, k) + CC(2, 3, k);
      double ci2 = CC(2, 1, k) + taur * ti2;
      CH(2, k, 1) = CC(2, 1, k) + ti2;
      double cr3 = taui * (CC(1, 2, k) - CC(1, 3, k));
      double ci3 = taui * (CC(2, 2, k) - CC(2, 3, k));
      CH(1, k, 2) = cr2 - ci3;
      CH(1, k, 3) = cr2 + ci3;
      CH(2, k, 2) = ci2 + cr3;
      CH(2, k, 3) = ci2 - cr3;
    }
  }
#undef CC
#undef CH
#undef WA1
#undef WA2
}

// passf5.f90 / passb5.f90
static void pass5(int ido, int l1, const double* cc_, double* ch_, const double* wa1_, const double* wa2_,
                  const double* wa3_, const double* wa4_, int sign) {
#define CC(i, j, k) cc_[((i) - 1) + ido * (((j) - 1) + 5 * ((k) - 1))]
#define CH(i, k, j) ch_[((i) - 1) + ido * (((k) - 1) + l1 * ((j) - 1))]
  const double pi = std::acos(-1.0);
  const double tr11 = std::cos(2.0 * pi / 5.0);
  const double ti11 = (sign < 0 ? -1.0 : 1.0) * std::sin(2.0 * pi / 5.0);
  const double tr12 = std::cos(4.0 * pi / 5.0);
  const double ti12 = (sign < 0 ? -1.0 : 1.0) * std::sin(4.0 * pi / 5.0);
  // the twiddle products of one output pair: passf5's w*d forward, passb5's conj(w)*d backward
  auto put = [&](int i, int k, int j, const double* wa, double dr, double di) {
    if (sign < 0) {
      CH(i - 1, k, j) = wa[(i - 1) - 1] * dr + wa[i - 1] * di;
      CH(i, k, j) = wa[(i - 1) - 1] * di - wa[i - 1] * dr;
    } else {
      CH(i - 1, k, j) = wa[(i - 1) - 1] * dr - wa[i - 1] * di;
      CH(i, k, j) = wa[(i - 1) - 1] * di + wa[i - 1] * dr;
    }
  };
  if (ido != 2) {
    for (int k = 1; k <= l1; ++k)
      for (int i = 2; i <= ido; i += 2) {
        double ti5 = CC(i, 2, k) - CC(i, 5, k);
        double ti2 = CC(i, 2, k) + CC(i, 5, k);
        double ti4 = CC(i, 3, k) - CC(i, 4, k);
        double ti3 = CC(i, 3, k) + CC(i, 4, k);
        double tr5 = CC(i - 1, 2, k) - CC(i - 1, 5, k);
        double tr2 = CC(i - 1, 2, k) + CC(i - 1, 5, k);
        double tr4 = CC(i - 1, 3, k) - CC(i - 1, 4, k);
        double tr3 = CC(i - 1, 3, k) + CC(i - 1, 4, k);
        CH(i - 1, k, 1) = CC(i - 1, 1, k) + tr2 + tr3;
        CH(i, k, 1) = CC(i, 1, k) + ti2 + ti3;
        double cr2 = CC(i - 1, 1, k) + tr11 * tr2 + tr12 * tr3;
        double ci2 = CC(i, 1, k) + tr11 * ti2 + tr12 * ti3;
        double cr3 = CC(i - 1, 1, k) + tr12 * tr2 + tr11 * tr3;
        double ci3 = CC(i, 1, k) + tr12 * ti2 + tr11 * ti3;
        double cr5 = ti11 * tr5 + ti12 * tr4;
        double ci5 = ti11 * ti5 + ti12 * ti4;
        double cr4 = ti12 * tr5 - ti11 * tr4;
        double ci4 = ti12 * ti5 - ti11 * ti4;
        double dr3 = cr3 - ci4;
        double dr4 = cr3 + ci4;
        double di3 = ci3 + cr4;
        double di4 = ci3 - cr4;
        double dr5 = cr2 + ci5;
        double dr2 = cr2 - ci5;
        double di5 = ci2 - cr5;
        double di2 = ci2 + cr5;
        put(i, k, 2, wa1_, dr2, di2);
        put(i, k, 3, wa2_, dr3, di3);
        put(i, k, 4, wa3_, dr4, di4);
        put(i, k, 5, wa4_, dr5, di5);
      }
  } else {
    for (int k = 1; k <= l1; ++k) {
      double ti5 = CC(2, 2, k) - CC(2, 5, k);
      double ti2 = CC(2, 2, k) + CC(2, 5, k);
      double ti4 = CC(2, 3, k) - CC(2, 4, k);
      double ti3 = CC(2, 3, k) + CC(2, 4, k);
      double tr5 = CC(1, 2, k) - CC(1, 5, k);
      double tr2 = CC(1, 2, k) + CC(1, 5, k);
      double tr4 = CC(1, 3, k) - CC(1, 4, k);
      double tr3 = CC(1, 3, k) + CC(1, 4, k);
      CH(1, k, 1) = CC(1, 1, k) + tr2 + tr3;
      CH(2, k, 1) = CC(2, 1, k) + ti2 + ti3;
      double cr2 = CC(1, 1, k) + tr11 * tr2 + tr12 * tr3;
      double ci2 = CC(2, 1, k) + tr11 * ti2 + tr12 * ti3;
      double cr3 = CC(1, 1, k) + tr12 * tr2 + tr11 * tr3;
      double ci3 = CC(2, 1, k) + tr12 * ti2 + tr11 * ti3;
      double cr5 = ti11 * tr5 + ti12 * tr4;
      double ci5 = ti11 * ti5 + ti12 * ti4;
      double cr4 = ti12 * tr5 - ti11 * tr4;
      double ci4 = ti12 * ti5 - ti11 * ti4;
      CH(1, k, 2) = cr2 - ci5;
      CH(1, k, 5) = cr2 + ci5;
      CH(2, k, 2) = ci2 + cr5;
      CH(2, k, 3) = ci3 + cr4;
      CH(1, k, 3) = cr3 - ci4;
      CH(1, k, 4) = cr3 + ci4;
      CH(2, k, 4) = ci3 - cr4;
      CH(2, k, 5) = ci2 - cr5;
    }
  }
#undef CC
#undef CH
}

// cfftf1.f90 / cfftb1.f90: apply the passes, ping-ponging between c and ch.
static void cfft1(const FftPlan& plan, double* c, double* ch, int sign) {
  const int n = plan.n;
  const std::vector<int>& ifac = plan.ifac;
  const double* wa = plan.wa.data() - 1;  // wa[1..]
  int nf = ifac[2];
  int na = 0, l1 = 1, iw = 1;
  for (int k1 = 1; k1 <= nf; ++k1) {
    int ip = ifac[k1 + 2];
    int l2 = ip * l1;
    int ido = n / l2;
    int idot = ido + ido;
    if (ip == 4) {
      int ix2 = iw + idot, ix3 = ix2 + idot;
      if (na != 0) pass4(idot, l1, ch, c, &wa[iw], &wa[ix2], &wa[ix3], sign);
      else pass4(idot, l1, c, ch, &wa[iw], &wa[ix2], &wa[ix3], sign);
      na = 1 - na;
    } else if (ip == 2) {
      if (na != 0) pass2(idot, l1, ch, c, &wa[iw], sign);
      else pass2(idot, l1, c, ch, &wa[iw], sign);
      na = 1 - na;
    } else if (ip == 3) {
      int ix2 = iw + idot;
      if (na != 0) pass3(idot, l1, ch, c, &wa[iw], &wa[ix2], sign);
      else pass3(idot, l1, c, ch, &wa[iw], &wa[ix2], sign);
      na = 1 - na;
    } else {  // ip == 5 (fft_plan_init rejects other factors)
      int ix2 = iw + idot, ix3 = ix2 + idot, ix4 = ix3 + idot;
      if (na != 0) pass5(idot, l1, ch, c, &wa[iw], &wa[ix2], &wa[ix3], &wa[ix4], sign);
      else pass5(idot, l1, c, ch, &wa[iw], &wa[ix2], &wa[ix3], &wa[ix4], sign);
      na = 1 - na;
    }
    l1 = l2;
    iw = iw + (ip - 1) * idot;
  }
  if (na == 0) return;
  for (int i = 0; i < 2 * n; ++i) c[i] = ch[i];
}

void zfftf(const FftPlan& plan, double* c, double* work) { cfft1(plan, c, work, -1); }
void zfftb(const FftPlan& plan, double* c, double* work) { cfft1(plan, c, work, +1); }

// fftnorth.F90:29-48 fftn_r2c: promote a real row to complex, forward transform, keep n/2+1.
void fftn_r2c(const FftPlan& plan, const double* in, double* out_complex, double* data, double* work) {
  const int n = plan.n;
  for (int i = 0; i < n; ++i) { data[2 * i] = in[i]; data[2 * i + 1] = 0.0; }
  zfftf(plan, data, work);
  for (int i = 0; i < n / 2 + 1; ++i) { out_complex[2 * i] = data[2 * i]; out_complex[2 * i + 1] = data[2 * i + 1]; }
}

// fftnorth.F90:54-73 fftn_c2r: Hermitian completion, backward transform, real part / n.
void fftn_c2r(const FftPlan& plan, const double* in_complex, double* out, double* data, double* work) {
  const int n = plan.n;
  for (int i = 0; i < n / 2 + 1; ++i) { data[2 * i] = in_complex[2 * i]; data[2 * i + 1] = in_complex[2 * i + 1]; }
  for (int i = n / 2 + 2; i <= n; ++i) {  // 1-based i; data(i) = conjg(in(n-i+2))
    int src = n - i + 2;
    data[2 * (i - 1)] = in_complex[2 * (src - 1)];
    data[2 * (i - 1) + 1] = -in_complex[2 * (src - 1) + 1];
  }
  zfftb(plan, data, work);
  for (int i = 0; i < n; ++i) out[i] = data[2 * i] / (double)n;
}

}  // namespace oracle
