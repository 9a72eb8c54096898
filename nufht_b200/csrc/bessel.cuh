// Device Bessel functions of the first kind in FP64, written for this project.
//
//   bessel_jn(n, x)      integer order n >= 0, x >= 0
//   bessel_jhalf(n, x)   order n + 1/2, 0 <= n <= 9, x >= 0
//   bessel_j_orders(...) J_0(z) .. J_nmax(z) at one argument (Miller's algorithm)
//
// Methods (absolute error target ~1e-15, checked against mpmath values):
//   * J_0 and J_1: Hankel's expansion for x >= 17 (bessel_j01_large), piecewise Chebyshev
//     expansions for x < 17 (bessel_j01_small); higher orders with x > n by the upward
//     recurrence J_{k+1} = (2k/x) J_k - J_{k-1}, stable while k < x;
//   * x <= 2 sqrt(n+1): power series  J_n(x) = sum_k (-x^2/4)^k (x/2)^n / (k! (n+k)!),
//     whose terms decrease from the first one in this range (no cancellation);
//   * otherwise: Miller's downward recurrence from an index N well above max(n, x),
//     normalised with the identity J_0 + 2 sum_k J_{2k} = 1, rescaling on overflow.
// Half-integer orders use J_{n+1/2}(x) = sqrt(2x/pi) j_n(x), with j_0 = sin x / x,
// j_1 = sin x / x^2 - cos x / x and upward recurrence (x >= n), or the power series of
// J_{n+1/2} for x < n.
#pragma once

#include <cuda_runtime.h>
#include <math.h>

#include "bessel_j01_table.h"

namespace hankel {

__device__ __forceinline__ int miller_start(int M) {
  int N = M + 16 + (int)sqrt(40.0 * (double)M);
  return (N + 1) & ~1;
}

// Hankel's expansion of J_0 and J_1 for x >= 17 (Abramowitz & Stegun 9.2.5-9.2.10)
//   J_nu(x) = sqrt(2/(pi x)) (P_nu cos chi - Q_nu sin chi),  chi = x - (nu/2 + 1/4) pi,
//   P_nu = sum_k (-1)^k a_2k(nu) / x^2k,  Q_nu = sum_k (-1)^k a_2k+1(nu) / x^2k+1,
//   a_0 = 1,  a_k = a_{k-1} (4 nu^2 - (2k-1)^2) / (8k),
// with 34 terms (at x >= 17 the terms keep decreasing past k = 34 and these leave a
// truncation error below 2e-16, checked against mpmath; larger arguments make the later
// terms smaller still).  P and Q are evaluated as polynomials in y = 1/x^2 by Horner's rule
// on coefficients computed at compile time from the recurrence: 34 multiply-adds, and
// cos chi, sin chi formed from sincos(x) so that the phase keeps full precision for arguments
// up to the largest k r of the transform.
struct HankelCoefs {
  double p[18];  // P: coefficient of y^m, terms k = 2m
  double q[17];  // Q / (1/x): coefficient of y^m, terms k = 2m + 1
};
__host__ __device__ constexpr HankelCoefs hankel_coefs(double mu) {  // mu = 4 nu^2
  HankelCoefs h{};
  double a = 1.0;
  h.p[0] = 1.0;
  for (int k = 1; k <= 34; ++k) {
    const double d = 2.0 * k - 1.0;
    a = a * (mu - d * d) / (8.0 * k);
    const double sg = ((k >> 1) & 1) ? -1.0 : 1.0;  // (-1)^floor(k/2)
    if (k & 1) h.q[(k - 1) / 2] = sg * a;
    else h.p[k / 2] = sg * a;
  }
  return h;
}

__device__ inline void bessel_j01_large(double x, double* J0, double* J1, bool need_j1 = true) {
  constexpr HankelCoefs h0 = hankel_coefs(0.0), h1 = hankel_coefs(4.0);
  const double ix = 1.0 / x, y = ix * ix;
  double p0 = h0.p[17], q0 = h0.q[16], p1 = h1.p[17], q1 = h1.q[16];
#pragma unroll
  for (int m = 16; m >= 0; --m) p0 = fma(p0, y, h0.p[m]);
#pragma unroll
  for (int m = 15; m >= 0; --m) q0 = fma(q0, y, h0.q[m]);
  q0 *= ix;
  if (need_j1) {
#pragma unroll
    for (int m = 16; m >= 0; --m) p1 = fma(p1, y, h1.p[m]);
#pragma unroll
    for (int m = 15; m >= 0; --m) q1 = fma(q1, y, h1.q[m]);
    q1 *= ix;
  }
  double sn, cn;
  sincos(x, &sn, &cn);
  const double r2 = 0.70710678118654752440;  // 1/sqrt(2)
  double amp = sqrt(2.0 / (M_PI * x));
  // chi0 = x - pi/4, chi1 = x - 3 pi/4
  double c0 = (cn + sn) * r2, s0 = (sn - cn) * r2;
  double c1 = (sn - cn) * r2, s1 = -(sn + cn) * r2;
  *J0 = amp * (p0 * c0 - q0 * s0);
  *J1 = amp * (p1 * c1 - q1 * s1);
}
constexpr double kHankelMinX = 17.0;

// J_0(x) and, when need_j1, J_1(x) for 0 <= x < 17 from the piecewise Chebyshev
// expansions of bessel_j01_table.h (intervals of 1/kJ01PerUnit, Clenshaw summation; error
// below 3e-16).
__device__ inline void bessel_j01_small(double x, double* J0, double* J1, bool need_j1 = true) {
  const double xs = x * kJ01PerUnit;  // exact: a power of two
  int a = (int)xs;
  a = a < 0 ? 0 : (a > kJ01Intervals - 1 ? kJ01Intervals - 1 : a);
  const double t = 2.0 * (xs - (double)a) - 1.0, t2 = 2.0 * t;
  const double* c0 = kJ01Cheb[0][a];
  double b1 = 0.0, b2 = 0.0;
#pragma unroll
  for (int k = kJ01Coefs - 1; k > 0; --k) {
    double bn = fma(t2, b1, c0[k] - b2);
    b2 = b1;
    b1 = bn;
  }
  *J0 = fma(t, b1, c0[0] - b2);
  if (!need_j1) return;
  const double* c1 = kJ01Cheb[1][a];
  double d1 = 0.0, d2 = 0.0;
#pragma unroll
  for (int k = kJ01Coefs - 1; k > 0; --k) {
    double dn = fma(t2, d1, c1[k] - d2);
    d2 = d1;
    d1 = dn;
  }
  *J1 = fma(t, d1, c1[0] - d2);
}

__device__ inline double bessel_jn(int n, double x) {
  double a = 0.0, b = 0.0;
  if (x >= kHankelMinX) {
    bessel_j01_large(x, &a, &b, n != 0);
  } else if (n <= 1 || x > (double)n) {
    bessel_j01_small(x, &a, &b, n != 0);
  }
  if (n == 0) return a;
  if (n == 1) return b;
  if (x > (double)n && (x >= kHankelMinX || x > 2.0 * sqrt((double)n + 1.0))) {
    // upward recurrence, stable while k < x
    const double tox = 2.0 / x;
    for (int k = 1; k < n; ++k) {
      double c = (double)k * tox * b - a;
      a = b;
      b = c;
    }
    return b;
  }
  if (x == 0.0) return 0.0;
  if (x <= 2.0 * sqrt((double)n + 1.0)) {
    double h = 0.5 * x, t = 1.0;
    for (int i = 1; i <= n; ++i) t *= h / (double)i;
    double s = t, q = -h * h;
    for (int k = 1; k < 200; ++k) {
      t *= q / ((double)k * (double)(n + k));
      s += t;
      if (fabs(t) <= 1e-17 * fabs(s)) break;
    }
    return s;
  }
  int N = miller_start(max(n, (int)ceil(x)));
  double tox = 2.0 / x, fkp1 = 0.0, fk = 1e-30, sum = 0.0, fn = 0.0;
  for (int k = N; k > 0; --k) {
    double fkm1 = (double)k * tox * fk - fkp1;
    fkp1 = fk;
    fk = fkm1;
    if (fabs(fk) > 1e250) {
      fk *= 1e-250;
      fkp1 *= 1e-250;
      sum *= 1e-250;
      fn *= 1e-250;
    }
    int km1 = k - 1;
    if (km1 == n) fn = fk;
    if (km1 > 0 && (km1 & 1) == 0) sum += fk;
  }
  return fn / (2.0 * sum + fk);
}

__device__ inline double bessel_jhalf(int n, double x) {
  const double nu = (double)n + 0.5;
  if (x == 0.0) return 0.0;
  if (x < (n > 1 ? (double)n : 1.0)) {
    double h = 0.5 * x;
    double t = exp(nu * log(h) - lgamma(nu + 1.0)), s = t, q = -h * h;
    for (int k = 1; k < 200; ++k) {
      t *= q / ((double)k * (nu + (double)k));
      s += t;
      if (fabs(t) <= 1e-17 * fabs(s)) break;
    }
    return s;
  }
  double sn, cs;
  sincos(x, &sn, &cs);
  double a = sn / x;
  double pre = sqrt(2.0 * x / M_PI);
  if (n == 0) return pre * a;
  double b = sn / (x * x) - cs / x;
  for (int k = 1; k < n; ++k) {
    double c = ((2.0 * k + 1.0) / x) * b - a;
    a = b;
    b = c;
  }
  return pre * b;
}

// J_nu(x) for the orders the transform accepts: nu2 = 2|nu| (integer); even nu2 means an
// integer order.
__device__ __forceinline__ double bessel_j(int nu2, double x) {
  return (nu2 & 1) ? bessel_jhalf(nu2 >> 1, x) : bessel_jn(nu2 >> 1, x);
}

// J_0(z) .. J_nmax(z) into out[0..nmax] (z > 0) by Miller's algorithm.
__device__ inline void bessel_j_orders(int nmax, double z, double* out) {
  int M = nmax;
  if ((double)M < z) M = (int)ceil(z);
  int N = miller_start(M);
  double tox = 2.0 / z, fkp1 = 0.0, fk = 1e-30, sum = 0.0;
  for (int i = 0; i <= nmax; ++i) out[i] = 0.0;
  for (int k = N; k > 0; --k) {
    double fkm1 = (double)k * tox * fk - fkp1;
    fkp1 = fk;
    fk = fkm1;
    if (fabs(fk) > 1e250) {
      fk *= 1e-250;
      fkp1 *= 1e-250;
      sum *= 1e-250;
      for (int i = k; i <= nmax; ++i) out[i] *= 1e-250;
    }
    int km1 = k - 1;
    if (km1 <= nmax) out[km1] = fk;
    if (km1 > 0 && (km1 & 1) == 0) sum += fk;
  }
  double inv = 1.0 / (2.0 * sum + fk);
  for (int i = 0; i <= nmax; ++i) out[i] *= inv;
}

}  // namespace hankel
