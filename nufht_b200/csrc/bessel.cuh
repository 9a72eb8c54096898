// Device Bessel functions of the first kind in FP64, written for this project.
//
//   bessel_jn(n, x)      integer order n >= 0, x >= 0
//   bessel_jhalf(n, x)   order n + 1/2, 0 <= n <= 9, x >= 0
//   bessel_j_orders(...) J_0(z) .. J_nmax(z) at one argument (Miller's algorithm)
//
// Methods (absolute error target ~1e-15, checked against mpmath values):
//   * x <= 2 sqrt(n+1): power series  J_n(x) = sum_k (-x^2/4)^k (x/2)^n / (k! (n+k)!),
//     whose terms decrease from the first one in this range (no cancellation);
//   * x > n: upward recurrence J_{k+1} = (2k/x) J_k - J_{k-1} from J_0, J_1 (CUDA's
//     j0()/j1()), stable while k < x;
//   * otherwise: Miller's downward recurrence from an index N well above max(n, x),
//     normalised with the identity J_0 + 2 sum_k J_{2k} = 1, rescaling on overflow.
// Half-integer orders use J_{n+1/2}(x) = sqrt(2x/pi) j_n(x), with j_0 = sin x / x,
// j_1 = sin x / x^2 - cos x / x and upward recurrence (x >= n), or the power series of
// J_{n+1/2} for x < n.
#pragma once

#include <cuda_runtime.h>
#include <math.h>

namespace hankel {

__device__ __forceinline__ int miller_start(int M) {
  int N = M + 16 + (int)sqrt(40.0 * (double)M);
  return (N + 1) & ~1;
}

__device__ inline double bessel_jn(int n, double x) {
  if (n == 0) return j0(x);
  if (n == 1) return j1(x);
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
  if (x > (double)n) {
    double a = j0(x), b = j1(x), tox = 2.0 / x;
    for (int k = 1; k < n; ++k) {
      double c = (double)k * tox * b - a;
      a = b;
      b = c;
    }
    return b;
  }
  int N = miller_start(n);
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
