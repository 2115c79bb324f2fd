// loglaw.cuh -- wall functions of the log-law (INDB(3,L) = 6) and fully
// rough (8) walls: the friction velocity of VF_CLOGLW (vf_cloglw.f:29-52)
// and VF_CLOGKS (vf_clogks.f:27-33), with the natural logarithm written
// out step by step so that the oracle's copy of the same steps gives the
// same bits.
#pragma once
#include "cadmas_dev.cuh"

namespace cadmas {

// ln x.  x = m 2^e with m in [sqrt(1/2), sqrt(2)) (frexp, exact), so
// ln x = e ln 2 + 2 atanh(s), s = (m - 1)/(m + 1), |s| <= 0.1716; the
// Maclaurin series 2 atanh(s) = 2 s (1 + z/3 + z^2/5 + ... + z^13/27),
// z = s^2 <= 0.0295, by Horner's rule; the first omitted term is below
// 2^-60 of the sum.  0 gives -inf, a negative or NaN argument NaN.
__device__ __forceinline__ double ln_series(double x) {
  if (!(x > 0.0)) return (x == 0.0) ? -HUGE_VAL : (x - x) / (x - x);
  if (x > 1.7976931348623157e308) return x;
  int e;
  double m = frexp(x, &e);
  if (m < 0.70710678118654752) {
    m = m * 2.0;
    e = e - 1;
  }
  const double s = (m - 1.0) / (m + 1.0);
  const double z = s * s;
  double p = 1.0 / 27.0;
#pragma unroll 1
  for (int k = 12; k >= 0; --k) p = p * z + 1.0 / (double)(2 * k + 1);
  return (double)e * 0.69314718055994531 + 2.0 * s * p;
}

// VF_CLOGLW: the friction velocity u* of u/u* = ln(DL u*/ANU0)/kappa + A
// for the tangential speed VA at distance DL from the wall, by Newton's
// method from u* = ANU0/DL (where the logarithm is zero), at most 20
// steps, |du*| < 1e-10 u*.  0 when VA < 1e-20 or ANU0 < 1e-20.  Returns
// false when the iteration did not converge ('NOT CONVERGED.').
__device__ __forceinline__ bool cloglw(double DL, double VA, double ANU0, double AKK0, double AKA0, double &VT) {
  const double ZERO = 1.0e-20;  // VF_A0PRM.h
  VT = 0.0;
  if (VA < ZERO || ANU0 < ZERO) return true;
  const double EPS = 1.0e-10;
  const double AKR = 1.0 / AKK0, ANR = 1.0 / ANU0;
  double X = ANU0 / DL, DX = 0.0;
#pragma unroll 1
  for (int it = 1; it <= 20; ++it) {
    const double W = ln_series(DL * X * ANR);
    const double F = X * AKR * W + X * AKA0 - VA;
    const double D = AKR * W + AKR + AKA0;
    DX = -F / D;
    X = X + DX;
    if (fabs(DX) < X * EPS) break;
  }
  if (fabs(DX) >= X * EPS) return false;  // (a NaN passes, as in the reference)
  VT = X;
  return true;
}

// VF_CLOGKS: u* = VA / (ln(DL/ks)/kappa + A + 3) on a fully rough wall of
// roughness ks; 0 when VA < 1e-20 or ANU0 < 1e-20.
__device__ __forceinline__ double clogks(double DL, double VA, double BKS, double ANU0, double AKK0, double AKA0) {
  const double ZERO = 1.0e-20;
  if (VA < ZERO || ANU0 < ZERO) return 0.0;
  const double X = ln_series(DL / BKS) / AKK0 + AKA0 + 3.0;
  return VA / X;
}

}  // namespace cadmas
