// wavetheory.cuh -- evaluation of a steady periodic wave given by its
// stream-function coefficients (FUNC STREAM N of WAVE-BC), shared by the
// host time part and the k_wave kernel.
//
// In the frame moving with the wave (celerity c), the stream function is
//   psi(X, z) = -UB (z + d) + sum_{j=1..N} B_j sinh(j k (z + d)) / cosh(j k d) cos(j k X),
// z measured from the still (mean) water level, d the depth.  The water
// velocity in the fixed frame at phase theta = k X is
//   u = c - UB + sum_j j k B_j cosh(j k (z + d)) / cosh(j k d) cos(j theta)
//   w =          sum_j j k B_j sinh(j k (z + d)) / cosh(j k d) sin(j theta)
// and the surface eta(theta) solves psi(theta, eta) = -Q.
//
// The hyperbolic functions are built here from one exponential written
// out with +, -, *, / and an exact power-of-two scaling, so the host, the
// kernels and an independent restatement give the same bits:
//   exp(x) = 2^n exp(r),  x = n ln2 + r,  |r| <= ln2/2 (Cody and Waite's
//   reduction with ln2 split into a 32-bit head and a tail), exp(r) by its
//   Taylor series to r^14 in Horner form (truncation below 2^-56).
#pragma once
#include <math.h>

namespace cadmas {

#ifdef __CUDACC__
#define WT_HD __host__ __device__
#else
#define WT_HD
#endif

constexpr int STREAM_NMAX = 22;

WT_HD inline double wt_exp(double x) {
  const double LN2_HEAD = 0.6931471803691238, LN2_TAIL = 1.9082149292705877e-10, INV_LN2 = 1.4426950408889634;
  const double t = x * INV_LN2;
  const double n = floor(t + 0.5);
  const double r = (x - n * LN2_HEAD) - n * LN2_TAIL;
  // Taylor coefficients 1/k!, k = 14 .. 0
  double p = 1.0 / 87178291200.0;
  p = p * r + 1.0 / 6227020800.0;
  p = p * r + 1.0 / 479001600.0;
  p = p * r + 1.0 / 39916800.0;
  p = p * r + 1.0 / 3628800.0;
  p = p * r + 1.0 / 362880.0;
  p = p * r + 1.0 / 40320.0;
  p = p * r + 1.0 / 5040.0;
  p = p * r + 1.0 / 720.0;
  p = p * r + 1.0 / 120.0;
  p = p * r + 1.0 / 24.0;
  p = p * r + 1.0 / 6.0;
  p = p * r + 0.5;
  p = p * r + 1.0;
  p = p * r + 1.0;
  return ldexp(p, (int)n);
}
WT_HD inline void wt_coshsinh(double x, double &ch, double &sh) {
  const double e = wt_exp(x), ei = 1.0 / e;
  ch = 0.5 * (e + ei);
  sh = 0.5 * (e - ei);
}

// Per-phase coefficients of the velocity series: cj = j k B_j cos(j theta)
// / cosh(j k d), sj = the same with sin, ub = c - UB.
struct WavePhase {
  int n;
  double k, d, ub;
  double cj[STREAM_NMAX], sj[STREAM_NMAX];
};

// u and w at height z above the still water level (z + d clamped at 0,
// as VF_SFMB2 does), each rounded to single precision as the REAL*4
// results of the reference's wave routines are.
WT_HD inline void wt_velocity(const WavePhase &ph, double z, double &u, double &w) {
  double zd = z + ph.d;
  if (zd < 0.0) zd = 0.0;
  double su = ph.ub, sw = 0.0;
  for (int j = 1; j <= ph.n; ++j) {
    double ch, sh;
    wt_coshsinh((double)j * ph.k * zd, ch, sh);
    su = su + ph.cj[j - 1] * ch;
    sw = sw + ph.sj[j - 1] * sh;
  }
  u = (double)(float)su;
  w = (double)(float)sw;
}

}  // namespace cadmas
