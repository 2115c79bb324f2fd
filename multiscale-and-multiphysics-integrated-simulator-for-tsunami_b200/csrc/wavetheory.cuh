// wavetheory.cuh -- per-face evaluation of the wave theories of the wave
// maker and the wave source (VF_CWMAK2 of FUNC STREAM N, STOKES, CNOIDAL),
// shared by the host time part and the k_wave / k_srcuv kernels.
//
// Two forms cover the three theories.  The series form holds the stream-
// function wave (in metres) and the fifth-order Stokes wave (in the
// centimetres of the reference's routine, vf_wstk0.f VF_STK2):
//   u = ub + sum_{j=1..n} cj cosh(j k (z + d)),   w = sum_j sj sinh(j k (z + d)),
// cj, sj the phase's cosine and sine terms.  The cnoidal form holds the
// third-order cnoidal wave (vf_wcnd0.f VF_CND2), polynomials in cn^2 and
// in Z^2 = (1 + z/d)^2:
//   u = sum_{i=4..1} cn^(2(i-1)) sum_{j=3..1} B(j,i) Z^(2(j-1)),
//   w = Z cn sn dn sum_{i=4..2} cn^(2(i-2)) sum_j BB(j,i) Z^(2(j-1)),
// in Horner order over j, then i.
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

// The phase's part of a theory, filled on the host (wavetheory.cu):
//   kind WT_SERIES: n terms cj, sj, the wave number k and depth d in the
//     theory's unit of length, ub the constant term; clamp: z + d held at
//     0 from below (the stream function, as VF_SFMB2 does);
//   kind WT_CNOIDAL: B(j,i) in cj and BB(j,i) in sj at (i-1)*3 + (j-1),
//     d the depth, cn2 = cn^2 and csd = cn sn dn at the phase.
// zs converts a height in metres to the theory's unit (1 or 100, cm) and
// us its velocities back to m/s (1 or 0.01).
enum { WT_SERIES = 0, WT_CNOIDAL = 1 };
struct WavePhase {
  int n, kind, clamp, pad;
  double zs, us;
  double k, d, ub;
  double cn2, csd;
  double cj[STREAM_NMAX], sj[STREAM_NMAX];
};

// u and w at height z above the still water level.  As in the reference,
// the height enters the theory's routine in single precision
// (REAL(ZC) or REAL(ZC*100.0D0), vf_cwmak2.f) and the velocities leave it
// in single precision, then scaled to m/s.
WT_HD inline void wt_velocity(const WavePhase &ph, double z, double &u, double &w) {
  const double zt = (double)(float)(z * ph.zs);
  double su, sw;
  if (ph.kind == WT_CNOIDAL) {
    const double Z = 1.0 + zt / ph.d, ZZ = Z * Z;
    su = 0.0;
    sw = 0.0;
    for (int i = 4; i >= 1; --i) {
      double pu = 0.0, pw = 0.0;
      for (int j = 3; j >= 1; --j) {
        pu = pu * ZZ + ph.cj[(i - 1) * 3 + (j - 1)];
        pw = pw * ZZ + ph.sj[(i - 1) * 3 + (j - 1)];
      }
      su = su * ph.cn2 + pu;
      if (i > 1) sw = sw * ph.cn2 + pw;
    }
    sw = sw * ph.csd * Z;
  } else {
    double zd = zt + ph.d;
    if (ph.clamp && zd < 0.0) zd = 0.0;
    su = ph.ub;
    sw = 0.0;
    for (int j = 1; j <= ph.n; ++j) {
      double ch, sh;
      wt_coshsinh((double)j * ph.k * zd, ch, sh);
      su = su + ph.cj[j - 1] * ch;
      sw = sw + ph.sj[j - 1] * sh;
    }
  }
  u = (double)(float)su * ph.us;
  w = (double)(float)sw * ph.us;
}

// The phase's data of one wave-maker column under oblique incidence: its
// level (VF_CWMAK1 at the column's phase) and the phase part.
struct WaveCol {
  double wvz;
  WavePhase ph;
};

}  // namespace cadmas
