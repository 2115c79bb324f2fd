// oracle.cpp -- CPU restatement of the CADMAS-SURF/3D SMAC step.
//
// TEST INFRASTRUCTURE ONLY (see oracle.h).  Every routine restates the
// Fortran routine it is named after, loop for loop and in the Fortran
// evaluation order (left to right, parentheses kept), from
//   Simulators/CADMAS-SURF-3D/Source code/<file>.f
// Built with -O2 -ffp-contract=off so that no fused multiply-add changes a
// rounding.  Loops run on the serial (NPROCS=1) index ranges: MYIS=2,
// MYIE=NUMI-1, MYJS=2, MYJE=NUMJ-1, MYMIS=MYMIE=MYMJS=MYMJE=1
// (vf_cpara.f:80-98).  Restated beyond the plain step: the droplet model
// VF_FDROPF (IDROP >= 1), FF-SLOPE advection (ISCMFF = 1), k-epsilon
// (LEQK = 1), log-law and rough walls (IB 6, 8) with VF_BWKELG, the
// matrix-table wave maker (MTBTYP 1, 2) and the fixed-water-level table
// (MTBTYP 3), the open (radiation) boundary and the adaptive time step
// VF_CDTCAL.  Options outside these (wave-source terms ISCTYP, temperature,
// scalars, time-dependent
// porosity IPRNT>1, the air-pressure model PVCP0) are not restated and
// are rejected.
#ifdef _OPENMP
#include <omp.h>
#endif
#include "oracle.h"

#include <chrono>
#include <cmath>
#include <cstring>
#include <vector>
#include <algorithm>

namespace {

typedef std::vector<double> vd;
typedef std::vector<int> vi;

struct Timer {
  std::chrono::steady_clock::time_point t0;
  void start() { t0 = std::chrono::steady_clock::now(); }
  double stop() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }
};

// gfortran's integer power (libgfortran pow_r8_i4: square and multiply).
static double ipow(double x, int n) {
  double pow = 1.0;
  if (n != 0) {
    unsigned u;
    if (n < 0) { u = (unsigned)(-n); x = pow / x; } else { u = (unsigned)n; }
    for (;;) {
      if (u & 1u) pow *= x;
      u >>= 1;
      if (u) x *= x; else break;
    }
  }
  return pow;
}

// MAX/MIN with the comparison the GPU kernels use (first operand on ties).
static inline double dmax(double a, double b) { return (a < b) ? b : a; }
static inline double dmin(double a, double b) { return (b < a) ? b : a; }

// Natural logarithm for the log-law wall functions, written out so that the
// GPU kernels can take the same steps: x = m 2^e with m in
// [sqrt(1/2), sqrt(2)) (frexp, exact), ln x = e ln 2 + 2 atanh(s),
// s = (m-1)/(m+1), |s| <= 0.1716, and the Maclaurin series
// 2 atanh(s) = 2 s (1 + z/3 + ... + z^13/27), z = s^2, by Horner's rule
// (the first omitted term is below 2^-60 of the sum).  Tests check it
// against libm.
static double ln_series(double x) {
  if (!(x > 0.0)) return (x == 0.0) ? -HUGE_VAL : (x - x) / (x - x);
  if (x > 1.7976931348623157e308) return x;
  int e;
  double m = std::frexp(x, &e);
  if (m < 0.70710678118654752) { m = m * 2.0; e = e - 1; }
  const double s = (m - 1.0) / (m + 1.0);
  const double z = s * s;
  double p = 1.0 / 27.0;
  for (int k = 12; k >= 0; --k) p = p * z + 1.0 / (double)(2 * k + 1);
  return (double)e * 0.69314718055994531 + 2.0 * s * p;
}

// VF_CLOGLW  vf_cloglw.f:29-52: Newton's method for the friction velocity
// of the log law from u* = ANU0/DL; false on 'NOT CONVERGED.'.
static bool cloglw(double DL, double VA, double ANU0, double AKK0, double AKA0, double &VT) {
  const double ZERO = 1.0e-20;
  VT = 0.0;
  if (VA < ZERO || ANU0 < ZERO) return true;
  const int NI = 20;
  const double EPS = 1.0e-10;
  const double AKR = 1.0 / AKK0, ANR = 1.0 / ANU0;
  double XX = ANU0 / DL, DX = 0.0;
  for (int I = 1; I <= NI; ++I) {
    const double W = ln_series(DL * XX * ANR);
    const double F = XX * AKR * W + XX * AKA0 - VA;
    const double D = AKR * W + AKR + AKA0;
    DX = -F / D;
    XX = XX + DX;
    if (std::fabs(DX) < XX * EPS) break;
  }
  if (std::fabs(DX) >= XX * EPS) return false;
  VT = XX;
  return true;
}

// VF_CLOGKS  vf_clogks.f:27-33
static double clogks(double DL, double VA, double BKS, double ANU0, double AKK0, double AKA0) {
  const double ZERO = 1.0e-20;
  if (VA < ZERO || ANU0 < ZERO) return 0.0;
  const double XX = ln_series(DL / BKS) / AKK0 + AKA0 + 3.0;
  return VA / XX;
}

// ------------------------------------------------ FF-SLOPE (ISCMFF = 1)
// Elementary functions of VF_CROOT3 from +,-,*,/ and sqrt only, so that
// the GPU kernels can evaluate the same operations in the same order and
// agree bit for bit (the library's cbrt/atan/cos differ between glibc
// and CUDA in the last bits).  Each is within a few ulps of the exact
// value on the arguments VF_CROOT3 gives it (tests check them against
// libm).
//
// Cube root: x = f 2^e with f in [0.5,1) (frexp, exact); m = f 2^r with
// r = e mod 3 in [0.5,4); Newton's method on y^3 = m from y0 = (m+2)/3,
// which lies above the root by the AM-GM inequality, so the iterates
// fall monotonically; six steps take the worst start (m = 4, 26% high)
// below one ulp.  The reference writes x**(1/3) with the exponent
// rounded to double, which differs from the cube root by a few ulps.
static double slope_cbrt(double x) {
  if (x == 0.0) return 0.0;
  int e;
  double f = std::frexp(x, &e);
  int r = ((e % 3) + 3) % 3;
  double m = std::ldexp(f, r);
  double y = (m + 2.0) / 3.0;
  for (int it = 0; it < 6; ++it) y = y - (y * y * y - m) / (3.0 * y * y);
  return std::ldexp(y, (e - r) / 3);
}

// Arctangent: odd symmetry; atan(a) = pi/2 - atan(1/a) for a > 1; two
// half-angle steps atan(a) = 2 atan(a / (1 + sqrt(1 + a^2))) bring a
// below tan(pi/16) = 0.199; then the Maclaurin series
// z - z^3/3 + z^5/5 - ... to the z^25 term by Horner's rule.
static double slope_atan(double y) {
  const double HALF_PI = 1.5707963267948966;
  double a = std::fabs(y);
  bool inv = a > 1.0;
  if (inv) a = 1.0 / a;
  a = a / (1.0 + std::sqrt(1.0 + a * a));
  a = a / (1.0 + std::sqrt(1.0 + a * a));
  double z2 = a * a;
  double p = 1.0 / 25.0;
  for (int n = 11; n >= 0; --n) p = 1.0 / (double)(2 * n + 1) - z2 * p;
  double t = 4.0 * (a * p);
  if (inv) t = HALF_PI - t;
  return (y < 0.0) ? -t : t;
}

// Cosine: the Maclaurin series in nested form
// 1 - x^2/(1*2) (1 - x^2/(3*4) (1 - ... (1 - x^2/(27*28)))), accurate
// to about 1e-15 for |x| <= 2.7; VF_CROOT3 calls it on
// (-pi/6, 5pi/6] only.
static double slope_cos(double x) {
  double x2 = x * x;
  double p = 1.0;
  for (int n = 14; n >= 1; --n) p = 1.0 - x2 * p / (double)((2 * n - 1) * (2 * n));
  return p;
}

// VF_CROOT2  vf_croot2.f:22-55
static void croot2(double AA, double BB, double CC, double &XX1, double &XX2, int &NRT) {
  if (AA == 0.0) {
    if (BB != 0.0) { XX1 = -CC / BB; XX2 = 0.0; NRT = 1; }
    else { XX1 = 0.0; XX2 = 0.0; NRT = 0; }
  } else {
    double B = 1.0 / AA;
    double A = 0.5 * BB * B;
    B = CC * B;
    double D = A * A - B;
    if (std::fabs(D) < 1.0e-20) { XX1 = -A; XX2 = 0.0; NRT = 1; }
    else if (D < 0.0) { XX1 = 0.0; XX2 = 0.0; NRT = 0; }
    else if (A >= 0.0) { XX1 = -A - std::sqrt(D); XX2 = B / XX1; NRT = 2; }
    else { XX1 = -A + std::sqrt(D); XX2 = B / XX1; NRT = 2; }
  }
}

// VF_CROOT3  vf_croot3.f:27-74 (Cardano)
static void croot3(double AA, double BB, double CC, double DD, double &XX1, double &XX2, double &XX3,
                   int &NRT) {
  const double PI = 3.141592653589794;  // VF_A0PRM.h
  if (AA == 0.0) {
    croot2(BB, CC, DD, XX1, XX2, NRT);
    XX3 = 0.0;
    return;
  }
  double C = 1.0 / AA;
  double A = BB * C;
  double B = CC * C;
  C = DD * C;
  double P = B / 3.0 - A * A / 9.0;
  double Q = C - A * B / 3.0 + 2.0 * A * A * A / 27.0;
  double D = Q * Q + 4.0 * P * P * P;
  if (D > 0.0) {
    double R1 = (Q <= 0.0) ? 0.5 * (-Q + std::sqrt(D)) : 0.5 * (-Q - std::sqrt(D));
    double R2 = -(P * P * P / R1);
    double R13 = slope_cbrt(std::fabs(R1));
    if (R1 < 0.0) R13 = -R13;
    double R23 = slope_cbrt(std::fabs(R2));
    if (R2 < 0.0) R23 = -R23;
    XX1 = R13 + R23 - A / 3.0;
    XX2 = 0.0; XX3 = 0.0; NRT = 1;
  } else {
    double T = (Q != 0.0) ? slope_atan(std::sqrt(-D) / (-Q)) : PI / 2.0;
    if (Q > 0.0) T = PI + T;
    double R = 2.0 * std::sqrt(-P);
    double S = -A / 3.0;
    XX1 = R * slope_cos(T / 3.0) + S;
    XX2 = -(R * slope_cos((PI - T) / 3.0)) + S;
    XX3 = -(R * slope_cos((PI + T) / 3.0)) + S;
    NRT = 3;
  }
}

// The root of VF_FSLP2A/3A in [XL-EP, XR+EP], else the midpoint (the
// reference's WARNING branch); false when there is no root (P.G ERROR).
static bool slope_pick(int NRT, double X1, double X2, double X3, double XL, double XR, double EP,
                       double &AA) {
  if (NRT == 0) return false;
  if (X1 >= XL - EP && X1 <= XR + EP) AA = X1;
  else if (NRT >= 2 && X2 >= XL - EP && X2 <= XR + EP) AA = X2;
  else if (NRT >= 3 && X3 >= XL - EP && X3 <= XR + EP) AA = X3;
  else AA = (XL + XR) / 2.0;
  return true;
}

// Axis order of VF_FSLP2A/2F (vf_fslp2a.f:30-41): L1 the axis of the
// smaller SD, the first on ties.
// VF_FSLP2A  vf_fslp2a.f:30-101: the plane offset AA (|SX| x + |SY| y =
// AA) that leaves FVAL of the DX*DY cell below the plane.  The volume
// 2|SX||SY| V(a) is the piecewise quadratic a^2 - (a-SD1)+^2 - (a-SD2)+^2;
// the interval holding VMX*FVAL is found from below and its quadratic
// solved by VF_CROOT2.
static bool fslp2a(double SX, double SY, double DX, double DY, double FVAL, double &AA) {
  double SS[2] = {std::fabs(SX), std::fabs(SY)}, DD[2] = {DX, DY};
  double SD[2] = {SS[0] * DX, SS[1] * DY};
  int L1 = 0, L2 = 1;
  if (!(SD[0] <= SD[1])) { L1 = 1; L2 = 0; }
  double CNS = 2.0 * SS[0] * SS[1];
  double XMX = SD[0] + SD[1];
  double VMX = DD[0] * DD[1] * CNS;
  double VIN = VMX * FVAL;
  double XL = 0.0, XR = SD[L1], A = 1.0, B = 0.0, C = 0.0;
  double VV = A * XR * XR;
  const double bp[3] = {SD[L1], SD[L2], XMX};
  int k = 0;
  while (!(VIN <= VV)) {
    if (++k == 3) return false;  // P.G ERROR(1)
    double Q = bp[k - 1];
    A = A - 1.0; B = B + 2.0 * Q; C = C - Q * Q;
    XL = XR; XR = bp[k];
    VV = (k == 2) ? VMX : A * XR * XR + B * XR + C;
  }
  double X1, X2; int NRT;
  croot2(A, B, C - VIN, X1, X2, NRT);
  return slope_pick(NRT > 2 ? 2 : NRT, X1, X2, 0.0, XL, XR, XMX * 1.0e-6, AA);  // P.G ERROR(2) if none
}

// VF_FSLP2F  vf_fslp2f.f:25-70: the water fraction below the plane AA.
static double fslp2f(double SX, double SY, double DX, double DY, double AA) {
  double SS[2] = {std::fabs(SX), std::fabs(SY)}, DD[2] = {DX, DY};
  double SD[2] = {SS[0] * DX, SS[1] * DY};
  int L1 = 0, L2 = 1;
  if (!(SD[0] <= SD[1])) { L1 = 1; L2 = 0; }
  double CNS = 2.0 * SS[0] * SS[1];
  double XMX = SD[0] + SD[1];
  double VMX = DD[0] * DD[1] * CNS;
  double A = 1.0, B = 0.0, C = 0.0, VV;
  if (AA <= 0.0) VV = 0.0;
  else if (AA >= XMX) VV = VMX;
  else if (AA <= SD[L1]) VV = A * AA * AA;
  else {
    double Q = SD[L1];
    A = A - 1.0; B = B + 2.0 * Q; C = C - Q * Q;
    if (AA <= SD[L2]) VV = A * AA * AA + B * AA + C;
    else {
      Q = SD[L2];
      A = A - 1.0; B = B + 2.0 * Q; C = C - Q * Q;
      VV = A * AA * AA + B * AA + C;
    }
  }
  return VV / VMX;
}

// Breakpoints of the piecewise cubic volume of VF_FSLP3A/3F, sorted
// SD(L1) <= SD(L2) <= SD(L3): six points before XMX, and the change of
// the cubic's leading coefficient at each (-1 where the plane passes a
// vertex on one axis, +1 on two).  The two orders are the two branches
// of vf_fslp3a.f:63 / vf_fslp3f.f:63.
struct SlopeCubic {
  double SS[3], SD[3], bp[7], XMX, VMX;
  int sg[6];
  SlopeCubic(double SX, double SY, double SZ, double DX, double DY, double DZ) {
    SS[0] = std::fabs(SX); SS[1] = std::fabs(SY); SS[2] = std::fabs(SZ);
    SD[0] = SS[0] * DX; SD[1] = SS[1] * DY; SD[2] = SS[2] * DZ;
    int L1 = 0, L2 = 1, L3 = 2, L;
    if (SD[L1] > SD[L2]) { L = L1; L1 = L2; L2 = L; }
    if (SD[L2] > SD[L3]) { L = L2; L2 = L3; L3 = L; }
    if (SD[L1] > SD[L2]) { L = L1; L1 = L2; L2 = L; }
    double CNS = 6.0 * SS[0] * SS[1] * SS[2];
    XMX = SD[0] + SD[1] + SD[2];
    VMX = DX * DY * DZ * CNS;
    bp[0] = SD[L1]; bp[1] = SD[L2];
    if (SD[L1] + SD[L2] <= SD[L3]) {
      bp[2] = SD[L1] + SD[L2]; bp[3] = SD[L3];
      const int s[6] = {-1, -1, 1, -1, 1, 1};
      for (int i = 0; i < 6; ++i) sg[i] = s[i];
    } else {
      bp[2] = SD[L3]; bp[3] = SD[L1] + SD[L2];
      const int s[6] = {-1, -1, -1, 1, 1, 1};
      for (int i = 0; i < 6; ++i) sg[i] = s[i];
    }
    bp[4] = SD[L1] + SD[L3]; bp[5] = SD[L2] + SD[L3]; bp[6] = XMX;
  }
  // A*x^3 + B*x^2 + C*x + D past the breakpoint Q
  static void pass(int s, double Q, double &A, double &B, double &C, double &D) {
    if (s < 0) { A = A - 1.0; B = B + 3.0 * Q; C = C - 3.0 * Q * Q; D = D + Q * Q * Q; }
    else { A = A + 1.0; B = B - 3.0 * Q; C = C + 3.0 * Q * Q; D = D - Q * Q * Q; }
  }
  static double poly(double A, double B, double C, double D, double x) {
    return A * x * x * x + B * x * x + C * x + D;
  }
};

// VF_FSLP3A  vf_fslp3a.f:30-266
static bool fslp3a(double SX, double SY, double SZ, double DX, double DY, double DZ, double FVAL, double &AA) {
  SlopeCubic c(SX, SY, SZ, DX, DY, DZ);
  double VIN = c.VMX * FVAL;
  double A = 1.0, B = 0.0, C = 0.0, D = 0.0, XL = 0.0, XR = c.bp[0];
  double VV = A * XR * XR * XR;
  int k = 0;
  while (!(VIN <= VV)) {
    if (++k == 7) return false;  // P.G ERROR(1)/(2)
    SlopeCubic::pass(c.sg[k - 1], XR, A, B, C, D);
    XL = XR; XR = c.bp[k];
    VV = (k == 6) ? c.VMX : SlopeCubic::poly(A, B, C, D, XR);
  }
  double X1, X2, X3; int NRT;
  croot3(A, B, C, D - VIN, X1, X2, X3, NRT);
  return slope_pick(NRT, X1, X2, X3, XL, XR, c.XMX * 1.0e-6, AA);  // P.G ERROR(3) if none
}

// VF_FSLP3F  vf_fslp3f.f:30-181
static double fslp3f(double SX, double SY, double SZ, double DX, double DY, double DZ, double AA) {
  SlopeCubic c(SX, SY, SZ, DX, DY, DZ);
  double VV;
  if (AA <= 0.0) VV = 0.0;
  else if (AA >= c.XMX) VV = c.VMX;
  else {
    double A = 1.0, B = 0.0, C = 0.0, D = 0.0, Q = c.bp[0];
    if (AA <= Q) VV = A * AA * AA * AA;
    else {
      int k = 1;
      for (;; ++k) {
        SlopeCubic::pass(c.sg[k - 1], Q, A, B, C, D);
        if (k == 6) break;
        Q = c.bp[k];
        if (AA <= Q) break;
      }
      VV = SlopeCubic::poly(A, B, C, D, AA);
    }
  }
  return VV / c.VMX;
}

// Warp tree of the GPU reduction: lane 0 after shfl_down by 16,8,4,2,1.
static double warp_tree(double *s) {
  for (int off = 16; off >= 1; off >>= 1)
    for (int l = 0; l < off; ++l) s[l] = s[l] + s[l + off];
  return s[0];
}

}  // namespace

struct orc_handle {
  int NI, NJ, NK, NB;
  // parallel loops only where a grid is large enough to pay for the threads
  bool par() const { return (long long)NI * NJ * NK >= 200000; }
  cadmas_params P;
  int sum_mode;
  // static
  vd XX, YY, ZZ, GGV, GGX, GGY, GGZ, GLV, GLX, GLY, GLZ, CD0, ANU;
  vi INDX, INDY, INDZ, INDB;
  bool have_static = false;
  // state
  vd UU, VV, WW, PP, FF, BCU, BCV, BCW, BCP, BCF, TBUB;
  vd BCVI;  // roughness of rough-wall faces
  vi NF, INDC, INDS, NLIM;
  // k-epsilon (LEQK != 0): AK, AE (here AEPS: AE names a solver vector
  // below), ANUT, BCK, BCE; the boundary types INDBK, INDBE and the input
  // boundary values BCK0, BCE0
  vd AK, AEPS, ANUT, BCK, BCE, BCK0, BCE0;
  vi INDBK, INDBE;
  int NUMS = 0;
  double TNOW = 0, DTNOW = 0;
  // wave maker, matrix table (WAVE-BC ... FUNC MATRIX): IBCTYP/BCTYP of
  // the four sides and the table of /VF_AFILEI/ (vf_iimdl.f:49-106)
  struct Wave {
    int on = 0, l1 = 0, l2 = 0;
    double d = 0, t = 0, a = 0;
    int theory = 0;             // FUNC STREAM N | STOKES | CNOIDAL: the wave `th`, not the table
    cadmas_wave_theory th{};
    double ang = 0, sx = 0, sy = 0;  // ANGLE: BCTYP(9..11,JD)
  } WV[4];
  struct Open { int on = 0; double c = 0; } OP[4];  // IBCTYP(1,JD) = 2 and BCTYP(6,JD)
  long long NLOG = 0;  // faces of type 6 or 8 (log-law, rough walls)
  // IBCTYP(2,JD) = -3 with MTBTYP 3: side JD fixes the water level
  bool FIXLVL(int JD) const { return JD >= 1 && JD <= 4 && WV[JD - 1].on && !WV[JD - 1].theory && MTBTYP == 3; }
  // a type 5 face on the domain boundary of the side its NS names
  bool fixlvl_face(int NS, int I, int J) const {
    if (NS < 1 || NS > 4 || !FIXLVL(NS)) return false;
    return NS == 1 ? I == 2 : NS == 2 ? I == NI : NS == 3 ? J == 2 : J == NJ;
  }
  int MTBTYP = 0, MTBNOW = 0;
  double DMTBT0 = 0;
  // wave source (MODEL WAVE-SRC, FUNC MATRIX): ISCTYP(1) = ISC (> 0 the x
  // line I, < 0 the y line -J), SCTYP(1,3,8) = SD, ST, SA; SRCUV(NUMIJ,NUMK)
  int ISC = 0;
  double SD = 0, ST = 0, SA = 0;
  int STHEORY = 0;              // ISCTYP(2) a wave theory (the wave STH), not the table
  cadmas_wave_theory STH{};
  vd SRCUV;
  int IWS() const { return ISC > 0 ? ISC : 0; }
  int JWS() const { return ISC < 0 ? -ISC : 0; }
  double SRC(int ij, int k) const { return SRCUV[(size_t)(ij - 1) + (size_t)(ISC > 0 ? NJ : NI) * (size_t)(k - 1)]; }
  vd DMTBTT, DMTBHH, DMTBZZ, DMTBUN, DMTBUT;
  int NNOW = 0;
  // work arrays WK01..WK17
  vd WK[18];
  // solver scratch
  vd DD, XW, Y2, R0, RR, PPv, AP, AE;
  cadmas_stats st;
  double tmr[5];

  // ---------------------------------------------------------------- helpers
  inline size_t id(int i, int j, int k) const {
    return (size_t)(i - 1) + (size_t)NI * ((size_t)(j - 1) + (size_t)NJ * (size_t)(k - 1));
  }
  inline double X_(int m, int i) const { return XX[(m - 1) + 6 * (i - 1)]; }
  inline double Y_(int m, int j) const { return YY[(m - 1) + 6 * (j - 1)]; }
  inline double Z_(int m, int k) const { return ZZ[(m - 1) + 6 * (k - 1)]; }
  inline int IB_(int m, int l) const { return INDB[(m - 1) + 4 * (l - 1)]; }
  void decode(int ijk, int &i, int &j, int &k) const {
    k = (ijk - 1) / (NI * NJ) + 1;
    ijk = ijk - NI * NJ * (k - 1);
    j = (ijk - 1) / NI + 1;
    i = ijk - NI * (j - 1);
  }

  // Global sum over cells of a masked contribution.  f(i,j,k,&c) returns
  // true when the cell contributes c.  The reference order loops K=2..NK-1,
  // J=2..NJ-1, I=2..NI-1 (e.g. vf_mzip.f:36-43); the GPU order is the row
  // tree described in oracle.h.  Cells outside the interior never
  // contribute in either order (their masks are false).
  template <class F> double gsum(F f) const {
    if (sum_mode == ORC_SUM_REF) {
      double s = 0.0, c;
      for (int k = 2; k <= NK - 1; ++k)
        for (int j = 2; j <= NJ - 1; ++j)
          for (int i = 2; i <= NI - 1; ++i)
            if (f(i, j, k, c)) s = s + c;
      return s;
    }
    const int NR = NJ * NK;
    std::vector<double> R(NR);
    double lane[32];
    for (int r = 0; r < NR; ++r) {
      int j = r % NJ + 1, k = r / NJ + 1;
      for (int l = 0; l < 32; ++l) {
        double s = 0.0, c;
        for (int i0 = l; i0 < NI; i0 += 32)
          if (f(i0 + 1, j, k, c)) s = s + c;
        lane[l] = s;
      }
      R[r] = warp_tree(lane);
    }
    double u[1024];
    for (int t = 0; t < 1024; ++t) {
      double s = 0.0;
      for (int r = t; r < NR; r += 1024) s = s + R[r];
      u[t] = s;
    }
    double w[32];
    for (int q = 0; q < 32; ++q) w[q] = warp_tree(u + 32 * q);
    return warp_tree(w);
  }

  // The same tree over the slabs of the GPU solver's tile-skewed layout
  // (layout tiles of TI x TJ columns, TJ halved with precond_split = 2):
  // tile b (x fastest), wavefront slab w = (k-2)+ti+tj, slab entry
  // t = ti + TIp*tj (TIp = TI rounded up to a multiple of 4; columns
  // ti >= TI are padding); lane l of a slab sums t = l, l+32, ... in order,
  // warp tree per slab, the slabs of each group of 8 (a thread block of the
  // GPU's slab kernels: slabs 8g .. 8g+7) added in slab order starting
  // from 0, then the 1024-thread tree over the groups.  This is the order
  // of the dot products of VF_M1BCGS in the GPU library.
  template <class F> double gsum_skew(F f) const {
    const int TI = std::min(P.precond_ti > 0 ? P.precond_ti : NI - 2, NI - 2);
    const int TJ = std::min(P.precond_tj > 0 ? P.precond_tj : NJ - 2, NJ - 2) /
                   (P.precond_split == 2 ? 2 : 1);  // rows of a layout tile
    const int TIp = (TI + 3) & ~3;
    const int T = TIp * TJ, W = (NK - 2) + (TI - 1) + (TJ - 1);
    const int ntx = (NI - 2 + TI - 1) / TI, nb = ntx * ((NJ - 2 + TJ - 1) / TJ);
    const long long NS = (long long)nb * W;
    std::vector<double> R(NS);
    double lane[32];
    for (long long sl = 0; sl < NS; ++sl) {
      const int b = (int)(sl / W), w = (int)(sl % W), bx = b % ntx, by = b / ntx;
      for (int l = 0; l < 32; ++l) {
        double s = 0.0, c;
        for (int t = l; t < T; t += 32) {
          const int ti = t % TIp, tj = t / TIp;
          const int I = 2 + bx * TI + ti, J = 2 + by * TJ + tj, k = 2 + w - ti - tj;
          if (ti >= TI || I > NI - 1 || J > NJ - 1 || k < 2 || k > NK - 1) continue;
          if (f(I, J, k, c)) s = s + c;
        }
        lane[l] = s;
      }
      R[sl] = warp_tree(lane);
    }
    const long long NG = (NS + 7) / 8;
    std::vector<double> G(NG);
    for (long long gi = 0; gi < NG; ++gi) {
      double s = 0.0;
      for (long long sl = 8 * gi; sl < 8 * gi + 8 && sl < NS; ++sl) s = s + R[sl];
      G[gi] = s;
    }
    double u[1024];
    for (int t = 0; t < 1024; ++t) {
      double s = 0.0;
      for (long long r = t; r < NG; r += 1024) s = s + G[r];
      u[t] = s;
    }
    double wv[32];
    for (int q = 0; q < 32; ++q) wv[q] = warp_tree(u + 32 * q);
    return warp_tree(wv);
  }

  template <class F> double solver_sum(F f) const {
    return sum_mode == ORC_SUM_GPU ? gsum_skew(f) : gsum(f);
  }

  // interior mask helper used by gsum callers
  inline bool interior(int i, int j, int k) const {
    return i >= 2 && i <= NI - 1 && j >= 2 && j <= NJ - 1 && k >= 2 && k <= NK - 1;
  }

  // ======================================================================
  // Momentum fluxes  VF_VFLXDU  vf_vflxdu.f:62-347
  void vflxdu(vd &FLUU, vd &FLUV, vd &FLUW) {
    const double SU = P.scmvp, SC = 1.0 - P.scmvp;
    const int LA = 3, LB = NI - 1;
    for (int K = 2; K <= NK - 1; ++K)
      for (int J = 2; J <= NJ - 1; ++J)
        for (int I = LA - 1; I <= LB; ++I) {
          if (INDC[id(I, J, K)] == -1) continue;
          double WIN = (GLX[id(I, J, K)] * UU[id(I, J, K)] + GLX[id(I + 1, J, K)] * UU[id(I + 1, J, K)]) * 0.5;
          double FG = WIN * (UU[id(I, J, K)] + UU[id(I + 1, J, K)]) * 0.5;
          double &F = FLUU[id(I, J, K)];
          F = F - SU * (dmax(WIN, 0.0) * UU[id(I, J, K)] - dmax(-WIN, 0.0) * UU[id(I + 1, J, K)]) - SC * FG;
          F = F + (GGX[id(I, J, K)] + GGX[id(I + 1, J, K)]) * ANU[id(I, J, K)] * X_(4, I) *
                      (UU[id(I + 1, J, K)] - UU[id(I, J, K)]);
        }
    // (Gy*v)*u  :93-213
    for (int K = 2; K <= NK; ++K)
      for (int J = 2; J <= NJ; ++J)
        for (int I = LA; I <= LB; ++I) {
          int IC = NF[id(I - 1, J - 1, K)] * NF[id(I, J - 1, K)] * NF[id(I - 1, J, K)] * NF[id(I, J, K)];
          int IT = INDX[id(I, J, K)], IBt = INDX[id(I, J - 1, K)];
          double &F = FLUV[id(I, J, K)];
          if (IC != 0 || (IT != 0 && IBt != 0)) {
          } else if (IT == 0 && IBt == 0) {
            double WIN = X_(6, I) * (X_(2, I - 1) * GLY[id(I, J, K)] * VV[id(I, J, K)] +
                                     X_(2, I) * GLY[id(I - 1, J, K)] * VV[id(I - 1, J, K)]);
            double FG = WIN * Y_(6, J) * (Y_(2, J - 1) * UU[id(I, J, K)] + Y_(2, J) * UU[id(I, J - 1, K)]);
            F = F - SU * (dmax(WIN, 0.0) * UU[id(I, J - 1, K)] - dmax(-WIN, 0.0) * UU[id(I, J, K)]) - SC * FG;
            double GG = X_(6, I) * (X_(2, I - 1) * GGY[id(I, J, K)] + X_(2, I) * GGY[id(I - 1, J, K)]);
            double ANR = Y_(6, J) * (Y_(2, J - 1) * ANU[id(I, J, K)] + Y_(2, J) * ANU[id(I, J - 1, K)]);
            double ANL = Y_(6, J) * (Y_(2, J - 1) * ANU[id(I - 1, J, K)] + Y_(2, J) * ANU[id(I - 1, J - 1, K)]);
            double AN = X_(6, I) * (X_(2, I - 1) * ANR + X_(2, I) * ANL);
            double D1 = Y_(5, J) * (UU[id(I, J, K)] - UU[id(I, J - 1, K)]);
            double D2 = X_(5, I) * (VV[id(I, J, K)] - VV[id(I - 1, J, K)]);
            F = F + GG * AN * (D1 + D2);
          } else {
            double BR, BL;
            int IS = INDY[id(I, J, K)];
            if (IS >= 1) {
              if (IB_(3, IS) == 1 || IB_(3, IS) == 4) BR = (IB_(2, IS) == 3) ? UU[id(I, J, K)] : UU[id(I, J - 1, K)];
              else BR = BCU[IS - 1];
            } else {
              BR = Y_(6, J) * (Y_(2, J - 1) * (UU[id(I, J, K)] + UU[id(I + 1, J, K)]) +
                               Y_(2, J) * (UU[id(I, J - 1, K)] + UU[id(I + 1, J - 1, K)])) * 0.5;
            }
            IS = INDY[id(I - 1, J, K)];
            if (IS >= 1) {
              if (IB_(3, IS) == 1 || IB_(3, IS) == 4) BL = (IB_(2, IS) == 3) ? UU[id(I, J, K)] : UU[id(I, J - 1, K)];
              else BL = BCU[IS - 1];
            } else {
              BL = Y_(6, J) * (Y_(2, J - 1) * (UU[id(I, J, K)] + UU[id(I - 1, J, K)]) +
                               Y_(2, J) * (UU[id(I, J - 1, K)] + UU[id(I - 1, J - 1, K)])) * 0.5;
            }
            double WIN = X_(6, I) * (X_(2, I - 1) * GLY[id(I, J, K)] * VV[id(I, J, K)] +
                                     X_(2, I) * GLY[id(I - 1, J, K)] * VV[id(I - 1, J, K)]);
            double FG = X_(6, I) * (X_(2, I) * GLY[id(I, J, K)] * VV[id(I, J, K)] * BR +
                                    X_(2, I - 1) * GLY[id(I - 1, J, K)] * VV[id(I - 1, J, K)] * BL);
            if (IT == 0 && WIN < 0.0) F = F - SU * WIN * UU[id(I, J, K)] - SC * FG;
            else if (IBt == 0 && WIN > 0.0) F = F - SU * WIN * UU[id(I, J - 1, K)] - SC * FG;
            else F = F - FG;
            double GG = X_(6, I) * (X_(2, I - 1) * GGY[id(I, J, K)] + X_(2, I) * GGY[id(I - 1, J, K)]);
            FG = X_(6, I) * (X_(2, I) * BR + X_(2, I - 1) * BL);
            double ANR, ANL;
            if (NF[id(I, J, K)] == -1) ANR = ANU[id(I, J - 1, K)];
            else if (NF[id(I, J - 1, K)] == -1) ANR = ANU[id(I, J, K)];
            else ANR = Y_(6, J) * (Y_(2, J - 1) * ANU[id(I, J, K)] + Y_(2, J) * ANU[id(I, J - 1, K)]);
            if (NF[id(I - 1, J, K)] == -1) ANL = ANU[id(I - 1, J - 1, K)];
            else if (NF[id(I - 1, J - 1, K)] == -1) ANL = ANU[id(I - 1, J, K)];
            else ANL = Y_(6, J) * (Y_(2, J - 1) * ANU[id(I - 1, J, K)] + Y_(2, J) * ANU[id(I - 1, J - 1, K)]);
            double AN = X_(6, I) * (X_(2, I - 1) * ANR + X_(2, I) * ANL);
            double D1 = (IT == 0) ? Y_(4, J) * (UU[id(I, J, K)] - FG) * 2.0
                                  : Y_(4, J - 1) * (FG - UU[id(I, J - 1, K)]) * 2.0;
            double D2 = X_(5, I) * (VV[id(I, J, K)] - VV[id(I - 1, J, K)]);
            F = F + GG * AN * (D1 + D2);
          }
        }
    // (Gz*w)*u  :215-345
    for (int K = 2; K <= NK; ++K)
      for (int J = 2; J <= NJ - 1; ++J)
        for (int I = LA; I <= LB; ++I) {
          int IC = NF[id(I - 1, J, K - 1)] * NF[id(I, J, K - 1)] * NF[id(I - 1, J, K)] * NF[id(I, J, K)];
          int IT = INDX[id(I, J, K)], IBt = INDX[id(I, J, K - 1)];
          double &F = FLUW[id(I, J, K)];
          if (IC != 0 || (IT != 0 && IBt != 0)) {
          } else if (IT == 0 && IBt == 0) {
            double WIN = X_(6, I) * (X_(2, I - 1) * GLZ[id(I, J, K)] * WW[id(I, J, K)] +
                                     X_(2, I) * GLZ[id(I - 1, J, K)] * WW[id(I - 1, J, K)]);
            double FG = WIN * Z_(6, K) * (Z_(2, K - 1) * UU[id(I, J, K)] + Z_(2, K) * UU[id(I, J, K - 1)]);
            F = F - SU * (dmax(WIN, 0.0) * UU[id(I, J, K - 1)] - dmax(-WIN, 0.0) * UU[id(I, J, K)]) - SC * FG;
            double GG = X_(6, I) * (X_(2, I - 1) * GGZ[id(I, J, K)] + X_(2, I) * GGZ[id(I - 1, J, K)]);
            double ANR = Z_(6, K) * (Z_(2, K - 1) * ANU[id(I, J, K)] + Z_(2, K) * ANU[id(I, J, K - 1)]);
            double ANL = Z_(6, K) * (Z_(2, K - 1) * ANU[id(I - 1, J, K)] + Z_(2, K) * ANU[id(I - 1, J, K - 1)]);
            double AN = X_(6, I) * (X_(2, I - 1) * ANR + X_(2, I) * ANL);
            double D1 = Z_(5, K) * (UU[id(I, J, K)] - UU[id(I, J, K - 1)]);
            double D2 = X_(5, I) * (WW[id(I, J, K)] - WW[id(I - 1, J, K)]);
            F = F + GG * AN * (D1 + D2);
          } else {
            double BR, BL;
            int IS = INDZ[id(I, J, K)];
            if (IS >= 1) {
              if (IB_(3, IS) == 1 || IB_(3, IS) == 4) BR = (IB_(2, IS) == 5) ? UU[id(I, J, K)] : UU[id(I, J, K - 1)];
              else BR = BCU[IS - 1];
            } else {
              BR = Z_(6, K) * (Z_(2, K - 1) * (UU[id(I, J, K)] + UU[id(I + 1, J, K)]) +
                               Z_(2, K) * (UU[id(I, J, K - 1)] + UU[id(I + 1, J, K - 1)])) * 0.5;
            }
            IS = INDZ[id(I - 1, J, K)];
            if (IS >= 1) {
              if (IB_(3, IS) == 1 || IB_(3, IS) == 4) BL = (IB_(2, IS) == 5) ? UU[id(I, J, K)] : UU[id(I, J, K - 1)];
              else BL = BCU[IS - 1];
            } else {
              BL = Z_(6, K) * (Z_(2, K - 1) * (UU[id(I, J, K)] + UU[id(I - 1, J, K)]) +
                               Z_(2, K) * (UU[id(I, J, K - 1)] + UU[id(I - 1, J, K - 1)])) * 0.5;
            }
            double WIN = X_(6, I) * (X_(2, I - 1) * GLZ[id(I, J, K)] * WW[id(I, J, K)] +
                                     X_(2, I) * GLZ[id(I - 1, J, K)] * WW[id(I - 1, J, K)]);
            double FG = X_(6, I) * (X_(2, I) * GLZ[id(I, J, K)] * WW[id(I, J, K)] * BR +
                                    X_(2, I - 1) * GLZ[id(I - 1, J, K)] * WW[id(I - 1, J, K)] * BL);
            if (IT == 0 && WIN < 0.0) F = F - SU * WIN * UU[id(I, J, K)] - SC * FG;
            else if (IBt == 0 && WIN > 0.0) F = F - SU * WIN * UU[id(I, J, K - 1)] - SC * FG;
            else F = F - FG;
            double GG = X_(6, I) * (X_(2, I - 1) * GGZ[id(I, J, K)] + X_(2, I) * GGZ[id(I - 1, J, K)]);
            FG = X_(6, I) * (X_(2, I) * BR + X_(2, I - 1) * BL);
            double ANR, ANL;
            if (NF[id(I, J, K)] == -1) ANR = ANU[id(I, J, K - 1)];
            else if (NF[id(I, J, K - 1)] == -1) ANR = ANU[id(I, J, K)];
            else ANR = Z_(6, K) * (Z_(2, K - 1) * ANU[id(I, J, K)] + Z_(2, K) * ANU[id(I, J, K - 1)]);
            if (NF[id(I - 1, J, K)] == -1) ANL = ANU[id(I - 1, J, K - 1)];
            else if (NF[id(I - 1, J, K - 1)] == -1) ANL = ANU[id(I - 1, J, K)];
            else ANL = Z_(6, K) * (Z_(2, K - 1) * ANU[id(I - 1, J, K)] + Z_(2, K) * ANU[id(I - 1, J, K - 1)]);
            double AN = X_(6, I) * (X_(2, I - 1) * ANR + X_(2, I) * ANL);
            double D1 = (IT == 0) ? Z_(4, K) * (UU[id(I, J, K)] - FG) * 2.0
                                  : Z_(4, K - 1) * (FG - UU[id(I, J, K - 1)]) * 2.0;
            double D2 = X_(5, I) * (WW[id(I, J, K)] - WW[id(I - 1, J, K)]);
            F = F + GG * AN * (D1 + D2);
          }
        }
  }

  // VF_VFLXDV  vf_vflxdv.f:62-347
  void vflxdv(vd &FLVU, vd &FLVV, vd &FLVW) {
    const double SU = P.scmvp, SC = 1.0 - P.scmvp;
    const int LA = 3, LB = NJ - 1;
    for (int K = 2; K <= NK - 1; ++K)
      for (int J = LA - 1; J <= LB; ++J)
        for (int I = 2; I <= NI - 1; ++I) {
          if (INDC[id(I, J, K)] == -1) continue;
          double WIN = (GLY[id(I, J, K)] * VV[id(I, J, K)] + GLY[id(I, J + 1, K)] * VV[id(I, J + 1, K)]) * 0.5;
          double FG = WIN * (VV[id(I, J, K)] + VV[id(I, J + 1, K)]) * 0.5;
          double &F = FLVV[id(I, J, K)];
          F = F - SU * (dmax(WIN, 0.0) * VV[id(I, J, K)] - dmax(-WIN, 0.0) * VV[id(I, J + 1, K)]) - SC * FG;
          F = F + (GGY[id(I, J, K)] + GGY[id(I, J + 1, K)]) * ANU[id(I, J, K)] * Y_(4, J) *
                      (VV[id(I, J + 1, K)] - VV[id(I, J, K)]);
        }
    // (Gx*u)*v
    for (int K = 2; K <= NK; ++K)
      for (int J = LA; J <= LB; ++J)
        for (int I = 2; I <= NI; ++I) {
          int IC = NF[id(I - 1, J - 1, K)] * NF[id(I - 1, J, K)] * NF[id(I, J - 1, K)] * NF[id(I, J, K)];
          int IT = INDY[id(I, J, K)], IBt = INDY[id(I - 1, J, K)];
          double &F = FLVU[id(I, J, K)];
          if (IC != 0 || (IT != 0 && IBt != 0)) {
          } else if (IT == 0 && IBt == 0) {
            double WIN = Y_(6, J) * (Y_(2, J - 1) * GLX[id(I, J, K)] * UU[id(I, J, K)] +
                                     Y_(2, J) * GLX[id(I, J - 1, K)] * UU[id(I, J - 1, K)]);
            double FG = WIN * X_(6, I) * (X_(2, I - 1) * VV[id(I, J, K)] + X_(2, I) * VV[id(I - 1, J, K)]);
            F = F - SU * (dmax(WIN, 0.0) * VV[id(I - 1, J, K)] - dmax(-WIN, 0.0) * VV[id(I, J, K)]) - SC * FG;
            double GG = Y_(6, J) * (Y_(2, J - 1) * GGX[id(I, J, K)] + Y_(2, J) * GGX[id(I, J - 1, K)]);
            double ANR = X_(6, I) * (X_(2, I - 1) * ANU[id(I, J, K)] + X_(2, I) * ANU[id(I - 1, J, K)]);
            double ANL = X_(6, I) * (X_(2, I - 1) * ANU[id(I, J - 1, K)] + X_(2, I) * ANU[id(I - 1, J - 1, K)]);
            double AN = Y_(6, J) * (Y_(2, J - 1) * ANR + Y_(2, J) * ANL);
            double D1 = X_(5, I) * (VV[id(I, J, K)] - VV[id(I - 1, J, K)]);
            double D2 = Y_(5, J) * (UU[id(I, J, K)] - UU[id(I, J - 1, K)]);
            F = F + GG * AN * (D1 + D2);
          } else {
            double BR, BL;
            int IS = INDX[id(I, J, K)];
            if (IS >= 1) {
              if (IB_(3, IS) == 1 || IB_(3, IS) == 4) BR = (IB_(2, IS) == 1) ? VV[id(I, J, K)] : VV[id(I - 1, J, K)];
              else BR = BCV[IS - 1];
            } else {
              BR = X_(6, I) * (X_(2, I - 1) * (VV[id(I, J, K)] + VV[id(I, J + 1, K)]) +
                               X_(2, I) * (VV[id(I - 1, J, K)] + VV[id(I - 1, J + 1, K)])) * 0.5;
            }
            IS = INDX[id(I, J - 1, K)];
            if (IS >= 1) {
              if (IB_(3, IS) == 1 || IB_(3, IS) == 4) BL = (IB_(2, IS) == 1) ? VV[id(I, J, K)] : VV[id(I - 1, J, K)];
              else BL = BCV[IS - 1];
            } else {
              BL = X_(6, I) * (X_(2, I - 1) * (VV[id(I, J, K)] + VV[id(I, J - 1, K)]) +
                               X_(2, I) * (VV[id(I - 1, J, K)] + VV[id(I - 1, J - 1, K)])) * 0.5;
            }
            double WIN = Y_(6, J) * (Y_(2, J - 1) * GLX[id(I, J, K)] * UU[id(I, J, K)] +
                                     Y_(2, J) * GLX[id(I, J - 1, K)] * UU[id(I, J - 1, K)]);
            double FG = Y_(6, J) * (Y_(2, J) * GLX[id(I, J, K)] * UU[id(I, J, K)] * BR +
                                    Y_(2, J - 1) * GLX[id(I, J - 1, K)] * UU[id(I, J - 1, K)] * BL);
            if (IT == 0 && WIN < 0.0) F = F - SU * WIN * VV[id(I, J, K)] - SC * FG;
            else if (IBt == 0 && WIN > 0.0) F = F - SU * WIN * VV[id(I - 1, J, K)] - SC * FG;
            else F = F - FG;
            double GG = Y_(6, J) * (Y_(2, J - 1) * GGX[id(I, J, K)] + Y_(2, J) * GGX[id(I, J - 1, K)]);
            FG = Y_(6, J) * (Y_(2, J) * BR + Y_(2, J - 1) * BL);
            double ANR, ANL;
            if (NF[id(I, J, K)] == -1) ANR = ANU[id(I - 1, J, K)];
            else if (NF[id(I - 1, J, K)] == -1) ANR = ANU[id(I, J, K)];
            else ANR = X_(6, I) * (X_(2, I - 1) * ANU[id(I, J, K)] + X_(2, I) * ANU[id(I - 1, J, K)]);
            if (NF[id(I, J - 1, K)] == -1) ANL = ANU[id(I - 1, J - 1, K)];
            else if (NF[id(I - 1, J - 1, K)] == -1) ANL = ANU[id(I, J - 1, K)];
            else ANL = X_(6, I) * (X_(2, I - 1) * ANU[id(I, J - 1, K)] + X_(2, I) * ANU[id(I - 1, J - 1, K)]);
            double AN = Y_(6, J) * (Y_(2, J - 1) * ANR + Y_(2, J) * ANL);
            double D1 = (IT == 0) ? X_(4, I) * (VV[id(I, J, K)] - FG) * 2.0
                                  : X_(4, I - 1) * (FG - VV[id(I - 1, J, K)]) * 2.0;
            double D2 = Y_(5, J) * (UU[id(I, J, K)] - UU[id(I, J - 1, K)]);
            F = F + GG * AN * (D1 + D2);
          }
        }
    // (Gz*w)*v
    for (int K = 2; K <= NK; ++K)
      for (int J = LA; J <= LB; ++J)
        for (int I = 2; I <= NI - 1; ++I) {
          int IC = NF[id(I, J - 1, K - 1)] * NF[id(I, J, K - 1)] * NF[id(I, J - 1, K)] * NF[id(I, J, K)];
          int IT = INDY[id(I, J, K)], IBt = INDY[id(I, J, K - 1)];
          double &F = FLVW[id(I, J, K)];
          if (IC != 0 || (IT != 0 && IBt != 0)) {
          } else if (IT == 0 && IBt == 0) {
            double WIN = Y_(6, J) * (Y_(2, J - 1) * GLZ[id(I, J, K)] * WW[id(I, J, K)] +
                                     Y_(2, J) * GLZ[id(I, J - 1, K)] * WW[id(I, J - 1, K)]);
            double FG = WIN * Z_(6, K) * (Z_(2, K - 1) * VV[id(I, J, K)] + Z_(2, K) * VV[id(I, J, K - 1)]);
            F = F - SU * (dmax(WIN, 0.0) * VV[id(I, J, K - 1)] - dmax(-WIN, 0.0) * VV[id(I, J, K)]) - SC * FG;
            double GG = Y_(6, J) * (Y_(2, J - 1) * GGZ[id(I, J, K)] + Y_(2, J) * GGZ[id(I, J - 1, K)]);
            double ANR = Z_(6, K) * (Z_(2, K - 1) * ANU[id(I, J, K)] + Z_(2, K) * ANU[id(I, J, K - 1)]);
            double ANL = Z_(6, K) * (Z_(2, K - 1) * ANU[id(I, J - 1, K)] + Z_(2, K) * ANU[id(I, J - 1, K - 1)]);
            double AN = Y_(6, J) * (Y_(2, J - 1) * ANR + Y_(2, J) * ANL);
            double D1 = Z_(5, K) * (VV[id(I, J, K)] - VV[id(I, J, K - 1)]);
            double D2 = Y_(5, J) * (WW[id(I, J, K)] - WW[id(I, J - 1, K)]);
            F = F + GG * AN * (D1 + D2);
          } else {
            double BR, BL;
            int IS = INDZ[id(I, J, K)];
            if (IS >= 1) {
              if (IB_(3, IS) == 1 || IB_(3, IS) == 4) BR = (IB_(2, IS) == 5) ? VV[id(I, J, K)] : VV[id(I, J, K - 1)];
              else BR = BCV[IS - 1];
            } else {
              BR = Z_(6, K) * (Z_(2, K - 1) * (VV[id(I, J, K)] + VV[id(I, J + 1, K)]) +
                               Z_(2, K) * (VV[id(I, J, K - 1)] + VV[id(I, J + 1, K - 1)])) * 0.5;
            }
            IS = INDZ[id(I, J - 1, K)];
            if (IS >= 1) {
              if (IB_(3, IS) == 1 || IB_(3, IS) == 4) BL = (IB_(2, IS) == 5) ? VV[id(I, J, K)] : VV[id(I, J, K - 1)];
              else BL = BCV[IS - 1];
            } else {
              BL = Z_(6, K) * (Z_(2, K - 1) * (VV[id(I, J, K)] + VV[id(I, J - 1, K)]) +
                               Z_(2, K) * (VV[id(I, J, K - 1)] + VV[id(I, J - 1, K - 1)])) * 0.5;
            }
            double WIN = Y_(6, J) * (Y_(2, J - 1) * GLZ[id(I, J, K)] * WW[id(I, J, K)] +
                                     Y_(2, J) * GLZ[id(I, J - 1, K)] * WW[id(I, J - 1, K)]);
            double FG = Y_(6, J) * (Y_(2, J) * GLZ[id(I, J, K)] * WW[id(I, J, K)] * BR +
                                    Y_(2, J - 1) * GLZ[id(I, J - 1, K)] * WW[id(I, J - 1, K)] * BL);
            if (IT == 0 && WIN < 0.0) F = F - SU * WIN * VV[id(I, J, K)] - SC * FG;
            else if (IBt == 0 && WIN > 0.0) F = F - SU * WIN * VV[id(I, J, K - 1)] - SC * FG;
            else F = F - FG;
            double GG = Y_(6, J) * (Y_(2, J - 1) * GGZ[id(I, J, K)] + Y_(2, J) * GGZ[id(I, J - 1, K)]);
            FG = Y_(6, J) * (Y_(2, J) * BR + Y_(2, J - 1) * BL);
            double ANR, ANL;
            if (NF[id(I, J, K)] == -1) ANR = ANU[id(I, J, K - 1)];
            else if (NF[id(I, J, K - 1)] == -1) ANR = ANU[id(I, J, K)];
            else ANR = Z_(6, K) * (Z_(2, K - 1) * ANU[id(I, J, K)] + Z_(2, K) * ANU[id(I, J, K - 1)]);
            if (NF[id(I, J - 1, K)] == -1) ANL = ANU[id(I, J - 1, K - 1)];
            else if (NF[id(I, J - 1, K - 1)] == -1) ANL = ANU[id(I, J - 1, K)];
            else ANL = Z_(6, K) * (Z_(2, K - 1) * ANU[id(I, J - 1, K)] + Z_(2, K) * ANU[id(I, J - 1, K - 1)]);
            double AN = Y_(6, J) * (Y_(2, J - 1) * ANR + Y_(2, J) * ANL);
            double D1 = (IT == 0) ? Z_(4, K) * (VV[id(I, J, K)] - FG) * 2.0
                                  : Z_(4, K - 1) * (FG - VV[id(I, J, K - 1)]) * 2.0;
            double D2 = Y_(5, J) * (WW[id(I, J, K)] - WW[id(I, J - 1, K)]);
            F = F + GG * AN * (D1 + D2);
          }
        }
  }

  // VF_VFLXDW  vf_vflxdw.f:58-342
  void vflxdw(vd &FLWU, vd &FLWV, vd &FLWW) {
    const double SU = P.scmvp, SC = 1.0 - P.scmvp;
    for (int K = 2; K <= NK - 1; ++K)
      for (int J = 2; J <= NJ - 1; ++J)
        for (int I = 2; I <= NI - 1; ++I) {
          if (INDC[id(I, J, K)] == -1) continue;
          double WIN = (GLZ[id(I, J, K)] * WW[id(I, J, K)] + GLZ[id(I, J, K + 1)] * WW[id(I, J, K + 1)]) * 0.5;
          double FG = WIN * (WW[id(I, J, K)] + WW[id(I, J, K + 1)]) * 0.5;
          double &F = FLWW[id(I, J, K)];
          F = F - SU * (dmax(WIN, 0.0) * WW[id(I, J, K)] - dmax(-WIN, 0.0) * WW[id(I, J, K + 1)]) - SC * FG;
          F = F + (GGZ[id(I, J, K)] + GGZ[id(I, J, K + 1)]) * ANU[id(I, J, K)] * Z_(4, K) *
                      (WW[id(I, J, K + 1)] - WW[id(I, J, K)]);
        }
    // (Gx*u)*w
    for (int K = 3; K <= NK - 1; ++K)
      for (int J = 2; J <= NJ - 1; ++J)
        for (int I = 2; I <= NI; ++I) {
          int IC = NF[id(I - 1, J, K - 1)] * NF[id(I - 1, J, K)] * NF[id(I, J, K - 1)] * NF[id(I, J, K)];
          int IT = INDZ[id(I, J, K)], IBt = INDZ[id(I - 1, J, K)];
          double &F = FLWU[id(I, J, K)];
          if (IC != 0 || (IT != 0 && IBt != 0)) {
          } else if (IT == 0 && IBt == 0) {
            double WIN = Z_(6, K) * (Z_(2, K - 1) * GLX[id(I, J, K)] * UU[id(I, J, K)] +
                                     Z_(2, K) * GLX[id(I, J, K - 1)] * UU[id(I, J, K - 1)]);
            double FG = WIN * X_(6, I) * (X_(2, I - 1) * WW[id(I, J, K)] + X_(2, I) * WW[id(I - 1, J, K)]);
            F = F - SU * (dmax(WIN, 0.0) * WW[id(I - 1, J, K)] - dmax(-WIN, 0.0) * WW[id(I, J, K)]) - SC * FG;
            double GG = Z_(6, K) * (Z_(2, K - 1) * GGX[id(I, J, K)] + Z_(2, K) * GGX[id(I, J, K - 1)]);
            double ANR = X_(6, I) * (X_(2, I - 1) * ANU[id(I, J, K)] + X_(2, I) * ANU[id(I - 1, J, K)]);
            double ANL = X_(6, I) * (X_(2, I - 1) * ANU[id(I, J, K - 1)] + X_(2, I) * ANU[id(I - 1, J, K - 1)]);
            double AN = Z_(6, K) * (Z_(2, K - 1) * ANR + Z_(2, K) * ANL);
            double D1 = X_(5, I) * (WW[id(I, J, K)] - WW[id(I - 1, J, K)]);
            double D2 = Z_(5, K) * (UU[id(I, J, K)] - UU[id(I, J, K - 1)]);
            F = F + GG * AN * (D1 + D2);
          } else {
            double BR, BL;
            int IS = INDX[id(I, J, K)];
            if (IS >= 1) {
              if (IB_(3, IS) == 1 || IB_(3, IS) == 4) BR = (IB_(2, IS) == 1) ? WW[id(I, J, K)] : WW[id(I - 1, J, K)];
              else BR = BCW[IS - 1];
            } else {
              BR = X_(6, I) * (X_(2, I - 1) * (WW[id(I, J, K)] + WW[id(I, J, K + 1)]) +
                               X_(2, I) * (WW[id(I - 1, J, K)] + WW[id(I - 1, J, K + 1)])) * 0.5;
            }
            IS = INDX[id(I, J, K - 1)];
            if (IS >= 1) {
              if (IB_(3, IS) == 1 || IB_(3, IS) == 4) BL = (IB_(2, IS) == 1) ? WW[id(I, J, K)] : WW[id(I - 1, J, K)];
              else BL = BCW[IS - 1];
            } else {
              BL = X_(6, I) * (X_(2, I - 1) * (WW[id(I, J, K)] + WW[id(I, J, K - 1)]) +
                               X_(2, I) * (WW[id(I - 1, J, K)] + WW[id(I - 1, J, K - 1)])) * 0.5;
            }
            double WIN = Z_(6, K) * (Z_(2, K - 1) * GLX[id(I, J, K)] * UU[id(I, J, K)] +
                                     Z_(2, K) * GLX[id(I, J, K - 1)] * UU[id(I, J, K - 1)]);
            double FG = Z_(6, K) * (Z_(2, K) * GLX[id(I, J, K)] * UU[id(I, J, K)] * BR +
                                    Z_(2, K - 1) * GLX[id(I, J, K - 1)] * UU[id(I, J, K - 1)] * BL);
            if (IT == 0 && WIN < 0.0) F = F - SU * WIN * WW[id(I, J, K)] - SC * FG;
            else if (IBt == 0 && WIN > 0.0) F = F - SU * WIN * WW[id(I - 1, J, K)] - SC * FG;
            else F = F - FG;
            double GG = Z_(6, K) * (Z_(2, K - 1) * GGX[id(I, J, K)] + Z_(2, K) * GGX[id(I, J, K - 1)]);
            FG = Z_(6, K) * (Z_(2, K) * BR + Z_(2, K - 1) * BL);
            double ANR, ANL;
            if (NF[id(I, J, K)] == -1) ANR = ANU[id(I - 1, J, K)];
            else if (NF[id(I - 1, J, K)] == -1) ANR = ANU[id(I, J, K)];
            else ANR = X_(6, I) * (X_(2, I - 1) * ANU[id(I, J, K)] + X_(2, I) * ANU[id(I - 1, J, K)]);
            if (NF[id(I, J, K - 1)] == -1) ANL = ANU[id(I - 1, J, K - 1)];
            else if (NF[id(I - 1, J, K - 1)] == -1) ANL = ANU[id(I, J, K - 1)];
            else ANL = X_(6, I) * (X_(2, I - 1) * ANU[id(I, J, K - 1)] + X_(2, I) * ANU[id(I - 1, J, K - 1)]);
            double AN = Z_(6, K) * (Z_(2, K - 1) * ANR + Z_(2, K) * ANL);
            double D1 = (IT == 0) ? X_(4, I) * (WW[id(I, J, K)] - FG) * 2.0
                                  : X_(4, I - 1) * (FG - WW[id(I - 1, J, K)]) * 2.0;
            double D2 = Z_(5, K) * (UU[id(I, J, K)] - UU[id(I, J, K - 1)]);
            F = F + GG * AN * (D1 + D2);
          }
        }
    // (Gy*v)*w
    for (int K = 3; K <= NK - 1; ++K)
      for (int J = 2; J <= NJ; ++J)
        for (int I = 2; I <= NI - 1; ++I) {
          int IC = NF[id(I, J - 1, K - 1)] * NF[id(I, J - 1, K)] * NF[id(I, J, K - 1)] * NF[id(I, J, K)];
          int IT = INDZ[id(I, J, K)], IBt = INDZ[id(I, J - 1, K)];
          double &F = FLWV[id(I, J, K)];
          if (IC != 0 || (IT != 0 && IBt != 0)) {
          } else if (IT == 0 && IBt == 0) {
            double WIN = Z_(6, K) * (Z_(2, K - 1) * GLY[id(I, J, K)] * VV[id(I, J, K)] +
                                     Z_(2, K) * GLY[id(I, J, K - 1)] * VV[id(I, J, K - 1)]);
            double FG = WIN * Y_(6, J) * (Y_(2, J - 1) * WW[id(I, J, K)] + Y_(2, J) * WW[id(I, J - 1, K)]);
            F = F - SU * (dmax(WIN, 0.0) * WW[id(I, J - 1, K)] - dmax(-WIN, 0.0) * WW[id(I, J, K)]) - SC * FG;
            double GG = Z_(6, K) * (Z_(2, K - 1) * GGY[id(I, J, K)] + Z_(2, K) * GGY[id(I, J, K - 1)]);
            double ANR = Y_(6, J) * (Y_(2, J - 1) * ANU[id(I, J, K)] + Y_(2, J) * ANU[id(I, J - 1, K)]);
            double ANL = Y_(6, J) * (Y_(2, J - 1) * ANU[id(I, J, K - 1)] + Y_(2, J) * ANU[id(I, J - 1, K - 1)]);
            double AN = Z_(6, K) * (Z_(2, K - 1) * ANR + Z_(2, K) * ANL);
            double D1 = Y_(5, J) * (WW[id(I, J, K)] - WW[id(I, J - 1, K)]);
            double D2 = Z_(5, K) * (VV[id(I, J, K)] - VV[id(I, J, K - 1)]);
            F = F + GG * AN * (D1 + D2);
          } else {
            double BR, BL;
            int IS = INDY[id(I, J, K)];
            if (IS >= 1) {
              if (IB_(3, IS) == 1 || IB_(3, IS) == 4) BR = (IB_(2, IS) == 3) ? WW[id(I, J, K)] : WW[id(I, J - 1, K)];
              else BR = BCW[IS - 1];
            } else {
              BR = Y_(6, J) * (Y_(2, J - 1) * (WW[id(I, J, K)] + WW[id(I, J, K + 1)]) +
                               Y_(2, J) * (WW[id(I, J - 1, K)] + WW[id(I, J - 1, K + 1)])) * 0.5;
            }
            IS = INDY[id(I, J, K - 1)];
            if (IS >= 1) {
              if (IB_(3, IS) == 1 || IB_(3, IS) == 4) BL = (IB_(2, IS) == 3) ? WW[id(I, J, K)] : WW[id(I, J - 1, K)];
              else BL = BCW[IS - 1];
            } else {
              BL = Y_(6, J) * (Y_(2, J - 1) * (WW[id(I, J, K)] + WW[id(I, J, K - 1)]) +
                               Y_(2, J) * (WW[id(I, J - 1, K)] + WW[id(I, J - 1, K - 1)])) * 0.5;
            }
            double WIN = Z_(6, K) * (Z_(2, K - 1) * GLY[id(I, J, K)] * VV[id(I, J, K)] +
                                     Z_(2, K) * GLY[id(I, J, K - 1)] * VV[id(I, J, K - 1)]);
            double FG = Z_(6, K) * (Z_(2, K) * GLY[id(I, J, K)] * VV[id(I, J, K)] * BR +
                                    Z_(2, K - 1) * GLY[id(I, J, K - 1)] * VV[id(I, J, K - 1)] * BL);
            if (IT == 0 && WIN < 0.0) F = F - SU * WIN * WW[id(I, J, K)] - SC * FG;
            else if (IBt == 0 && WIN > 0.0) F = F - SU * WIN * WW[id(I, J - 1, K)] - SC * FG;
            else F = F - FG;
            double GG = Z_(6, K) * (Z_(2, K - 1) * GGY[id(I, J, K)] + Z_(2, K) * GGY[id(I, J, K - 1)]);
            FG = Z_(6, K) * (Z_(2, K) * BR + Z_(2, K - 1) * BL);
            double ANR, ANL;
            if (NF[id(I, J, K)] == -1) ANR = ANU[id(I, J - 1, K)];
            else if (NF[id(I, J - 1, K)] == -1) ANR = ANU[id(I, J, K)];
            else ANR = Y_(6, J) * (Y_(2, J - 1) * ANU[id(I, J, K)] + Y_(2, J) * ANU[id(I, J - 1, K)]);
            if (NF[id(I, J, K - 1)] == -1) ANL = ANU[id(I, J - 1, K - 1)];
            else if (NF[id(I, J - 1, K - 1)] == -1) ANL = ANU[id(I, J, K - 1)];
            else ANL = Y_(6, J) * (Y_(2, J - 1) * ANU[id(I, J, K - 1)] + Y_(2, J) * ANU[id(I, J - 1, K - 1)]);
            double AN = Z_(6, K) * (Z_(2, K - 1) * ANR + Z_(2, K) * ANL);
            double D1 = (IT == 0) ? Y_(4, J) * (WW[id(I, J, K)] - FG) * 2.0
                                  : Y_(4, J - 1) * (FG - WW[id(I, J - 1, K)]) * 2.0;
            double D2 = Z_(5, K) * (VV[id(I, J, K)] - VV[id(I, J, K - 1)]);
            F = F + GG * AN * (D1 + D2);
          }
        }
  }

  // VF_VGENE  vf_vgene.f:84-332 (IDRGN<=0 drag, wave source, no T/C)
  void vgene(vd &QU, vd &QV, vd &QW) {
    const double RI = 1.0 / P.rho0;
    for (int K = 2; K <= NK - 1; ++K)
      for (int J = 2; J <= NJ - 1; ++J)
        for (int I = 3; I <= NI - 1; ++I) {
          int I1 = I - 1;
          if (!(INDX[id(I, J, K)] == 0 && NF[id(I1, J, K)] * NF[id(I, J, K)] == 0)) continue;
          double GV = X_(6, I) * (X_(2, I) * GGV[id(I, J, K)] + X_(2, I1) * GGV[id(I1, J, K)]);
          double CD = X_(6, I) * (X_(2, I) * CD0[id(I, J, K)] + X_(2, I1) * CD0[id(I1, J, K)]);
          double &Q = QU[id(I, J, K)];
          Q = Q + GV * RI * X_(5, I) * (PP[id(I1, J, K)] - PP[id(I, J, K)]);
          double U = UU[id(I, J, K)];
          double V = X_(6, I) * (X_(2, I1) * (VV[id(I, J, K)] + VV[id(I, J + 1, K)]) +
                                 X_(2, I) * (VV[id(I1, J, K)] + VV[id(I1, J + 1, K)])) * 0.5;
          double W = X_(6, I) * (X_(2, I1) * (WW[id(I, J, K)] + WW[id(I, J, K + 1)]) +
                                 X_(2, I) * (WW[id(I1, J, K)] + WW[id(I1, J, K + 1)])) * 0.5;
          double UVW = std::sqrt(U * U + V * V + W * W);
          Q = Q - 0.5 * CD * X_(5, I) * (1.0 - GGX[id(I, J, K)]) * U * UVW;
          // wave source  vf_vgene.f:149-152
          const int IWS_ = IWS();
          if (IWS_ != 0 && (IWS_ == I || IWS_ + 1 == I)) {
            double QS = 2.0 * X_(4, IWS_) * SRC(J, K);
            Q = Q + UU[id(I, J, K)] * QS * X_(2, IWS_) * X_(5, I) * 0.5;
          }
        }
    for (int K = 2; K <= NK - 1; ++K)
      for (int J = 3; J <= NJ - 1; ++J)
        for (int I = 2; I <= NI - 1; ++I) {
          int J1 = J - 1;
          if (!(INDY[id(I, J, K)] == 0 && NF[id(I, J1, K)] * NF[id(I, J, K)] == 0)) continue;
          double GV = Y_(6, J) * (Y_(2, J) * GGV[id(I, J, K)] + Y_(2, J1) * GGV[id(I, J1, K)]);
          double CD = Y_(6, J) * (Y_(2, J) * CD0[id(I, J, K)] + Y_(2, J1) * CD0[id(I, J1, K)]);
          double &Q = QV[id(I, J, K)];
          Q = Q + GV * RI * Y_(5, J) * (PP[id(I, J1, K)] - PP[id(I, J, K)]);
          double U = Y_(6, J) * (Y_(2, J1) * (UU[id(I, J, K)] + UU[id(I + 1, J, K)]) +
                                 Y_(2, J) * (UU[id(I, J1, K)] + UU[id(I + 1, J1, K)])) * 0.5;
          double V = VV[id(I, J, K)];
          double W = Y_(6, J) * (Y_(2, J1) * (WW[id(I, J, K)] + WW[id(I, J, K + 1)]) +
                                 Y_(2, J) * (WW[id(I, J1, K)] + WW[id(I, J1, K + 1)])) * 0.5;
          double UVW = std::sqrt(U * U + V * V + W * W);
          Q = Q - 0.5 * CD * Y_(5, J) * (1.0 - GGY[id(I, J, K)]) * V * UVW;
          // wave source  vf_vgene.f:225-228
          const int JWS_ = JWS();
          if (JWS_ != 0 && (JWS_ == J || JWS_ + 1 == J)) {
            double QS = 2.0 * Y_(4, JWS_) * SRC(I, K);
            Q = Q + VV[id(I, J, K)] * QS * Y_(2, JWS_) * Y_(5, J) * 0.5;
          }
        }
    for (int K = 3; K <= NK - 1; ++K) {
      int K1 = K - 1;
      for (int J = 2; J <= NJ - 1; ++J)
        for (int I = 2; I <= NI - 1; ++I) {
          if (!(INDZ[id(I, J, K)] == 0 && NF[id(I, J, K1)] * NF[id(I, J, K)] == 0)) continue;
          double GV = Z_(6, K) * (Z_(2, K) * GGV[id(I, J, K)] + Z_(2, K1) * GGV[id(I, J, K1)]);
          double CD = Z_(6, K) * (Z_(2, K) * CD0[id(I, J, K)] + Z_(2, K1) * CD0[id(I, J, K1)]);
          double &Q = QW[id(I, J, K)];
          Q = Q + GV * RI * Z_(5, K) * (PP[id(I, J, K1)] - PP[id(I, J, K)]);
          double U = Z_(6, K) * (Z_(2, K1) * (UU[id(I, J, K)] + UU[id(I + 1, J, K)]) +
                                 Z_(2, K) * (UU[id(I, J, K1)] + UU[id(I + 1, J, K1)])) * 0.5;
          double V = Z_(6, K) * (Z_(2, K1) * (VV[id(I, J, K)] + VV[id(I, J + 1, K)]) +
                                 Z_(2, K) * (VV[id(I, J, K1)] + VV[id(I, J + 1, K1)])) * 0.5;
          double W = WW[id(I, J, K)];
          double UVW = std::sqrt(U * U + V * V + W * W);
          Q = Q - 0.5 * CD * Z_(5, K) * (1.0 - GGZ[id(I, J, K)]) * W * UVW;
          Q = Q - GV * P.grz0;
          // wave source  vf_vgene.f:304-315
          if (IWS() == I) {
            double Q1 = 2.0 * X_(4, I) * SRC(J, K - 1);
            double Q2 = 2.0 * X_(4, I) * SRC(J, K);
            Q = Q + Z_(5, K) * (Q2 - Q1) * P.anu0 / 3.0;
            Q = Q + WW[id(I, J, K)] * (Q1 + Q2) * 0.5;
          }
          if (JWS() == J) {
            double Q1 = 2.0 * Y_(4, J) * SRC(I, K - 1);
            double Q2 = 2.0 * Y_(4, J) * SRC(I, K);
            Q = Q + Z_(5, K) * (Q2 - Q1) * P.anu0 / 3.0;
            Q = Q + WW[id(I, J, K)] * (Q1 + Q2) * 0.5;
          }
          double DR = 0.0;  // no temperature / concentration (vf_vgene.f:318-327)
          Q = Q - GV * P.grz0 * DR / P.rho0;
        }
    }
  }

  // Sponge of VF_VEULER (vf_veuler.f:77-113 parameters, :131-166 profile)
  struct Sponge {
    int IPA = 0, IP[4];
    double W[4], PX[4], PZ[4];
  };
  Sponge sponge() const {
    Sponge s;
    for (int d = 0; d < 4; ++d) {
      s.IP[d] = P.idamp[d];
      s.W[d] = s.PX[d] = s.PZ[d] = 0.0;
      if (s.IP[d] >= 0) {
        s.IPA = s.IPA + 1;
        double D = std::sqrt(P.grz0 / P.damp[d][3]);
        s.W[d] = P.damp[d][2];
        s.PX[d] = (double)(s.IP[d] + 1) * P.damp[d][0] * D;
        s.PZ[d] = (double)(s.IP[d] + 1) * P.damp[d][1] * D;
      }
    }
    return s;
  }
  double sponge_dmax(const Sponge &s, double X, double Y, bool z) const {
    double DMAX = 0.0, D;
    const double *PP_ = z ? s.PZ : s.PX;
    if (s.IP[0] >= 0) { D = X - P.glxmin; if (D <= s.W[0]) { D = PP_[0] * ipow(1.0 - D / s.W[0], s.IP[0]); if (D > DMAX) DMAX = D; } }
    if (s.IP[1] >= 0) { D = P.glxmax - X; if (D <= s.W[1]) { D = PP_[1] * ipow(1.0 - D / s.W[1], s.IP[1]); if (D > DMAX) DMAX = D; } }
    if (s.IP[2] >= 0) { D = Y - P.glymin; if (D <= s.W[2]) { D = PP_[2] * ipow(1.0 - D / s.W[2], s.IP[2]); if (D > DMAX) DMAX = D; } }
    if (s.IP[3] >= 0) { D = P.glymax - Y; if (D <= s.W[3]) { D = PP_[3] * ipow(1.0 - D / s.W[3], s.IP[3]); if (D > DMAX) DMAX = D; } }
    return DMAX;
  }

  // VF_VEULER  vf_veuler.f:115-284  (GLV0 = GLV, GGV0 = GGV for IPRNT<=1)
  void veuler(const vd &FLUU, const vd &FLUV, const vd &FLUW, const vd &QU,
              const vd &FLVU, const vd &FLVV, const vd &FLVW, const vd &QV,
              const vd &FLWU, const vd &FLWV, const vd &FLWW, const vd &QW) {
    Sponge s = sponge();
    const double DT = DTNOW, VM = P.vvmax;
    for (int K = 2; K <= NK - 1; ++K)
      for (int J = 2; J <= NJ - 1; ++J)
        for (int I = 3; I <= NI - 1; ++I) {
          if (!(INDX[id(I, J, K)] == 0 && NF[id(I - 1, J, K)] * NF[id(I, J, K)] == 0)) continue;
          double GV = X_(6, I) * (X_(2, I) * GLV[id(I, J, K)] + X_(2, I - 1) * GLV[id(I - 1, J, K)]);
          double GV0 = X_(6, I) * (X_(2, I) * GLV[id(I, J, K)] + X_(2, I - 1) * GLV[id(I - 1, J, K)]);
          double DU = (X_(5, I) * (FLUU[id(I, J, K)] - FLUU[id(I - 1, J, K)]) +
                       Y_(4, J) * (FLUV[id(I, J + 1, K)] - FLUV[id(I, J, K)]) +
                       Z_(4, K) * (FLUW[id(I, J, K + 1)] - FLUW[id(I, J, K)]) + QU[id(I, J, K)]);
          double &U = UU[id(I, J, K)];
          U = (GV * U + DT * DU) / GV0;
          if (U > VM) U = VM;
          if (U < -VM) U = -VM;
          if (s.IPA != 0) {
            double X = X_(1, I), Y = (Y_(1, J) + Y_(1, J + 1)) * 0.5;
            double DMAX = sponge_dmax(s, X, Y, false);
            double G = X_(6, I) * (X_(2, I) * GGV[id(I, J, K)] + X_(2, I - 1) * GGV[id(I - 1, J, K)]);
            double D = GV0 / (GV0 + DT * G * DMAX);
            U = U * D;
          }
        }
    for (int K = 2; K <= NK - 1; ++K)
      for (int J = 3; J <= NJ - 1; ++J)
        for (int I = 2; I <= NI - 1; ++I) {
          if (!(INDY[id(I, J, K)] == 0 && NF[id(I, J - 1, K)] * NF[id(I, J, K)] == 0)) continue;
          double GV = Y_(6, J) * (Y_(2, J) * GLV[id(I, J, K)] + Y_(2, J - 1) * GLV[id(I, J - 1, K)]);
          double GV0 = Y_(6, J) * (Y_(2, J) * GLV[id(I, J, K)] + Y_(2, J - 1) * GLV[id(I, J - 1, K)]);
          double DV = (X_(4, I) * (FLVU[id(I + 1, J, K)] - FLVU[id(I, J, K)]) +
                       Y_(5, J) * (FLVV[id(I, J, K)] - FLVV[id(I, J - 1, K)]) +
                       Z_(4, K) * (FLVW[id(I, J, K + 1)] - FLVW[id(I, J, K)]) + QV[id(I, J, K)]);
          double &V = VV[id(I, J, K)];
          V = (GV * V + DT * DV) / GV0;
          if (V > VM) V = VM;
          if (V < -VM) V = -VM;
          if (s.IPA != 0) {
            double X = (X_(1, I) + X_(1, I + 1)) * 0.5, Y = Y_(1, J);
            double DMAX = sponge_dmax(s, X, Y, false);
            double G = Y_(6, J) * (Y_(2, J) * GGV[id(I, J, K)] + Y_(2, J - 1) * GGV[id(I, J - 1, K)]);
            double D = GV0 / (GV0 + DT * G * DMAX);
            V = V * D;
          }
        }
    for (int K = 3; K <= NK - 1; ++K)
      for (int J = 2; J <= NJ - 1; ++J)
        for (int I = 2; I <= NI - 1; ++I) {
          if (!(INDZ[id(I, J, K)] == 0 && NF[id(I, J, K - 1)] * NF[id(I, J, K)] == 0)) continue;
          double GV = Z_(6, K) * (Z_(2, K) * GLV[id(I, J, K)] + Z_(2, K - 1) * GLV[id(I, J, K - 1)]);
          double GV0 = Z_(6, K) * (Z_(2, K) * GLV[id(I, J, K)] + Z_(2, K - 1) * GLV[id(I, J, K - 1)]);
          double DW = (X_(4, I) * (FLWU[id(I + 1, J, K)] - FLWU[id(I, J, K)]) +
                       Y_(4, J) * (FLWV[id(I, J + 1, K)] - FLWV[id(I, J, K)]) +
                       Z_(5, K) * (FLWW[id(I, J, K)] - FLWW[id(I, J, K - 1)]) + QW[id(I, J, K)]);
          double &W = WW[id(I, J, K)];
          W = (GV * W + DT * DW) / GV0;
          if (W > VM) W = VM;
          if (W < -VM) W = -VM;
          if (s.IPA != 0) {
            double X = (X_(1, I) + X_(1, I + 1)) * 0.5, Y = (Y_(1, J) + Y_(1, J + 1)) * 0.5;
            double DMAX = sponge_dmax(s, X, Y, true);
            double G = Z_(6, K) * (Z_(2, K) * GGV[id(I, J, K)] + Z_(2, K - 1) * GGV[id(I, J, K - 1)]);
            double D = GV0 / (GV0 + DT * G * DMAX);
            W = W * D;
          }
        }
  }

  // VF_BWUWN  vf_bwuwn.f:93-160 (slip, no-slip, fixed, free); wave and
  // open faces (IB=5,7) by side afterwards (bwuwn_wave, bwuwn_open).
  // UB, VB, WB are the velocities of the step's start.
  int bwuwn(const vd &UB, const vd &VB, const vd &WB) {
    for (int L = 1; L <= NB; ++L) {
      int I, J, K;
      decode(IB_(1, L), I, J, K);
      int NS = IB_(2, L), IB = IB_(3, L);
      if (IB == 1 || IB == 6 || IB == 8) {
        if (NS == 1 || NS == 2) { BCU[L - 1] = 0.0; UU[id(I, J, K)] = 0.0; }
        else if (NS == 3 || NS == 4) { BCV[L - 1] = 0.0; VV[id(I, J, K)] = 0.0; }
        else { BCW[L - 1] = 0.0; WW[id(I, J, K)] = 0.0; }
      } else if (IB == 2) {
        BCU[L - 1] = 0.0; BCV[L - 1] = 0.0; BCW[L - 1] = 0.0;
        if (NS == 1 || NS == 2) UU[id(I, J, K)] = BCU[L - 1];
        else if (NS == 3 || NS == 4) VV[id(I, J, K)] = BCV[L - 1];
        else WW[id(I, J, K)] = BCW[L - 1];
      } else if (IB == 3) {
        if (NS == 1 || NS == 2) UU[id(I, J, K)] = BCU[L - 1];
        else if (NS == 3 || NS == 4) VV[id(I, J, K)] = BCV[L - 1];
        else WW[id(I, J, K)] = BCW[L - 1];
      } else if (IB == 4) {
        double VAL;
        if (NS == 1) { VAL = UU[id(I + 1, J, K)]; BCU[L - 1] = VAL; UU[id(I, J, K)] = VAL; }
        else if (NS == 2) { VAL = UU[id(I - 1, J, K)]; BCU[L - 1] = VAL; UU[id(I, J, K)] = VAL; }
        else if (NS == 3) { VAL = VV[id(I, J + 1, K)]; BCV[L - 1] = VAL; VV[id(I, J, K)] = VAL; }
        else if (NS == 4) { VAL = VV[id(I, J - 1, K)]; BCV[L - 1] = VAL; VV[id(I, J, K)] = VAL; }
        else if (NS == 5) { VAL = WW[id(I, J, K + 1)]; BCW[L - 1] = VAL; WW[id(I, J, K)] = VAL; }
        else if (NS == 6) { VAL = WW[id(I, J, K - 1)]; BCW[L - 1] = VAL; WW[id(I, J, K)] = VAL; }
      } else if (IB == 5) {  // vf_bwuwn.f:161-216 (fixed water level only)
        if (fixlvl_face(NS, I, J)) {
          double VAL;
          if (NS == 1) { VAL = UU[id(I + 1, J, K)]; BCU[L - 1] = VAL; UU[id(I, J, K)] = VAL; }
          else if (NS == 2) { VAL = UU[id(I - 1, J, K)]; BCU[L - 1] = VAL; UU[id(I, J, K)] = VAL; }
          else if (NS == 3) { VAL = VV[id(I, J + 1, K)]; BCV[L - 1] = VAL; VV[id(I, J, K)] = VAL; }
          else { VAL = VV[id(I, J - 1, K)]; BCV[L - 1] = VAL; VV[id(I, J, K)] = VAL; }
        } else if (NS > 4) {
          return CADMAS_EPG;
        }
      } else if (IB == 7) {
        // vf_bwuwn.f:234-235: set below by side
      } else {
        return CADMAS_EPG;
      }
    }
    int rc = bwuwn_wave();
    if (rc) return rc;
    return bwuwn_open(UB, VB, WB);
  }

  // VF_BWUWN open-boundary part  vf_bwuwn.f:481-598 (IBCTYP(1,JD) = 2,
  // one rank: IP = JP = 0 and the rank's range is the whole side)
  int bwuwn_open(const vd &UB, const vd &VB, const vd &WB) {
    bool any = false;
    for (int JD = 1; JD <= 4; ++JD) {
      if (!OP[JD - 1].on) continue;
      any = true;
      const double C = OP[JD - 1].c;
      if (JD == 1 || JD == 2) {
        int I, IC, I2;
        if (JD == 1) { I = 2; IC = 2; I2 = 3; }
        else { I = NI; IC = NI - 1; I2 = IC; }
        double ALN, ALT;
        if (NNOW == 0) { ALN = 1.0; ALT = 1.0; }
        else { ALN = std::min(C * DTNOW / X_(2, IC), 1.0); ALT = std::min(ALN * 2.0, 1.0); }
        for (int K = 2; K <= NK - 1; ++K)
          for (int J = 2; J <= NJ - 1; ++J) {
            const int L = INDX[id(I, J, K)];
            if (L < 1) continue;
            if (NF[id(IC, J, K)] == 0) {
              const double VC = (VB[id(IC, J, K)] + VB[id(IC, J + 1, K)]) * 0.5;
              const double WC = (WB[id(IC, J, K)] + WB[id(IC, J, K + 1)]) * 0.5;
              BCU[L - 1] = (1.0 - ALN) * BCU[L - 1] + ALN * UB[id(I2, J, K)];
              BCV[L - 1] = (1.0 - ALT) * BCV[L - 1] + ALT * VC;
              BCW[L - 1] = (1.0 - ALT) * BCW[L - 1] + ALT * WC;
              UU[id(I, J, K)] = BCU[L - 1];
            } else {
              BCU[L - 1] = 0.0; BCV[L - 1] = 0.0; BCW[L - 1] = 0.0;
              UU[id(I, J, K)] = 0.0;
            }
          }
        for (int K = 2; K <= NK - 1; ++K)
          for (int J = 2; J <= NJ - 1; ++J) {
            const int L = INDX[id(I, J, K)];
            if (L < 1) continue;
            const int NW = NF[id(IC, J, K)];
            if (NW == 5) {
              const int L2 = INDX[id(I, J, K - 1)];
              if (L2 < 1) return CADMAS_EPG;
              BCU[L - 1] = BCU[L2 - 1]; BCV[L - 1] = BCV[L2 - 1]; BCW[L - 1] = BCW[L2 - 1];
              UU[id(I, J, K)] = BCU[L - 1];
            } else if (NW == 6) {
              const int L2 = INDX[id(I, J, K + 1)];
              if (L2 < 1) return CADMAS_EPG;
              BCU[L - 1] = BCU[L2 - 1]; BCV[L - 1] = BCV[L2 - 1]; BCW[L - 1] = BCW[L2 - 1];
              UU[id(I, J, K)] = 0.0;
            }
          }
      } else {
        int J, JC, J2;
        if (JD == 3) { J = 2; JC = 2; J2 = 3; }
        else { J = NJ; JC = NJ - 1; J2 = JC; }
        double ALN, ALT;
        if (NNOW == 0) { ALN = 1.0; ALT = 1.0; }
        else { ALN = std::min(C * DTNOW / Y_(2, JC), 1.0); ALT = std::min(ALN * 2.0, 1.0); }
        for (int K = 2; K <= NK - 1; ++K)
          for (int I = 2; I <= NI - 1; ++I) {
            const int L = INDY[id(I, J, K)];
            if (L < 1) continue;
            if (NF[id(I, JC, K)] == 0) {
              const double UC = (UB[id(I, JC, K)] + UB[id(I + 1, JC, K)]) * 0.5;
              const double WC = (WB[id(I, JC, K)] + WB[id(I, JC, K + 1)]) * 0.5;
              BCU[L - 1] = (1.0 - ALT) * BCU[L - 1] + ALT * UC;
              BCV[L - 1] = (1.0 - ALN) * BCV[L - 1] + ALN * VB[id(I, J2, K)];
              BCW[L - 1] = (1.0 - ALT) * BCW[L - 1] + ALT * WC;
              VV[id(I, J, K)] = BCV[L - 1];
            } else {
              BCU[L - 1] = 0.0; BCV[L - 1] = 0.0; BCW[L - 1] = 0.0;
              VV[id(I, J, K)] = 0.0;
            }
          }
        for (int K = 2; K <= NK - 1; ++K)
          for (int I = 2; I <= NI - 1; ++I) {
            const int L = INDY[id(I, J, K)];
            if (L < 1) continue;
            const int NW = NF[id(I, JC, K)];
            if (NW == 5 || NW == 6) {
              const int L2 = INDY[id(I, J, NW == 5 ? K - 1 : K + 1)];
              if (L2 < 1) return CADMAS_EPG;
              BCU[L - 1] = BCU[L2 - 1]; BCV[L - 1] = BCV[L2 - 1]; BCW[L - 1] = BCW[L2 - 1];
              VV[id(I, J, K)] = BCV[L - 1];
            }
          }
      }
    }
    if (!any)
      for (int L = 1; L <= NB; ++L)
        if (IB_(3, L) == 7) return CADMAS_EINVAL;  // open faces on no open side
    return CADMAS_OK;
  }

  // VF_CWMTB1  vf_cwmtb1.f:26-69
  bool cwmtb1(double WVT, double &W1, double &W2, double &WVZ) {
    const int MTBTT = (int)DMTBTT.size();
    auto TT = [&](int i) { return DMTBTT[i - 1]; };
    if (MTBNOW <= 0) MTBNOW = MTBTT - 1;
    if (WVT <= TT(1)) {
      MTBNOW = 1; W1 = 1.0; W2 = 0.0;
    } else if (WVT >= TT(MTBTT)) {
      MTBNOW = MTBTT - 1; W1 = 0.0; W2 = 1.0;
    } else {
      int IP = 0;
      W1 = W2 = 0.0;
      for (int I = MTBNOW; I >= 1 && IP == 0; --I) {
        if (TT(I) <= WVT && WVT <= TT(I + 1)) {
          IP = I;
          W2 = 1.0 / (TT(I + 1) - TT(I));
          W1 = (TT(I + 1) - WVT) * W2;
          W2 = (WVT - TT(I)) * W2;
        }
      }
      for (int I = MTBTT - 1; I >= MTBNOW + 1 && IP == 0; --I) {
        if (TT(I) <= WVT && WVT <= TT(I + 1)) {
          IP = I;
          W2 = 1.0 / (TT(I + 1) - TT(I));
          W1 = (TT(I + 1) - WVT) * W2;
          W2 = (WVT - TT(I)) * W2;
        }
      }
      if (IP == 0) return false;
      MTBNOW = IP;
    }
    WVZ = (MTBTYP != 2) ? W1 * DMTBHH[MTBNOW - 1] + W2 * DMTBHH[MTBNOW] : 0.0;
    return true;
  }

  // VF_CWMTB2  vf_cwmtb2.f:26-66
  bool cwmtb2(int &KM, double WT1, double WT2, double ZC, double &UN, double &UT) const {
    const int MTBZZ = (int)DMTBZZ.size();
    auto ZT = [&](int k) { return DMTBZZ[k - 1]; };
    auto TUN = [&](int k, int i) { return DMTBUN[(k - 1) + (size_t)MTBZZ * (i - 1)]; };
    auto TUT = [&](int k, int i) { return DMTBUT[(k - 1) + (size_t)MTBZZ * (i - 1)]; };
    double W1, W2;
    if (ZC <= ZT(1)) {
      KM = 1; W1 = 1.0; W2 = 0.0;
    } else if (ZC >= ZT(MTBZZ)) {
      KM = MTBZZ - 1; W1 = 0.0; W2 = 1.0;
    } else {
      int KP = 0;
      W1 = W2 = 0.0;
      for (int K = KM; K <= MTBZZ - 1 && KP == 0; ++K) {
        if (ZT(K) <= ZC && ZC <= ZT(K + 1)) {
          KP = K;
          W2 = 1.0 / (ZT(K + 1) - ZT(K));
          W1 = (ZT(K + 1) - ZC) * W2;
          W2 = (ZC - ZT(K)) * W2;
        }
      }
      if (KP == 0) return false;
      KM = KP;
    }
    const int KM1 = KM + 1, IM = MTBNOW, IM1 = MTBNOW + 1;
    double P1 = W1 * TUN(KM, IM) + W2 * TUN(KM1, IM);
    double P2 = W1 * TUN(KM, IM1) + W2 * TUN(KM1, IM1);
    UN = WT1 * P1 + WT2 * P2;
    P1 = W1 * TUT(KM, IM) + W2 * TUT(KM1, IM);
    P2 = W1 * TUT(KM, IM1) + W2 * TUT(KM1, IM1);
    UT = WT1 * P1 + WT2 * P2;
    return true;
  }

  // VF_BWFFSF  vf_bwffsf.f:43-128: F of the column next to each side whose
  // table fixes the water level (MTBTYP 3) from WVLVL + the table's level
  int bwffsf() {
    if (MTBTYP != 3) return CADMAS_OK;
    const double PI = 3.141592653589794, ZERO = 1.0e-20;
    for (int JD = 1; JD <= 4; ++JD) {
      const Wave &w = WV[JD - 1];
      if (!w.on || w.theory) continue;
      const double T = w.t, T0 = DMTBT0;
      double A = w.a;
      float R4TN = (float)(T0 - TNOW / T);
      R4TN = R4TN - (float)(int)R4TN;
      if (R4TN < 0.0f) R4TN = R4TN + 1.0f;
      double AW = 1.0;
      if (A >= ZERO) {
        A = TNOW / T / A;
        if (A < 1.0) AW = 0.5 * std::sin(PI * (A - 0.5)) + 0.5;
      }
      double WMT1, WMT2, WVZ;
      if (!cwmtb1((double)R4TN, WMT1, WMT2, WVZ)) return CADMAS_EPG;
      const double WL = P.wvlvl + WVZ * AW;
      for (int K = 2; K <= NK - 1; ++K) {
        double VAL;
        if (Z_(1, K) > WL) VAL = 0.0;
        else if (Z_(1, K + 1) < WL) VAL = 1.0;
        else VAL = (WL - Z_(1, K)) / (Z_(1, K + 1) - Z_(1, K));
        for (int n = w.l1; n <= w.l2; ++n) {
          const size_t c = (JD <= 2) ? id(JD == 1 ? 2 : NI - 1, n, K) : id(n, JD == 3 ? 2 : NJ - 1, K);
          if (NF[c] != -1) FF[c] = VAL;
        }
      }
    }
    return CADMAS_OK;
  }

  // ---- the stream-function wave (FUNC STREAM N) at a phase: VF_CWMAK1's
  // level and VF_CWMAK2's velocities, evaluated from the coefficients of
  // the wave (the series of psi = -UB (z+d) + sum B_j sinh(jk(z+d)) /
  // cosh(jkd) cos(jkX), the moving frame; fixed-frame velocities c - UB +
  // ...).  exp by the reduction x = n ln2 + r and r's Taylor series to
  // r^14, 2^n applied by ldexp; cosh, sinh from it; the level by Newton's
  // method on psi = -Q from 0; results rounded to single precision.
  static double sw_exp(double x) {
    const double L2H = 0.6931471803691238, L2T = 1.9082149292705877e-10, IL2 = 1.4426950408889634;
    const double n = std::floor(x * IL2 + 0.5);
    const double r = (x - n * L2H) - n * L2T;
    const double inv_fact[15] = {1.0, 1.0, 0.5, 1.0 / 6.0, 1.0 / 24.0, 1.0 / 120.0, 1.0 / 720.0, 1.0 / 5040.0,
                                 1.0 / 40320.0, 1.0 / 362880.0, 1.0 / 3628800.0, 1.0 / 39916800.0,
                                 1.0 / 479001600.0, 1.0 / 6227020800.0, 1.0 / 87178291200.0};
    double p = inv_fact[14];
    for (int i = 13; i >= 0; --i) p = p * r + inv_fact[i];
    return std::ldexp(p, (int)n);
  }
  static void sw_chsh(double x, double &ch, double &sh) {
    const double e = sw_exp(x), ei = 1.0 / e;
    ch = 0.5 * (e + ei);
    sh = 0.5 * (e - ei);
  }
  static double sw_level(const cadmas_stream_wave &s, double wvt) {
    const double th = 2.0 * 3.141592653589793 * wvt, d = s.depth, k = s.k;
    double e = 0.0;
    for (int it = 0; it < 60; ++it) {
      double f = -s.ubar * (e + d) + s.q, df = -s.ubar;
      for (int j = 1; j <= s.order; ++j) {
        double chd, shd, ch, sh;
        sw_chsh((double)j * k * d, chd, shd);
        sw_chsh((double)j * k * (e + d), ch, sh);
        const double cs = std::cos((double)j * th);
        f = f + s.b[j - 1] * sh / chd * cs;
        df = df + (double)j * k * s.b[j - 1] * ch / chd * cs;
      }
      const double de = f / df;
      e = e - de;
      if (std::fabs(de) < 1e-14 * d) break;
    }
    return (double)(float)e;
  }
  static void sw_velocity(const cadmas_stream_wave &s, double wvt, double z, double &u, double &w) {
    const double th = 2.0 * 3.141592653589793 * wvt;
    double zd = (double)(float)z + s.depth;  // REAL(ZC) (vf_cwmak2.f)
    if (zd < 0.0) zd = 0.0;
    double su = s.celerity - s.ubar, sv = 0.0;
    for (int j = 1; j <= s.order; ++j) {
      double chd, shd, ch, sh;
      sw_chsh((double)j * s.k * s.depth, chd, shd);
      const double a = (double)j * s.k * s.b[j - 1] / chd;
      const double cj = a * std::cos((double)j * th), sj = a * std::sin((double)j * th);
      sw_chsh((double)j * s.k * zd, ch, sh);
      su = su + cj * ch;
      sv = sv + sj * sh;
    }
    u = (double)(float)su;
    w = (double)(float)sv;
  }

  // ---- Stokes (fifth order, VF_STK1/2 of vf_wstk0.f) and cnoidal (third
  // order, VF_CND1/2 of vf_wcnd0.f) at a phase from their coefficients, in
  // the routines' centimetres: the level sum a_i cos(i theta) or the
  // polynomial in cn^2; the velocities b0 + sum b_i cosh(i k (z+d))
  // cos(i theta), sum b_i sinh(...) sin(i theta), or the polynomials in
  // cn^2 and (1 + z/d)^2 times Z cn sn dn for w.  Jacobi's functions at
  // u = 4 K x by the arithmetic-geometric mean (Abramowitz and Stegun
  // 16.4), the moduli from the theta series of the smaller nome.  Heights
  // enter as REAL(ZC*100), results leave in single precision, times 0.01.
  static void th_jacobi(double ql, double x, double &cn, double &sn, double &dn) {
    const double PI = 3.141592653589793;
    double t2, t3, t4;
    auto thetas = [&](double q) {
      double s2 = 0.0, s3 = 0.0, s4 = 0.0;
      for (int n = 6; n >= 1; --n) {
        s3 = s3 + std::pow(q, (double)(n * n));
        s4 = s4 + ((n & 1) ? -1.0 : 1.0) * std::pow(q, (double)(n * n));
      }
      for (int n = 6; n >= 0; --n) s2 = s2 + std::pow(q, (double)(n * (n + 1)));
      t2 = 2.0 * std::pow(q, 0.25) * s2;
      t3 = 1.0 + 2.0 * s3;
      t4 = 1.0 + 2.0 * s4;
    };
    double k, kp;
    if (ql >= PI) {
      thetas(std::exp(-ql));
      k = (t2 / t3) * (t2 / t3);
      kp = (t4 / t3) * (t4 / t3);
    } else {
      thetas(std::exp(-PI * PI / ql));
      kp = (t2 / t3) * (t2 / t3);
      k = (t4 / t3) * (t4 / t3);
    }
    double x1 = x - std::floor(x + 0.5), sig = 1.0;
    if (x1 > 0.25) { x1 = x1 - 0.5; sig = -1.0; }
    else if (x1 < -0.25) { x1 = x1 + 0.5; sig = -1.0; }
    std::vector<double> a(1, 1.0), c(1, k);
    double b = kp;
    while ((int)a.size() < 47 && std::fabs(c.back()) > 1e-15 * a.back()) {
      const double an = a.back();
      a.push_back(0.5 * (an + b));
      c.push_back(0.5 * (an - b));
      b = std::sqrt(an * b);
    }
    const int N = (int)a.size() - 1;
    double phi = std::ldexp(2.0 * PI * x1, N), phi1 = phi;
    for (int m = N; m >= 1; --m) {
      phi1 = phi;
      phi = 0.5 * (phi + std::asin(c[m] / a[m] * std::sin(phi)));
    }
    sn = sig * std::sin(phi);
    cn = sig * std::cos(phi);
    dn = (N == 0) ? 1.0 : std::cos(phi) / std::cos(phi1 - phi);
  }
  // VF_CWMAK1  vf_cwmak1.f: the level at phase wvt (m)
  static double th_level(const cadmas_wave_theory &t, double wvt) {
    if (t.type >= 1) return sw_level(t.stream, wvt);
    double zs = 0.0;
    if (t.type == -2) {
      const double th = 2.0 * 3.141592653589793 * wvt;
      for (int i = 1; i <= 5; ++i) zs = zs + t.stokes.a[i - 1] * std::cos((double)i * th);
    } else {
      double cn, sn, dn;
      th_jacobi(t.cnoidal.ql, wvt / 2.0, cn, sn, dn);
      const double cn2 = cn * cn;
      for (int L = 4; L >= 1; --L) zs = zs * cn2 + t.cnoidal.a[L - 1];
    }
    return (double)(float)zs * 0.01;
  }
  // VF_CWMAK2  vf_cwmak2.f: normal and vertical velocity at height z (m/s)
  static void th_velocity(const cadmas_wave_theory &t, double wvt, double z, double &u, double &w) {
    if (t.type >= 1) { sw_velocity(t.stream, wvt, z, u, w); return; }
    const double zt = (double)(float)(z * 100.0);
    double su, sv;
    if (t.type == -2) {
      const double th = 2.0 * 3.141592653589793 * wvt, zd = zt + t.depth * 100.0;
      su = t.stokes.b0;
      sv = 0.0;
      for (int i = 1; i <= 5; ++i) {
        const double cj = t.stokes.b[i - 1] * std::cos((double)i * th);
        const double sj = t.stokes.b[i - 1] * std::sin((double)i * th);
        double ch, sh;
        sw_chsh((double)i * t.stokes.k * zd, ch, sh);
        su = su + cj * ch;
        sv = sv + sj * sh;
      }
    } else {
      double cn, sn, dn;
      th_jacobi(t.cnoidal.ql, wvt / 2.0, cn, sn, dn);
      const double cn2 = cn * cn, csd = cn * sn * dn;
      const double Z = 1.0 + zt / t.cnoidal.d, ZZ = Z * Z;
      su = 0.0;
      sv = 0.0;
      for (int K = 4; K >= 1; --K) {
        double pu = 0.0, pw = 0.0;
        for (int L = 3; L >= 1; --L) {
          pu = pu * ZZ + t.cnoidal.b[(K - 1) * 3 + (L - 1)];
          pw = pw * ZZ + t.cnoidal.bb[(K - 1) * 3 + (L - 1)];
        }
        su = su * cn2 + pu;
        if (K > 1) sv = sv * cn2 + pw;
      }
      sv = sv * csd * Z;
    }
    u = (double)(float)su * 0.01;
    w = (double)(float)sv * 0.01;
  }

  // VF_BWUWN wave-maker part  vf_bwuwn.f:259-470: the matrix-table inflow
  // (IBCTYP(2,JD) = -3, MTBTYP 1 or 2) or a wave theory (IBCTYP(2,JD) =
  // N >= 1, -1, -2: VF_CWMAK1/VF_CWMAK2), normal or oblique incidence
  // (BCTYP(9..11,JD)), one rank.
  int bwuwn_wave() {
    const double PI = 3.141592653589794, ZERO = 1.0e-20;
    for (int JD = 1; JD <= 4; ++JD) {
      const Wave &w = WV[JD - 1];
      if (!w.on) continue;
      const double D = w.d, T = w.t, T0 = w.theory ? w.th.phase0 : DMTBT0;
      double A = w.a;
      float R4TN = (float)(T0 - TNOW / T);
      R4TN = R4TN - (float)(int)R4TN;
      if (R4TN < 0.0f) R4TN = R4TN + 1.0f;
      double AW = 1.0;
      if (A >= ZERO) {
        A = TNOW / T / A;
        if (A < 1.0) AW = 0.5 * std::sin(PI * (A - 0.5)) + 0.5;
      }
      const double WVT = (double)R4TN;
      double WMT1 = 0.0, WMT2 = 0.0, WVZ;
      if (w.theory) WVZ = th_level(w.th, WVT);
      else if (!cwmtb1(WVT, WMT1, WMT2, WVZ)) return CADMAS_EPG;
      double SA = w.ang, SB, SC;
      const int ISA = (std::fabs(SA) <= ZERO) ? 0 : 1;
      if (ISA == 0) {
        if (JD == 1) { SA = 1.0; SB = 0.0; }
        else if (JD == 2) { SA = -1.0; SB = 0.0; }
        else if (JD == 3) { SA = 0.0; SB = 1.0; }
        else { SA = 0.0; SB = -1.0; }
        SC = 0.0;
      } else {
        if (!w.theory) return CADMAS_EPG;  // vf_bwuwn.f:351-356
        if (JD == 2) SA = SA + 180.0;
        else if (JD == 3) SA = SA + 90.0;
        else if (JD == 4) SA = SA + 270.0;
        SA = SA * PI / 180.0;
        SB = std::sin(SA);
        SA = std::cos(SA);
        SC = -(SA * w.sx + SB * w.sy);
      }
      const double DL = w.th.length;
      if (!w.theory && MTBTYP == 3) continue;  // vf_bwuwn.f:330: no velocities from a level table
      const int MT = w.theory ? 1 : MTBTYP;
      const bool xs = (JD == 1 || JD == 2);
      const int I0 = (JD == 1) ? 2 : NI, IC0 = (JD == 1) ? 2 : NI - 1;
      const int J0 = (JD == 3) ? 2 : NJ, JC0 = (JD == 3) ? 2 : NJ - 1;
      for (int n = w.l1; n <= w.l2; ++n) {
        const int I = xs ? I0 : n, J = xs ? n : J0, IC = xs ? IC0 : n, JC = xs ? n : JC0;
        if (xs ? (J < 2 || J > NJ - 1) : (I < 2 || I > NI - 1)) continue;
        double WVTC = WVT;
        if (ISA != 0) {  // this line's phase and level (vf_bwuwn.f:345-356, 418-430)
          const double X0 = xs ? X_(1, I) : (X_(1, I) + X_(1, I + 1)) * 0.5;
          const double Y0 = xs ? (Y_(1, J) + Y_(1, J + 1)) * 0.5 : Y_(1, J);
          const double RR = (SA * X0 + SB * Y0 + SC) / std::sqrt(SA * SA + SB * SB);
          float R4 = (float)(T0 - (TNOW / T - RR / DL));
          R4 = R4 - (float)(int)R4;
          if (R4 < 0.0f) R4 = R4 + 1.0f;
          WVTC = (double)R4;
          WVZ = th_level(w.th, WVTC);
        }
        double VWS;
        if (MT != 1) {
          VWS = 1.0;
        } else {
          double VAL = 0.0;
          for (int K = 2; K <= NK - 1; ++K) {
            const int NW = NF[id(IC, JC, K)];
            if (NW == -1) VAL = VAL + Z_(2, K) * 1.0;
            else if (NW == 0) VAL = VAL + Z_(2, K) * FF[id(IC, JC, K)];
            else if (NW != 8) { VAL = VAL + Z_(2, K) * FF[id(IC, JC, K)]; break; }
          }
          VAL = VAL - (P.wvlvl - Z_(1, 2));
          VWS = (WVZ + D) / (VAL + D);
        }
        int KMT = 1;
        for (int K = 2; K <= NK - 1; ++K) {
          const int L = xs ? INDX[id(I, J, K)] : INDY[id(I, J, K)];
          if (L < 1) continue;
          double ZC = (Z_(1, K) + Z_(1, K + 1)) * 0.5 - P.wvlvl;
          ZC = VWS * (ZC + D) - D;
          double UN, UT;
          if (w.theory) th_velocity(w.th, WVTC, ZC, UN, UT);
          else if (!cwmtb2(KMT, WMT1, WMT2, ZC, UN, UT)) return CADMAS_EPG;
          BCU[L - 1] = UN * VWS * AW * SA;
          BCV[L - 1] = UN * VWS * AW * SB;
          BCW[L - 1] = UT * VWS * AW;
          if (xs) UU[id(I, J, K)] = BCU[L - 1];
          else VV[id(I, J, K)] = BCV[L - 1];
        }
      }
    }
    return CADMAS_OK;
  }

  // VF_VPCOEF  vf_vpcoef.f:117-437 (IPRNT<=1: GGV0=GGV; PVCP0<0: PPS=0)
  int vpcoef(vd &AD, vd &ALI, vd &ALJ, vd &ALK, vd &AUI, vd &AUJ, vd &AUK, vd &BB) {
    std::fill(AD.begin(), AD.end(), 0.0);
    std::fill(ALI.begin(), ALI.end(), 0.0); std::fill(ALJ.begin(), ALJ.end(), 0.0);
    std::fill(ALK.begin(), ALK.end(), 0.0); std::fill(AUI.begin(), AUI.end(), 0.0);
    std::fill(AUJ.begin(), AUJ.end(), 0.0); std::fill(AUK.begin(), AUK.end(), 0.0);
    std::fill(BB.begin(), BB.end(), 0.0);
    const double DTI = 1.0 / DTNOW, TR = DTNOW / P.rho0, PPS = 0.0;
    for (int K = 1; K <= NK; ++K)
      for (int J = 1; J <= NJ; ++J)
        for (int I = 1; I <= NI; ++I) {
          size_t c = id(I, J, K);
          int N = NF[c];
          if (INDC[c] == -1) {
            AD[c] = 1.0; ALI[c] = 0.0; ALJ[c] = 0.0; ALK[c] = 0.0;
            AUI[c] = 0.0; AUJ[c] = 0.0; AUK[c] = 0.0; BB[c] = 0.0;
          } else if (N == 0) {
            int IM = I - 1, IP = I + 1, JM = J - 1, JP = J + 1, KM = K - 1, KP = K + 1;
            double AXY = X_(2, I) * Y_(2, J), AXZ = X_(2, I) * Z_(2, K), AYZ = Y_(2, J) * Z_(2, K);
            double AVL = X_(2, I) * Y_(2, J) * Z_(2, K);
            double AIM, AIP, AJM, AJP, AKM, AKP, GV;
            int IS = INDX[c];
            if (IS == 0) {
              GV = X_(6, I) * (X_(2, I) * GGV[c] / GLV[c] + X_(2, IM) * GGV[id(IM, J, K)] / GLV[id(IM, J, K)]);
              AIM = AYZ * X_(5, I) * GGX[c] * GV; ALI[c] = -AIM;
            } else if (IS >= 1) {
              if (IB_(3, IS) == 4 || (IB_(3, IS) == 5 && I == 2 && FIXLVL(1))) { AIM = 2.0 * AYZ * X_(4, I) * GGX[c] * GGV[c] / GLV[c]; ALI[c] = 0.0; }
              else { AIM = 0.0; ALI[c] = 0.0; }
            } else return CADMAS_EPG;
            IS = INDX[id(IP, J, K)];
            if (IS == 0) {
              GV = X_(6, IP) * (X_(2, IP) * GGV[id(IP, J, K)] / GLV[id(IP, J, K)] + X_(2, I) * GGV[c] / GLV[c]);
              AIP = AYZ * X_(5, IP) * GGX[id(IP, J, K)] * GV; AUI[c] = -AIP;
            } else if (IS >= 1) {
              if (IB_(3, IS) == 4 || (IB_(3, IS) == 5 && IP == NI && FIXLVL(2))) { AIP = 2.0 * AYZ * X_(4, I) * GGX[id(IP, J, K)] * GGV[c] / GLV[c]; AUI[c] = 0.0; }
              else { AIP = 0.0; AUI[c] = 0.0; }
            } else return CADMAS_EPG;
            IS = INDY[c];
            if (IS == 0) {
              GV = Y_(6, J) * (Y_(2, J) * GGV[c] / GLV[c] + Y_(2, JM) * GGV[id(I, JM, K)] / GLV[id(I, JM, K)]);
              AJM = AXZ * Y_(5, J) * GGY[c] * GV; ALJ[c] = -AJM;
            } else if (IS >= 1) {
              if (IB_(3, IS) == 4 || (IB_(3, IS) == 5 && J == 2 && FIXLVL(3))) { AJM = 2.0 * AXZ * Y_(4, J) * GGY[c] * GGV[c] / GLV[c]; ALJ[c] = 0.0; }
              else { AJM = 0.0; ALJ[c] = 0.0; }
            } else return CADMAS_EPG;
            IS = INDY[id(I, JP, K)];
            if (IS == 0) {
              GV = Y_(6, JP) * (Y_(2, JP) * GGV[id(I, JP, K)] / GLV[id(I, JP, K)] + Y_(2, J) * GGV[c] / GLV[c]);
              AJP = AXZ * Y_(5, JP) * GGY[id(I, JP, K)] * GV; AUJ[c] = -AJP;
            } else if (IS >= 1) {
              if (IB_(3, IS) == 4 || (IB_(3, IS) == 5 && JP == NJ && FIXLVL(4))) { AJP = 2.0 * AXZ * Y_(4, J) * GGY[id(I, JP, K)] * GGV[c] / GLV[c]; AUJ[c] = 0.0; }
              else { AJP = 0.0; AUJ[c] = 0.0; }
            } else return CADMAS_EPG;
            IS = INDZ[c];
            if (IS == 0) {
              GV = Z_(6, K) * (Z_(2, K) * GGV[c] / GLV[c] + Z_(2, KM) * GGV[id(I, J, KM)] / GLV[id(I, J, KM)]);
              AKM = AXY * Z_(5, K) * GGZ[c] * GV; ALK[c] = -AKM;
            } else if (IS >= 1) {
              if (IB_(3, IS) != 4) { AKM = 0.0; ALK[c] = 0.0; }
              else { AKM = 2.0 * AXY * Z_(4, K) * GGZ[c] * GGV[c] / GLV[c]; ALK[c] = 0.0; }
            } else return CADMAS_EPG;
            IS = INDZ[id(I, J, KP)];
            if (IS == 0) {
              GV = Z_(6, KP) * (Z_(2, KP) * GGV[id(I, J, KP)] / GLV[id(I, J, KP)] + Z_(2, K) * GGV[c] / GLV[c]);
              AKP = AXY * Z_(5, KP) * GGZ[id(I, J, KP)] * GV; AUK[c] = -AKP;
            } else if (IS >= 1) {
              if (IB_(3, IS) != 4) { AKP = 0.0; AUK[c] = 0.0; }
              else { AKP = 2.0 * AXY * Z_(4, K) * GGZ[id(I, J, KP)] * GGV[c] / GLV[c]; AUK[c] = 0.0; }
            } else return CADMAS_EPG;
            AD[c] = AKM + AJM + AIM + AIP + AJP + AKP;
            double VD = AYZ * (GGX[id(IP, J, K)] * UU[id(IP, J, K)] - GGX[c] * UU[c]) +
                        AXZ * (GGY[id(I, JP, K)] * VV[id(I, JP, K)] - GGY[c] * VV[c]) +
                        AXY * (GGZ[id(I, J, KP)] * WW[id(I, J, KP)] - GGZ[c] * WW[c]);
            double VQ = -(GGV[c] - GGV[c]) * DTI * AVL;
            if (IWS() == I) VQ = 2.0 * Z_(2, K) * SRC(J, K) * Y_(2, J);  // vf_vpcoef.f:349-350
            if (JWS() == J) VQ = 2.0 * Z_(2, K) * SRC(I, K) * X_(2, I);
            BB[c] = VD - VQ;
          } else if (N == 5) {
            double PSI = Z_(3, K) / (0.5 * Z_(2, K - 1) + FF[c] * Z_(2, K));
            AD[c] = 1.0; ALI[c] = 0.0; ALJ[c] = 0.0; ALK[c] = PSI - 1.0; AUI[c] = 0.0; AUJ[c] = 0.0; AUK[c] = 0.0;
            BB[c] = -TR * ((1.0 - PSI) * PP[id(I, J, K - 1)] + PSI * PPS - PP[c]);
          } else if (N == 6) {
            double PSI = Z_(3, K + 1) / (0.5 * Z_(2, K + 1) + FF[c] * Z_(2, K));
            AD[c] = 1.0; ALI[c] = 0.0; ALJ[c] = 0.0; ALK[c] = 0.0; AUI[c] = 0.0; AUJ[c] = 0.0; AUK[c] = PSI - 1.0;
            BB[c] = -TR * ((1.0 - PSI) * PP[id(I, J, K + 1)] + PSI * PPS - PP[c]);
          } else if (N == 3) {
            double PSI = Y_(3, J) / (0.5 * Y_(2, J - 1) + FF[c] * Y_(2, J));
            AD[c] = 1.0; ALI[c] = 0.0; ALJ[c] = PSI - 1.0; ALK[c] = 0.0; AUI[c] = 0.0; AUJ[c] = 0.0; AUK[c] = 0.0;
            BB[c] = -TR * ((1.0 - PSI) * PP[id(I, J - 1, K)] + PSI * PPS - PP[c]);
          } else if (N == 4) {
            double PSI = Y_(3, J + 1) / (0.5 * Y_(2, J + 1) + FF[c] * Y_(2, J));
            AD[c] = 1.0; ALI[c] = 0.0; ALJ[c] = 0.0; ALK[c] = 0.0; AUI[c] = 0.0; AUJ[c] = PSI - 1.0; AUK[c] = 0.0;
            BB[c] = -TR * ((1.0 - PSI) * PP[id(I, J + 1, K)] + PSI * PPS - PP[c]);
          } else if (N == 1) {
            double PSI = X_(3, I) / (0.5 * X_(2, I - 1) + FF[c] * X_(2, I));
            AD[c] = 1.0; ALI[c] = PSI - 1.0; ALJ[c] = 0.0; ALK[c] = 0.0; AUI[c] = 0.0; AUJ[c] = 0.0; AUK[c] = 0.0;
            BB[c] = -TR * ((1.0 - PSI) * PP[id(I - 1, J, K)] + PSI * PPS - PP[c]);
          } else if (N == 2) {
            double PSI = X_(3, I + 1) / (0.5 * X_(2, I + 1) + FF[c] * X_(2, I));
            AD[c] = 1.0; ALI[c] = 0.0; ALJ[c] = 0.0; ALK[c] = 0.0; AUI[c] = PSI - 1.0; AUJ[c] = 0.0; AUK[c] = 0.0;
            BB[c] = -TR * ((1.0 - PSI) * PP[id(I + 1, J, K)] + PSI * PPS - PP[c]);
          } else {
            return CADMAS_EPG;
          }
        }
    return CADMAS_OK;
  }

  // ----------------------------------------------------------- solver
  // Block decomposition of the interior for the preconditioner
  // (emulated PARALLEL X/Y ranks; tile = one rank's MYIS..MYIE x MYJS..MYJE).
  struct Tile { int is, ie, js, je; };
  std::vector<Tile> tiles() const {
    int ti = P.precond_ti > 0 ? P.precond_ti : (NI - 2);
    int tj = P.precond_tj > 0 ? P.precond_tj : (NJ - 2);
    std::vector<Tile> t;
    for (int js = 2; js <= NJ - 1; js += tj)
      for (int is = 2; is <= NI - 1; is += ti)
        t.push_back({is, std::min(NI - 1, is + ti - 1), js, std::min(NJ - 1, js + tj - 1)});
    return t;
  }

  // VF_MZDCMP  vf_mzdcmp.f:53-67, per tile.  A neighbour outside the tile
  // is a halo cell of the rank: DD=0 there and its coefficients are 0
  // (VF_VPCOEF zeroes the arrays and the halo exchanges are disabled), so
  // its term is coef*0*0.
  bool mzdcmp(const vd &AD, const vd &ALI, const vd &ALJ, const vd &ALK, const vd &AUI,
              const vd &AUJ, const vd &AUK, vd &DDo, const int *IC) {
    const double U = (P.icgtyp != 0) ? P.cgpara : 0.0;
    int npos = 1;
    const std::vector<Tile> tl = tiles();
    // tiles are independent (block-Jacobi): one thread per tile
#pragma omp parallel for schedule(dynamic) reduction(&& : npos) if (par())
    for (size_t n = 0; n < tl.size(); ++n) {
      const Tile &t = tl[n];
      for (int K = 2; K <= NK - 1; ++K)
        for (int J = t.js; J <= t.je; ++J)
          for (int I = t.is; I <= t.ie; ++I) {
            size_t c = id(I, J, K);
            if (IC[c] == -1) continue;
            double d1 = 0.0, a1 = 0.0, d2 = 0.0, a2 = 0.0, d3 = 0.0, a3 = 0.0;
            if (I > t.is) { size_t n = id(I - 1, J, K); d1 = DDo[n]; a1 = AUI[n] + U * (AUJ[n] + AUK[n]); }
            else { a1 = 0.0 + U * (0.0 + 0.0); }
            if (J > t.js) { size_t n = id(I, J - 1, K); d2 = DDo[n]; a2 = AUJ[n] + U * (AUI[n] + AUK[n]); }
            else { a2 = 0.0 + U * (0.0 + 0.0); }
            { size_t n = id(I, J, K - 1); d3 = DDo[n]; a3 = AUK[n] + U * (AUI[n] + AUJ[n]); }
            DDo[c] = 1.0 / (AD[c] - ALI[c] * d1 * a1 - ALJ[c] * d2 * a2 - ALK[c] * d3 * a3);
            if (DDo[c] <= 0.0) npos = 0;
          }
    }
    return npos != 0;
  }
  // VF_MZFRWD vf_mzfrwd.f:37-48 then VF_MZBKWD vf_mzbkwd.f:37-47, per tile.
  void mzminv(const vd &DDv, const vd &ALI, const vd &ALJ, const vd &ALK, const vd &AUI,
              const vd &AUJ, const vd &AUK, vd &X, const vd &Yv, const int *IC) {
    const std::vector<Tile> tl = tiles();
#pragma omp parallel for schedule(dynamic) if (par())
    for (size_t n = 0; n < tl.size(); ++n) {
      const Tile &t = tl[n];
      for (int K = 2; K <= NK - 1; ++K)
        for (int J = t.js; J <= t.je; ++J)
          for (int I = t.is; I <= t.ie; ++I) {
            size_t c = id(I, J, K);
            if (IC[c] == -1) continue;
            double d1 = 0.0, x1 = 0.0, d2 = 0.0, x2 = 0.0;
            if (I > t.is) { d1 = DDv[id(I - 1, J, K)]; x1 = X[id(I - 1, J, K)]; }
            if (J > t.js) { d2 = DDv[id(I, J - 1, K)]; x2 = X[id(I, J - 1, K)]; }
            double d3 = DDv[id(I, J, K - 1)], x3 = X[id(I, J, K - 1)];
            X[c] = Yv[c] - ALI[c] * d1 * x1 - ALJ[c] * d2 * x2 - ALK[c] * d3 * x3;
          }
      for (int K = NK - 1; K >= 2; --K)
        for (int J = t.je; J >= t.js; --J)
          for (int I = t.ie; I >= t.is; --I) {
            size_t c = id(I, J, K);
            if (IC[c] == -1) continue;
            double x1 = (I < t.ie) ? X[id(I + 1, J, K)] : 0.0;
            double x2 = (J < t.je) ? X[id(I, J + 1, K)] : 0.0;
            double x3 = X[id(I, J, K + 1)];
            X[c] = (X[c] - AUI[c] * x1 - AUJ[c] * x2 - AUK[c] * x3) * DDv[c];
          }
    }
  }
  // VF_MZAX  vf_mzax.f:42-56
  void mzax(const vd &AD, const vd &ALI, const vd &ALJ, const vd &ALK, const vd &AUI,
            const vd &AUJ, const vd &AUK, const vd &X, vd &Yv, const int *IC) {
#pragma omp parallel for schedule(static) if (par())
    for (int K = 2; K <= NK - 1; ++K)
      for (int J = 2; J <= NJ - 1; ++J)
        for (int I = 2; I <= NI - 1; ++I) {
          size_t c = id(I, J, K);
          if (IC[c] == -1) continue;
          Yv[c] = AD[c] * X[c] + ALI[c] * X[id(I - 1, J, K)] + ALJ[c] * X[id(I, J - 1, K)] +
                  ALK[c] * X[id(I, J, K - 1)] + AUI[c] * X[id(I + 1, J, K)] + AUJ[c] * X[id(I, J + 1, K)] +
                  AUK[c] * X[id(I, J, K + 1)];
        }
  }
  // VF_MZIP  vf_mzip.f:32-43 (+ VF_P1SUMD): per-rank partial sums in ref
  // order, the row tree in GPU order.
  double mzip(const vd &X, const vd &Yv, const int *IC) {
    if (sum_mode == ORC_SUM_REF) {
      // each emulated rank's partial in parallel, then the ranks in order
      const std::vector<Tile> tl = tiles();
      std::vector<double> part(tl.size());
#pragma omp parallel for schedule(dynamic) if (par())
      for (size_t n = 0; n < tl.size(); ++n) {
        const Tile &t = tl[n];
        double s = 0.0;
        for (int K = 2; K <= NK - 1; ++K)
          for (int J = t.js; J <= t.je; ++J)
            for (int I = t.is; I <= t.ie; ++I) {
              size_t c = id(I, J, K);
              if (IC[c] != -1) s = s + X[c] * Yv[c];
            }
        part[n] = s;
      }
      double S = 0.0;
      for (double s : part) S = S + s;
      return S;
    }
    return gsum_skew([&](int i, int j, int k, double &c) {
      size_t q = id(i, j, k);
      if (IC[q] == -1) return false;
      c = X[q] * Yv[q];
      return true;
    });
  }

  // VF_M1BCGS  vf_m1bcgs.f:76-266
  void m1bcgs(const vd &AD, const vd &ALI, const vd &ALJ, const vd &ALK, const vd &AUI,
              const vd &AUJ, const vd &AUK, const vd &BB, vd &X0, const int *IC,
              double &BNORM, double &XNORM, int &ITER) {
    size_t N = X0.size();
    XW = X0;
    DD.assign(N, 0.0); Y2.assign(N, 0.0); R0.assign(N, 0.0); RR.assign(N, 0.0);
    PPv.assign(N, 0.0); AP.assign(N, 0.0); AE.assign(N, 0.0);
    ITER = -1; BNORM = 0.0; XNORM = 0.0;
    if (!mzdcmp(AD, ALI, ALJ, ALK, AUI, AUJ, AUK, DD, IC)) return;
    const double EPSA2 = P.cgepsa * P.cgepsa, EPSR2 = P.cgepsr * P.cgepsr, DIV2 = P.cgdiv * P.cgdiv;
    mzminv(DD, ALI, ALJ, ALK, AUI, AUJ, AUK, Y2, BB, IC);
    BNORM = mzip(Y2, Y2, IC);
    ITER = 0;
    mzax(AD, ALI, ALJ, ALK, AUI, AUJ, AUK, XW, Y2, IC);
#pragma omp parallel for schedule(static) if (par())
    for (size_t c = 0; c < N; ++c) if (IC[c] != -1) Y2[c] = BB[c] - Y2[c];
    mzminv(DD, ALI, ALJ, ALK, AUI, AUJ, AUK, R0, Y2, IC);
    double S = mzip(R0, R0, IC);
    XNORM = S;
    if (!(XNORM <= BNORM * EPSR2 + EPSA2)) {
#pragma omp parallel for schedule(static) if (par())
      for (size_t c = 0; c < N; ++c) if (IC[c] != -1) { RR[c] = R0[c]; PPv[c] = R0[c]; }
      for (;;) {
        ITER = ITER + 1;
        if (ITER > P.icgmax) break;
        mzax(AD, ALI, ALJ, ALK, AUI, AUJ, AUK, PPv, Y2, IC);
        mzminv(DD, ALI, ALJ, ALK, AUI, AUJ, AUK, AP, Y2, IC);
        double W1 = mzip(R0, AP, IC);
        double ALPHA = S / W1;
#pragma omp parallel for schedule(static) if (par())
        for (size_t c = 0; c < N; ++c) if (IC[c] != -1) RR[c] = RR[c] - ALPHA * AP[c];
        mzax(AD, ALI, ALJ, ALK, AUI, AUJ, AUK, RR, Y2, IC);
        mzminv(DD, ALI, ALJ, ALK, AUI, AUJ, AUK, AE, Y2, IC);
        W1 = mzip(RR, AE, IC);
        double W2 = mzip(AE, AE, IC);
        double OMEGA = W1 / W2;
#pragma omp parallel for schedule(static) if (par())
        for (size_t c = 0; c < N; ++c)
          if (IC[c] != -1) {
            XW[c] = XW[c] + (ALPHA * PPv[c] + OMEGA * RR[c]);
            RR[c] = RR[c] - OMEGA * AE[c];
          }
        XNORM = mzip(RR, RR, IC);
        if (XNORM <= BNORM * EPSR2 + EPSA2) break;
        if (XNORM > DIV2) { ITER = -2; break; }
        W1 = mzip(R0, RR, IC);
        double BETA = W1 * ALPHA / (S * OMEGA);
#pragma omp parallel for schedule(static) if (par())
        for (size_t c = 0; c < N; ++c)
          if (IC[c] != -1) PPv[c] = RR[c] + BETA * (PPv[c] - OMEGA * AP[c]);
        S = W1;
      }
    }
    BNORM = std::sqrt(BNORM);
    XNORM = std::sqrt(XNORM);
    if (ITER >= 0)
      for (size_t c = 0; c < N; ++c) if (IC[c] != -1) X0[c] = XW[c];
  }
  inline bool interior_c(size_t c) const {
    int i = (int)(c % NI) + 1, j = (int)((c / NI) % NJ) + 1, k = (int)(c / ((size_t)NI * NJ)) + 1;
    return interior(i, j, k);
  }

  // ||b - A x||_2 / ||b||_2 over INDC != -1 (diagnostic of the metric)
  double true_relres(const vd &AD, const vd &ALI, const vd &ALJ, const vd &ALK, const vd &AUI,
                     const vd &AUJ, const vd &AUK, const vd &BB, const vd &X, const int *IC) {
    double rn = solver_sum([&](int I, int J, int K, double &c) {
      if (!interior(I, J, K)) return false;
      size_t q = id(I, J, K);
      if (IC[q] == -1) return false;
      double ax = AD[q] * X[q] + ALI[q] * X[id(I - 1, J, K)] + ALJ[q] * X[id(I, J - 1, K)] +
                  ALK[q] * X[id(I, J, K - 1)] + AUI[q] * X[id(I + 1, J, K)] + AUJ[q] * X[id(I, J + 1, K)] +
                  AUK[q] * X[id(I, J, K + 1)];
      double r = BB[q] - ax;
      c = r * r;
      return true;
    });
    double bn = solver_sum([&](int I, int J, int K, double &c) {
      size_t q = id(I, J, K);
      if (!interior(I, J, K) || IC[q] == -1) return false;
      c = BB[q] * BB[q];
      return true;
    });
    return bn > 0.0 ? std::sqrt(rn) / std::sqrt(bn) : 0.0;
  }

  // VF_VMODIF  vf_vmodif.f:58-215 (wave faces with matrix data not restated)
  void vmodif(const vd &PT) {
    for (int K = 2; K <= NK - 1; ++K)
      for (int J = 2; J <= NJ - 1; ++J)
        for (int I = 2; I <= NI; ++I) {
          if (NF[id(I - 1, J, K)] * NF[id(I, J, K)] != 0) continue;
          int IS = INDX[id(I, J, K)];
          if (IS == 0) {
            double GV = X_(6, I) * (X_(2, I) * GGV[id(I, J, K)] / GLV[id(I, J, K)] +
                                    X_(2, I - 1) * GGV[id(I - 1, J, K)] / GLV[id(I - 1, J, K)]);
            UU[id(I, J, K)] = UU[id(I, J, K)] + X_(5, I) * GV * (PT[id(I, J, K)] - PT[id(I - 1, J, K)]);
          } else if (IS > 0 && (IB_(3, IS) == 4 || (IB_(3, IS) == 5 && fixlvl_face(IB_(2, IS), I, J)))) {
            if (IB_(2, IS) == 1)
              UU[id(I, J, K)] = UU[id(I, J, K)] + 2.0 * X_(4, I) * GGV[id(I, J, K)] / GLV[id(I, J, K)] * PT[id(I, J, K)];
            else
              UU[id(I, J, K)] = UU[id(I, J, K)] - 2.0 * X_(4, I - 1) * GGV[id(I - 1, J, K)] / GLV[id(I - 1, J, K)] * PT[id(I - 1, J, K)];
            BCU[IS - 1] = UU[id(I, J, K)];
          }
        }
    for (int K = 2; K <= NK - 1; ++K)
      for (int J = 2; J <= NJ; ++J)
        for (int I = 2; I <= NI - 1; ++I) {
          if (NF[id(I, J - 1, K)] * NF[id(I, J, K)] != 0) continue;
          int IS = INDY[id(I, J, K)];
          if (IS == 0) {
            double GV = Y_(6, J) * (Y_(2, J) * GGV[id(I, J, K)] / GLV[id(I, J, K)] +
                                    Y_(2, J - 1) * GGV[id(I, J - 1, K)] / GLV[id(I, J - 1, K)]);
            VV[id(I, J, K)] = VV[id(I, J, K)] + Y_(5, J) * GV * (PT[id(I, J, K)] - PT[id(I, J - 1, K)]);
          } else if (IS > 0 && (IB_(3, IS) == 4 || (IB_(3, IS) == 5 && fixlvl_face(IB_(2, IS), I, J)))) {
            if (IB_(2, IS) == 3)
              VV[id(I, J, K)] = VV[id(I, J, K)] + 2.0 * Y_(4, J) * GGV[id(I, J, K)] / GLV[id(I, J, K)] * PT[id(I, J, K)];
            else
              VV[id(I, J, K)] = VV[id(I, J, K)] - 2.0 * Y_(4, J - 1) * GGV[id(I, J - 1, K)] / GLV[id(I, J - 1, K)] * PT[id(I, J - 1, K)];
            BCV[IS - 1] = VV[id(I, J, K)];
          }
        }
    for (int K = 2; K <= NK; ++K)
      for (int J = 2; J <= NJ - 1; ++J)
        for (int I = 2; I <= NI - 1; ++I) {
          if (NF[id(I, J, K - 1)] * NF[id(I, J, K)] != 0) continue;
          int IS = INDZ[id(I, J, K)];
          if (IS == 0) {
            double GV = Z_(6, K) * (Z_(2, K) * GGV[id(I, J, K)] / GLV[id(I, J, K)] +
                                    Z_(2, K - 1) * GGV[id(I, J, K - 1)] / GLV[id(I, J, K - 1)]);
            WW[id(I, J, K)] = WW[id(I, J, K)] + Z_(5, K) * GV * (PT[id(I, J, K)] - PT[id(I, J, K - 1)]);
          } else if (IS > 0 && IB_(3, IS) == 4) {
            if (IB_(2, IS) == 5)
              WW[id(I, J, K)] = WW[id(I, J, K)] + 2.0 * Z_(4, K) * GGV[id(I, J, K)] / GLV[id(I, J, K)] * PT[id(I, J, K)];
            else
              WW[id(I, J, K)] = WW[id(I, J, K)] - 2.0 * Z_(4, K - 1) * GGV[id(I, J, K - 1)] / GLV[id(I, J, K - 1)] * PT[id(I, J, K - 1)];
            BCW[IS - 1] = WW[id(I, J, K)];
          }
        }
    const double RT = P.rho0 / DTNOW;
    for (int K = 2; K <= NK - 1; ++K)
      for (int J = 2; J <= NJ - 1; ++J)
        for (int I = 2; I <= NI - 1; ++I)
          if (INDC[id(I, J, K)] != -1) PP[id(I, J, K)] = PP[id(I, J, K)] - RT * PT[id(I, J, K)];
  }

  // VF_BSUWT  vf_bsuwt.f:41-470 (one axis; 'a' is the face array, the
  // surface directions checked are the other two axes).
  // Written out per axis below to keep the Fortran operand order.
  void bsuwt() {
    const int S0 = (P.ibsuw0 == 0);
    // x faces
    for (int K = 2; K <= NK - 1; ++K)
      for (int J = 2; J <= NJ - 1; ++J)
        for (int I = 3; I <= NI - 1; ++I) {
          if (INDX[id(I, J, K)] != 0) continue;
          int I1 = I - 1, NL = NF[id(I1, J, K)], NR = NF[id(I, J, K)];
          if (NL == 8 && NR == 8) { UU[id(I, J, K)] = 0.0; continue; }
          if (!(NL != 0 && NR != 0)) continue;
          double DL = 0, VL = 0, DR = 0, VR = 0, V0;
          if (NL == 3 || NR == 3) {
            V0 = UU[id(I, J - 1, K)];
            if (S0) { int L1 = J - 1, L2 = J - 2;
              if (NF[id(I1, L1, K)] != -1 && NF[id(I, L1, K)] != -1)
                if (NF[id(I1, L2, K)] != -1 && NF[id(I, L2, K)] != -1)
                  if (NF[id(I1, L2, K)] == 0 || NF[id(I, L2, K)] == 0)
                    V0 = V0 + (V0 - UU[id(I, L2, K)]) * Y_(3, J) / Y_(3, L1); }
            if (NL == 3) { DL = Y_(3, J); VL = V0; }
            if (NR == 3) { DR = Y_(3, J); VR = V0; }
          }
          if (NL == 4 || NR == 4) {
            V0 = UU[id(I, J + 1, K)];
            if (S0) { int L1 = J + 1, L2 = J + 2;
              if (NF[id(I1, L1, K)] != -1 && NF[id(I, L1, K)] != -1)
                if (NF[id(I1, L2, K)] != -1 && NF[id(I, L2, K)] != -1)
                  if (NF[id(I1, L2, K)] == 0 || NF[id(I, L2, K)] == 0)
                    V0 = V0 + (V0 - UU[id(I, L2, K)]) * Y_(3, L1) / Y_(3, L2); }
            if (NL == 4) { DL = Y_(3, J + 1); VL = V0; }
            if (NR == 4) { DR = Y_(3, J + 1); VR = V0; }
          }
          if (NL == 5 || NR == 5) {
            V0 = UU[id(I, J, K - 1)];
            if (S0) { int L1 = K - 1, L2 = K - 2;
              if (NF[id(I1, J, L1)] != -1 && NF[id(I, J, L1)] != -1)
                if (NF[id(I1, J, L2)] != -1 && NF[id(I, J, L2)] != -1)
                  if (NF[id(I1, J, L2)] == 0 || NF[id(I, J, L2)] == 0)
                    V0 = V0 + (V0 - UU[id(I, J, L2)]) * Z_(3, K) / Z_(3, L1); }
            if (NL == 5) { DL = Z_(3, K); VL = V0; }
            if (NR == 5) { DR = Z_(3, K); VR = V0; }
          }
          if (NL == 6 || NR == 6) {
            V0 = UU[id(I, J, K + 1)];
            if (S0) { int L1 = K + 1, L2 = K + 2;
              if (NF[id(I1, J, L1)] != -1 && NF[id(I, J, L1)] != -1)
                if (NF[id(I1, J, L2)] != -1 && NF[id(I, J, L2)] != -1)
                  if (NF[id(I1, J, L2)] == 0 || NF[id(I, J, L2)] == 0)
                    V0 = V0 + (V0 - UU[id(I, J, L2)]) * Z_(3, L1) / Z_(3, L2); }
            if (NL == 6) { DL = Z_(3, K + 1); VL = V0; }
            if (NR == 6) { DR = Z_(3, K + 1); VR = V0; }
          }
          if (NL == 8) UU[id(I, J, K)] = VR;
          else if (NR == 8) UU[id(I, J, K)] = VL;
          else UU[id(I, J, K)] = (DR * VL + DL * VR) / (DR + DL);
        }
    // y faces
    for (int K = 2; K <= NK - 1; ++K)
      for (int J = 3; J <= NJ - 1; ++J)
        for (int I = 2; I <= NI - 1; ++I) {
          if (INDY[id(I, J, K)] != 0) continue;
          int J1 = J - 1, NL = NF[id(I, J1, K)], NR = NF[id(I, J, K)];
          if (NL == 8 && NR == 8) { VV[id(I, J, K)] = 0.0; continue; }
          if (!(NL != 0 && NR != 0)) continue;
          double DL = 0, VL = 0, DR = 0, VR = 0, V0;
          if (NL == 1 || NR == 1) {
            V0 = VV[id(I - 1, J, K)];
            if (S0) { int L1 = I - 1, L2 = I - 2;
              if (NF[id(L1, J1, K)] != -1 && NF[id(L1, J, K)] != -1)
                if (NF[id(L2, J1, K)] != -1 && NF[id(L2, J, K)] != -1)
                  if (NF[id(L2, J1, K)] == 0 || NF[id(L2, J, K)] == 0)
                    V0 = V0 + (V0 - VV[id(L2, J, K)]) * X_(3, I) / X_(3, L1); }
            if (NL == 1) { DL = X_(3, I); VL = V0; }
            if (NR == 1) { DR = X_(3, I); VR = V0; }
          }
          if (NL == 2 || NR == 2) {
            V0 = VV[id(I + 1, J, K)];
            if (S0) { int L1 = I + 1, L2 = I + 2;
              if (NF[id(L1, J1, K)] != -1 && NF[id(L1, J, K)] != -1)
                if (NF[id(L2, J1, K)] != -1 && NF[id(L2, J, K)] != -1)
                  if (NF[id(L2, J1, K)] == 0 || NF[id(L2, J, K)] == 0)
                    V0 = V0 + (V0 - VV[id(L2, J, K)]) * X_(3, L1) / X_(3, L2); }
            if (NL == 2) { DL = X_(3, I + 1); VL = V0; }
            if (NR == 2) { DR = X_(3, I + 1); VR = V0; }
          }
          if (NL == 5 || NR == 5) {
            V0 = VV[id(I, J, K - 1)];
            if (S0) { int L1 = K - 1, L2 = K - 2;
              if (NF[id(I, J1, L1)] != -1 && NF[id(I, J, L1)] != -1)
                if (NF[id(I, J1, L2)] != -1 && NF[id(I, J, L2)] != -1)
                  if (NF[id(I, J1, L2)] == 0 || NF[id(I, J, L2)] == 0)
                    V0 = V0 + (V0 - VV[id(I, J, L2)]) * Z_(3, K) / Z_(3, L1); }
            if (NL == 5) { DL = Z_(3, K); VL = V0; }
            if (NR == 5) { DR = Z_(3, K); VR = V0; }
          }
          if (NL == 6 || NR == 6) {
            V0 = VV[id(I, J, K + 1)];
            if (S0) { int L1 = K + 1, L2 = K + 2;
              if (NF[id(I, J1, L1)] != -1 && NF[id(I, J, L1)] != -1)
                if (NF[id(I, J1, L2)] != -1 && NF[id(I, J, L2)] != -1)
                  if (NF[id(I, J1, L2)] == 0 || NF[id(I, J, L2)] == 0)
                    V0 = V0 + (V0 - VV[id(I, J, L2)]) * Z_(3, L1) / Z_(3, L2); }
            if (NL == 6) { DL = Z_(3, K + 1); VL = V0; }
            if (NR == 6) { DR = Z_(3, K + 1); VR = V0; }
          }
          if (NL == 8) VV[id(I, J, K)] = VR;
          else if (NR == 8) VV[id(I, J, K)] = VL;
          else VV[id(I, J, K)] = (DR * VL + DL * VR) / (DR + DL);
        }
    // z faces
    for (int K = 3; K <= NK - 1; ++K)
      for (int J = 2; J <= NJ - 1; ++J)
        for (int I = 2; I <= NI - 1; ++I) {
          if (INDZ[id(I, J, K)] != 0) continue;
          int K1 = K - 1, NL = NF[id(I, J, K1)], NR = NF[id(I, J, K)];
          if (NL == 8 && NR == 8) { WW[id(I, J, K)] = 0.0; continue; }
          if (!(NL != 0 && NR != 0)) continue;
          double DL = 0, VL = 0, DR = 0, VR = 0, V0;
          if (NL == 1 || NR == 1) {
            V0 = WW[id(I - 1, J, K)];
            if (S0) { int L1 = I - 1, L2 = I - 2;
              if (NF[id(L1, J, K1)] != -1 && NF[id(L1, J, K)] != -1)
                if (NF[id(L2, J, K1)] != -1 && NF[id(L2, J, K)] != -1)
                  if (NF[id(L2, J, K1)] == 0 || NF[id(L2, J, K)] == 0)
                    V0 = V0 + (V0 - WW[id(L2, J, K)]) * X_(3, I) / X_(3, L1); }
            if (NL == 1) { DL = X_(3, I); VL = V0; }
            if (NR == 1) { DR = X_(3, I); VR = V0; }
          }
          if (NL == 2 || NR == 2) {
            V0 = WW[id(I + 1, J, K)];
            if (S0) { int L1 = I + 1, L2 = I + 2;
              if (NF[id(L1, J, K1)] != -1 && NF[id(L1, J, K)] != -1)
                if (NF[id(L2, J, K1)] != -1 && NF[id(L2, J, K)] != -1)
                  if (NF[id(L2, J, K1)] == 0 || NF[id(L2, J, K)] == 0)
                    V0 = V0 + (V0 - WW[id(L2, J, K)]) * X_(3, L1) / X_(3, L2); }
            if (NL == 2) { DL = X_(3, I + 1); VL = V0; }
            if (NR == 2) { DR = X_(3, I + 1); VR = V0; }
          }
          if (NL == 3 || NR == 3) {
            V0 = WW[id(I, J - 1, K)];
            if (S0) { int L1 = J - 1, L2 = J - 2;
              if (NF[id(I, L1, K1)] != -1 && NF[id(I, L1, K)] != -1)
                if (NF[id(I, L2, K1)] != -1 && NF[id(I, L2, K)] != -1)
                  if (NF[id(I, L2, K1)] == 0 || NF[id(I, L2, K)] == 0)
                    V0 = V0 + (V0 - WW[id(I, L2, K)]) * Y_(3, J) / Y_(3, L1); }
            if (NL == 3) { DL = Y_(3, J); VL = V0; }
            if (NR == 3) { DR = Y_(3, J); VR = V0; }
          }
          if (NL == 4 || NR == 4) {
            V0 = WW[id(I, J + 1, K)];
            if (S0) { int L1 = J + 1, L2 = J + 2;
              if (NF[id(I, L1, K1)] != -1 && NF[id(I, L1, K)] != -1)
                if (NF[id(I, L2, K1)] != -1 && NF[id(I, L2, K)] != -1)
                  if (NF[id(I, L2, K1)] == 0 || NF[id(I, L2, K)] == 0)
                    V0 = V0 + (V0 - WW[id(I, L2, K)]) * Y_(3, L1) / Y_(3, L2); }
            if (NL == 4) { DL = Y_(3, J + 1); VL = V0; }
            if (NR == 4) { DR = Y_(3, J + 1); VR = V0; }
          }
          if (NL == 8) WW[id(I, J, K)] = VR;
          else if (NR == 8) WW[id(I, J, K)] = VL;
          else WW[id(I, J, K)] = (DR * VL + DL * VR) / (DR + DL);
        }
  }

  // VF_BSUWT2  vf_bsuwt2.f:36-107
  void bsuwt2() {
    for (int L = 0; L < NUMS; ++L) {
      int I, J, K;
      decode(INDS[L], I, J, K);
      int NF0 = NF[id(I, J, K)];
      int L1, L2, LB;
      if (NF0 == 5 || NF0 == 6) {
        LB = (NF0 == 5) ? K - 1 : K + 1;
        L1 = I; L2 = I;
        if (NF[id(I - 1, J, K)] == 8 && INDX[id(I, J, LB)] != 0) L2 = L2 + 1;
        if (NF[id(I + 1, J, K)] == 8 && INDX[id(I + 1, J, LB)] != 0) L1 = L1 + 1;
        UU[id(L1, J, K)] = UU[id(L2, J, K)];
        L1 = J; L2 = J;
        if (NF[id(I, J - 1, K)] == 8 && INDY[id(I, J, LB)] != 0) L2 = L2 + 1;
        if (NF[id(I, J + 1, K)] == 8 && INDY[id(I, J + 1, LB)] != 0) L1 = L1 + 1;
        VV[id(I, L1, K)] = VV[id(I, L2, K)];
      } else if (NF0 == 3 || NF0 == 4) {
        LB = (NF0 == 3) ? J - 1 : J + 1;
        L1 = I; L2 = I;
        if (NF[id(I - 1, J, K)] == 8 && INDX[id(I, LB, K)] != 0) L2 = L2 + 1;
        if (NF[id(I + 1, J, K)] == 8 && INDX[id(I + 1, LB, K)] != 0) L1 = L1 + 1;
        UU[id(L1, J, K)] = UU[id(L2, J, K)];
        L1 = K; L2 = K;
        if (NF[id(I, J, K - 1)] == 8 && INDZ[id(I, LB, K)] != 0) L2 = L2 + 1;
        if (NF[id(I, J, K + 1)] == 8 && INDZ[id(I, LB, K + 1)] != 0) L1 = L1 + 1;
        WW[id(I, J, L1)] = WW[id(I, J, L2)];
      } else if (NF0 == 1 || NF0 == 2) {
        LB = (NF0 == 1) ? I - 1 : I + 1;
        L1 = J; L2 = J;
        if (NF[id(I, J - 1, K)] == 8 && INDY[id(LB, J, K)] != 0) L2 = L2 + 1;
        if (NF[id(I, J + 1, K)] == 8 && INDY[id(LB, J + 1, K)] != 0) L1 = L1 + 1;
        VV[id(I, L1, K)] = VV[id(I, L2, K)];
        L1 = K; L2 = K;
        if (NF[id(I, J, K - 1)] == 8 && INDZ[id(LB, J, K)] != 0) L2 = L2 + 1;
        if (NF[id(I, J, K + 1)] == 8 && INDZ[id(LB, J, K + 1)] != 0) L1 = L1 + 1;
        WW[id(I, J, L1)] = WW[id(I, J, L2)];
      }
    }
  }

  // VF_BSUWN  vf_bsuwn.f:57-118
  void bsuwn() {
    for (int L = 0; L < NUMS; ++L) {
      int I, J, K;
      decode(INDS[L], I, J, K);
      int NF0 = NF[id(I, J, K)];
      int I1 = I + 1, J1 = J + 1, K1 = K + 1;
      double FXP = GGX[id(I1, J, K)] * UU[id(I1, J, K)], FXM = GGX[id(I, J, K)] * UU[id(I, J, K)];
      double FYP = GGY[id(I, J1, K)] * VV[id(I, J1, K)], FYM = GGY[id(I, J, K)] * VV[id(I, J, K)];
      double FZP = GGZ[id(I, J, K1)] * WW[id(I, J, K1)], FZM = GGZ[id(I, J, K)] * WW[id(I, J, K)];
      if (NF0 == 5) WW[id(I, J, K1)] = (FZM - Z_(2, K) * (X_(4, I) * (FXP - FXM) + Y_(4, J) * (FYP - FYM))) / GGZ[id(I, J, K1)];
      else if (NF0 == 6) WW[id(I, J, K)] = (FZP + Z_(2, K) * (X_(4, I) * (FXP - FXM) + Y_(4, J) * (FYP - FYM))) / GGZ[id(I, J, K)];
      else if (NF0 == 3) VV[id(I, J1, K)] = (FYM - Y_(2, J) * (X_(4, I) * (FXP - FXM) + Z_(4, K) * (FZP - FZM))) / GGY[id(I, J1, K)];
      else if (NF0 == 4) VV[id(I, J, K)] = (FYP + Y_(2, J) * (X_(4, I) * (FXP - FXM) + Z_(4, K) * (FZP - FZM))) / GGY[id(I, J, K)];
      else if (NF0 == 1) UU[id(I1, J, K)] = (FXM - X_(2, I) * (Y_(4, J) * (FYP - FYM) + Z_(4, K) * (FZP - FZM))) / GGX[id(I1, J, K)];
      else if (NF0 == 2) UU[id(I, J, K)] = (FXP + X_(2, I) * (Y_(4, J) * (FYP - FYM) + Z_(4, K) * (FZP - FZM))) / GGX[id(I, J, K)];
    }
    // wave source  vf_bsuwn.f:81-118
    const int IWS_ = IWS(), JWS_ = JWS();
    if (IWS_ != 0 || JWS_ != 0) {
      for (int J = 2; J <= NJ - 1; ++J)
        for (int I = 2; I <= NI - 1; ++I) {
          if (!(IWS_ == I || JWS_ == J)) continue;
          for (int K = 2; K <= NK - 1; ++K) {
            const int N = NF[id(I, J, K)];
            if (N == -1 || N == 0) continue;
            if (N == 8) continue;
            double Q = 0.0;
            if (IWS_ == I) Q = 2.0 * X_(4, I) * SRC(J, K);
            if (JWS_ == J) Q = 2.0 * Y_(4, J) * SRC(I, K);
            if (N == 1) UU[id(I + 1, J, K)] = UU[id(I + 1, J, K)] + X_(2, I) * Q / GGX[id(I + 1, J, K)];
            else if (N == 2) UU[id(I, J, K)] = UU[id(I, J, K)] - X_(2, I) * Q / GGX[id(I, J, K)];
            else if (N == 3) VV[id(I, J + 1, K)] = VV[id(I, J + 1, K)] + Y_(2, J) * Q / GGY[id(I, J + 1, K)];
            else if (N == 4) VV[id(I, J, K)] = VV[id(I, J, K)] - Y_(2, J) * Q / GGY[id(I, J, K)];
            else if (N == 5) WW[id(I, J, K + 1)] = WW[id(I, J, K + 1)] + Z_(2, K) * Q / GGZ[id(I, J, K + 1)];
            else if (N == 6) WW[id(I, J, K)] = WW[id(I, J, K)] - Z_(2, K) * Q / GGZ[id(I, J, K)];
            break;
          }
        }
    }
  }

  // VF_BSUWN3  vf_bsuwn3.f:37-340; written for the z case and mapped by
  // a small accessor per axis so that every operand keeps its position.
  void bsuwn3() {
    const int S0 = (P.ibsuw0 == 0);
    for (int L = 0; L < NUMS; ++L) {
      int I, J, K;
      decode(INDS[L], I, J, K);
      int NF0 = NF[id(I, J, K)];
      int IS1 = 0, IS2 = 0, IS3 = 0, IS4 = 0;
      double D0, V0, D1 = 0, V1 = 0, D2 = 0, V2 = 0, D3 = 0, V3 = 0, D4 = 0, V4 = 0;
      auto lat = [&](int &isx, double &dx, double &vx, size_t a, size_t b, double d, double v) {
        if (NF[a] == 0 || NF[b] == 0)
          if (NF[a] != -1 && NF[b] != -1) { isx = 1; dx = d; vx = v; }
      };
      if (NF0 == 5) {
        D0 = Z_(2, K); V0 = WW[id(I, J, K)]; int L1 = K + 1;
        lat(IS1, D1, V1, id(I - 1, J, K), id(I - 1, J, L1), X_(3, I), WW[id(I - 1, J, L1)]);
        lat(IS2, D2, V2, id(I + 1, J, K), id(I + 1, J, L1), X_(3, I + 1), WW[id(I + 1, J, L1)]);
        lat(IS3, D3, V3, id(I, J - 1, K), id(I, J - 1, L1), Y_(3, J), WW[id(I, J - 1, L1)]);
        lat(IS4, D4, V4, id(I, J + 1, K), id(I, J + 1, L1), Y_(3, J + 1), WW[id(I, J + 1, L1)]);
        int ISS = IS1 + IS2 + IS3 + IS4;
        if (ISS <= 0) {
          if (S0 && NF[id(I, J, K - 2)] == 0) V0 = V0 + (V0 - WW[id(I, J, K - 1)]) * Z_(2, K) / Z_(2, K - 1);
          WW[id(I, J, K + 1)] = V0;
        } else {
          double DS = D0 + D1 + D2 + D3 + D4;
          WW[id(I, J, K + 1)] = ((DS - D0) * V0 + (DS - D1) * V1 + (DS - D2) * V2 + (DS - D3) * V3 + (DS - D4) * V4) / DS / (double)ISS;
        }
      } else if (NF0 == 6) {
        D0 = Z_(2, K); V0 = WW[id(I, J, K + 1)]; int L1 = K - 1;
        lat(IS1, D1, V1, id(I - 1, J, K), id(I - 1, J, L1), X_(3, I), WW[id(I - 1, J, K)]);
        lat(IS2, D2, V2, id(I + 1, J, K), id(I + 1, J, L1), X_(3, I + 1), WW[id(I + 1, J, K)]);
        lat(IS3, D3, V3, id(I, J - 1, K), id(I, J - 1, L1), Y_(3, J), WW[id(I, J - 1, K)]);
        lat(IS4, D4, V4, id(I, J + 1, K), id(I, J + 1, L1), Y_(3, J + 1), WW[id(I, J + 1, K)]);
        int ISS = IS1 + IS2 + IS3 + IS4;
        if (ISS <= 0) {
          if (S0 && NF[id(I, J, K + 2)] == 0) V0 = V0 + (V0 - WW[id(I, J, K + 2)]) * Z_(2, K) / Z_(2, K + 1);
          WW[id(I, J, K)] = V0;
        } else {
          double DS = D0 + D1 + D2 + D3 + D4;
          WW[id(I, J, K)] = ((DS - D0) * V0 + (DS - D1) * V1 + (DS - D2) * V2 + (DS - D3) * V3 + (DS - D4) * V4) / DS / (double)ISS;
        }
      } else if (NF0 == 3) {
        D0 = Y_(2, J); V0 = VV[id(I, J, K)]; int L1 = J + 1;
        lat(IS1, D1, V1, id(I - 1, J, K), id(I - 1, L1, K), X_(3, I), VV[id(I - 1, L1, K)]);
        lat(IS2, D2, V2, id(I + 1, J, K), id(I + 1, L1, K), X_(3, I + 1), VV[id(I + 1, L1, K)]);
        lat(IS3, D3, V3, id(I, J, K - 1), id(I, L1, K - 1), Z_(3, K), VV[id(I, L1, K - 1)]);
        lat(IS4, D4, V4, id(I, J, K + 1), id(I, L1, K + 1), Z_(3, K + 1), VV[id(I, L1, K + 1)]);
        int ISS = IS1 + IS2 + IS3 + IS4;
        if (ISS <= 0) {
          if (S0 && NF[id(I, J - 2, K)] == 0) V0 = V0 + (V0 - VV[id(I, J - 1, K)]) * Y_(2, J) / Y_(2, J - 1);
          VV[id(I, J + 1, K)] = V0;
        } else {
          double DS = D0 + D1 + D2 + D3 + D4;
          VV[id(I, J + 1, K)] = ((DS - D0) * V0 + (DS - D1) * V1 + (DS - D2) * V2 + (DS - D3) * V3 + (DS - D4) * V4) / DS / (double)ISS;
        }
      } else if (NF0 == 4) {
        D0 = Y_(2, J); V0 = VV[id(I, J + 1, K)]; int L1 = J - 1;
        lat(IS1, D1, V1, id(I - 1, J, K), id(I - 1, L1, K), X_(3, I), VV[id(I - 1, J, K)]);
        lat(IS2, D2, V2, id(I + 1, J, K), id(I + 1, L1, K), X_(3, I + 1), VV[id(I + 1, J, K)]);
        lat(IS3, D3, V3, id(I, J, K - 1), id(I, L1, K - 1), Z_(3, K), VV[id(I, J, K - 1)]);
        lat(IS4, D4, V4, id(I, J, K + 1), id(I, L1, K + 1), Z_(3, K + 1), VV[id(I, J, K + 1)]);
        int ISS = IS1 + IS2 + IS3 + IS4;
        if (ISS <= 0) {
          if (S0 && NF[id(I, J + 2, K)] == 0) V0 = V0 + (V0 - VV[id(I, J + 2, K)]) * Y_(2, J) / Y_(2, J + 1);
          VV[id(I, J, K)] = V0;
        } else {
          double DS = D0 + D1 + D2 + D3 + D4;
          VV[id(I, J, K)] = ((DS - D0) * V0 + (DS - D1) * V1 + (DS - D2) * V2 + (DS - D3) * V3 + (DS - D4) * V4) / DS / (double)ISS;
        }
      } else if (NF0 == 1) {
        D0 = X_(2, I); V0 = UU[id(I, J, K)]; int L1 = I + 1;
        lat(IS1, D1, V1, id(I, J - 1, K), id(L1, J - 1, K), Y_(3, J), UU[id(L1, J - 1, K)]);
        lat(IS2, D2, V2, id(I, J + 1, K), id(L1, J + 1, K), Y_(3, J + 1), UU[id(L1, J + 1, K)]);
        lat(IS3, D3, V3, id(I, J, K - 1), id(L1, J, K - 1), Z_(3, K), UU[id(L1, J, K - 1)]);
        lat(IS4, D4, V4, id(I, J, K + 1), id(L1, J, K + 1), Z_(3, K + 1), UU[id(L1, J, K + 1)]);
        int ISS = IS1 + IS2 + IS3 + IS4;
        if (ISS <= 0) {
          if (S0 && NF[id(I - 2, J, K)] == 0) V0 = V0 + (V0 - UU[id(I - 1, J, K)]) * X_(2, I) / X_(2, I - 1);
          UU[id(I + 1, J, K)] = V0;
        } else {
          double DS = D0 + D1 + D2 + D3 + D4;
          UU[id(I + 1, J, K)] = ((DS - D0) * V0 + (DS - D1) * V1 + (DS - D2) * V2 + (DS - D3) * V3 + (DS - D4) * V4) / DS / (double)ISS;
        }
      } else if (NF0 == 2) {
        D0 = X_(2, I); V0 = UU[id(I + 1, J, K)]; int L1 = I - 1;
        lat(IS1, D1, V1, id(I, J - 1, K), id(L1, J - 1, K), Y_(3, J), UU[id(I, J - 1, K)]);
        lat(IS2, D2, V2, id(I, J + 1, K), id(L1, J + 1, K), Y_(3, J + 1), UU[id(I, J + 1, K)]);
        lat(IS3, D3, V3, id(I, J, K - 1), id(L1, J, K - 1), Z_(3, K), UU[id(I, J, K - 1)]);
        lat(IS4, D4, V4, id(I, J, K + 1), id(L1, J, K + 1), Z_(3, K + 1), UU[id(I, J, K + 1)]);
        int ISS = IS1 + IS2 + IS3 + IS4;
        if (ISS <= 0) {
          if (S0 && NF[id(I + 2, J, K)] == 0) V0 = V0 + (V0 - UU[id(I + 2, J, K)]) * X_(2, I) / X_(2, I + 1);
          UU[id(I, J, K)] = V0;
        } else {
          double DS = D0 + D1 + D2 + D3 + D4;
          UU[id(I, J, K)] = ((DS - D0) * V0 + (DS - D1) * V1 + (DS - D2) * V2 + (DS - D3) * V3 + (DS - D4) * V4) / DS / (double)ISS;
        }
      }
    }
  }

  // VF_BWUWT  vf_bwuwt.f:41-118 (slip/free, no-slip, fixed; wave faces
  // without matrix data and radiation faces untouched)
  // (vf_bwuwt.f:41-181; IB 5 acts for MTBTYP 3 only, IB 2, 3, 7 keep BC)
  int bwuwt() {
    for (int L = 1; L <= NB; ++L) {
      int I, J, K;
      decode(IB_(1, L), I, J, K);
      int NS = IB_(2, L), IB = IB_(3, L);
      if (IB == 6 || IB == 8) {  // vf_bwuwt.f:116-176
        double V1, V2, DL, AN;
        if (NS == 1) {
          V1 = (VV[id(I, J, K)] + VV[id(I, J + 1, K)]) * 0.5; V2 = (WW[id(I, J, K)] + WW[id(I, J, K + 1)]) * 0.5;
          DL = X_(2, I) * 0.5; AN = ANU[id(I, J, K)];
        } else if (NS == 2) {
          V1 = (VV[id(I - 1, J, K)] + VV[id(I - 1, J + 1, K)]) * 0.5; V2 = (WW[id(I - 1, J, K)] + WW[id(I - 1, J, K + 1)]) * 0.5;
          DL = X_(2, I - 1) * 0.5; AN = ANU[id(I - 1, J, K)];
        } else if (NS == 3) {
          V1 = (UU[id(I, J, K)] + UU[id(I + 1, J, K)]) * 0.5; V2 = (WW[id(I, J, K)] + WW[id(I, J, K + 1)]) * 0.5;
          DL = Y_(2, J) * 0.5; AN = ANU[id(I, J, K)];
        } else if (NS == 4) {
          V1 = (UU[id(I, J - 1, K)] + UU[id(I + 1, J - 1, K)]) * 0.5; V2 = (WW[id(I, J - 1, K)] + WW[id(I, J - 1, K + 1)]) * 0.5;
          DL = Y_(2, J - 1) * 0.5; AN = ANU[id(I, J - 1, K)];
        } else if (NS == 5) {
          V1 = (UU[id(I, J, K)] + UU[id(I + 1, J, K)]) * 0.5; V2 = (VV[id(I, J, K)] + VV[id(I, J + 1, K)]) * 0.5;
          DL = Z_(2, K) * 0.5; AN = ANU[id(I, J, K)];
        } else {
          V1 = (UU[id(I, J, K - 1)] + UU[id(I + 1, J, K - 1)]) * 0.5; V2 = (VV[id(I, J, K - 1)] + VV[id(I, J + 1, K - 1)]) * 0.5;
          DL = Z_(2, K - 1) * 0.5; AN = ANU[id(I, J, K - 1)];
        }
        const double ZERO = 1.0e-20;
        double VA = std::sqrt(V1 * V1 + V2 * V2), VT;
        if (VA < ZERO || AN < ZERO) {
          V1 = 0.0; V2 = 0.0; DL = 1.0; AN = 1.0; VA = 1.0; VT = 1.0;
        } else if (IB == 6) {
          if (!cloglw(DL, VA, P.anu0, P.akk0, P.aka0, VT)) return CADMAS_ENOTCONV;
        } else {
          VT = clogks(DL, VA, BCVI[L - 1], P.anu0, P.akk0, P.aka0);
        }
        VA = DL / AN * VT * VT / VA;
        V1 = V1 - VA * V1;
        V2 = V2 - VA * V2;
        if (NS == 1 || NS == 2) { BCV[L - 1] = V1; BCW[L - 1] = V2; }
        else if (NS == 3 || NS == 4) { BCU[L - 1] = V1; BCW[L - 1] = V2; }
        else { BCU[L - 1] = V1; BCV[L - 1] = V2; }
      } else if (IB == 1 || IB == 4 || (IB == 5 && fixlvl_face(NS, I, J))) {  // vf_bwuwt.f:51-115
        if (NS == 1) { BCV[L - 1] = (VV[id(I, J, K)] + VV[id(I, J + 1, K)]) * 0.5; BCW[L - 1] = (WW[id(I, J, K)] + WW[id(I, J, K + 1)]) * 0.5; }
        else if (NS == 2) { BCV[L - 1] = (VV[id(I - 1, J, K)] + VV[id(I - 1, J + 1, K)]) * 0.5; BCW[L - 1] = (WW[id(I - 1, J, K)] + WW[id(I - 1, J, K + 1)]) * 0.5; }
        else if (NS == 3) { BCU[L - 1] = (UU[id(I, J, K)] + UU[id(I + 1, J, K)]) * 0.5; BCW[L - 1] = (WW[id(I, J, K)] + WW[id(I, J, K + 1)]) * 0.5; }
        else if (NS == 4) { BCU[L - 1] = (UU[id(I, J - 1, K)] + UU[id(I + 1, J - 1, K)]) * 0.5; BCW[L - 1] = (WW[id(I, J - 1, K)] + WW[id(I, J - 1, K + 1)]) * 0.5; }
        else if (NS == 5) { BCU[L - 1] = (UU[id(I, J, K)] + UU[id(I + 1, J, K)]) * 0.5; BCV[L - 1] = (VV[id(I, J, K)] + VV[id(I, J + 1, K)]) * 0.5; }
        else if (NS == 6) { BCU[L - 1] = (UU[id(I, J, K - 1)] + UU[id(I + 1, J, K - 1)]) * 0.5; BCV[L - 1] = (VV[id(I, J, K - 1)] + VV[id(I, J + 1, K - 1)]) * 0.5; }
      }
    }
    return CADMAS_OK;
  }
  // VF_BWPP  vf_bwpp.f:28-51
  void bwpp() {
    for (int L = 1; L <= NB; ++L) {
      int I, J, K;
      decode(IB_(1, L), I, J, K);
      int NS = IB_(2, L);
      if (NS == 1) BCP[L - 1] = PP[id(I, J, K)];
      else if (NS == 2) BCP[L - 1] = PP[id(I - 1, J, K)];
      else if (NS == 3) BCP[L - 1] = PP[id(I, J, K)];
      else if (NS == 4) BCP[L - 1] = PP[id(I, J - 1, K)];
      else if (NS == 5) BCP[L - 1] = PP[id(I, J, K)];
      else if (NS == 6) BCP[L - 1] = PP[id(I, J, K - 1)];
    }
  }

  // ---------------------------------------------------------------- VOF
  // VF_FCONV  vf_fconv.f:56-206
  void fconv(vd &FLFU, vd &FLFV, vd &FLFW) {
    const double DT = DTNOW, FL = P.flower;
    auto face = [&](double C, int N, double FDa, int ndm, double FDMa, double Vd, double Vo, double bcf,
                    int na, double FAa, int dirA, int dirB, int dirC, int dirD, double &FL_, int &lim) {
      (void)dirA;
      double AC = std::fabs(C), FD, FDMW, V, FA;
      if (N != -1) { FD = FDa; FDMW = 1.0; if (ndm != -1) FDMW = FDMa; V = Vd; }
      else { FD = bcf; FDMW = 1.0; V = Vo; }
      FA = (na != -1) ? FAa : FD;
      double FAD = FA;
      if (N == -1 || N == dirA || N == dirB || N == dirC || N == dirD)
        if (FDMW != 0.0 && FA != 0.0) FAD = FD;
      double FDM = dmax(FDMW, FD);
      if (FDMW < FL && FA < FL) FDM = dmax(FDM, 0.1);
      double CFX = dmax((FDM - FAD) * AC - (FDM - FD) * V, 0.0);
      double FVX = FAD * AC + CFX;
      double FVM = FD * V;
      FL_ = dmin(FVX, FVM);
      lim = (FVX > FVM);
    };
    for (int K = 2; K <= NK - 1; ++K)
      for (int J = 2; J <= NJ - 1; ++J)
        for (int I = 2; I <= NI; ++I) {
          if (INDX[id(I, J, K)] == -1) continue;
          double C = DT * GGX[id(I, J, K)] * UU[id(I, J, K)];
          int LSN, LA, LD, LDM;
          if (C >= 0.0) { LSN = 1; LA = I; LD = I - 1; LDM = I - 2; } else { LSN = -1; LA = I - 1; LD = I; LDM = I + 1; }
          int N = NF[id(LD, J, K)];
          int ndm = (N != -1) ? NF[id(LDM, J, K)] : -1;
          double fdm = (N != -1 && ndm != -1) ? FF[id(LDM, J, K)] : 0.0;
          double vd_ = (N != -1) ? X_(2, LD) * GGV[id(LD, J, K)] : 0.0;
          double bcf = (N == -1) ? BCF[INDX[id(I, J, K)] - 1] : 0.0;
          int na = NF[id(LA, J, K)];
          double fl; int lim;
          face(C, N, (N != -1) ? FF[id(LD, J, K)] : 0.0, ndm, fdm, vd_, X_(2, LD), bcf, na,
               (na != -1) ? FF[id(LA, J, K)] : 0.0, 3, 4, 5, 6, fl, lim);
          FLFU[id(I, J, K)] = FLFU[id(I, J, K)] - (double)LSN * fl;
          if (lim) NLIM[id(LD, J, K)] = 1;
        }
    for (int K = 2; K <= NK - 1; ++K)
      for (int J = 2; J <= NJ; ++J)
        for (int I = 2; I <= NI - 1; ++I) {
          if (INDY[id(I, J, K)] == -1) continue;
          double C = DT * GGY[id(I, J, K)] * VV[id(I, J, K)];
          int LSN, LA, LD, LDM;
          if (C >= 0.0) { LSN = 1; LA = J; LD = J - 1; LDM = J - 2; } else { LSN = -1; LA = J - 1; LD = J; LDM = J + 1; }
          int N = NF[id(I, LD, K)];
          int ndm = (N != -1) ? NF[id(I, LDM, K)] : -1;
          double fdm = (N != -1 && ndm != -1) ? FF[id(I, LDM, K)] : 0.0;
          double vd_ = (N != -1) ? Y_(2, LD) * GGV[id(I, LD, K)] : 0.0;
          double bcf = (N == -1) ? BCF[INDY[id(I, J, K)] - 1] : 0.0;
          int na = NF[id(I, LA, K)];
          double fl; int lim;
          face(C, N, (N != -1) ? FF[id(I, LD, K)] : 0.0, ndm, fdm, vd_, Y_(2, LD), bcf, na,
               (na != -1) ? FF[id(I, LA, K)] : 0.0, 1, 2, 5, 6, fl, lim);
          FLFV[id(I, J, K)] = FLFV[id(I, J, K)] - (double)LSN * fl;
          if (lim) NLIM[id(I, LD, K)] = 1;
        }
    for (int K = 2; K <= NK; ++K)
      for (int J = 2; J <= NJ - 1; ++J)
        for (int I = 2; I <= NI - 1; ++I) {
          if (INDZ[id(I, J, K)] == -1) continue;
          double C = DT * GGZ[id(I, J, K)] * WW[id(I, J, K)];
          int LSN, LA, LD, LDM;
          if (C >= 0.0) { LSN = 1; LA = K; LD = K - 1; LDM = K - 2; } else { LSN = -1; LA = K - 1; LD = K; LDM = K + 1; }
          int N = NF[id(I, J, LD)];
          int ndm = (N != -1) ? NF[id(I, J, LDM)] : -1;
          double fdm = (N != -1 && ndm != -1) ? FF[id(I, J, LDM)] : 0.0;
          double vd_ = (N != -1) ? Z_(2, LD) * GGV[id(I, J, LD)] : 0.0;
          double bcf = (N == -1) ? BCF[INDZ[id(I, J, K)] - 1] : 0.0;
          int na = NF[id(I, J, LA)];
          double fl; int lim;
          face(C, N, (N != -1) ? FF[id(I, J, LD)] : 0.0, ndm, fdm, vd_, Z_(2, LD), bcf, na,
               (na != -1) ? FF[id(I, J, LA)] : 0.0, 1, 2, 3, 4, fl, lim);
          FLFW[id(I, J, K)] = FLFW[id(I, J, K)] - (double)LSN * fl;
          if (lim) NLIM[id(I, J, LD)] = 1;
        }
  }

  // VF_FCONVS  vf_fconvs.f:72-387: slope normals and plane offsets of
  // the surface cells.  ISTYP = 0 (none), 3, 5, 6 or 7 (bits of the
  // normal components with |S| >= 1e-4, two or more of them).
  int ist_count[8] = {0, 0, 0, 0, 0, 0, 0, 0};  // cells of each slope type, summed over the run
  int fslope(std::vector<int> &IST, vd &SX, vd &SY, vd &SZ, vd &SA) {
    const size_t N = UU.size();
    IST.assign(N, 0); SX.assign(N, 0.0); SY.assign(N, 0.0); SZ.assign(N, 0.0); SA.assign(N, 0.0);
    const double ZERO = 1.0e-20;
    int rc = CADMAS_OK;
    // one side of one axis (vf_fconvs.f:86-123 and its five copies):
    // the neighbour's F (FO) and distance (DO) towards it.  a/b are the
    // NF0 values of the cross-axis pair, e/o their cross-axis offsets;
    // sgn = -1 for the minus side (metric entries of this cell), +1 for
    // the plus side (of the neighbour); m3/m6 the 3rd and 6th metric
    // entries, d2 the neighbour's width, DD0 this cell's.
    auto side = [&](int NF0, double FF0, size_t cL, int NFL, double BCFv, const int *ns, const long long *off,
                    double DD0, double d2, double m3, double m6, double &FO, double &DO) {
      double FFL = FF[cL];
      if (NFL == -1) { FO = BCFv; DO = DD0 * 0.5; }
      else if (NFL == 8) {
        if (NF0 == ns[0] || NF0 == ns[1] || NF0 == ns[2] || NF0 == ns[3]) { FO = FF0; DO = 0.0; }
        else { FO = 0.0; DO = DD0 * 0.5; }
      } else if (NFL == 0) {
        FO = FFL; DO = DD0 * 0.5;
        for (int q = 0; q < 4; ++q)
          if (NF0 == ns[q]) {
            size_t cq = (size_t)((long long)cL + off[q]);
            if (NF[cq] != -1) { FO = FO + FF[cq]; DO = m3; }
            break;
          }
      } else {
        FO = m6 * (d2 * FF0 + DD0 * FFL);
        DO = DD0 * 0.5;
      }
    };
    const long long sI = 1, sJ = NI, sK = (long long)NI * NJ;
    for (int K = 2; K <= NK - 1; ++K)
      for (int J = 2; J <= NJ - 1; ++J)
        for (int I = 2; I <= NI - 1; ++I) {
          const size_t c = id(I, J, K);
          const int NF0 = NF[c];
          const double FF0 = FF[c];
          if (!(NF0 > 0 && FF0 >= P.flower && FF0 <= P.fupper)) continue;
          double FM, FP, DM, DP, S1, S2, S3;
          auto bc = [&](int l, double &v) {
            if (l < 1 || l > NB) return false;
            v = BCF[l - 1];
            return true;
          };
          double bm = 0.0, bp = 0.0;
          // x: cross-axis partners NF0 = 3 (J+1), 4 (J-1), 5 (K+1), 6 (K-1)
          {
            const int ns[4] = {3, 4, 5, 6};
            const long long off[4] = {sJ, -sJ, sK, -sK};
            int nm = NF[c - sI], np = NF[c + sI];
            if (nm == -1 && !bc(INDX[c], bm)) return CADMAS_EPG;
            if (np == -1 && !bc(INDX[c + sI], bp)) return CADMAS_EPG;
            side(NF0, FF0, c - sI, nm, bm, ns, off, X_(2, I), X_(2, I - 1), X_(3, I), X_(6, I), FM, DM);
            side(NF0, FF0, c + sI, np, bp, ns, off, X_(2, I), X_(2, I + 1), X_(3, I + 1), X_(6, I + 1), FP, DP);
            S1 = (DM + DP <= ZERO) ? 0.0 : (FM - FP) / (DM + DP);
          }
          {
            const int ns[4] = {1, 2, 5, 6};
            const long long off[4] = {sI, -sI, sK, -sK};
            int nm = NF[c - sJ], np = NF[c + sJ];
            if (nm == -1 && !bc(INDY[c], bm)) return CADMAS_EPG;
            if (np == -1 && !bc(INDY[c + sJ], bp)) return CADMAS_EPG;
            side(NF0, FF0, c - sJ, nm, bm, ns, off, Y_(2, J), Y_(2, J - 1), Y_(3, J), Y_(6, J), FM, DM);
            side(NF0, FF0, c + sJ, np, bp, ns, off, Y_(2, J), Y_(2, J + 1), Y_(3, J + 1), Y_(6, J + 1), FP, DP);
            S2 = (DM + DP <= ZERO) ? 0.0 : (FM - FP) / (DM + DP);
          }
          {
            const int ns[4] = {1, 2, 3, 4};
            const long long off[4] = {sI, -sI, sJ, -sJ};
            int nm = NF[c - sK], np = NF[c + sK];
            if (nm == -1 && !bc(INDZ[c], bm)) return CADMAS_EPG;
            if (np == -1 && !bc(INDZ[c + sK], bp)) return CADMAS_EPG;
            side(NF0, FF0, c - sK, nm, bm, ns, off, Z_(2, K), Z_(2, K - 1), Z_(3, K), Z_(6, K), FM, DM);
            side(NF0, FF0, c + sK, np, bp, ns, off, Z_(2, K), Z_(2, K + 1), Z_(3, K + 1), Z_(6, K + 1), FP, DP);
            S3 = (DM + DP <= ZERO) ? 0.0 : (FM - FP) / (DM + DP);
          }
          double RN = S1 * S1 + S2 * S2 + S3 * S3;
          if (RN >= ZERO) {
            RN = 1.0 / std::sqrt(RN);
            S1 = S1 * RN; S2 = S2 * RN; S3 = S3 * RN;
            int I1 = std::fabs(S1) >= 1.0e-4, I2 = std::fabs(S2) >= 1.0e-4, I3 = std::fabs(S3) >= 1.0e-4;
            if (I1 + I2 + I3 >= 2) { IST[c] = I1 + 2 * I2 + 4 * I3; SX[c] = S1; SY[c] = S2; SZ[c] = S3; }
          }
          ist_count[IST[c]]++;
          bool ok = true;
          switch (IST[c]) {
            case 0: break;
            case 3: ok = fslp2a(SX[c], SY[c], X_(2, I), Y_(2, J), FF[c], SA[c]); break;
            case 5: ok = fslp2a(SX[c], SZ[c], X_(2, I), Z_(2, K), FF[c], SA[c]); break;
            case 6: ok = fslp2a(SY[c], SZ[c], Y_(2, J), Z_(2, K), FF[c], SA[c]); break;
            default: ok = fslp3a(SX[c], SY[c], SZ[c], X_(2, I), Y_(2, J), Z_(2, K), FF[c], SA[c]); break;
          }
          if (!ok) rc = CADMAS_EPG;
        }
    return rc;
  }

  // VF_FCONVS  vf_fconvs.f:395-635: the face fluxes; a face whose donor
  // has a slope type usable across it (X: 3, 5, 7; Y: 3, 6, 7; Z: 5, 6,
  // 7) and INDX <= 1 takes the water under the donor's plane in the
  // swept strip, every other face the donor-acceptor flux of VF_FCONV.
  int fconvs(vd &FLFU, vd &FLFV, vd &FLFW) {
    std::vector<int> IST;
    vd SX, SY, SZ, SA;
    int rc = fslope(IST, SX, SY, SZ, SA);
    if (rc) return rc;
    const double DT = DTNOW, FL = P.flower;
    auto da = [&](double C, int N, double FDa, int ndm, double FDMa, double Vd, double Vo, double bcf, int na,
                  double FAa, int d1, int d2, int d3, int d4) {
      double AC = std::fabs(C), FD, FDMW, V, FA;
      if (N != -1) { FD = FDa; FDMW = 1.0; if (ndm != -1) FDMW = FDMa; V = Vd; }
      else { FD = bcf; FDMW = 1.0; V = Vo; }
      FA = (na != -1) ? FAa : FD;
      double FAD = FA;
      if (N == -1 || N == d1 || N == d2 || N == d3 || N == d4)
        if (FDMW != 0.0 && FA != 0.0) FAD = FD;
      double FDM = dmax(FDMW, FD);
      if (FDMW < FL && FA < FL) FDM = dmax(FDM, 0.1);
      double CFX = dmax((FDM - FAD) * AC - (FDM - FD) * V, 0.0);
      double FVX = FAD * AC + CFX;
      double FVM = FD * V;
      return dmin(FVX, FVM);
    };
    // Slope branch: the water that leaves is the donor's water below its
    // plane in the strip of width AC next to the face, capped at the
    // donor's content.  VF_FSLP2F/3F measure from the water side of the
    // cell: when the normal points along the flow (LSW = 1) the water
    // side is away from the face, and the strip's water is the donor's
    // water minus that of the other DX-AC.
    for (int K = 2; K <= NK - 1; ++K)
      for (int J = 2; J <= NJ - 1; ++J)
        for (int I = 2; I <= NI; ++I) {
          const size_t c = id(I, J, K);
          if (INDX[c] == -1) continue;
          double C = DT * GGX[c] * UU[c];
          int LSN, LA, LD, LDM;
          if (C >= 0.0) { LSN = 1; LA = I; LD = I - 1; LDM = I - 2; } else { LSN = -1; LA = I - 1; LD = I; LDM = I + 1; }
          const size_t d = id(LD, J, K);
          const int ist = IST[d];
          double fl;
          if (INDX[c] > 1 || ist <= 0 || ist == 6) {
            int N = NF[d];
            int ndm = (N != -1) ? NF[id(LDM, J, K)] : -1;
            double fdm = (N != -1 && ndm != -1) ? FF[id(LDM, J, K)] : 0.0;
            double vd_ = (N != -1) ? X_(2, LD) * GGV[d] : 0.0;
            double bcf = (N == -1) ? BCF[INDX[c] - 1] : 0.0;
            int na = NF[id(LA, J, K)];
            fl = da(C, N, (N != -1) ? FF[d] : 0.0, ndm, fdm, vd_, X_(2, LD), bcf, na,
                    (na != -1) ? FF[id(LA, J, K)] : 0.0, 3, 4, 5, 6);
          } else {
            double AC = std::fabs(C);
            int LSW = LSN;
            if (SX[d] < 0.0) LSW = -LSW;
            double DD0 = AC;
            if (LSW == 1) DD0 = X_(2, LD) - AC;
            double DFF;
            if (ist == 3) DFF = fslp2f(SX[d], SY[d], DD0, Y_(2, J), SA[d]);
            else if (ist == 5) DFF = fslp2f(SX[d], SZ[d], DD0, Z_(2, K), SA[d]);
            else DFF = fslp3f(SX[d], SY[d], SZ[d], DD0, Y_(2, J), Z_(2, K), SA[d]);
            double VG = X_(2, LD) * FF[d];
            double FVX = DFF * DD0;
            if (LSW == 1) FVX = VG - FVX;
            VG = VG * GGV[d];
            fl = dmin(FVX, VG);
          }
          FLFU[c] = FLFU[c] - (double)LSN * fl;
        }
    for (int K = 2; K <= NK - 1; ++K)
      for (int J = 2; J <= NJ; ++J)
        for (int I = 2; I <= NI - 1; ++I) {
          const size_t c = id(I, J, K);
          if (INDY[c] == -1) continue;
          double C = DT * GGY[c] * VV[c];
          int LSN, LA, LD, LDM;
          if (C >= 0.0) { LSN = 1; LA = J; LD = J - 1; LDM = J - 2; } else { LSN = -1; LA = J - 1; LD = J; LDM = J + 1; }
          const size_t d = id(I, LD, K);
          const int ist = IST[d];
          double fl;
          if (INDY[c] > 1 || ist <= 0 || ist == 5) {
            int N = NF[d];
            int ndm = (N != -1) ? NF[id(I, LDM, K)] : -1;
            double fdm = (N != -1 && ndm != -1) ? FF[id(I, LDM, K)] : 0.0;
            double vd_ = (N != -1) ? Y_(2, LD) * GGV[d] : 0.0;
            double bcf = (N == -1) ? BCF[INDY[c] - 1] : 0.0;
            int na = NF[id(I, LA, K)];
            fl = da(C, N, (N != -1) ? FF[d] : 0.0, ndm, fdm, vd_, Y_(2, LD), bcf, na,
                    (na != -1) ? FF[id(I, LA, K)] : 0.0, 1, 2, 5, 6);
          } else {
            double AC = std::fabs(C);
            int LSW = LSN;
            if (SY[d] < 0.0) LSW = -LSW;
            double DD0 = AC;
            if (LSW == 1) DD0 = Y_(2, LD) - AC;
            double DFF;
            if (ist == 3) DFF = fslp2f(SX[d], SY[d], X_(2, I), DD0, SA[d]);
            else if (ist == 6) DFF = fslp2f(SY[d], SZ[d], DD0, Z_(2, K), SA[d]);
            else DFF = fslp3f(SX[d], SY[d], SZ[d], X_(2, I), DD0, Z_(2, K), SA[d]);
            double VG = Y_(2, LD) * FF[d];
            double FVX = DFF * DD0;
            if (LSW == 1) FVX = VG - FVX;
            VG = VG * GGV[d];
            fl = dmin(FVX, VG);
          }
          FLFV[c] = FLFV[c] - (double)LSN * fl;
        }
    for (int K = 2; K <= NK; ++K)
      for (int J = 2; J <= NJ - 1; ++J)
        for (int I = 2; I <= NI - 1; ++I) {
          const size_t c = id(I, J, K);
          if (INDZ[c] == -1) continue;
          double C = DT * GGZ[c] * WW[c];
          int LSN, LA, LD, LDM;
          if (C >= 0.0) { LSN = 1; LA = K; LD = K - 1; LDM = K - 2; } else { LSN = -1; LA = K - 1; LD = K; LDM = K + 1; }
          const size_t d = id(I, J, LD);
          const int ist = IST[d];
          double fl;
          if (INDZ[c] > 1 || ist <= 0 || ist == 3) {
            int N = NF[d];
            int ndm = (N != -1) ? NF[id(I, J, LDM)] : -1;
            double fdm = (N != -1 && ndm != -1) ? FF[id(I, J, LDM)] : 0.0;
            double vd_ = (N != -1) ? Z_(2, LD) * GGV[d] : 0.0;
            double bcf = (N == -1) ? BCF[INDZ[c] - 1] : 0.0;
            int na = NF[id(I, J, LA)];
            fl = da(C, N, (N != -1) ? FF[d] : 0.0, ndm, fdm, vd_, Z_(2, LD), bcf, na,
                    (na != -1) ? FF[id(I, J, LA)] : 0.0, 1, 2, 3, 4);
          } else {
            double AC = std::fabs(C);
            int LSW = LSN;
            if (SZ[d] < 0.0) LSW = -LSW;
            double DD0 = AC;
            if (LSW == 1) DD0 = Z_(2, LD) - AC;
            double DFF;
            if (ist == 5) DFF = fslp2f(SX[d], SZ[d], X_(2, I), DD0, SA[d]);
            else if (ist == 6) DFF = fslp2f(SY[d], SZ[d], Y_(2, J), DD0, SA[d]);
            else DFF = fslp3f(SX[d], SY[d], SZ[d], X_(2, I), Y_(2, J), DD0, SA[d]);
            double VG = Z_(2, LD) * FF[d];
            double FVX = DFF * DD0;
            if (LSW == 1) FVX = VG - FVX;
            VG = VG * GGV[d];
            fl = dmin(FVX, VG);
          }
          FLFW[c] = FLFW[c] - (double)LSN * fl;
        }
    return CADMAS_OK;
  }

  // VF_FGENE  vf_fgene.f:42-70: QF of the wave source's line
  void fgene(vd &QF) const {
    const int IWS_ = IWS(), JWS_ = JWS();
    if (IWS_ == 0 && JWS_ == 0) return;
    for (int J = 2; J <= NJ - 1; ++J)
      for (int I = 2; I <= NI - 1; ++I)
        for (int K = 2; K <= NK - 1; ++K) {
          if (IWS_ == I) {
            const size_t c = id(I, J, K);
            if (NF[c] == -1) {
            } else if (NF[c] == 0) {
              double Q = 2.0 * X_(4, I) * SRC(J, K);
              QF[c] = QF[c] + FF[c] * Q;
            } else if (NF[c] != 8) {
              double Q = 2.0 * X_(4, I) * SRC(J, K);
              QF[c] = QF[c] + FF[c] * Q;
              break;
            }
          }
          if (JWS_ == J) {
            const size_t c = id(I, J, K);
            if (NF[c] == -1) {
            } else if (NF[c] == 0) {
              double Q = 2.0 * Y_(4, J) * SRC(I, K);
              QF[c] = QF[c] + FF[c] * Q;
            } else if (NF[c] != 8) {
              double Q = 2.0 * Y_(4, J) * SRC(I, K);
              QF[c] = QF[c] + FF[c] * Q;
              break;
            }
          }
        }
  }

  // VF_FEULER  vf_feuler.f:43-56 (GGV0 = GGV, LOOPS = 1); QF from VF_FGENE
  void feuler(const vd &FLFU, const vd &FLFV, const vd &FLFW) {
    vd QF;
    if (ISC != 0) { QF.assign(FF.size(), 0.0); fgene(QF); }
    for (int K = 2; K <= NK - 1; ++K)
      for (int J = 2; J <= NJ - 1; ++J)
        for (int I = 2; I <= NI - 1; ++I) {
          size_t c = id(I, J, K);
          if (NF[c] == -1) continue;
          double G0 = GGV[c] - (GGV[c] - GGV[c]) * 1.0;
          const double qf = ISC != 0 ? QF[c] : 0.0;
          double DF = (X_(4, I) * (FLFU[id(I + 1, J, K)] - FLFU[c]) + Y_(4, J) * (FLFV[id(I, J + 1, K)] - FLFV[c]) +
                       Z_(4, K) * (FLFW[id(I, J, K + 1)] - FLFW[c]) + DTNOW * qf);
          FF[c] = (G0 * FF[c] + DF) / GGV[c];
        }
  }

  // VF_FMOD1  vf_fmod1.f:37-200
  void fmod1() {
    std::fill(NLIM.begin(), NLIM.end(), 0);
    auto ends = [&](int I, int J, int K, int N, int &IE, int &JE, int &KE, int &IF, int &JF, int &KF) {
      IE = I; JE = J; KE = K; IF = I; JF = J; KF = K;
      if (N == 5) { KE = K + 1; KF = K - 1; }
      else if (N == 6) { KE = K - 1; KF = K + 1; }
      else if (N == 3) { JE = J + 1; JF = J - 1; }
      else if (N == 4) { JE = J - 1; JF = J + 1; }
      else if (N == 1) { IE = I + 1; IF = I - 1; }
      else if (N == 2) { IE = I - 1; IF = I + 1; }
    };
    for (int L = 0; L < NUMS; ++L) {
      int I, J, K, IE, JE, KE, IF, JF, KF;
      decode(INDS[L], I, J, K);
      ends(I, J, K, NF[id(I, J, K)], IE, JE, KE, IF, JF, KF);
      NLIM[id(IE, JE, KE)] += 1;
      NLIM[id(IF, JF, KF)] += 1;
    }
    for (int L = 0; L < NUMS; ++L) {
      int I, J, K, IE, JE, KE, IF, JF, KF;
      decode(INDS[L], I, J, K);
      ends(I, J, K, NF[id(I, J, K)], IE, JE, KE, IF, JF, KF);
      size_t e = id(IE, JE, KE), s = id(I, J, K), f = id(IF, JF, KF);
      double VE = X_(2, IE) * Y_(2, JE) * Z_(2, KE) * GGV[e];
      double VS = X_(2, I) * Y_(2, J) * Z_(2, K) * GGV[s];
      double VF = X_(2, IF) * Y_(2, JF) * Z_(2, KF) * GGV[f];
      double SS = VS * FF[s];
      if (NLIM[e] == 1) SS = SS + VE * FF[e];
      if (NLIM[f] == 1) SS = SS + VF * FF[f];
      double DS;
      if (NLIM[f] == 1) { DS = dmin(VF, SS); SS = SS - DS; FF[f] = DS / VF; }
      DS = dmin(VS, SS); SS = SS - DS; FF[s] = DS / VS;
      if (NLIM[e] == 1) { DS = dmin(VE, SS); SS = SS - DS; FF[e] = DS / VE; }
      if (SS > 0.0) {
        if (NLIM[e] == 1) FF[e] = FF[e] + SS / VE;
        else FF[s] = FF[s] + SS / VS;
      }
    }
    for (int L = 0; L < NUMS; ++L) {
      int I, J, K, IE, JE, KE, IF, JF, KF;
      decode(INDS[L], I, J, K);
      ends(I, J, K, NF[id(I, J, K)], IE, JE, KE, IF, JF, KF);
      size_t e = id(IE, JE, KE), s = id(I, J, K), f = id(IF, JF, KF);
      double VE = X_(2, IE) * Y_(2, JE) * Z_(2, KE) * GGV[e];
      double VS = X_(2, I) * Y_(2, J) * Z_(2, K) * GGV[s];
      double VF = X_(2, IF) * Y_(2, JF) * Z_(2, KF) * GGV[f];
      if (FF[s] > 1.0) { FF[e] = FF[e] + VS * (FF[s] - 1.0) / VE; FF[s] = 1.0; }
      if (FF[s] < 0.0) { FF[f] = FF[f] + VS * FF[s] / VF; FF[s] = 0.0; }
    }
  }

  // VF_FCUT01  vf_fcut01.f:34-56; in GPU order the cut-off of each cell is
  // applied first and both sums use the row tree.
  void fcut01(double &FSUM, double &FCUT) {
    if (sum_mode == ORC_SUM_REF) {
      FSUM = 0.0; FCUT = 0.0;
      for (int K = 2; K <= NK - 1; ++K)
        for (int J = 2; J <= NJ - 1; ++J)
          for (int I = 2; I <= NI - 1; ++I) {
            size_t c = id(I, J, K);
            if (NF[c] == -1) continue;
            double V = X_(2, I) * Y_(2, J) * Z_(2, K) * GGV[c];
            if (FF[c] > P.fupper) { FCUT = FCUT + (FF[c] - 1.0) * V; FF[c] = 1.0; }
            else if (FF[c] < P.flower) { FCUT = FCUT + (FF[c] - 0.0) * V; FF[c] = 0.0; }
            FSUM = FSUM + FF[c] * V;
          }
      return;
    }
    vd cut(FF.size(), 0.0);
    std::vector<char> hc(FF.size(), 0);
    for (int K = 2; K <= NK - 1; ++K)
      for (int J = 2; J <= NJ - 1; ++J)
        for (int I = 2; I <= NI - 1; ++I) {
          size_t c = id(I, J, K);
          if (NF[c] == -1) continue;
          double V = X_(2, I) * Y_(2, J) * Z_(2, K) * GGV[c];
          if (FF[c] > P.fupper) { cut[c] = (FF[c] - 1.0) * V; hc[c] = 1; FF[c] = 1.0; }
          else if (FF[c] < P.flower) { cut[c] = (FF[c] - 0.0) * V; hc[c] = 1; FF[c] = 0.0; }
        }
    FCUT = gsum([&](int I, int J, int K, double &c) {
      size_t q = id(I, J, K);
      if (!interior(I, J, K) || NF[q] == -1 || !hc[q]) return false;
      c = cut[q]; return true;
    });
    FSUM = gsum([&](int I, int J, int K, double &c) {
      size_t q = id(I, J, K);
      if (!interior(I, J, K) || NF[q] == -1) return false;
      double V = X_(2, I) * Y_(2, J) * Z_(2, K) * GGV[q];
      c = FF[q] * V; return true;
    });
  }

  // VF_BWFF  vf_bwff.f:31-89
  int bwff() {
    for (int L = 1; L <= NB; ++L) {
      int I, J, K;
      decode(IB_(1, L), I, J, K);
      int NS = IB_(2, L), IB = IB_(4, L);
      if (IB == 1) {
      } else if (IB == 2 || IB == 5 || IB == 7) {
        if (NS == 1) BCF[L - 1] = FF[id(I, J, K)];
        else if (NS == 2) BCF[L - 1] = FF[id(I - 1, J, K)];
        else if (NS == 3) BCF[L - 1] = FF[id(I, J, K)];
        else if (NS == 4) BCF[L - 1] = FF[id(I, J - 1, K)];
        else if (IB == 2 && NS == 5) BCF[L - 1] = FF[id(I, J, K)];
        else if (IB == 2 && NS == 6) BCF[L - 1] = FF[id(I, J, K - 1)];
        else return CADMAS_EPG;
      } else return CADMAS_EPG;
    }
    return CADMAS_OK;
  }

  // VF_BSUWEM  vf_bsuwem.f:37-103
  void bsuwem() {
    std::fill(NLIM.begin(), NLIM.end(), 0);
    for (int L = 0; L < NUMS; ++L) {
      int I, J, K;
      decode(INDS[L], I, J, K);
      int N = NF[id(I, J, K)];
      if (N == 5 || N == 6) { NLIM[id(I + 1, J, K)]++; NLIM[id(I - 1, J, K)]++; NLIM[id(I, J + 1, K)]++; NLIM[id(I, J - 1, K)]++; }
      else if (N == 3 || N == 4) { NLIM[id(I + 1, J, K)]++; NLIM[id(I - 1, J, K)]++; NLIM[id(I, J, K + 1)]++; NLIM[id(I, J, K - 1)]++; }
      else { NLIM[id(I, J + 1, K)]++; NLIM[id(I, J - 1, K)]++; NLIM[id(I, J, K + 1)]++; NLIM[id(I, J, K - 1)]++; }
    }
    for (int K = 2; K <= NK - 1; ++K)
      for (int J = 2; J <= NJ - 1; ++J)
        for (int I = 2; I <= NI - 1; ++I) {
          if (!(NLIM[id(I, J, K)] >= 2 && NF[id(I, J, K)] == 8)) continue;
          if (NF[id(I - 1, J, K)] == 8 && NLIM[id(I - 1, J, K)] < 2)
            if (NF[id(I + 1, J, K)] != 8) UU[id(I, J, K)] = UU[id(I + 1, J, K)];
          if (NF[id(I + 1, J, K)] == 8 && NLIM[id(I + 1, J, K)] < 2)
            if (NF[id(I - 1, J, K)] != 8) UU[id(I + 1, J, K)] = UU[id(I, J, K)];
          if (NF[id(I, J - 1, K)] == 8 && NLIM[id(I, J - 1, K)] < 2)
            if (NF[id(I, J + 1, K)] != 8) VV[id(I, J, K)] = VV[id(I, J + 1, K)];
          if (NF[id(I, J + 1, K)] == 8 && NLIM[id(I, J + 1, K)] < 2)
            if (NF[id(I, J - 1, K)] != 8) VV[id(I, J + 1, K)] = VV[id(I, J, K)];
          if (NF[id(I, J, K - 1)] == 8 && NLIM[id(I, J, K - 1)] < 2)
            if (NF[id(I, J, K + 1)] != 8) WW[id(I, J, K)] = WW[id(I, J, K + 1)];
          if (NF[id(I, J, K + 1)] == 8 && NLIM[id(I, J, K + 1)] < 2)
            if (NF[id(I, J, K - 1)] != 8) WW[id(I, J, K + 1)] = WW[id(I, J, K)];
        }
  }

  // VF_FNFINI  vf_fnfini.f:36-197
  int fnfini() {
    for (int K = 2; K <= NK - 1; ++K)
      for (int J = 1; J <= NJ; ++J)
        for (int I = 1; I <= NI; ++I)
          if (NF[id(I, J, K)] != -1) NF[id(I, J, K)] = 0;
    const double FU = P.fupper;
    for (int K = 2; K <= NK - 1; ++K)
      for (int J = 2; J <= NJ - 1; ++J)
        for (int I = 2; I <= NI - 1; ++I) {
          size_t c = id(I, J, K);
          if (NF[c] == -1 || !(FF[c] < P.flower)) continue;
          int IX1 = INDX[c], IX2 = INDX[id(I + 1, J, K)], IY1 = INDY[c], IY2 = INDY[id(I, J + 1, K)];
          int IZ1 = INDZ[c], IZ2 = INDZ[id(I, J, K + 1)];
          double FX1 = IX1 >= 1 ? BCF[IX1 - 1] : FF[id(I - 1, J, K)];
          double FX2 = IX2 >= 1 ? BCF[IX2 - 1] : FF[id(I + 1, J, K)];
          double FY1 = IY1 >= 1 ? BCF[IY1 - 1] : FF[id(I, J - 1, K)];
          double FY2 = IY2 >= 1 ? BCF[IY2 - 1] : FF[id(I, J + 1, K)];
          double FZ1 = IZ1 >= 1 ? BCF[IZ1 - 1] : FF[id(I, J, K - 1)];
          double FZ2 = IZ2 >= 1 ? BCF[IZ2 - 1] : FF[id(I, J, K + 1)];
          if (!(FZ1 > FU && IZ1 == 0) && !(FY1 > FU && IY1 == 0) && !(FY2 > FU && IY2 == 0) &&
              !(FX1 > FU && IX1 == 0) && !(FX2 > FU && IX2 == 0) && !(FZ2 > FU && IZ2 == 0))
            NF[c] = 8;
        }
    const int ICAP = 100000;
    for (int ITER = 1;; ++ITER) {
      if (ITER > ICAP) return CADMAS_ECAP;
      int NS = 0;
      INDS.clear();
      for (int K = 2; K <= NK - 1; ++K)
        for (int J = 2; J <= NJ - 1; ++J)
          for (int I = 2; I <= NI - 1; ++I) {
            size_t c = id(I, J, K);
            if (NF[c] == -1 || NF[c] == 8) continue;
            if (NF[id(I, J, K + 1)] == 8 || NF[id(I, J + 1, K)] == 8 || NF[id(I, J - 1, K)] == 8 ||
                NF[id(I + 1, J, K)] == 8 || NF[id(I - 1, J, K)] == 8 || NF[id(I, J, K - 1)] == 8) {
              NS++;
              INDS.push_back(I + NI * (J - 1) + NI * NJ * (K - 1));
              NF[c] = 7;
            }
          }
      std::vector<int> keep;
      for (int L = 0; L < NS; ++L) {
        int I, J, K;
        decode(INDS[L], I, J, K);
        if (NF[id(I, J, K + 1)] != 0 && NF[id(I, J + 1, K)] != 0 && NF[id(I, J - 1, K)] != 0 &&
            NF[id(I + 1, J, K)] != 0 && NF[id(I - 1, J, K)] != 0 && NF[id(I, J, K - 1)] != 0)
          NF[id(I, J, K)] = 8;
        else keep.push_back(INDS[L]);
      }
      INDS = keep;
      NUMS = (int)INDS.size();
      int NCH = 0;
      for (int L = 0; L < NUMS; ++L) {
        int I, J, K;
        decode(INDS[L], I, J, K);
        auto nf = [&](int a, int b, int c) { return NF[id(a, b, c)]; };
        if (nf(I, J, K - 1) != 0 || nf(I, J, K + 1) != 8)
          if (nf(I - 1, J, K) != 0 || nf(I + 1, J, K) != 8)
            if (nf(I + 1, J, K) != 0 || nf(I - 1, J, K) != 8)
              if (nf(I, J - 1, K) != 0 || nf(I, J + 1, K) != 8)
                if (nf(I, J + 1, K) != 0 || nf(I, J - 1, K) != 8)
                  if (nf(I, J, K + 1) != 0 || nf(I, J, K - 1) != 8) { NF[id(I, J, K)] = -7; NCH++; }
      }
      if (NCH <= 0) break;
      for (int L = 0; L < NUMS; ++L) {
        int I, J, K;
        decode(INDS[L], I, J, K);
        if (NF[id(I, J, K)] == -7) NF[id(I, J, K)] = 8;
      }
    }
    return CADMAS_OK;
  }

  // VF_FBUBUP  vf_fbubup.f:35-51
  void fbubup() {
    for (int K = NK - 2; K >= 2; --K) {
      double DTBUB = Z_(2, K) / P.wbub;
      if (!(TNOW - TBUB[K - 1] > DTBUB)) continue;
      int K1 = K + 1;
      for (int J = 2; J <= NJ - 1; ++J)
        for (int I = 2; I <= NI - 1; ++I) {
          size_t c = id(I, J, K), u = id(I, J, K1);
          if (FF[c] < P.fupper && NF[c] == 0 && NF[u] != -1) {
            double V0 = Z_(2, K) * GGV[c], V1 = Z_(2, K1) * GGV[u];
            double FMOVE = dmin((1.0 - FF[c]) * V0, FF[u] * V1);
            FF[u] = FF[u] - FMOVE / V1;
            FF[c] = FF[c] + FMOVE / V0;
          }
        }
      TBUB[K - 1] = TBUB[K - 1] + DTBUB;
    }
  }

  // VF_CDTCAL  vf_cdtcal.f:46-147 (no temperature or scalars: WK01 = ANU).
  // Reference order: the running DT = V/MAX(FL1..FL6, V/DT) in K,J,I order.
  // GPU order: the smallest of the cells' limits taken directly.
  double cdtcal(double dtinit, double dtmin, double dtmax, double dtsafe) {
    double DT = dtmax / dtsafe, M = DT;
    for (int K = 2; K <= NK - 1; ++K)
      for (int J = 2; J <= NJ - 1; ++J)
        for (int I = 2; I <= NI - 1; ++I) {
          const size_t c = id(I, J, K);
          if (NF[c] == -1) continue;
          const double DX = X_(2, I), DY = Y_(2, J), DZ = Z_(2, K);
          const double DXY = DX * DY, DXZ = DX * DZ, DYZ = DY * DZ, FC = FF[c];
          double V = GGV[c] * DX * DY * DZ;
          double FL[6] = {std::fabs(DYZ * GGX[c] * UU[c]), std::fabs(DYZ * GGX[id(I + 1, J, K)] * UU[id(I + 1, J, K)]),
                          std::fabs(DXZ * GGY[c] * VV[c]), std::fabs(DXZ * GGY[id(I, J + 1, K)] * VV[id(I, J + 1, K)]),
                          std::fabs(DXY * GGZ[c] * WW[c]), std::fabs(DXY * GGZ[id(I, J, K + 1)] * WW[id(I, J, K + 1)])};
          const int ind[6] = {INDX[c], INDX[id(I + 1, J, K)], INDY[c], INDY[id(I, J + 1, K)], INDZ[c],
                              INDZ[id(I, J, K + 1)]};
          for (int q = 0; q < 6; ++q)
            if (ind[q] >= 1 && dmax(FC, BCF[ind[q] - 1]) <= 0.0) FL[q] = 0.0;
          double FM = FL[0];
          for (int q = 1; q < 6; ++q) FM = dmax(FM, FL[q]);
          const double V2 = 0.5 / (1.0 / (DX * DX) + 1.0 / (DY * DY) + 1.0 / (DZ * DZ));
          if (sum_mode == ORC_SUM_REF) {
            DT = V / dmax(FM, V / DT);
            DT = V2 / dmax(ANU[c], V2 / DT);
          } else {
            if (FM > 0.0) M = dmin(M, V / FM);
            if (ANU[c] > 0.0) M = dmin(M, V2 / ANU[c]);
          }
        }
    if (sum_mode != ORC_SUM_REF) DT = M;
    const double W = (NNOW == 0) ? dtinit : DTNOW;
    return dmax(dmin(DT * dtsafe, 1.20 * W), dtmin);
  }

  // ----------------------------------------------------------- droplets
  // DROPTX..DROPWW of the TimerDoor droplet model; vf_cinit.f:412-427
  // starts every cell at (-1e10, 0, 0, 0, 0, 0).
  vd DTX, DTY, DTZ, DUU, DVV, DWW;
  vd DW[7];  // weighted sums of a directional pass
  void drop_clear(size_t c) {
    DTX[c] = -1.0e10; DTY[c] = 0.0; DTZ[c] = 0.0; DUU[c] = 0.0; DVV[c] = 0.0; DWW[c] = 0.0;
  }
  void drop_alloc() {
    const size_t N = (size_t)NI * NJ * NK;
    for (vd *a : {&DTX, &DTY, &DTZ, &DUU, &DVV, &DWW}) a->assign(N, 0.0);
    std::fill(DTX.begin(), DTX.end(), -1.0e10);
  }

  // VF_FDROPF  vf_fdropf.f:69-290.  A droplet cell is a gas cell (NF=8)
  // holding water (F > FLOWER).  A new one (DROPTX < 0) takes the mean
  // cell-centre velocity of the neighbours along its 12 edges that are
  // fluid and reachable past an open face, else of its 6 face neighbours
  // that are fluid or surface, else its own; on an obstacle it is at
  // rest.  An old one resting on an obstacle slides down the slope of the
  // porosity around it.  Every other cell loses its droplet values.
  void drop_start() {
    const double FL = P.flower;
    for (int K = 2; K <= NK - 1; ++K)
      for (int J = 2; J <= NJ - 1; ++J)
        for (int I = 2; I <= NI - 1; ++I) {
          const size_t c = id(I, J, K);
          if (!(FF[c] > FL && NF[c] == 8)) { drop_clear(c); continue; }
          if (DTX[c] < 0.0) {
            DTX[c] = TNOW; DTY[c] = TNOW; DTZ[c] = TNOW;
            int IP = 0;
            double UP = 0.0, VP = 0.0, WP = 0.0;
            auto take = [&](int i, int j, int k) {
              IP = IP + 1;
              UP = UP + 0.5 * (UU[id(i + 1, j, k)] + UU[id(i, j, k)]);
              VP = VP + 0.5 * (VV[id(i, j + 1, k)] + VV[id(i, j, k)]);
              WP = WP + 0.5 * (WW[id(i, j, k + 1)] + WW[id(i, j, k)]);
            };
            // edge neighbour (i1,j1,k1) reached past face cell a or b
            auto edge = [&](int i1, int j1, int k1, size_t a, size_t b) {
              if (NF[id(i1, j1, k1)] == 0 && (NF[a] != -1 || NF[b] != -1)) take(i1, j1, k1);
            };
            for (int dk = -1; dk <= 1; dk += 2)  // x-z plane (:79-114)
              for (int di = -1; di <= 1; di += 2) edge(I + di, J, K + dk, id(I + di, J, K), id(I, J, K + dk));
            for (int dj = -1; dj <= 1; dj += 2)  // x-y plane (:115-150)
              for (int di = -1; di <= 1; di += 2) edge(I + di, J + dj, K, id(I + di, J, K), id(I, J + dj, K));
            for (int dk = -1; dk <= 1; dk += 2)  // y-z plane (:151-186)
              for (int dj = -1; dj <= 1; dj += 2) edge(I, J + dj, K + dk, id(I, J + dj, K), id(I, J, K + dk));
            if (IP == 0) {  // face neighbours, fluid or surface (:188-231)
              const int nb[6][3] = {{-1, 0, 0}, {1, 0, 0}, {0, 0, -1}, {0, 0, 1}, {0, -1, 0}, {0, 1, 0}};
              for (auto &d : nb) {
                const int N1 = NF[id(I + d[0], J + d[1], K + d[2])];
                if (N1 != -1 && N1 != 8) take(I + d[0], J + d[1], K + d[2]);
              }
            }
            if (IP >= 1) {
              const double CP = 1.0 / (double)IP;
              DUU[c] = UP * CP; DVV[c] = VP * CP; DWW[c] = WP * CP;
            } else {
              DUU[c] = 0.5 * (UU[c] + UU[id(I + 1, J, K)]);
              DVV[c] = 0.5 * (VV[c] + VV[id(I, J + 1, K)]);
              DWW[c] = 0.5 * (WW[c] + WW[id(I, J, K + 1)]);
            }
            if (NF[id(I, J, K - 1)] == -1) { DUU[c] = 0.0; DVV[c] = 0.0; DWW[c] = 0.0; }
          } else if (NF[id(I, J, K - 1)] == -1) {  // sliding on an obstacle (:253-280)
            auto h = [&](size_t n) { return NF[n] == -1 ? 1.0 : 1.0 - GGV[n]; };
            double HX = 0.5 * (h(id(I + 1, J, K)) - h(id(I - 1, J, K))) * Z_(2, K);
            double HY = 0.5 * (h(id(I, J + 1, K)) - h(id(I, J - 1, K))) * Z_(2, K);
            HX = HX / X_(2, I);
            HY = HY / Y_(2, J);
            const double DN = 1.0 / (HX * HX + HY * HY + 1.0);
            HX = -(P.grz0 * HX * DN);
            HY = -(P.grz0 * HY * DN);
            DUU[c] = DUU[c] + DTNOW * HX;
            DVV[c] = DVV[c] + DTNOW * HY;
          }
        }
  }

  // VF_FDROPF  vf_fdropf.f:292-610: droplet water moves one cell along
  // axis ax (0 x, 1 y, 2 z), towards + (L = 1) or - (L = 2), once the time
  // to cross its cell has passed since the droplet last moved that way; the
  // droplet values of the cells that keep or receive water become the
  // water-weighted means.  The line is swept against the motion so water
  // moves at most one cell per pass.
  void drop_move(int ax, int L) {
    const double FL = P.flower, G = P.grz0;
    // WKTX..WKFF (the reference lends WK05..WK11; separate arrays here keep
    // the step's Poisson system readable by orc_get_poisson)
    vd &WTX = DW[0], &WTY = DW[1], &WTZ = DW[2], &WUU = DW[3], &WVV = DW[4], &WWW = DW[5], &WFF = DW[6];
    for (vd *a : {&WTX, &WTY, &WTZ, &WUU, &WVV, &WWW, &WFF})
      if (a->size() != FF.size()) a->assign(FF.size(), 0.0);
    for (int K = 2; K <= NK - 1; ++K)
      for (int J = 2; J <= NJ - 1; ++J)
        for (int I = 2; I <= NI - 1; ++I) {
          const size_t c = id(I, J, K);
          WTX[c] = 0.0; WTY[c] = 0.0; WTZ[c] = 0.0; WUU[c] = 0.0; WVV[c] = 0.0; WWW[c] = 0.0; WFF[c] = 0.0;
        }
    const int NA = ax == 0 ? NI : (ax == 1 ? NJ : NK);
    const int st = (L == 1) ? NA - 1 : 2, en = (L == 1) ? 2 : NA - 1, dl = (L == 1) ? -1 : 1;
    const double SG = (L == 1) ? 1.0 : -1.0;
    auto cell = [&](int I, int J, int K) {
      const int I1 = I - (ax == 0 ? dl : 0), J1 = J - (ax == 1 ? dl : 0), K1 = K - (ax == 2 ? dl : 0);
      const size_t c = id(I, J, K), c1 = id(I1, J1, K1);
      double DT = 0.0;
      const bool drop = FF[c] > FL && NF[c] == 8 && NF[c1] != -1;
      bool go = false;
      if (ax < 2) {
        const double D = ax == 0 ? DUU[c] : DVV[c];
        if (drop && SG * D > 0.0) {
          DT = (ax == 0 ? X_(2, I) : Y_(2, J)) / std::fabs(D);
          go = (TNOW - (ax == 0 ? DTX[c] : DTY[c])) > DT;
          if (!go) DT = 0.0;
        }
      } else if (drop) {
        const double X = std::sqrt(2.0 * G * Z_(2, K)), W = DWW[c];
        if (L == 1) {
          if (W > X) DT = (W - std::sqrt(W * W - X * X)) / G;
        } else if (W <= X) {
          if (W <= 0.0) DT = (W + std::sqrt(W * W + X * X)) / G;
          else DT = 2.0 * W / G;
        }
        go = DT > 0.0 && (TNOW - DTZ[c]) > DT;
        if (!go) DT = 0.0;
      }
      const double TX = DTX[c] + (ax == 0 ? DT : 0.0), TY = DTY[c] + (ax == 1 ? DT : 0.0),
                   TZ = DTZ[c] + (ax == 2 ? DT : 0.0), WW2 = ax == 2 ? DWW[c] - DT * G : DWW[c];
      // the unshifted values enter as they are (x + 0.0 would turn -0 into +0)
      auto tx = [&]() { return ax == 0 ? TX : DTX[c]; };
      auto ty = [&]() { return ax == 1 ? TY : DTY[c]; };
      auto tz = [&]() { return ax == 2 ? TZ : DTZ[c]; };
      auto ww = [&]() { return ax == 2 ? WW2 : DWW[c]; };
      if (go) {
        const double V0 = X_(2, I) * Y_(2, J) * Z_(2, K) * GGV[c];
        const double V1 = X_(2, I1) * Y_(2, J1) * Z_(2, K1) * GGV[c1];
        const double FMOVE = dmin((1.0 - FF[c1]) * V1, FF[c] * V0);
        FF[c] = FF[c] - FMOVE / V0;
        FF[c1] = FF[c1] + FMOVE / V1;
        if (NF[c1] == 8) {
          WTX[c1] = WTX[c1] + FMOVE * tx(); WTY[c1] = WTY[c1] + FMOVE * ty();
          WTZ[c1] = WTZ[c1] + FMOVE * tz(); WUU[c1] = WUU[c1] + FMOVE * DUU[c];
          WVV[c1] = WVV[c1] + FMOVE * DVV[c]; WWW[c1] = WWW[c1] + FMOVE * ww();
          WFF[c1] = WFF[c1] + FMOVE;
        }
      }
      if (FF[c] > FL && NF[c] == 8) {
        const double FOLD = FF[c] * X_(2, I) * Y_(2, J) * Z_(2, K) * GGV[c];
        WTX[c] = WTX[c] + FOLD * tx(); WTY[c] = WTY[c] + FOLD * ty();
        WTZ[c] = WTZ[c] + FOLD * tz(); WUU[c] = WUU[c] + FOLD * DUU[c];
        WVV[c] = WVV[c] + FOLD * DVV[c]; WWW[c] = WWW[c] + FOLD * ww();
        WFF[c] = WFF[c] + FOLD;
      } else {
        drop_clear(c);
      }
    };
    // the reference's loop nests: the swept index outermost
    for (int a = st; dl > 0 ? a <= en : a >= en; a += dl) {
      if (ax == 0) { for (int K = 2; K <= NK - 1; ++K) for (int J = 2; J <= NJ - 1; ++J) cell(a, J, K); }
      else if (ax == 1) { for (int K = 2; K <= NK - 1; ++K) for (int I = 2; I <= NI - 1; ++I) cell(I, a, K); }
      else { for (int J = 2; J <= NJ - 1; ++J) for (int I = 2; I <= NI - 1; ++I) cell(I, J, a); }
    }
    for (int K = 2; K <= NK - 1; ++K)
      for (int J = 2; J <= NJ - 1; ++J)
        for (int I = 2; I <= NI - 1; ++I) {
          const size_t c = id(I, J, K);
          if (!(FF[c] > FL && NF[c] == 8)) continue;
          const double W = 1.0 / WFF[c];
          DTX[c] = WTX[c] * W; DTY[c] = WTY[c] * W; DTZ[c] = WTZ[c] * W;
          DUU[c] = WUU[c] * W; DVV[c] = WVV[c] * W; DWW[c] = WWW[c] * W;
          if (ax == 2 && L == 1) {  // stopped under a ceiling (:590-597)
            const double X = std::sqrt(2.0 * G * Z_(2, K));
            if (NF[id(I, J, K + 1)] == -1 && DWW[c] > X) { DUU[c] = 0.0; DVV[c] = 0.0; DWW[c] = 0.0; }
          }
        }
  }

  // VF_FDROPF  vf_fdropf.f:63-671
  void fdropf() {
    if (DTX.size() != FF.size()) drop_alloc();
    drop_start();
    for (int ax = 0; ax < 3; ++ax)
      for (int L = 1; L <= 2; ++L) drop_move(ax, L);
  }

  // VF_FNFPRV  vf_fnfprv.f:34-225
  int fnfprv() {
    for (int L = 0; L < NUMS; ++L) {
      int I, J, K;
      decode(INDS[L], I, J, K);
      size_t c = id(I, J, K);
      double FM = -1.0, FS;
      auto bf = [&](int ind, double f) { return ind >= 1 ? BCF[ind - 1] : f; };
      int KB = K - 1;
      if (NF[id(I, J, KB)] == 0 && NF[id(I, J, K + 1)] == 8) {
        FS = 2.0 * FF[id(I, J, KB)];
        FS = FS + bf(INDX[id(I, J, KB)], FF[id(I - 1, J, KB)]);
        FS = FS + bf(INDX[id(I + 1, J, KB)], FF[id(I + 1, J, KB)]);
        FS = FS + bf(INDY[id(I, J, KB)], FF[id(I, J - 1, KB)]);
        FS = FS + bf(INDY[id(I, J + 1, KB)], FF[id(I, J + 1, KB)]);
        if (FS > FM) { NF[c] = 5; FM = FS; }
      }
      KB = K + 1;
      if (NF[id(I, J, KB)] == 0 && NF[id(I, J, K - 1)] == 8) {
        FS = 2.0 * FF[id(I, J, KB)];
        FS = FS + bf(INDX[id(I, J, KB)], FF[id(I - 1, J, KB)]);
        FS = FS + bf(INDX[id(I + 1, J, KB)], FF[id(I + 1, J, KB)]);
        FS = FS + bf(INDY[id(I, J, KB)], FF[id(I, J - 1, KB)]);
        FS = FS + bf(INDY[id(I, J + 1, KB)], FF[id(I, J + 1, KB)]);
        if (FS > FM) { NF[c] = 6; FM = FS; }
      }
      int JB = J - 1;
      if (NF[id(I, JB, K)] == 0 && NF[id(I, J + 1, K)] == 8) {
        FS = 2.0 * FF[id(I, JB, K)];
        FS = FS + bf(INDX[id(I, JB, K)], FF[id(I - 1, JB, K)]);
        FS = FS + bf(INDX[id(I + 1, JB, K)], FF[id(I + 1, JB, K)]);
        FS = FS + bf(INDZ[id(I, JB, K)], FF[id(I, JB, K - 1)]);
        FS = FS + bf(INDZ[id(I, JB, K + 1)], FF[id(I, JB, K + 1)]);
        if (FS > FM) { NF[c] = 3; FM = FS; }
      }
      JB = J + 1;
      if (NF[id(I, JB, K)] == 0 && NF[id(I, J - 1, K)] == 8) {
        FS = 2.0 * FF[id(I, JB, K)];
        FS = FS + bf(INDX[id(I, JB, K)], FF[id(I - 1, JB, K)]);
        FS = FS + bf(INDX[id(I + 1, JB, K)], FF[id(I + 1, JB, K)]);
        FS = FS + bf(INDZ[id(I, JB, K)], FF[id(I, JB, K - 1)]);
        FS = FS + bf(INDZ[id(I, JB, K + 1)], FF[id(I, JB, K + 1)]);
        if (FS > FM) { NF[c] = 4; FM = FS; }
      }
      int IB = I - 1;
      if (NF[id(IB, J, K)] == 0 && NF[id(I + 1, J, K)] == 8) {
        FS = 2.0 * FF[id(IB, J, K)];
        FS = FS + bf(INDY[id(IB, J, K)], FF[id(IB, J - 1, K)]);
        FS = FS + bf(INDY[id(IB, J + 1, K)], FF[id(IB, J + 1, K)]);
        FS = FS + bf(INDZ[id(IB, J, K)], FF[id(IB, J, K - 1)]);
        FS = FS + bf(INDZ[id(IB, J, K + 1)], FF[id(IB, J, K + 1)]);
        if (FS > FM) { NF[c] = 1; FM = FS; }
      }
      IB = I + 1;
      if (NF[id(IB, J, K)] == 0 && NF[id(I - 1, J, K)] == 8) {
        FS = 2.0 * FF[id(IB, J, K)];
        FS = FS + bf(INDY[id(IB, J, K)], FF[id(IB, J - 1, K)]);
        FS = FS + bf(INDY[id(IB, J + 1, K)], FF[id(IB, J + 1, K)]);
        FS = FS + bf(INDZ[id(IB, J, K)], FF[id(IB, J, K - 1)]);
        FS = FS + bf(INDZ[id(IB, J, K + 1)], FF[id(IB, J, K + 1)]);
        if (FS > FM) { NF[c] = 2; FM = FS; }
      }
      if (NF[c] == 7) return CADMAS_EPG;
    }
    return CADMAS_OK;
  }

  // VF_CINDC  vf_cindc.f:35-53
  void cindc() {
    for (int K = 2; K <= NK - 1; ++K)
      for (int J = 2; J <= NJ - 1; ++J)
        for (int I = 2; I <= NI - 1; ++I) {
          int n = NF[id(I, J, K)];
          INDC[id(I, J, K)] = (n == 8 || n == -1) ? -1 : 0;
        }
  }

  // VF_BSPPFL  vf_bsppfl.f:40-67 (NF0 = NF before FNFINI, kept in NLIM)
  void bsppfl() {
    vd PP0 = PP;
    for (int K = 2; K <= NK - 1; ++K)
      for (int J = 2; J <= NJ - 1; ++J)
        for (int I = 2; I <= NI - 1; ++I) {
          if (!(NF[id(I, J, K)] == 0 && NLIM[id(I, J, K)] == 8)) continue;
          double SUMF = 0.0, SUMP = 0.0;
          for (int KP = -1; KP <= 1; ++KP)
            for (int JP = -1; JP <= 1; ++JP)
              for (int IP = -1; IP <= 1; ++IP) {
                size_t q = id(I + IP, J + JP, K + KP);
                if (NF[q] == 0) { double F = FF[q]; SUMF = SUMF + F; SUMP = SUMP + F * PP0[q]; }
              }
          PP[id(I, J, K)] = (SUMF < 1.0e-20) ? 0.0 : SUMP / SUMF;
        }
  }

  // VF_BSPP  vf_bspp.f:33-61 (PVCP0 < 0)
  void bspp() {
    const double PPS = 0.0;
    for (int K = 2; K <= NK - 1; ++K)
      for (int J = 2; J <= NJ - 1; ++J)
        for (int I = 2; I <= NI - 1; ++I) {
          size_t c = id(I, J, K);
          int n = NF[c];
          double PSI;
          if (n == 8) PP[c] = 0.0;
          else if (n == 5) { PSI = Z_(3, K) / (0.5 * Z_(2, K - 1) + FF[c] * Z_(2, K)); PP[c] = (1.0 - PSI) * PP[id(I, J, K - 1)] + PSI * PPS; }
          else if (n == 6) { PSI = Z_(3, K + 1) / (0.5 * Z_(2, K + 1) + FF[c] * Z_(2, K)); PP[c] = (1.0 - PSI) * PP[id(I, J, K + 1)] + PSI * PPS; }
          else if (n == 3) { PSI = Y_(3, J) / (0.5 * Y_(2, J - 1) + FF[c] * Y_(2, J)); PP[c] = (1.0 - PSI) * PP[id(I, J - 1, K)] + PSI * PPS; }
          else if (n == 4) { PSI = Y_(3, J + 1) / (0.5 * Y_(2, J + 1) + FF[c] * Y_(2, J)); PP[c] = (1.0 - PSI) * PP[id(I, J + 1, K)] + PSI * PPS; }
          else if (n == 1) { PSI = X_(3, I) / (0.5 * X_(2, I - 1) + FF[c] * X_(2, I)); PP[c] = (1.0 - PSI) * PP[id(I - 1, J, K)] + PSI * PPS; }
          else if (n == 2) { PSI = X_(3, I + 1) / (0.5 * X_(2, I + 1) + FF[c] * X_(2, I)); PP[c] = (1.0 - PSI) * PP[id(I + 1, J, K)] + PSI * PPS; }
        }
  }

  // VF_CDIV00  vf_cdiv00.f:38-56
  double cdiv00() {
    double v = gsum([&](int I, int J, int K, double &c) {
      if (!interior(I, J, K)) return false;
      size_t q = id(I, J, K);
      if (INDC[q] == -1) return false;
      double VD = Y_(2, J) * Z_(2, K) * (GGX[id(I + 1, J, K)] * UU[id(I + 1, J, K)] - GGX[q] * UU[q]) +
                  X_(2, I) * Z_(2, K) * (GGY[id(I, J + 1, K)] * VV[id(I, J + 1, K)] - GGY[q] * VV[q]) +
                  X_(2, I) * Y_(2, J) * (GGZ[id(I, J, K + 1)] * WW[id(I, J, K + 1)] - GGZ[q] * WW[q]);
      c = VD * VD;
      return true;
    });
    return std::sqrt(v);
  }

  // VF_CWMSRC  vf_cwmsrc.f:46-143 (N = -3, the matrix table, or a wave
  // theory) at TDMY = TNOW: SRCUV of every line of the source
  int cwmsrc() {
    const double PI = 3.141592653589794, ZERO = 1.0e-20;
    const int IJ1 = 2, IJ2 = (ISC > 0 ? NJ : NI) - 1;
    const double D = SD, T = ST, T0 = STHEORY ? STH.phase0 : DMTBT0;
    double A = SA;
    float R4TN = (float)(T0 - TNOW / T);
    R4TN = R4TN - (float)(int)R4TN;
    if (R4TN < 0.0f) R4TN = R4TN + 1.0f;
    double AW = 1.0;
    if (A >= ZERO) {
      A = TNOW / T / A;
      if (A < 1.0) AW = 0.5 * std::sin(PI * (A - 0.5)) + 0.5;
    }
    const double WVT = (double)R4TN;
    double WMT1 = 0.0, WMT2 = 0.0, WVZ;
    if (STHEORY) WVZ = th_level(STH, WVT);
    else if (!cwmtb1(WVT, WMT1, WMT2, WVZ)) return CADMAS_EPG;
    const int NIJ = ISC > 0 ? NJ : NI;
    for (int IJ = IJ1; IJ <= IJ2; ++IJ) {
      const int I = ISC > 0 ? ISC : IJ, J = ISC > 0 ? IJ : -ISC;
      double VWS;
      if (STHEORY || MTBTYP == 1) {
        double VAL = 0.0;
        for (int K = 2; K <= NK - 1; ++K) {
          const int NW = NF[id(I, J, K)];
          if (NW == -1) VAL = VAL + Z_(2, K) * 1.0;
          else if (NW == 0) VAL = VAL + Z_(2, K) * FF[id(I, J, K)];
          else if (NW != 8) { VAL = VAL + Z_(2, K) * FF[id(I, J, K)]; break; }
        }
        VAL = VAL - (P.wvlvl - Z_(1, 2));
        VWS = (WVZ + D) / (VAL + D);
      } else {
        VWS = 1.0;
      }
      int KMT = 1;
      for (int K = 2; K <= NK - 1; ++K) {
        double ZC = (Z_(1, K) + Z_(1, K + 1)) * 0.5 - P.wvlvl;
        ZC = VWS * (ZC + D) - D;
        double UN, UT;
        if (STHEORY) th_velocity(STH, WVT, ZC, UN, UT);
        else if (!cwmtb2(KMT, WMT1, WMT2, ZC, UN, UT)) return CADMAS_EPG;
        SRCUV[(size_t)(IJ - 1) + (size_t)NIJ * (size_t)(K - 1)] = UN * VWS * AW;
      }
    }
    return CADMAS_OK;
  }

  // ---------------------------------------------------------------- drivers
  // VF_V1CAL  vf_v1cal.f:118-297 (ILOOP = 1), after the time loop's
  // VF_CWMSRC (vf_a1main.f:1035-1040)
  int v1cal() {
    Timer T;
    size_t N = UU.size();
    if (ISC != 0) { const int rs = cwmsrc(); if (rs) return rs; }
    T.start();
    for (int w = 1; w <= 12; ++w) WK[w].assign(N, 0.0);
    WK[13] = UU; WK[14] = VV; WK[15] = WW;
    vflxdu(WK[1], WK[2], WK[3]);
    vflxdv(WK[5], WK[6], WK[7]);
    vflxdw(WK[9], WK[10], WK[11]);
    vgene(WK[4], WK[8], WK[12]);
    veuler(WK[1], WK[2], WK[3], WK[4], WK[5], WK[6], WK[7], WK[8], WK[9], WK[10], WK[11], WK[12]);
    int rc = bwuwn(WK[13], WK[14], WK[15]);
    if (rc) return rc;
    tmr[0] += T.stop();
    T.start();
    rc = vpcoef(WK[1], WK[2], WK[3], WK[4], WK[5], WK[6], WK[7], WK[8]);
    if (rc) return rc;
    tmr[1] += T.stop();
    T.start();
    // VF_VPSOL vf_vpsol.f:52-76
    WK[9].assign(N, 0.0);
    double bn, xn; int it;
    m1bcgs(WK[1], WK[2], WK[3], WK[4], WK[5], WK[6], WK[7], WK[8], WK[9], INDC.data(), bn, xn, it);
    st.cgbnrm = bn; st.cgxnrm = xn; st.icgitr = it;
    tmr[2] += T.stop();
    if (it > P.icgmax) return CADMAS_ENOTCONV;
    if (it == -2) return CADMAS_EDIVERGE;
    if (it == -1) return CADMAS_EPIVOT;
    if (P.diag_relres) st.true_relres = true_relres(WK[1], WK[2], WK[3], WK[4], WK[5], WK[6], WK[7], WK[8], WK[9], INDC.data());
    T.start();
    vmodif(WK[9]);
    bsuwt(); bsuwt2(); bsuwn();
    int rcw = bwuwt();
    if (rcw) return rcw;
    bwpp();
    tmr[3] += T.stop();
    return CADMAS_OK;
  }

  // ------------------------------------------------------------ k-epsilon
  // VF_SCONVD  vf_sconvd.f:37-175 (ISW = -1: SU = SCMK): donor-cell flux
  // of CC through the faces next to a fluid cell.
  void sconvd(const vd &CC, const vd &BCC, const vi &INDBC, vd &FU, vd &FV, vd &FW) {
    const double SU = P.scmk, SC = 1.0 - SU;
    const size_t sI = 1, sJ = NI, sK = (size_t)NI * NJ;
    auto face = [&](size_t c, size_t m, double WIN, int IND, double w6, double wm, double wc, double &FL) {
      if (IND == 0) {
        double FLC = WIN * w6 * (wm * CC[c] + wc * CC[m]);
        FL = FL - SU * (dmax(WIN, 0.0) * CC[m] - dmax(-WIN, 0.0) * CC[c]) - SC * FLC;
      } else if (INDBC[IND - 1] >= 1) {
        double FLC = WIN * BCC[IND - 1];
        if (NF[c] == 0) {
          if (WIN >= 0.0) FL = FL - FLC;
          else FL = FL - SU * WIN * CC[c] - SC * FLC;
        } else {
          if (WIN <= 0.0) FL = FL - FLC;
          else FL = FL - SU * WIN * CC[m] - SC * FLC;
        }
      }
    };
    for (int K = 2; K <= NK - 1; ++K)
      for (int J = 2; J <= NJ - 1; ++J)
        for (int I = 2; I <= NI; ++I) {
          size_t c = id(I, J, K);
          if (NF[c - sI] * NF[c] == 0) face(c, c - sI, GGX[c] * UU[c], INDX[c], X_(6, I), X_(2, I - 1), X_(2, I), FU[c]);
        }
    for (int K = 2; K <= NK - 1; ++K)
      for (int J = 2; J <= NJ; ++J)
        for (int I = 2; I <= NI - 1; ++I) {
          size_t c = id(I, J, K);
          if (NF[c - sJ] * NF[c] == 0) face(c, c - sJ, GGY[c] * VV[c], INDY[c], Y_(6, J), Y_(2, J - 1), Y_(2, J), FV[c]);
        }
    for (int K = 2; K <= NK; ++K)
      for (int J = 2; J <= NJ - 1; ++J)
        for (int I = 2; I <= NI - 1; ++I) {
          size_t c = id(I, J, K);
          if (NF[c - sK] * NF[c] == 0) face(c, c - sK, GGZ[c] * WW[c], INDZ[c], Z_(6, K), Z_(2, K - 1), Z_(2, K), FW[c]);
        }
  }

  // VF_SDIFF  vf_sdiff.f:47-159 (ISW = -1: AL = 1): diffusive flux with
  // the diffusivity DD of the cells.
  void sdiff(const vd &CC, const vd &BCC, const vd &DDv, vd &FU, vd &FV, vd &FW) {
    const double AL = 1.0;
    const size_t sI = 1, sJ = NI, sK = (size_t)NI * NJ;
    // w6, wm, wc: metric 6 and the widths of the face's two cells; w5 the
    // metric 5 of the face; w4c, w4m the metric 4 of the two cells
    auto face = [&](size_t c, size_t m, double G, int IND, double w6, double wm, double wc, double w5, double w4c,
                    double w4m, double &FL) {
      if (IND == 0) {
        double D = w6 * (wm * DDv[c] + wc * DDv[m]);
        D = D * AL;
        FL = FL + G * D * w5 * (CC[c] - CC[m]);
      } else {
        double CW = BCC[IND - 1];
        if (NF[c] == 0) {
          double D = DDv[c] * AL;
          FL = FL + G * D * w4c * (CC[c] - CW) * 2.0;
        } else {
          double D = DDv[m] * AL;
          FL = FL + G * D * w4m * (CW - CC[m]) * 2.0;
        }
      }
    };
    for (int K = 2; K <= NK - 1; ++K)
      for (int J = 2; J <= NJ - 1; ++J)
        for (int I = 2; I <= NI; ++I) {
          size_t c = id(I, J, K);
          if (NF[c - sI] * NF[c] == 0)
            face(c, c - sI, GGX[c], INDX[c], X_(6, I), X_(2, I - 1), X_(2, I), X_(5, I), X_(4, I), X_(4, I - 1), FU[c]);
        }
    for (int K = 2; K <= NK - 1; ++K)
      for (int J = 2; J <= NJ; ++J)
        for (int I = 2; I <= NI - 1; ++I) {
          size_t c = id(I, J, K);
          if (NF[c - sJ] * NF[c] == 0)
            face(c, c - sJ, GGY[c], INDY[c], Y_(6, J), Y_(2, J - 1), Y_(2, J), Y_(5, J), Y_(4, J), Y_(4, J - 1), FV[c]);
        }
    for (int K = 2; K <= NK; ++K)
      for (int J = 2; J <= NJ - 1; ++J)
        for (int I = 2; I <= NI - 1; ++I) {
          size_t c = id(I, J, K);
          if (NF[c - sK] * NF[c] == 0)
            face(c, c - sK, GGZ[c], INDZ[c], Z_(6, K), Z_(2, K - 1), Z_(2, K), Z_(5, K), Z_(4, K), Z_(4, K - 1), FW[c]);
        }
  }

  // VF_KGENE  vf_kgene.f:51-182: production and dissipation of the fluid
  // cells (GT = 0: no buoyancy term).
  void kgene(vd &QK, vd &QE) {
    const double ZERO = 1.0e-20;
    for (int K = 2; K <= NK - 1; ++K)
      for (int J = 2; J <= NJ - 1; ++J)
        for (int I = 2; I <= NI - 1; ++I) {
          size_t c = id(I, J, K);
          if (NF[c] != 0) continue;
          const int IM = I - 1, IP = I + 1, JM = J - 1, JP = J + 1, KM = K - 1, KP = K + 1;
          double UXM = UU[id(I, J, K)], UXP = UU[id(IP, J, K)];
          double VYM = VV[id(I, J, K)], VYP = VV[id(I, JP, K)];
          double WZM = WW[id(I, J, K)], WZP = WW[id(I, J, KP)];
          double VXM, WXM, VXP, WXP, UYM, WYM, UYP, WYP, UZM, VZM, UZP, VZP;
          int IND = INDX[id(I, J, K)];
          if (IND == 0) {
            VXM = 0.5 * X_(6, I) * (X_(2, IM) * (VV[id(I, J, K)] + VV[id(I, JP, K)]) + X_(2, I) * (VV[id(IM, J, K)] + VV[id(IM, JP, K)]));
            WXM = 0.5 * X_(6, I) * (X_(2, IM) * (WW[id(I, J, K)] + WW[id(I, J, KP)]) + X_(2, I) * (WW[id(IM, J, K)] + WW[id(IM, J, KP)]));
          } else { VXM = BCV[IND - 1]; WXM = BCW[IND - 1]; }
          IND = INDX[id(IP, J, K)];
          if (IND == 0) {
            VXP = 0.5 * X_(6, IP) * (X_(2, I) * (VV[id(IP, J, K)] + VV[id(IP, JP, K)]) + X_(2, IP) * (VV[id(I, J, K)] + VV[id(I, JP, K)]));
            WXP = 0.5 * X_(6, IP) * (X_(2, I) * (WW[id(IP, J, K)] + WW[id(IP, J, KP)]) + X_(2, IP) * (WW[id(I, J, K)] + WW[id(I, J, KP)]));
          } else { VXP = BCV[IND - 1]; WXP = BCW[IND - 1]; }
          IND = INDY[id(I, J, K)];
          if (IND == 0) {
            UYM = 0.5 * Y_(6, J) * (Y_(2, JM) * (UU[id(I, J, K)] + UU[id(IP, J, K)]) + Y_(2, J) * (UU[id(I, JM, K)] + UU[id(IP, JM, K)]));
            WYM = 0.5 * Y_(6, J) * (Y_(2, JM) * (WW[id(I, J, K)] + WW[id(I, J, KP)]) + Y_(2, J) * (WW[id(I, JM, K)] + WW[id(I, JM, KP)]));
          } else { UYM = BCU[IND - 1]; WYM = BCW[IND - 1]; }
          IND = INDY[id(I, JP, K)];
          if (IND == 0) {
            UYP = 0.5 * Y_(6, JP) * (Y_(2, J) * (UU[id(I, JP, K)] + UU[id(IP, JP, K)]) + Y_(2, JP) * (UU[id(I, J, K)] + UU[id(IP, J, K)]));
            WYP = 0.5 * Y_(6, JP) * (Y_(2, J) * (WW[id(I, JP, K)] + WW[id(I, JP, KP)]) + Y_(2, JP) * (WW[id(I, J, K)] + WW[id(I, J, KP)]));
          } else { UYP = BCU[IND - 1]; WYP = BCW[IND - 1]; }
          IND = INDZ[id(I, J, K)];
          if (IND == 0) {
            UZM = 0.5 * Z_(6, K) * (Z_(2, KM) * (UU[id(I, J, K)] + UU[id(IP, J, K)]) + Z_(2, K) * (UU[id(I, J, KM)] + UU[id(IP, J, KM)]));
            VZM = 0.5 * Z_(6, K) * (Z_(2, KM) * (VV[id(I, J, K)] + VV[id(I, JP, K)]) + Z_(2, K) * (VV[id(I, J, KM)] + VV[id(I, JP, KM)]));
          } else { UZM = BCU[IND - 1]; VZM = BCV[IND - 1]; }
          IND = INDZ[id(I, J, KP)];
          if (IND == 0) {
            UZP = 0.5 * Z_(6, KP) * (Z_(2, K) * (UU[id(I, J, KP)] + UU[id(IP, J, KP)]) + Z_(2, KP) * (UU[id(I, J, K)] + UU[id(IP, J, K)]));
            VZP = 0.5 * Z_(6, KP) * (Z_(2, K) * (VV[id(I, J, KP)] + VV[id(I, JP, KP)]) + Z_(2, KP) * (VV[id(I, J, K)] + VV[id(I, JP, K)]));
          } else { UZP = BCU[IND - 1]; VZP = BCV[IND - 1]; }
          double DLR = X_(4, I);
          double DUDX = DLR * (UXP - UXM), DVDX = DLR * (VXP - VXM), DWDX = DLR * (WXP - WXM);
          DLR = Y_(4, J);
          double DUDY = DLR * (UYP - UYM), DVDY = DLR * (VYP - VYM), DWDY = DLR * (WYP - WYM);
          DLR = Z_(4, K);
          double DUDZ = DLR * (UZP - UZM), DVDZ = DLR * (VZP - VZM), DWDZ = DLR * (WZP - WZM);
          double GS = ANUT[c] * (2.0 * (DUDX * DUDX + DVDY * DVDY + DWDZ * DWDZ) + ipow(DUDY + DVDX, 2) +
                                 ipow(DVDZ + DWDY, 2) + ipow(DWDX + DUDZ, 2));
          double GT = 0.0;
          double GST = GS + GT;
          double RF = -GT / dmax(GST, ZERO);
          double AK0 = dmax(AK[c], P.akmink);
          double AE0 = AEPS[c];
          double AEK = AE0 / AK0;
          double GG = GGV[c];
          QK[c] = QK[c] + GG * (GST - AE0);
          QE[c] = QE[c] + GG * (P.akc1 * AEK * GST * (1.0 + P.akc3 * RF) - P.akc2 * AEK * AE0);
        }
  }

  // VF_SEULER  vf_seuler.f:43-56 (GGV0 = GGV): Euler step of the fluid cells.
  void seuler(vd &CC, const vd &FU, const vd &FV, const vd &FW, const vd &QC) {
    for (int K = 2; K <= NK - 1; ++K)
      for (int J = 2; J <= NJ - 1; ++J)
        for (int I = 2; I <= NI - 1; ++I) {
          size_t c = id(I, J, K);
          if (NF[c] != 0) continue;
          double G0 = GGV[c] - (GGV[c] - GGV[c]) * 1.0;
          double DS = (X_(4, I) * (FU[id(I + 1, J, K)] - FU[c]) + Y_(4, J) * (FV[id(I, J + 1, K)] - FV[c]) +
                       Z_(4, K) * (FW[id(I, J, K + 1)] - FW[c]) + QC[c]);
          CC[c] = (G0 * CC[c] + DTNOW * DS) / GGV[c];
        }
  }

  // VF_BSSS  vf_bsss.f:27-66: gas cells 0, surface cells the mean of their
  // fluid neighbours (none is written in the pass, so it is in place).
  void bsss(vd &SC) {
    for (int K = 2; K <= NK - 1; ++K)
      for (int J = 2; J <= NJ - 1; ++J)
        for (int I = 2; I <= NI - 1; ++I) {
          size_t c = id(I, J, K);
          if (NF[c] == 8) SC[c] = 0.0;
          else if (NF[c] >= 1) {
            int N = 0;
            double S = 0.0;
            const size_t nb[6] = {id(I - 1, J, K), id(I + 1, J, K), id(I, J - 1, K), id(I, J + 1, K), id(I, J, K - 1),
                                  id(I, J, K + 1)};
            for (int q = 0; q < 6; ++q)
              if (NF[nb[q]] == 0) { N = N + 1; S = S + SC[nb[q]]; }
            SC[c] = S / (double)N;
          }
        }
  }

  // VF_BWKE  vf_bwke.f:33-108: boundary values of k and e.
  int bwke() {
    for (int L = 1; L <= NB; ++L) {
      int I, J, K;
      decode(IB_(1, L), I, J, K);
      const int NS = IB_(2, L), IBK = std::abs(INDBK[L - 1]), IBE = std::abs(INDBE[L - 1]);
      size_t c;
      if (NS == 1) c = id(I, J, K);
      else if (NS == 2) c = id(I - 1, J, K);
      else if (NS == 3) c = id(I, J, K);
      else if (NS == 4) c = id(I, J - 1, K);
      else if (NS == 5) c = id(I, J, K);
      else c = id(I, J, K - 1);
      const double AKC = AK[c], AEC = AEPS[c];
      if (IBK == 1) BCK[L - 1] = BCK[L - 1];
      else if (IBK == 2 || IBK == 6 || IBK == 8) BCK[L - 1] = AKC;
      else return CADMAS_EPG;
      if (IBE == 1) BCE[L - 1] = BCE[L - 1];
      else if (IBE == 2 || IBE == 6 || IBE == 8) BCE[L - 1] = AEC;
      else return CADMAS_EPG;
    }
    return CADMAS_OK;
  }

  // VF_CNUT0  vf_cnut0.f:37-49 and VF_CNU00  vf_cnu00.f:52-61: the eddy
  // viscosity C_mu k^2 / max(e, AKMINE) and ANU = ANU0 + ANUT.
  void cnut0() {
    for (int K = 2; K <= NK - 1; ++K)
      for (int J = 2; J <= NJ - 1; ++J)
        for (int I = 2; I <= NI - 1; ++I) {
          size_t c = id(I, J, K);
          if (NF[c] != -1) {
            double W = dmax(AEPS[c], P.akmine);
            ANUT[c] = P.akcmu * AK[c] * AK[c] / W;
          } else ANUT[c] = 0.0;
        }
  }
  void cnu00() {
    for (int K = 2; K <= NK - 1; ++K)
      for (int J = 2; J <= NJ - 1; ++J)
        for (int I = 2; I <= NI - 1; ++I) {
          size_t c = id(I, J, K);
          ANU[c] = (NF[c] != -1) ? P.anu0 + ANUT[c] : 0.0;
        }
  }

  // VF_K1CAL  vf_k1cal.f:84-170 (ISCMK = 0; VF_BWKELG acts on log-law and
  // rough walls only, which cadmas_create refuses)
  // VF_BWKELG  vf_bwkelg.f:30-160: k and e of the fluid cells next to
  // log-law (6) or rough (8) faces from the faces' friction velocities.
  // The z count tests the y faces for two log-law faces, as the reference.
  int bwkelg() {
    const double ZERO = 1.0e-20;
    const double CMR = 1.0 / std::sqrt(P.akcmu), CKR = 1.0 / P.akk0;
    bool bad = false;
    for (int K = 2; K <= NK - 1; ++K)
      for (int J = 2; J <= NJ - 1; ++J)
        for (int I = 2; I <= NI - 1; ++I) {
          const size_t c = id(I, J, K);
          if (NF[c] != 0) continue;
          const int LXM = INDX[c], LXP = INDX[id(I + 1, J, K)], LYM = INDY[c], LYP = INDY[id(I, J + 1, K)];
          const int LZM = INDZ[c], LZP = INDZ[id(I, J, K + 1)];
          int IXM = 0, IXP = 0, IYM = 0, IYP = 0, IZM = 0, IZP = 0;
          if (LXM >= 1) IXM = IB_(3, LXM);
          if (LXP >= 1) IXP = IB_(3, LXP);
          if (LYM >= 1) IYM = IB_(3, LYM);
          if (LYP >= 1) IYP = IB_(3, LYP);
          if (LZM >= 1) IZM = IB_(3, LZM);
          if (LZP >= 1) IZP = IB_(3, LZP);
          if (!(IXM == 6 || IXP == 6 || IYM == 6 || IYP == 6 || IZM == 6 || IZP == 6 || IXM == 8 || IXP == 8 ||
                IYM == 8 || IYP == 8 || IZM == 8 || IZP == 8))
            continue;
          const double UC = (UU[c] + UU[id(I + 1, J, K)]) * 0.5;
          const double VC = (VV[c] + VV[id(I, J + 1, K)]) * 0.5;
          const double WC = (WW[c] + WW[id(I, J, K + 1)]) * 0.5;
          const double VX = std::sqrt(VC * VC + WC * WC);
          const double VY = std::sqrt(UC * UC + WC * WC);
          const double VZ = std::sqrt(UC * UC + VC * VC);
          const double DX = X_(2, I) * 0.5, DY = Y_(2, J) * 0.5, DZ = Z_(2, K) * 0.5;
          double SX = 0.0, UT = 0.0;
          if (IXM == 6 || IXP == 6) {
            if (VX >= ZERO && P.anu0 >= ZERO) bad |= !cloglw(DX, VX, P.anu0, P.akk0, P.aka0, UT);
            SX = 1.0;
            if (IXM == 6 && IXP == 6) SX = 2.0;
          }
          double SY = 0.0, VT = 0.0;
          if (IYM == 6 || IYP == 6) {
            if (VY >= ZERO && P.anu0 >= ZERO) bad |= !cloglw(DY, VY, P.anu0, P.akk0, P.aka0, VT);
            SY = 1.0;
            if (IYM == 6 && IYP == 6) SY = 2.0;
          }
          double SZ = 0.0, WT = 0.0;
          if (IZM == 6 || IZP == 6) {
            if (VZ >= ZERO && P.anu0 >= ZERO) bad |= !cloglw(DZ, VZ, P.anu0, P.akk0, P.aka0, WT);
            SZ = 1.0;
            if (IYM == 6 && IYP == 6) SZ = 2.0;
          }
          double SXM = 0.0, UTM = 0.0, SXP = 0.0, UTP = 0.0, SYM = 0.0, VTM = 0.0, SYP = 0.0, VTP = 0.0;
          double SZM = 0.0, WTM = 0.0, SZP = 0.0, WTP = 0.0;
          if (IXM == 8) { if (VX >= ZERO) UTM = clogks(DX, VX, BCVI[LXM - 1], P.anu0, P.akk0, P.aka0); SXM = 1.0; }
          if (IXP == 8) { if (VX >= ZERO) UTP = clogks(DX, VX, BCVI[LXP - 1], P.anu0, P.akk0, P.aka0); SXP = 1.0; }
          if (IYM == 8) { if (VY >= ZERO) VTM = clogks(DY, VY, BCVI[LYM - 1], P.anu0, P.akk0, P.aka0); SYM = 1.0; }
          if (IYP == 8) { if (VY >= ZERO) VTP = clogks(DY, VY, BCVI[LYP - 1], P.anu0, P.akk0, P.aka0); SYP = 1.0; }
          if (IZM == 8) { if (VZ >= ZERO) WTM = clogks(DZ, VZ, BCVI[LZM - 1], P.anu0, P.akk0, P.aka0); SZM = 1.0; }
          if (IZP == 8) { if (VZ >= ZERO) WTP = clogks(DZ, VZ, BCVI[LZP - 1], P.anu0, P.akk0, P.aka0); SZP = 1.0; }
          const double SR = 1.0 / (SX + SY + SZ + SXM + SXP + SYM + SYP + SZM + SZP);
          AK[c] = CMR * (UT * UT * SX + VT * VT * SY + WT * WT * SZ + UTM * UTM * SXM + UTP * UTP * SXP +
                         VTM * VTM * SYM + VTP * VTP * SYP + WTM * WTM * SZM + WTP * WTP * SZP) * SR;
          AEPS[c] = CKR * (UT * UT * UT / DX * SX + VT * VT * VT / DY * SY + WT * WT * WT / DZ * SZ +
                           UTM * UTM * UTM / DX * SXM + UTP * UTP * UTP / DX * SXP + VTM * VTM * VTM / DY * SYM +
                           VTP * VTP * VTP / DY * SYP + WTM * WTM * WTM / DZ * SZM + WTP * WTP * WTP / DZ * SZP) * SR;
        }
    return bad ? CADMAS_ENOTCONV : CADMAS_OK;
  }

  int k1cal() {
    const size_t N = UU.size();
    vd FLKU(N, 0.0), FLKV(N, 0.0), FLKW(N, 0.0), QK(N, 0.0), FLEU(N, 0.0), FLEV(N, 0.0), FLEW(N, 0.0),
        QE(N, 0.0), WKNU(N, 0.0);
    sconvd(AK, BCK, INDBK, FLKU, FLKV, FLKW);
    sconvd(AEPS, BCE, INDBE, FLEU, FLEV, FLEW);
    double W = 1.0 / P.aksgk;
    for (int K = 2; K <= NK - 1; ++K)
      for (int J = 2; J <= NJ - 1; ++J)
        for (int I = 2; I <= NI - 1; ++I)
          if (NF[id(I, J, K)] != -1) WKNU[id(I, J, K)] = P.anu0 + ANUT[id(I, J, K)] * W;
    sdiff(AK, BCK, WKNU, FLKU, FLKV, FLKW);
    W = 1.0 / P.aksge;
    for (int K = 2; K <= NK - 1; ++K)
      for (int J = 2; J <= NJ - 1; ++J)
        for (int I = 2; I <= NI - 1; ++I)
          if (NF[id(I, J, K)] != -1) WKNU[id(I, J, K)] = P.anu0 + ANUT[id(I, J, K)] * W;
    sdiff(AEPS, BCE, WKNU, FLEU, FLEV, FLEW);
    kgene(QK, QE);
    seuler(AK, FLKU, FLKV, FLKW, QK);
    seuler(AEPS, FLEU, FLEV, FLEW, QE);
    if (NLOG > 0) {  // vf_k1cal.f:147-149
      const int rcl = bwkelg();
      if (rcl) return rcl;
    }
    for (int K = 2; K <= NK - 1; ++K)
      for (int J = 2; J <= NJ - 1; ++J)
        for (int I = 2; I <= NI - 1; ++I) {
          size_t c = id(I, J, K);
          if (NF[c] == 0) {
            if (AEPS[c] < P.akmine) { AK[c] = P.akmink; AEPS[c] = P.akmine; }
            else if (AK[c] < P.akmink) AK[c] = P.akmink;
          }
        }
    bsss(AK);
    bsss(AEPS);
    return bwke();
  }

  // After VF_F1CAL (vf_a1main.f:1119-1127): the new NF's surface and gas
  // values, the eddy viscosity, boundary values.
  int kpost() {
    if (NLOG > 0) {  // vf_a1main.f:1120
      const int rcl = bwkelg();
      if (rcl) return rcl;
    }
    bsss(AK);
    bsss(AEPS);
    cnut0();
    cnu00();
    int rc = bwke();
    if (rc) return rc;
    return bwuwt();
  }

  // VF_CINIT's k-epsilon part (vf_cinit.f:295-315, 359-364; the boundary
  // part 397-401 is kinit_bc)
  void kinit() {
    const size_t N = UU.size();
    AK.assign(N, 0.0); AEPS.assign(N, 0.0); ANUT.assign(N, 0.0);
    for (int K = 2; K <= NK - 1; ++K)
      for (int J = 2; J <= NJ - 1; ++J)
        for (int I = 2; I <= NI - 1; ++I)
          if (INDC[id(I, J, K)] != -1) { AK[id(I, J, K)] = P.akinik; AEPS[id(I, J, K)] = P.akinie; }
    cnut0();
    std::fill(ANU.begin(), ANU.end(), 0.0);
    cnu00();
  }
  int kinit_bc() {
    BCK = BCK0; BCE = BCE0;
    bsss(AK);
    bsss(AEPS);
    return bwke();
  }

  // VF_F1CAL  vf_f1cal.f:121-243
  int f1cal() {
    Timer T;
    T.start();
    size_t N = UU.size();
    vd FLFU(N, 0.0), FLFV(N, 0.0), FLFW(N, 0.0);
    std::fill(NLIM.begin(), NLIM.end(), 0);
    if (P.iscmff == 0) fconv(FLFU, FLFV, FLFW);  // vf_f1cal.f:138-146
    else {
      int rcs = fconvs(FLFU, FLFV, FLFW);
      if (rcs) return rcs;
    }
    feuler(FLFU, FLFV, FLFW);
    {
      const int rl = bwffsf();  // vf_f1cal.f:180
      if (rl) return rl;
    }
    fmod1();
    double fs, fc;
    fcut01(fs, fc);
    st.fsum = fs; st.fcut = fc;
    int rc = bwff();
    if (rc) return rc;
    bsuwn3();
    bsuwem();
    NLIM = NF;
    rc = fnfini();
    if (rc) return rc;
    if (P.wbub >= 1.0e-20) {
      fbubup();
      rc = fnfini();
      if (rc) return rc;
    }
    if (P.idrop >= 1) {  // vf_f1cal.f:212-217
      fdropf();
      rc = fnfini();
      if (rc) return rc;
    }
    rc = fnfprv();
    if (rc) return rc;
    cindc();
    bsppfl();
    bsuwt(); bsuwt2(); bsuwn3(); bspp();
    int rcw = bwuwt();
    if (rcw) return rcw;
    bwpp();
    st.nums = NUMS;
    tmr[4] += T.stop();
    return CADMAS_OK;
  }
};

// ============================================================================
extern "C" {

orc_handle *orc_create(const cadmas_dims *d, const cadmas_params *p, int sum_mode) {
  if (!d || !p || d->numi < 5 || d->numj < 3 || d->numk < 5 || d->numb < 0) return nullptr;
  orc_handle *h = new orc_handle();
  h->NI = d->numi; h->NJ = d->numj; h->NK = d->numk; h->NB = d->numb;
  h->P = *p;
  h->sum_mode = sum_mode;
  size_t N = (size_t)h->NI * h->NJ * h->NK;
  h->UU.assign(N, 0); h->VV.assign(N, 0); h->WW.assign(N, 0); h->PP.assign(N, 0); h->FF.assign(N, 0);
  h->NF.assign(N, -1); h->INDC.assign(N, -1); h->NLIM.assign(N, 0);
  size_t B = (size_t)std::max(h->NB, 1);
  h->BCU.assign(B, 0); h->BCV.assign(B, 0); h->BCW.assign(B, 0); h->BCP.assign(B, 0); h->BCF.assign(B, 0);
  h->BCVI.assign(B, 0.0);
  h->TBUB.assign(h->NK, 0.0);
  std::memset(&h->st, 0, sizeof(h->st));
  h->st.true_relres = -1.0;
  return h;
}

void orc_destroy(orc_handle *h) { delete h; }

int orc_upload_static(orc_handle *h, const cadmas_static *s) {
  size_t N = (size_t)h->NI * h->NJ * h->NK;
  h->XX.assign(s->xx, s->xx + 6 * h->NI);
  h->YY.assign(s->yy, s->yy + 6 * h->NJ);
  h->ZZ.assign(s->zz, s->zz + 6 * h->NK);
  h->GGV.assign(s->ggv, s->ggv + N); h->GGX.assign(s->ggx, s->ggx + N);
  h->GGY.assign(s->ggy, s->ggy + N); h->GGZ.assign(s->ggz, s->ggz + N);
  h->GLV.assign(s->glv, s->glv + N); h->GLX.assign(s->glx, s->glx + N);
  h->GLY.assign(s->gly, s->gly + N); h->GLZ.assign(s->glz, s->glz + N);
  h->CD0.assign(s->cd0, s->cd0 + N); h->ANU.assign(s->anu, s->anu + N);
  h->INDX.assign(s->indx, s->indx + N); h->INDY.assign(s->indy, s->indy + N);
  h->INDZ.assign(s->indz, s->indz + N);
  h->INDB.assign(s->indb, s->indb + 4 * (size_t)h->NB);
  if (h->NB == 0) h->INDB.assign(4, 0);
  h->BCVI.assign((size_t)std::max(h->NB, 1), 0.0);
  if (s->bcvi && h->NB > 0) h->BCVI.assign(s->bcvi, s->bcvi + h->NB);
  h->NLOG = 0;
  for (int L = 1; L <= h->NB; ++L) h->NLOG += (h->IB_(3, L) == 6 || h->IB_(3, L) == 8);
  if (h->P.leqk != 0) {
    if (!s->indbk || !s->indbe || !s->bck || !s->bce) return CADMAS_EINVAL;
    const size_t B = (size_t)h->NB;
    h->INDBK.assign(s->indbk, s->indbk + B); h->INDBE.assign(s->indbe, s->indbe + B);
    h->BCK0.assign(s->bck, s->bck + B); h->BCE0.assign(s->bce, s->bce + B);
    h->BCK = h->BCK0; h->BCE = h->BCE0;
    h->AK.assign(N, 0.0); h->AEPS.assign(N, 0.0); h->ANUT.assign(N, 0.0);
  }
  h->have_static = true;
  return CADMAS_OK;
}

int orc_set_state(orc_handle *h, const cadmas_state *s) {
  size_t N = (size_t)h->NI * h->NJ * h->NK, B = (size_t)h->NB;
  if (s->uu) h->UU.assign(s->uu, s->uu + N);
  if (s->vv) h->VV.assign(s->vv, s->vv + N);
  if (s->ww) h->WW.assign(s->ww, s->ww + N);
  if (s->pp) h->PP.assign(s->pp, s->pp + N);
  if (s->ff) h->FF.assign(s->ff, s->ff + N);
  if (s->nf) h->NF.assign(s->nf, s->nf + N);
  if (s->indc) h->INDC.assign(s->indc, s->indc + N);
  if (s->bcu) std::copy(s->bcu, s->bcu + B, h->BCU.begin());
  if (s->bcv) std::copy(s->bcv, s->bcv + B, h->BCV.begin());
  if (s->bcw) std::copy(s->bcw, s->bcw + B, h->BCW.begin());
  if (s->bcp) std::copy(s->bcp, s->bcp + B, h->BCP.begin());
  if (s->bcf) std::copy(s->bcf, s->bcf + B, h->BCF.begin());
  if (s->tbub) h->TBUB.assign(s->tbub, s->tbub + h->NK);
  h->TNOW = s->tnow; h->NNOW = s->nnow;
  // rebuild INDS in the order FNFINI produces (ascending linear index)
  h->INDS.clear();
  for (int K = 2; K <= h->NK - 1; ++K)
    for (int J = 2; J <= h->NJ - 1; ++J)
      for (int I = 2; I <= h->NI - 1; ++I) {
        int n = h->NF[h->id(I, J, K)];
        if (n >= 1 && n <= 7) h->INDS.push_back(I + h->NI * (J - 1) + h->NI * h->NJ * (K - 1));
      }
  h->NUMS = (int)h->INDS.size();
  return CADMAS_OK;
}

int orc_get_state(orc_handle *h, cadmas_state *s) {
  size_t B = (size_t)h->NB;
  if (s->uu) std::copy(h->UU.begin(), h->UU.end(), s->uu);
  if (s->vv) std::copy(h->VV.begin(), h->VV.end(), s->vv);
  if (s->ww) std::copy(h->WW.begin(), h->WW.end(), s->ww);
  if (s->pp) std::copy(h->PP.begin(), h->PP.end(), s->pp);
  if (s->ff) std::copy(h->FF.begin(), h->FF.end(), s->ff);
  if (s->nf) std::copy(h->NF.begin(), h->NF.end(), s->nf);
  if (s->indc) std::copy(h->INDC.begin(), h->INDC.end(), s->indc);
  if (s->bcu) std::copy(h->BCU.begin(), h->BCU.begin() + B, s->bcu);
  if (s->bcv) std::copy(h->BCV.begin(), h->BCV.begin() + B, s->bcv);
  if (s->bcw) std::copy(h->BCW.begin(), h->BCW.begin() + B, s->bcw);
  if (s->bcp) std::copy(h->BCP.begin(), h->BCP.begin() + B, s->bcp);
  if (s->bcf) std::copy(h->BCF.begin(), h->BCF.begin() + B, s->bcf);
  if (s->tbub) std::copy(h->TBUB.begin(), h->TBUB.end(), s->tbub);
  s->tnow = h->TNOW; s->nnow = h->NNOW;
  return CADMAS_OK;
}

// VF_CINIT vf_cinit.f:202-283 and the BC calls that follow it.
int orc_init_state(orc_handle *h, int hydrostatic) {
  if (!h->have_static) return CADMAS_ENOSTATIC;
  {
    const int rl = h->bwffsf();  // vf_cinit.f:177
    if (rl) return rl;
  }
  double fs, fc;
  h->fcut01(fs, fc);
  h->st.fsum = fs; h->st.fcut = fc;
  int rc = h->bwff();
  if (rc) return rc;
  rc = h->fnfini();
  if (rc) return rc;
  rc = h->fnfprv();
  if (rc) return rc;
  std::fill(h->INDC.begin(), h->INDC.end(), -1);
  h->cindc();
  if (hydrostatic) {
    std::fill(h->PP.begin(), h->PP.end(), 0.0);
    for (int K = 2; K <= h->NK - 1; ++K) {
      double VAL = h->P.rho0 * h->P.grz0 * (h->P.wvlvl - (h->Z_(1, K) + h->Z_(1, K + 1)) * 0.5);
      for (int J = 2; J <= h->NJ - 1; ++J)
        for (int I = 2; I <= h->NI - 1; ++I)
          if (h->INDC[h->id(I, J, K)] != -1) h->PP[h->id(I, J, K)] = VAL;
    }
  }
  {  // vf_cinit.f:376-390: the present velocities stand for the previous step's
    const vd ub = h->UU, vb = h->VV, wb = h->WW;
    rc = h->bwuwn(ub, vb, wb);
  }
  if (rc) return rc;
  if (h->P.leqk != 0) h->kinit();  // vf_cinit.f:295-315, 359-364
  h->bsuwt(); h->bsuwt2(); h->bsuwn3(); h->bspp();
  rc = h->bwuwt();
  if (rc) return rc;
  h->bwpp();
  if (h->P.leqk != 0) {  // vf_cinit.f:397-401
    rc = h->kinit_bc();
    if (rc) return rc;
  }
  std::fill(h->TBUB.begin(), h->TBUB.end(), 0.0);
  h->drop_alloc();  // vf_cinit.f:416-427
  h->st.nums = h->NUMS;
  return CADMAS_OK;
}

int orc_step(orc_handle *h, double dt) {
  if (!h->have_static) return CADMAS_ENOSTATIC;
  for (double &t : h->tmr) t = 0.0;
  h->DTNOW = dt;
  h->NNOW = h->NNOW + 1;
  h->TNOW = h->TNOW + h->DTNOW;
  int rc = h->v1cal();
  if (rc == CADMAS_OK && h->P.leqk != 0) rc = h->k1cal();  // vf_a1main.f:1093-1100
  if (rc == CADMAS_OK) rc = h->f1cal();
  if (rc == CADMAS_OK && h->P.leqk != 0) rc = h->kpost();  // vf_a1main.f:1119-1127
  h->st.last_status = rc;
  return rc;
}

int orc_get_stats(orc_handle *h, cadmas_stats *st) { *st = h->st; return CADMAS_OK; }

int orc_divnorm(orc_handle *h, double *val) {
  *val = h->cdiv00();
  h->st.divnorm = *val;
  return CADMAS_OK;
}

int orc_m1bcgs(orc_handle *h, const double *ad, const double *ali, const double *alj,
               const double *alk, const double *aui, const double *auj, const double *auk,
               const double *bb, double *x0, const int *indc, int *iter, double *bnorm,
               double *xnorm) {
  size_t N = (size_t)h->NI * h->NJ * h->NK;
  vd AD(ad, ad + N), ALI(ali, ali + N), ALJ(alj, alj + N), ALK(alk, alk + N), AUI(aui, aui + N),
      AUJ(auj, auj + N), AUK(auk, auk + N), BB(bb, bb + N), X(x0, x0 + N);
  h->m1bcgs(AD, ALI, ALJ, ALK, AUI, AUJ, AUK, BB, X, indc, *bnorm, *xnorm, *iter);
  std::copy(X.begin(), X.end(), x0);
  return CADMAS_OK;
}

int orc_get_poisson(orc_handle *h, int which, double *out) {
  if (which < 0 || which > 8) return CADMAS_EINVAL;
  const vd &a = h->WK[which + 1];
  if (a.empty()) return CADMAS_EINVAL;
  std::copy(a.begin(), a.end(), out);
  return CADMAS_OK;
}

// VF_COMAK0  vf_comak0.f:24-55 with BCTYP(6,JD) = WLN/T (vf_csetup.f:139-143)
int orc_open_speed(double depth, double period, double grav, double *c) {
  if (!c || !(depth > 0.0) || !(period > 0.0) || !(grav > 0.0)) return CADMAS_EINVAL;
  const double PI = 3.141592653589794;
  const double D = 4.0 * PI * PI * depth / grav / period / period;
  double X = D >= 1.0 ? D : std::sqrt(D);
  for (int ITR = 1; ITR <= 10; ++ITR) {
    const double EXPX = std::exp(X), EXPXI = 1.0 / EXPX;
    const double COTHX = (EXPX + EXPXI) / (EXPX - EXPXI);
    const double DX = (X - D * COTHX) / (1.0 + D * (COTHX * COTHX - 1.0));
    X = X - DX;
    if (std::fabs(DX / X) <= 1.0e-10) break;
  }
  *c = 2.0 * PI * depth / X / period;
  return std::isfinite(*c) ? CADMAS_OK : CADMAS_EINVAL;
}

int orc_set_open(orc_handle *h, int side, double depth, double period) {
  if (!h || side < 1 || side > 4 || h->WV[side - 1].on) return CADMAS_EINVAL;
  double c;
  const int rc = orc_open_speed(depth, period, h->P.grz0, &c);
  if (rc) return rc;
  h->OP[side - 1].on = 1;
  h->OP[side - 1].c = c;
  return CADMAS_OK;
}

int orc_set_wave(orc_handle *h, const cadmas_wave_bc *w, const cadmas_wave_table *t) {
  if (!h || !w || !t || w->side < 1 || w->side > 4 || t->ntt < 2 || t->nzz < 2) return CADMAS_EINVAL;
  if (h->OP[w->side - 1].on) return CADMAS_EINVAL;
  if (t->mtbtyp < 1 || t->mtbtyp > 3) return CADMAS_EINVAL;
  h->DMTBTT.assign(t->tt, t->tt + t->ntt);
  h->DMTBHH.assign(t->hh, t->hh + t->ntt);
  h->DMTBZZ.assign(t->zz, t->zz + t->nzz);
  h->DMTBUN.assign(t->un, t->un + (size_t)t->nzz * t->ntt);
  h->DMTBUT.assign(t->ut, t->ut + (size_t)t->nzz * t->ntt);
  h->MTBTYP = t->mtbtyp;
  h->DMTBT0 = t->phase0;
  orc_handle::Wave &v = h->WV[w->side - 1];
  v.on = 1; v.l1 = w->first; v.l2 = w->last; v.d = w->depth; v.t = w->period; v.a = w->ramp;
  v.theory = 0;
  return CADMAS_OK;
}

int orc_set_wave_theory(orc_handle *h, const cadmas_wave_bc *w, const cadmas_stream_wave *sw) {
  if (!h || !w || !sw || w->side < 1 || w->side > 4 || sw->order < 1 || sw->order > CADMAS_STREAM_NMAX)
    return CADMAS_EINVAL;
  if (h->OP[w->side - 1].on) return CADMAS_EINVAL;
  cadmas_wave_theory th;
  std::memset(&th, 0, sizeof(th));
  th.type = sw->order;
  th.depth = sw->depth; th.period = sw->period; th.height = sw->height;
  th.length = (double)(float)sw->length;  // WVLENG = DBLE(R4L) (vf_cwmak0.f:50)
  th.phase0 = sw->phase0;
  th.stream = *sw;
  return orc_set_wave_func(h, w, &th);
}

int orc_set_wave_func(orc_handle *h, const cadmas_wave_bc *w, const cadmas_wave_theory *th) {
  if (!h || !w || !th || w->side < 1 || w->side > 4 || th->type == 0 || th->type < -2 || th->type > CADMAS_STREAM_NMAX)
    return CADMAS_EINVAL;
  if (h->OP[w->side - 1].on) return CADMAS_EINVAL;
  orc_handle::Wave &v = h->WV[w->side - 1];
  v.on = 1; v.l1 = w->first; v.l2 = w->last; v.d = w->depth; v.t = w->period; v.a = w->ramp;
  v.theory = 1; v.th = *th;
  return CADMAS_OK;
}

// VF_CWMAK1/VF_CWMAK2 of a solved wave theory at one phase and height
int orc_wave_eval(const cadmas_wave_theory *t, double phase, double z, double *eta, double *u, double *w) {
  if (!t || t->type == 0 || t->type < -2 || t->type > CADMAS_STREAM_NMAX) return CADMAS_EINVAL;
  if (eta) *eta = orc_handle::th_level(*t, phase);
  double uu, ww;
  orc_handle::th_velocity(*t, phase, z, uu, ww);
  if (u) *u = uu;
  if (w) *w = ww;
  return CADMAS_OK;
}

int orc_set_wave_angle(orc_handle *h, int side, double angle, double sx, double sy) {
  if (!h || side < 1 || side > 4 || !h->WV[side - 1].on || !h->WV[side - 1].theory) return CADMAS_EINVAL;
  orc_handle::Wave &v = h->WV[side - 1];
  v.ang = angle; v.sx = sx; v.sy = sy;
  return CADMAS_OK;
}

int orc_set_wave_source_func(orc_handle *h, const cadmas_wave_src *src, const cadmas_wave_theory *th) {
  if (!h || !src || src->line == 0 || !th || th->type == 0 || th->type < -2 || th->type > CADMAS_STREAM_NMAX)
    return CADMAS_EINVAL;
  h->ISC = src->line;
  h->SD = src->depth; h->ST = src->period; h->SA = src->ramp;
  h->STHEORY = 1;
  h->STH = *th;
  h->SRCUV.assign((size_t)(src->line > 0 ? h->NJ : h->NI) * h->NK, 0.0);
  return CADMAS_OK;
}

int orc_set_wave_source(orc_handle *h, const cadmas_wave_src *src, const cadmas_wave_table *t) {
  if (!h || !src || src->line == 0) return CADMAS_EINVAL;
  if (t) {
    if (t->ntt < 2 || t->nzz < 2 || t->mtbtyp < 1 || t->mtbtyp > 3) return CADMAS_EINVAL;
    h->DMTBTT.assign(t->tt, t->tt + t->ntt);
    h->DMTBHH.assign(t->hh, t->hh + t->ntt);
    h->DMTBZZ.assign(t->zz, t->zz + t->nzz);
    h->DMTBUN.assign(t->un, t->un + (size_t)t->nzz * t->ntt);
    h->DMTBUT.assign(t->ut, t->ut + (size_t)t->nzz * t->ntt);
    h->MTBTYP = t->mtbtyp;
    h->DMTBT0 = t->phase0;
  }
  if (h->DMTBZZ.empty() || h->MTBTYP == 3) return CADMAS_EINVAL;  // vf_csetup.f:267
  h->STHEORY = 0;
  h->ISC = src->line;
  h->SD = src->depth; h->ST = src->period; h->SA = src->ramp;
  h->SRCUV.assign((size_t)(src->line > 0 ? h->NJ : h->NI) * h->NK, 0.0);
  return CADMAS_OK;
}

int orc_get_timers(orc_handle *h, double *t5) {
  for (int i = 0; i < 5; ++i) t5[i] = h->tmr[i];
  return CADMAS_OK;
}

int orc_get_drop(orc_handle *h, double *tx, double *ty, double *tz, double *uu, double *vv, double *ww) {
  if (h->DTX.size() != h->FF.size()) h->drop_alloc();
  double *dst[6] = {tx, ty, tz, uu, vv, ww};
  const vd *src[6] = {&h->DTX, &h->DTY, &h->DTZ, &h->DUU, &h->DVV, &h->DWW};
  for (int a = 0; a < 6; ++a)
    if (dst[a]) std::copy(src[a]->begin(), src[a]->end(), dst[a]);
  return CADMAS_OK;
}

int orc_set_drop(orc_handle *h, const double *tx, const double *ty, const double *tz, const double *uu,
                 const double *vv, const double *ww) {
  if (h->DTX.size() != h->FF.size()) h->drop_alloc();
  const double *src[6] = {tx, ty, tz, uu, vv, ww};
  vd *dst[6] = {&h->DTX, &h->DTY, &h->DTZ, &h->DUU, &h->DVV, &h->DWW};
  for (int a = 0; a < 6; ++a)
    if (src[a]) std::copy(src[a], src[a] + dst[a]->size(), dst[a]->begin());
  return CADMAS_OK;
}

int orc_set_time(orc_handle *h, double tnow, double dtnow, int nnow) {
  h->TNOW = tnow; h->DTNOW = dtnow; h->NNOW = nnow;
  return CADMAS_OK;
}

int orc_cdtcal(orc_handle *h, double dtinit, double dtmin, double dtmax, double dtsafe, double *dt) {
  if (!h->have_static) return CADMAS_ENOSTATIC;
  *dt = h->cdtcal(dtinit, dtmin, dtmax, dtsafe);
  return CADMAS_OK;
}

int orc_get_turb(orc_handle *h, double *ak, double *ae, double *anut, double *anu, double *bck, double *bce) {
  if (h->P.leqk == 0) return CADMAS_EINVAL;
  auto put = [](const vd &v, double *o) { if (o) std::copy(v.begin(), v.end(), o); };
  put(h->AK, ak); put(h->AEPS, ae); put(h->ANUT, anut); put(h->ANU, anu); put(h->BCK, bck); put(h->BCE, bce);
  return CADMAS_OK;
}

int orc_set_turb(orc_handle *h, const double *ak, const double *ae, const double *bck, const double *bce) {
  if (h->P.leqk == 0 || !ak || !ae || !bck || !bce) return CADMAS_EINVAL;
  const size_t N = (size_t)h->NI * h->NJ * h->NK, B = (size_t)h->NB;
  h->AK.assign(ak, ak + N); h->AEPS.assign(ae, ae + N);
  h->BCK.assign(bck, bck + B); h->BCE.assign(bce, bce + B);
  h->cnut0();  // vf_ir1inp.f:339-340
  h->cnu00();
  return CADMAS_OK;
}

int orc_slope_counts(orc_handle *h, int *counts) {
  for (int i = 0; i < 8; ++i) counts[i] = h->ist_count[i];
  return CADMAS_OK;
}

double orc_slope_fn(int fn, double x) {
  switch (fn) {
    case 0: return slope_cbrt(x);
    case 1: return slope_atan(x);
    default: return slope_cos(x);
  }
}

double orc_ln(double x) { return ln_series(x); }

int orc_cloglw(double dl, double va, double anu0, double akk0, double aka0, double *vt) {
  return cloglw(dl, va, anu0, akk0, aka0, *vt) ? CADMAS_OK : CADMAS_ENOTCONV;
}

double orc_clogks(double dl, double va, double ks, double anu0, double akk0, double aka0) {
  return clogks(dl, va, ks, anu0, akk0, aka0);
}

int orc_fslp(int dim, const double *s, const double *d, double fval, double *aa, double *fback) {
  bool ok;
  if (dim == 2) {
    ok = fslp2a(s[0], s[1], d[0], d[1], fval, *aa);
    if (ok) *fback = fslp2f(s[0], s[1], d[0], d[1], *aa);
  } else {
    ok = fslp3a(s[0], s[1], s[2], d[0], d[1], d[2], fval, *aa);
    if (ok) *fback = fslp3f(s[0], s[1], s[2], d[0], d[1], d[2], *aa);
  }
  return ok ? CADMAS_OK : CADMAS_EPG;
}

int orc_croot3(double a, double b, double c, double d, double *x, int *nrt) {
  croot3(a, b, c, d, x[0], x[1], x[2], *nrt);
  return CADMAS_OK;
}

int orc_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

}  // extern "C"
