// k_slope.cu -- FF-SLOPE advection of F, VF_FCONVS (vf_fconvs.f), the
// scheme VF_F1CAL uses when ISCMFF != 0 (vf_f1cal.f:138-146).
//
//   k_fslope   vf_fconvs.f:72-387  per cell: the slope normal of a surface
//              cell, its type ISTYP (0, 3, 5, 6, 7) and the plane offset
//              SA from VF_FSLP2A / VF_FSLP3A; every cell is written, so
//              the arrays need no clearing
//   k_fconvs   vf_fconvs.f:395-635 the three face fluxes of each cell: by
//              slope (VF_FSLP2F / VF_FSLP3F) where the donor has a type
//              usable across the face and INDX <= 1, else the
//              donor-acceptor flux of VF_FCONV
//
// The cubic of VF_FSLP3A is solved by Cardano's method (VF_CROOT3), which
// needs a cube root, an arctangent and a cosine.  The ones here are built
// from +,-,*,/ and sqrt (methods named at each), so that the oracle, which
// evaluates the same operations in the same order, agrees bit for bit;
// the CUDA and glibc versions of cbrt/atan/cos differ in the last bits.
#include "cadmas_dev.cuh"
#include "kernels.h"
#include "vof_face.cuh"

namespace cadmas {

#define A(a, i, j, k) a[cid(g, i, j, k)]
#define XX_(m, i) gx(g, m, i)
#define YY_(m, j) gy(g, m, j)
#define ZZ_(m, k) gz(g, m, k)

// ------------------------------------------------- elementary functions
// Cube root of x >= 0: x = f 2^e, f in [0.5,1) (frexp, exact); m = f 2^r,
// r = e mod 3, in [0.5,4); Newton's method on y^3 = m from y0 = (m+2)/3,
// above the root by the AM-GM inequality, six steps.
__device__ __forceinline__ double slope_cbrt(double x) {
  if (x == 0.0) return 0.0;
  int e;
  double f = frexp(x, &e);
  int r = ((e % 3) + 3) % 3;
  double m = ldexp(f, r);
  double y = (m + 2.0) / 3.0;
#pragma unroll 1
  for (int it = 0; it < 6; ++it) y = y - (y * y * y - m) / (3.0 * y * y);
  return ldexp(y, (e - r) / 3);
}

// Arctangent: odd symmetry; pi/2 - atan(1/a) for a > 1; two half-angle
// steps a / (1 + sqrt(1 + a^2)); Maclaurin series to z^25 by Horner.
__device__ __forceinline__ double slope_atan(double y) {
  const double HALF_PI = 1.5707963267948966;
  double a = fabs(y);
  bool inv = a > 1.0;
  if (inv) a = 1.0 / a;
  a = a / (1.0 + sqrt(1.0 + a * a));
  a = a / (1.0 + sqrt(1.0 + a * a));
  double z2 = a * a;
  double p = 1.0 / 25.0;
#pragma unroll 1
  for (int n = 11; n >= 0; --n) p = 1.0 / (double)(2 * n + 1) - z2 * p;
  double t = 4.0 * (a * p);
  if (inv) t = HALF_PI - t;
  return (y < 0.0) ? -t : t;
}

// Cosine: Maclaurin series nested as 1 - x^2/(1*2) (1 - x^2/(3*4) (...)),
// 14 levels, for |x| <= 2.7.
__device__ __forceinline__ double slope_cos(double x) {
  double x2 = x * x;
  double p = 1.0;
#pragma unroll 1
  for (int n = 14; n >= 1; --n) p = 1.0 - x2 * p / (double)((2 * n - 1) * (2 * n));
  return p;
}

// ------------------------------------------------------------- roots
// VF_CROOT2  vf_croot2.f:22-55
__device__ void croot2(double AA, double BB, double CC, double &XX1, double &XX2, int &NRT) {
  if (AA == 0.0) {
    if (BB != 0.0) { XX1 = -CC / BB; XX2 = 0.0; NRT = 1; }
    else { XX1 = 0.0; XX2 = 0.0; NRT = 0; }
  } else {
    double B = 1.0 / AA;
    double A = 0.5 * BB * B;
    B = CC * B;
    double D = A * A - B;
    if (fabs(D) < 1.0e-20) { XX1 = -A; XX2 = 0.0; NRT = 1; }
    else if (D < 0.0) { XX1 = 0.0; XX2 = 0.0; NRT = 0; }
    else if (A >= 0.0) { XX1 = -A - sqrt(D); XX2 = B / XX1; NRT = 2; }
    else { XX1 = -A + sqrt(D); XX2 = B / XX1; NRT = 2; }
  }
}

// VF_CROOT3  vf_croot3.f:27-74 (Cardano)
__device__ void croot3(double AA, double BB, double CC, double DD, double &XX1, double &XX2, double &XX3,
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
    double R1 = (Q <= 0.0) ? 0.5 * (-Q + sqrt(D)) : 0.5 * (-Q - sqrt(D));
    double R2 = -(P * P * P / R1);
    double R13 = slope_cbrt(fabs(R1));
    if (R1 < 0.0) R13 = -R13;
    double R23 = slope_cbrt(fabs(R2));
    if (R2 < 0.0) R23 = -R23;
    XX1 = R13 + R23 - A / 3.0;
    XX2 = 0.0; XX3 = 0.0; NRT = 1;
  } else {
    double T = (Q != 0.0) ? slope_atan(sqrt(-D) / (-Q)) : PI / 2.0;
    if (Q > 0.0) T = PI + T;
    double R = 2.0 * sqrt(-P);
    double S = -A / 3.0;
    XX1 = R * slope_cos(T / 3.0) + S;
    XX2 = -(R * slope_cos((PI - T) / 3.0)) + S;
    XX3 = -(R * slope_cos((PI + T) / 3.0)) + S;
    NRT = 3;
  }
}

// The root in [XL-EP, XR+EP], else the midpoint (the reference's WARNING);
// false when there is none (P.G ERROR).
__device__ __forceinline__ bool slope_pick(int NRT, double X1, double X2, double X3, double XL, double XR,
                                           double EP, double &AA) {
  if (NRT == 0) return false;
  if (X1 >= XL - EP && X1 <= XR + EP) AA = X1;
  else if (NRT >= 2 && X2 >= XL - EP && X2 <= XR + EP) AA = X2;
  else if (NRT >= 3 && X3 >= XL - EP && X3 <= XR + EP) AA = X3;
  else AA = (XL + XR) / 2.0;
  return true;
}

// ------------------------------------------------------ plane <-> volume
// VF_FSLP2A  vf_fslp2a.f:30-101: the offset AA of |SX| x + |SY| y = AA that
// leaves FVAL of the DX*DY cell below the plane; the area 2|SX||SY| V(a) is
// the piecewise quadratic a^2 - (a-SD1)+^2 - (a-SD2)+^2.
__device__ bool fslp2a(double SX, double SY, double DX, double DY, double FVAL, double &AA) {
  const double SS0 = fabs(SX), SS1 = fabs(SY);
  const double SD0 = SS0 * DX, SD1 = SS1 * DY;
  const bool lo0 = SD0 <= SD1;
  const double SL1 = lo0 ? SD0 : SD1, SL2 = lo0 ? SD1 : SD0;
  double CNS = 2.0 * SS0 * SS1;
  double XMX = SD0 + SD1;
  double VMX = DX * DY * CNS;
  double VIN = VMX * FVAL;
  double XL = 0.0, XR = SL1, A = 1.0, B = 0.0, C = 0.0;
  double VV = A * XR * XR;
  int k = 0;
  while (!(VIN <= VV)) {
    if (++k == 3) return false;
    double Q = (k == 1) ? SL1 : SL2;
    A = A - 1.0; B = B + 2.0 * Q; C = C - Q * Q;
    XL = XR; XR = (k == 1) ? SL2 : XMX;
    VV = (k == 2) ? VMX : A * XR * XR + B * XR + C;
  }
  double X1, X2; int NRT;
  croot2(A, B, C - VIN, X1, X2, NRT);
  return slope_pick(NRT, X1, X2, 0.0, XL, XR, XMX * 1.0e-6, AA);
}

// VF_FSLP2F  vf_fslp2f.f:25-70: the water fraction below the plane AA.
__device__ double fslp2f(double SX, double SY, double DX, double DY, double AA) {
  const double SS0 = fabs(SX), SS1 = fabs(SY);
  const double SD0 = SS0 * DX, SD1 = SS1 * DY;
  const bool lo0 = SD0 <= SD1;
  const double SL1 = lo0 ? SD0 : SD1, SL2 = lo0 ? SD1 : SD0;
  double CNS = 2.0 * SS0 * SS1;
  double XMX = SD0 + SD1;
  double VMX = DX * DY * CNS;
  double A = 1.0, B = 0.0, C = 0.0, VV;
  if (AA <= 0.0) VV = 0.0;
  else if (AA >= XMX) VV = VMX;
  else if (AA <= SL1) VV = A * AA * AA;
  else {
    double Q = SL1;
    A = A - 1.0; B = B + 2.0 * Q; C = C - Q * Q;
    if (AA <= SL2) VV = A * AA * AA + B * AA + C;
    else {
      Q = SL2;
      A = A - 1.0; B = B + 2.0 * Q; C = C - Q * Q;
      VV = A * AA * AA + B * AA + C;
    }
  }
  return VV / VMX;
}

// The piecewise cubic of VF_FSLP3A/3F: breakpoints after sorting
// SD(L1) <= SD(L2) <= SD(L3) and the change of the leading coefficient at
// each (-1 at a vertex on one axis, +1 on two); the two orders are the
// branches at vf_fslp3a.f:63 / vf_fslp3f.f:63.
struct SlopeCubic {
  double bp[7], XMX, VMX;
  unsigned neg;  // bit k set: the coefficient falls by one at bp[k]
  __device__ SlopeCubic(double SX, double SY, double SZ, double DX, double DY, double DZ) {
    double SS[3] = {fabs(SX), fabs(SY), fabs(SZ)};
    double SD[3] = {SS[0] * DX, SS[1] * DY, SS[2] * DZ};
    int L1 = 0, L2 = 1, L3 = 2, L;
    if (SD[L1] > SD[L2]) { L = L1; L1 = L2; L2 = L; }
    if (SD[L2] > SD[L3]) { L = L2; L2 = L3; L3 = L; }
    if (SD[L1] > SD[L2]) { L = L1; L1 = L2; L2 = L; }
    double CNS = 6.0 * SS[0] * SS[1] * SS[2];
    XMX = SD[0] + SD[1] + SD[2];
    VMX = DX * DY * DZ * CNS;
    bp[0] = SD[L1]; bp[1] = SD[L2];
    if (SD[L1] + SD[L2] <= SD[L3]) { bp[2] = SD[L1] + SD[L2]; bp[3] = SD[L3]; neg = 0x0Bu; }
    else { bp[2] = SD[L3]; bp[3] = SD[L1] + SD[L2]; neg = 0x07u; }
    bp[4] = SD[L1] + SD[L3]; bp[5] = SD[L2] + SD[L3]; bp[6] = XMX;
  }
  __device__ static void pass(bool down, double Q, double &A, double &B, double &C, double &D) {
    if (down) { A = A - 1.0; B = B + 3.0 * Q; C = C - 3.0 * Q * Q; D = D + Q * Q * Q; }
    else { A = A + 1.0; B = B - 3.0 * Q; C = C + 3.0 * Q * Q; D = D - Q * Q * Q; }
  }
  __device__ static double poly(double A, double B, double C, double D, double x) {
    return A * x * x * x + B * x * x + C * x + D;
  }
};

// VF_FSLP3A  vf_fslp3a.f:30-266
__device__ bool fslp3a(double SX, double SY, double SZ, double DX, double DY, double DZ, double FVAL, double &AA) {
  SlopeCubic c(SX, SY, SZ, DX, DY, DZ);
  double VIN = c.VMX * FVAL;
  double A = 1.0, B = 0.0, C = 0.0, D = 0.0, XL = 0.0, XR = c.bp[0];
  double VV = A * XR * XR * XR;
  int k = 0;
  while (!(VIN <= VV)) {
    if (++k == 7) return false;
    SlopeCubic::pass((c.neg >> (k - 1)) & 1u, XR, A, B, C, D);
    XL = XR; XR = c.bp[k];
    VV = (k == 6) ? c.VMX : SlopeCubic::poly(A, B, C, D, XR);
  }
  double X1, X2, X3; int NRT;
  croot3(A, B, C, D - VIN, X1, X2, X3, NRT);
  return slope_pick(NRT, X1, X2, X3, XL, XR, c.XMX * 1.0e-6, AA);
}

// VF_FSLP3F  vf_fslp3f.f:30-181
__device__ double fslp3f(double SX, double SY, double SZ, double DX, double DY, double DZ, double AA) {
  SlopeCubic c(SX, SY, SZ, DX, DY, DZ);
  double VV;
  if (AA <= 0.0) VV = 0.0;
  else if (AA >= c.XMX) VV = c.VMX;
  else {
    double A = 1.0, B = 0.0, C = 0.0, D = 0.0, Q = c.bp[0];
    if (AA <= Q) VV = A * AA * AA * AA;
    else {
      for (int k = 1;; ++k) {
        SlopeCubic::pass((c.neg >> (k - 1)) & 1u, Q, A, B, C, D);
        if (k == 6) break;
        Q = c.bp[k];
        if (AA <= Q) break;
      }
      VV = SlopeCubic::poly(A, B, C, D, AA);
    }
  }
  return VV / c.VMX;
}

// ------------------------------------------------------------ k_fslope
// One side of one axis (vf_fconvs.f:86-123 and its five copies): the F
// (FO) and distance (DO) towards the neighbour cL.  ns: the NF0 values
// whose cross-axis partner (offset off[q] from cL) is merged; DD0 this
// cell's width, d2 the neighbour's, m3 / m6 the 3rd / 6th metric entries.
__device__ __forceinline__ void slope_side(const Fld &f, int NF0, double FF0, long long cL, int NFL, double BCFv,
                                           int n0, int n1, int n2, int n3, long long o0, long long o1,
                                           long long o2, long long o3, double DD0, double d2, double m3,
                                           double m6, double &FO, double &DO) {
  double FFL = f.ff[cL];
  if (NFL == -1) { FO = BCFv; DO = DD0 * 0.5; }
  else if (NFL == 8) {
    if (NF0 == n0 || NF0 == n1 || NF0 == n2 || NF0 == n3) { FO = FF0; DO = 0.0; }
    else { FO = 0.0; DO = DD0 * 0.5; }
  } else if (NFL == 0) {
    FO = FFL; DO = DD0 * 0.5;
    long long o = -1;
    bool hit = true;
    if (NF0 == n0) o = o0;
    else if (NF0 == n1) o = o1;
    else if (NF0 == n2) o = o2;
    else if (NF0 == n3) o = o3;
    else hit = false;
    if (hit) {
      const long long cq = cL + o;
      if (f.nf[cq] != -1) { FO = FO + f.ff[cq]; DO = m3; }
    }
  } else {
    FO = m6 * (d2 * FF0 + DD0 * FFL);
    DO = DD0 * 0.5;
  }
}

__global__ void k_fslope(Geo g, Fld f, Prm p, int *IST, double *SX, double *SY, double *SZ, double *SA, int *err) {
  const double ZERO = 1.0e-20;
  ROW_LOOP_BEGIN(g)
  const long long c = cid(g, I, J, K);
  int ist = 0;
  double s1 = 0.0, s2 = 0.0, s3 = 0.0, sa = 0.0;
  const int NI = g.NI, NJ = g.NJ, NK = g.NK;
  if (I >= 2 && I <= NI - 1 && J >= 2 && J <= NJ - 1 && K >= 2 && K <= NK - 1) {
    const int NF0 = f.nf[c];
    const double FF0 = f.ff[c];
    if (NF0 > 0 && FF0 >= p.flower && FF0 <= p.fupper) {
      const long long sI = 1, sJ = NI, sK = (long long)NI * NJ;
      const int NB = g.NB;
      bool bad = false;
      auto bcf = [&](int l) {
        if (l < 1 || l > NB) { bad = true; return 0.0; }
        return f.bcf[l - 1];
      };
      double FM, FP, DM, DP, S1, S2, S3;
      {
        int nm = f.nf[c - sI], np = f.nf[c + sI];
        double bm = (nm == -1) ? bcf(f.indx[c]) : 0.0, bp = (np == -1) ? bcf(f.indx[c + sI]) : 0.0;
        slope_side(f, NF0, FF0, c - sI, nm, bm, 3, 4, 5, 6, sJ, -sJ, sK, -sK, XX_(2, I), XX_(2, I - 1),
                   XX_(3, I), XX_(6, I), FM, DM);
        slope_side(f, NF0, FF0, c + sI, np, bp, 3, 4, 5, 6, sJ, -sJ, sK, -sK, XX_(2, I), XX_(2, I + 1),
                   XX_(3, I + 1), XX_(6, I + 1), FP, DP);
        S1 = (DM + DP <= ZERO) ? 0.0 : (FM - FP) / (DM + DP);
      }
      {
        int nm = f.nf[c - sJ], np = f.nf[c + sJ];
        double bm = (nm == -1) ? bcf(f.indy[c]) : 0.0, bp = (np == -1) ? bcf(f.indy[c + sJ]) : 0.0;
        slope_side(f, NF0, FF0, c - sJ, nm, bm, 1, 2, 5, 6, sI, -sI, sK, -sK, YY_(2, J), YY_(2, J - 1),
                   YY_(3, J), YY_(6, J), FM, DM);
        slope_side(f, NF0, FF0, c + sJ, np, bp, 1, 2, 5, 6, sI, -sI, sK, -sK, YY_(2, J), YY_(2, J + 1),
                   YY_(3, J + 1), YY_(6, J + 1), FP, DP);
        S2 = (DM + DP <= ZERO) ? 0.0 : (FM - FP) / (DM + DP);
      }
      {
        int nm = f.nf[c - sK], np = f.nf[c + sK];
        double bm = (nm == -1) ? bcf(f.indz[c]) : 0.0, bp = (np == -1) ? bcf(f.indz[c + sK]) : 0.0;
        slope_side(f, NF0, FF0, c - sK, nm, bm, 1, 2, 3, 4, sI, -sI, sJ, -sJ, ZZ_(2, K), ZZ_(2, K - 1),
                   ZZ_(3, K), ZZ_(6, K), FM, DM);
        slope_side(f, NF0, FF0, c + sK, np, bp, 1, 2, 3, 4, sI, -sI, sJ, -sJ, ZZ_(2, K), ZZ_(2, K + 1),
                   ZZ_(3, K + 1), ZZ_(6, K + 1), FP, DP);
        S3 = (DM + DP <= ZERO) ? 0.0 : (FM - FP) / (DM + DP);
      }
      if (bad) atomicOr(err, ERR_PG);
      double RN = S1 * S1 + S2 * S2 + S3 * S3;
      if (!bad && RN >= ZERO) {
        RN = 1.0 / sqrt(RN);
        S1 = S1 * RN; S2 = S2 * RN; S3 = S3 * RN;
        int I1 = fabs(S1) >= 1.0e-4, I2 = fabs(S2) >= 1.0e-4, I3 = fabs(S3) >= 1.0e-4;
        if (I1 + I2 + I3 >= 2) { ist = I1 + 2 * I2 + 4 * I3; s1 = S1; s2 = S2; s3 = S3; }
      }
      bool ok = true;
      if (ist == 3) ok = fslp2a(s1, s2, XX_(2, I), YY_(2, J), FF0, sa);
      else if (ist == 5) ok = fslp2a(s1, s3, XX_(2, I), ZZ_(2, K), FF0, sa);
      else if (ist == 6) ok = fslp2a(s2, s3, YY_(2, J), ZZ_(2, K), FF0, sa);
      else if (ist == 7) ok = fslp3a(s1, s2, s3, XX_(2, I), YY_(2, J), ZZ_(2, K), FF0, sa);
      if (!ok) atomicOr(err, ERR_PG);
    }
  }
  IST[c] = ist; SX[c] = s1; SY[c] = s2; SZ[c] = s3; SA[c] = sa;
  ROW_LOOP_END
}

// ------------------------------------------------------------ k_fconvs
// The slope flux of a face whose donor d has type ist: the water below the
// donor's plane in the strip of width AC next to the face (vf_fconvs.f:
// 448-470 and its y/z copies), capped at the donor's content.  w is the
// donor's width across the face; DFF comes from VF_FSLP2F/3F with the
// strip's width DD0 in place of that width.
template <int AX>
__device__ __forceinline__ double slope_flux(const Geo &g, const Fld &f, const int ist, const long long d, int I,
                                             int J, int K, int LSN, double AC, double w, const double *SX,
                                             const double *SY, const double *SZ, const double *SA) {
  const double sx = SX[d], sy = SY[d], sz = SZ[d], sa = SA[d];
  const double sn = (AX == 0) ? sx : (AX == 1) ? sy : sz;
  int LSW = LSN;
  if (sn < 0.0) LSW = -LSW;
  double DD0 = AC;
  if (LSW == 1) DD0 = w - AC;
  double DFF;
  if (AX == 0) {
    if (ist == 3) DFF = fslp2f(sx, sy, DD0, YY_(2, J), sa);
    else if (ist == 5) DFF = fslp2f(sx, sz, DD0, ZZ_(2, K), sa);
    else DFF = fslp3f(sx, sy, sz, DD0, YY_(2, J), ZZ_(2, K), sa);
  } else if (AX == 1) {
    if (ist == 3) DFF = fslp2f(sx, sy, XX_(2, I), DD0, sa);
    else if (ist == 6) DFF = fslp2f(sy, sz, DD0, ZZ_(2, K), sa);
    else DFF = fslp3f(sx, sy, sz, XX_(2, I), DD0, ZZ_(2, K), sa);
  } else {
    if (ist == 5) DFF = fslp2f(sx, sz, XX_(2, I), DD0, sa);
    else if (ist == 6) DFF = fslp2f(sy, sz, YY_(2, J), DD0, sa);
    else DFF = fslp3f(sx, sy, sz, XX_(2, I), YY_(2, J), DD0, sa);
  }
  double VG = w * f.ff[d];
  double FVX = DFF * DD0;
  if (LSW == 1) FVX = VG - FVX;
  VG = VG * f.ggv[d];
  return dmin(FVX, VG);
}

__global__ void k_fconvs(Geo g, Fld f, Prm p, const int *IST, const double *SX, const double *SY, const double *SZ,
                         const double *SA, double *FLFU, double *FLFV, double *FLFW) {
  const double DT = p.dtnow, FL = p.flower;
  const int *NF = f.nf;
  const double *FF = f.ff, *GGV = f.ggv;
  ROW_LOOP_BEGIN(g)
  const long long c = cid(g, I, J, K);
  const int NI = g.NI, NJ = g.NJ, NK = g.NK;
  double fu = 0.0, fv = 0.0, fw = 0.0;
  if (K >= 2 && K <= NK - 1 && J >= 2 && J <= NJ - 1 && I >= 2 && f.indx[c] != -1) {
    double C = DT * f.ggx[c] * f.uu[c];
    int LSN, LA, LD, LDM;
    if (C >= 0.0) { LSN = 1; LA = I; LD = I - 1; LDM = I - 2; } else { LSN = -1; LA = I - 1; LD = I; LDM = I + 1; }
    const long long d = cid(g, LD, J, K);
    const int ist = IST[d];
    double fl;
    if (f.indx[c] > 1 || ist <= 0 || ist == 6) {
      int N = NF[d];
      int ndm = (N != -1) ? A(NF, LDM, J, K) : -1;
      double fdm = (N != -1 && ndm != -1) ? A(FF, LDM, J, K) : 0.0;
      double vd = (N != -1) ? XX_(2, LD) * GGV[d] : 0.0;
      double bcf = (N == -1) ? f.bcf[f.indx[c] - 1] : 0.0;
      int na = A(NF, LA, J, K);
      fl = fconv_face(C, N, (N != -1) ? FF[d] : 0.0, ndm, fdm, vd, XX_(2, LD), bcf, na,
                      (na != -1) ? A(FF, LA, J, K) : 0.0, 3, 4, 5, 6, FL);
    } else {
      fl = slope_flux<0>(g, f, ist, d, I, J, K, LSN, fabs(C), XX_(2, LD), SX, SY, SZ, SA);
    }
    fu = 0.0 - (double)LSN * fl;
  }
  if (K >= 2 && K <= NK - 1 && J >= 2 && I >= 2 && I <= NI - 1 && f.indy[c] != -1) {
    double C = DT * f.ggy[c] * f.vv[c];
    int LSN, LA, LD, LDM;
    if (C >= 0.0) { LSN = 1; LA = J; LD = J - 1; LDM = J - 2; } else { LSN = -1; LA = J - 1; LD = J; LDM = J + 1; }
    const long long d = cid(g, I, LD, K);
    const int ist = IST[d];
    double fl;
    if (f.indy[c] > 1 || ist <= 0 || ist == 5) {
      int N = NF[d];
      int ndm = (N != -1) ? A(NF, I, LDM, K) : -1;
      double fdm = (N != -1 && ndm != -1) ? A(FF, I, LDM, K) : 0.0;
      double vd = (N != -1) ? YY_(2, LD) * GGV[d] : 0.0;
      double bcf = (N == -1) ? f.bcf[f.indy[c] - 1] : 0.0;
      int na = A(NF, I, LA, K);
      fl = fconv_face(C, N, (N != -1) ? FF[d] : 0.0, ndm, fdm, vd, YY_(2, LD), bcf, na,
                      (na != -1) ? A(FF, I, LA, K) : 0.0, 1, 2, 5, 6, FL);
    } else {
      fl = slope_flux<1>(g, f, ist, d, I, J, K, LSN, fabs(C), YY_(2, LD), SX, SY, SZ, SA);
    }
    fv = 0.0 - (double)LSN * fl;
  }
  if (K >= 2 && J >= 2 && J <= NJ - 1 && I >= 2 && I <= NI - 1 && f.indz[c] != -1) {
    double C = DT * f.ggz[c] * f.ww[c];
    int LSN, LA, LD, LDM;
    if (C >= 0.0) { LSN = 1; LA = K; LD = K - 1; LDM = K - 2; } else { LSN = -1; LA = K - 1; LD = K; LDM = K + 1; }
    const long long d = cid(g, I, J, LD);
    const int ist = IST[d];
    double fl;
    if (f.indz[c] > 1 || ist <= 0 || ist == 3) {
      int N = NF[d];
      int ndm = (N != -1) ? A(NF, I, J, LDM) : -1;
      double fdm = (N != -1 && ndm != -1) ? A(FF, I, J, LDM) : 0.0;
      double vd = (N != -1) ? ZZ_(2, LD) * GGV[d] : 0.0;
      double bcf = (N == -1) ? f.bcf[f.indz[c] - 1] : 0.0;
      int na = A(NF, I, J, LA);
      fl = fconv_face(C, N, (N != -1) ? FF[d] : 0.0, ndm, fdm, vd, ZZ_(2, LD), bcf, na,
                      (na != -1) ? A(FF, I, J, LA) : 0.0, 1, 2, 3, 4, FL);
    } else {
      fl = slope_flux<2>(g, f, ist, d, I, J, K, LSN, fabs(C), ZZ_(2, LD), SX, SY, SZ, SA);
    }
    fw = 0.0 - (double)LSN * fl;
  }
  FLFU[c] = fu; FLFV[c] = fv; FLFW[c] = fw;
  ROW_LOOP_END
}

#undef A
#undef XX_
#undef YY_
#undef ZZ_

void launch_fconvs(cudaStream_t s, const Geo &g, const Fld &f, const Prm &p, int *ist, double *sx, double *sy,
                   double *sz, double *sa, double *flfu, double *flfv, double *flfw, int *err) {
  k_fslope<<<row_blocks(g), ROW_THREADS, 0, s>>>(g, f, p, ist, sx, sy, sz, sa, err);
  count_launch();
  k_fconvs<<<row_blocks(g), ROW_THREADS, 0, s>>>(g, f, p, ist, sx, sy, sz, sa, flfu, flfv, flfw);
  count_launch();
}

}  // namespace cadmas
