// k_bc.cu -- free-surface and wall boundary rules applied inside the step.
//
//   k_bsuwt   VF_BSUWT  (vf_bsuwt.f:41-470)  tangential velocity on faces
//             between non-fluid cells (linear extrapolation, IBSUW0=0)
//   k_bsuwt2  VF_BSUWT2 (vf_bsuwt2.f:36-107)
//   k_bsuwn   VF_BSUWN  (vf_bsuwn.f:57-86)   normal velocity from continuity
//   k_bsuwn3  VF_BSUWN3 (vf_bsuwn3.f:37-340)
//   k_bsuwem_count/fix  VF_BSUWEM (vf_bsuwem.f:37-103)
//   k_bspp    VF_BSPP   (vf_bspp.f:33-61)     gas p = 0, surface p by
//             interpolation to the free-surface pressure 0
//   k_bwuwt   VF_BWUWT  (vf_bwuwt.f:41-118)  boundary tangential values
//   k_bwpp    VF_BWPP   (vf_bwpp.f:28-51)
//   k_bwff    VF_BWFF   (vf_bwff.f:31-89)
//   k_cdiv    VF_CDIV00 (vf_cdiv00.f:38-56)  row partials of |VD|^2
//
// All of these update their arrays in place with one thread per cell or
// face.  The sequential loops of the reference have no order dependence
// here: the faces a rule writes lie between a surface (or non-fluid) cell
// and a gas cell, while the faces it reads lie next to a fluid cell, and
// FNFPRV guarantees that the fluid-side neighbour of a surface cell has
// NF=0, so no written value is read by another thread of the same pass.
#include "cadmas_dev.cuh"
#include "kernels.h"
#include "loglaw.cuh"

namespace cadmas {

#define A(a, i, j, k) a[cid(g, i, j, k)]
#define XX_(m, i) gx(g, m, i)
#define YY_(m, j) gy(g, m, j)
#define ZZ_(m, k) gz(g, m, k)

__device__ __forceinline__ bool inb(const Geo &g, int I, int J, int K) {
  return I >= 1 && I <= g.NI && J >= 1 && J <= g.NJ && K >= 1 && K <= g.NK;
}

// ------------------------------------------------------------ VF_BSUWT
// The three face rules between surface and non-fluid cells, apart from
// the common cases (gas on both sides: 0; fluid on a side: unchanged),
// which the kernel handles inline with all its loads issued together.
__device__ __noinline__ double bsuwt_x(const Geo &g, const int *NF, const double *UU, int S0, int I, int J, int K,
                                       int NL, int NR) {
  const int NI = g.NI, NJ = g.NJ, NK = g.NK;
  (void)NI;
  const int I1 = I - 1;
  double DL = 0, VL = 0, DR = 0, VR = 0, V0;
  if (NL == 3 || NR == 3) {
    V0 = A(UU, I, J - 1, K);
    if (S0) { int L1 = J - 1, L2 = J - 2;
      if (L2 >= 1 && A(NF, I1, L1, K) != -1 && A(NF, I, L1, K) != -1)
        if (A(NF, I1, L2, K) != -1 && A(NF, I, L2, K) != -1)
          if (A(NF, I1, L2, K) == 0 || A(NF, I, L2, K) == 0)
            V0 = V0 + (V0 - A(UU, I, L2, K)) * YY_(3, J) / YY_(3, L1); }
    if (NL == 3) { DL = YY_(3, J); VL = V0; }
    if (NR == 3) { DR = YY_(3, J); VR = V0; }
  }
  if (NL == 4 || NR == 4) {
    V0 = A(UU, I, J + 1, K);
    if (S0) { int L1 = J + 1, L2 = J + 2;
      if (L2 <= NJ && A(NF, I1, L1, K) != -1 && A(NF, I, L1, K) != -1)
        if (A(NF, I1, L2, K) != -1 && A(NF, I, L2, K) != -1)
          if (A(NF, I1, L2, K) == 0 || A(NF, I, L2, K) == 0)
            V0 = V0 + (V0 - A(UU, I, L2, K)) * YY_(3, L1) / YY_(3, L2); }
    if (NL == 4) { DL = YY_(3, J + 1); VL = V0; }
    if (NR == 4) { DR = YY_(3, J + 1); VR = V0; }
  }
  if (NL == 5 || NR == 5) {
    V0 = A(UU, I, J, K - 1);
    if (S0) { int L1 = K - 1, L2 = K - 2;
      if (L2 >= 1 && A(NF, I1, J, L1) != -1 && A(NF, I, J, L1) != -1)
        if (A(NF, I1, J, L2) != -1 && A(NF, I, J, L2) != -1)
          if (A(NF, I1, J, L2) == 0 || A(NF, I, J, L2) == 0)
            V0 = V0 + (V0 - A(UU, I, J, L2)) * ZZ_(3, K) / ZZ_(3, L1); }
    if (NL == 5) { DL = ZZ_(3, K); VL = V0; }
    if (NR == 5) { DR = ZZ_(3, K); VR = V0; }
  }
  if (NL == 6 || NR == 6) {
    V0 = A(UU, I, J, K + 1);
    if (S0) { int L1 = K + 1, L2 = K + 2;
      if (L2 <= NK && A(NF, I1, J, L1) != -1 && A(NF, I, J, L1) != -1)
        if (A(NF, I1, J, L2) != -1 && A(NF, I, J, L2) != -1)
          if (A(NF, I1, J, L2) == 0 || A(NF, I, J, L2) == 0)
            V0 = V0 + (V0 - A(UU, I, J, L2)) * ZZ_(3, L1) / ZZ_(3, L2); }
    if (NL == 6) { DL = ZZ_(3, K + 1); VL = V0; }
    if (NR == 6) { DR = ZZ_(3, K + 1); VR = V0; }
  }
  if (NL == 8) return VR;
  if (NR == 8) return VL;
  return (DR * VL + DL * VR) / (DR + DL);
}
__device__ __noinline__ double bsuwt_y(const Geo &g, const int *NF, const double *VV, int S0, int I, int J, int K,
                                       int NL, int NR) {
  const int NI = g.NI, NJ = g.NJ, NK = g.NK;
  (void)NJ;
  const int J1 = J - 1;
  double DL = 0, VL = 0, DR = 0, VR = 0, V0;
  if (NL == 1 || NR == 1) {
    V0 = A(VV, I - 1, J, K);
    if (S0) { int L1 = I - 1, L2 = I - 2;
      if (L2 >= 1 && A(NF, L1, J1, K) != -1 && A(NF, L1, J, K) != -1)
        if (A(NF, L2, J1, K) != -1 && A(NF, L2, J, K) != -1)
          if (A(NF, L2, J1, K) == 0 || A(NF, L2, J, K) == 0)
            V0 = V0 + (V0 - A(VV, L2, J, K)) * XX_(3, I) / XX_(3, L1); }
    if (NL == 1) { DL = XX_(3, I); VL = V0; }
    if (NR == 1) { DR = XX_(3, I); VR = V0; }
  }
  if (NL == 2 || NR == 2) {
    V0 = A(VV, I + 1, J, K);
    if (S0) { int L1 = I + 1, L2 = I + 2;
      if (L2 <= NI && A(NF, L1, J1, K) != -1 && A(NF, L1, J, K) != -1)
        if (A(NF, L2, J1, K) != -1 && A(NF, L2, J, K) != -1)
          if (A(NF, L2, J1, K) == 0 || A(NF, L2, J, K) == 0)
            V0 = V0 + (V0 - A(VV, L2, J, K)) * XX_(3, L1) / XX_(3, L2); }
    if (NL == 2) { DL = XX_(3, I + 1); VL = V0; }
    if (NR == 2) { DR = XX_(3, I + 1); VR = V0; }
  }
  if (NL == 5 || NR == 5) {
    V0 = A(VV, I, J, K - 1);
    if (S0) { int L1 = K - 1, L2 = K - 2;
      if (L2 >= 1 && A(NF, I, J1, L1) != -1 && A(NF, I, J, L1) != -1)
        if (A(NF, I, J1, L2) != -1 && A(NF, I, J, L2) != -1)
          if (A(NF, I, J1, L2) == 0 || A(NF, I, J, L2) == 0)
            V0 = V0 + (V0 - A(VV, I, J, L2)) * ZZ_(3, K) / ZZ_(3, L1); }
    if (NL == 5) { DL = ZZ_(3, K); VL = V0; }
    if (NR == 5) { DR = ZZ_(3, K); VR = V0; }
  }
  if (NL == 6 || NR == 6) {
    V0 = A(VV, I, J, K + 1);
    if (S0) { int L1 = K + 1, L2 = K + 2;
      if (L2 <= NK && A(NF, I, J1, L1) != -1 && A(NF, I, J, L1) != -1)
        if (A(NF, I, J1, L2) != -1 && A(NF, I, J, L2) != -1)
          if (A(NF, I, J1, L2) == 0 || A(NF, I, J, L2) == 0)
            V0 = V0 + (V0 - A(VV, I, J, L2)) * ZZ_(3, L1) / ZZ_(3, L2); }
    if (NL == 6) { DL = ZZ_(3, K + 1); VL = V0; }
    if (NR == 6) { DR = ZZ_(3, K + 1); VR = V0; }
  }
  if (NL == 8) return VR;
  if (NR == 8) return VL;
  return (DR * VL + DL * VR) / (DR + DL);
}
__device__ __noinline__ double bsuwt_z(const Geo &g, const int *NF, const double *WW, int S0, int I, int J, int K,
                                       int NL, int NR) {
  const int NI = g.NI, NJ = g.NJ, NK = g.NK;
  (void)NK;
  const int K1 = K - 1;
  double DL = 0, VL = 0, DR = 0, VR = 0, V0;
  if (NL == 1 || NR == 1) {
    V0 = A(WW, I - 1, J, K);
    if (S0) { int L1 = I - 1, L2 = I - 2;
      if (L2 >= 1 && A(NF, L1, J, K1) != -1 && A(NF, L1, J, K) != -1)
        if (A(NF, L2, J, K1) != -1 && A(NF, L2, J, K) != -1)
          if (A(NF, L2, J, K1) == 0 || A(NF, L2, J, K) == 0)
            V0 = V0 + (V0 - A(WW, L2, J, K)) * XX_(3, I) / XX_(3, L1); }
    if (NL == 1) { DL = XX_(3, I); VL = V0; }
    if (NR == 1) { DR = XX_(3, I); VR = V0; }
  }
  if (NL == 2 || NR == 2) {
    V0 = A(WW, I + 1, J, K);
    if (S0) { int L1 = I + 1, L2 = I + 2;
      if (L2 <= NI && A(NF, L1, J, K1) != -1 && A(NF, L1, J, K) != -1)
        if (A(NF, L2, J, K1) != -1 && A(NF, L2, J, K) != -1)
          if (A(NF, L2, J, K1) == 0 || A(NF, L2, J, K) == 0)
            V0 = V0 + (V0 - A(WW, L2, J, K)) * XX_(3, L1) / XX_(3, L2); }
    if (NL == 2) { DL = XX_(3, I + 1); VL = V0; }
    if (NR == 2) { DR = XX_(3, I + 1); VR = V0; }
  }
  if (NL == 3 || NR == 3) {
    V0 = A(WW, I, J - 1, K);
    if (S0) { int L1 = J - 1, L2 = J - 2;
      if (L2 >= 1 && A(NF, I, L1, K1) != -1 && A(NF, I, L1, K) != -1)
        if (A(NF, I, L2, K1) != -1 && A(NF, I, L2, K) != -1)
          if (A(NF, I, L2, K1) == 0 || A(NF, I, L2, K) == 0)
            V0 = V0 + (V0 - A(WW, I, L2, K)) * YY_(3, J) / YY_(3, L1); }
    if (NL == 3) { DL = YY_(3, J); VL = V0; }
    if (NR == 3) { DR = YY_(3, J); VR = V0; }
  }
  if (NL == 4 || NR == 4) {
    V0 = A(WW, I, J + 1, K);
    if (S0) { int L1 = J + 1, L2 = J + 2;
      if (L2 <= NJ && A(NF, I, L1, K1) != -1 && A(NF, I, L1, K) != -1)
        if (A(NF, I, L2, K1) != -1 && A(NF, I, L2, K) != -1)
          if (A(NF, I, L2, K1) == 0 || A(NF, I, L2, K) == 0)
            V0 = V0 + (V0 - A(WW, I, L2, K)) * YY_(3, L1) / YY_(3, L2); }
    if (NL == 4) { DL = YY_(3, J + 1); VL = V0; }
    if (NR == 4) { DR = YY_(3, J + 1); VR = V0; }
  }
  if (NL == 8) return VR;
  if (NR == 8) return VL;
  return (DR * VL + DL * VR) / (DR + DL);
}

__global__ void __launch_bounds__(ROW_THREADS, 4) k_bsuwt(Geo g, Fld f, Prm p) {
  const int S0 = (p.ibsuw0 == 0);
  const int *NF = f.nf;
  ROW_LOOP_BEGIN(g)
  const long long c = cid(g, I, J, K);
  const int NI = g.NI, NJ = g.NJ, NK = g.NK;
  // x faces K=2..NK-1, J=2..NJ-1, I=3..NI-1; y faces K=2..NK-1, J=3..NJ-1,
  // I=2..NI-1; z faces K=3..NK-1, J=2..NJ-1, I=2..NI-1
  const bool bx = K >= 2 && K <= NK - 1 && J >= 2 && J <= NJ - 1 && I >= 3 && I <= NI - 1;
  const bool by = K >= 2 && K <= NK - 1 && J >= 3 && J <= NJ - 1 && I >= 2 && I <= NI - 1;
  const bool bz = K >= 3 && K <= NK - 1 && J >= 2 && J <= NJ - 1 && I >= 2 && I <= NI - 1;
  if (bx || by || bz) {
    const int ix = bx ? f.indx[c] : 1, iy = by ? f.indy[c] : 1, iz = bz ? f.indz[c] : 1;
    const int NR = NF[c];
    const int NLx = bx ? A(NF, I - 1, J, K) : 0, NLy = by ? A(NF, I, J - 1, K) : 0,
              NLz = bz ? A(NF, I, J, K - 1) : 0;
    if (ix == 0) {
      if (NLx == 8 && NR == 8) f.uu[c] = 0.0;
      else if (NLx != 0 && NR != 0) f.uu[c] = bsuwt_x(g, NF, f.uu, S0, I, J, K, NLx, NR);
    }
    if (iy == 0) {
      if (NLy == 8 && NR == 8) f.vv[c] = 0.0;
      else if (NLy != 0 && NR != 0) f.vv[c] = bsuwt_y(g, NF, f.vv, S0, I, J, K, NLy, NR);
    }
    if (iz == 0) {
      if (NLz == 8 && NR == 8) f.ww[c] = 0.0;
      else if (NLz != 0 && NR != 0) f.ww[c] = bsuwt_z(g, NF, f.ww, S0, I, J, K, NLz, NR);
    }
  }
  ROW_LOOP_END
}

__device__ __forceinline__ bool surf_interior(const Geo &g, int I, int J, int K) {
  return I >= 2 && I <= g.NI - 1 && J >= 2 && J <= g.NJ - 1 && K >= 2 && K <= g.NK - 1;
}

// ----------------------------------------------------------- VF_BSUWT2
__global__ void k_bsuwt2(Geo g, Fld f) {
  const int *NF = f.nf;
  double *UU = f.uu, *VV = f.vv, *WW = f.ww;
  ROW_LOOP_BEGIN(g)
  const long long c = cid(g, I, J, K);
  const int NF0 = NF[c];
  if (NF0 >= 1 && NF0 <= 6 && surf_interior(g, I, J, K)) {
    int L1, L2, LB;
    if (NF0 == 5 || NF0 == 6) {
      LB = (NF0 == 5) ? K - 1 : K + 1;
      L1 = I; L2 = I;
      if (A(NF, I - 1, J, K) == 8 && A(f.indx, I, J, LB) != 0) L2 = L2 + 1;
      if (A(NF, I + 1, J, K) == 8 && A(f.indx, I + 1, J, LB) != 0) L1 = L1 + 1;
      A(UU, L1, J, K) = A(UU, L2, J, K);
      L1 = J; L2 = J;
      if (A(NF, I, J - 1, K) == 8 && A(f.indy, I, J, LB) != 0) L2 = L2 + 1;
      if (A(NF, I, J + 1, K) == 8 && A(f.indy, I, J + 1, LB) != 0) L1 = L1 + 1;
      A(VV, I, L1, K) = A(VV, I, L2, K);
    } else if (NF0 == 3 || NF0 == 4) {
      LB = (NF0 == 3) ? J - 1 : J + 1;
      L1 = I; L2 = I;
      if (A(NF, I - 1, J, K) == 8 && A(f.indx, I, LB, K) != 0) L2 = L2 + 1;
      if (A(NF, I + 1, J, K) == 8 && A(f.indx, I + 1, LB, K) != 0) L1 = L1 + 1;
      A(UU, L1, J, K) = A(UU, L2, J, K);
      L1 = K; L2 = K;
      if (A(NF, I, J, K - 1) == 8 && A(f.indz, I, LB, K) != 0) L2 = L2 + 1;
      if (A(NF, I, J, K + 1) == 8 && A(f.indz, I, LB, K + 1) != 0) L1 = L1 + 1;
      A(WW, I, J, L1) = A(WW, I, J, L2);
    } else {
      LB = (NF0 == 1) ? I - 1 : I + 1;
      L1 = J; L2 = J;
      if (A(NF, I, J - 1, K) == 8 && A(f.indy, LB, J, K) != 0) L2 = L2 + 1;
      if (A(NF, I, J + 1, K) == 8 && A(f.indy, LB, J + 1, K) != 0) L1 = L1 + 1;
      A(VV, I, L1, K) = A(VV, I, L2, K);
      L1 = K; L2 = K;
      if (A(NF, I, J, K - 1) == 8 && A(f.indz, LB, J, K) != 0) L2 = L2 + 1;
      if (A(NF, I, J, K + 1) == 8 && A(f.indz, LB, J, K + 1) != 0) L1 = L1 + 1;
      A(WW, I, J, L1) = A(WW, I, J, L2);
    }
  }
  ROW_LOOP_END
}

// ------------------------------------------------------------ VF_BSUWN
__global__ void k_bsuwn(Geo g, Fld f) {
  double *UU = f.uu, *VV = f.vv, *WW = f.ww;
  const double *GGX = f.ggx, *GGY = f.ggy, *GGZ = f.ggz;
  ROW_LOOP_BEGIN(g)
  const long long c = cid(g, I, J, K);
  const int NF0 = f.nf[c];
  if (NF0 >= 1 && NF0 <= 6 && surf_interior(g, I, J, K)) {
    const int I1 = I + 1, J1 = J + 1, K1 = K + 1;
    double FXP = A(GGX, I1, J, K) * A(UU, I1, J, K), FXM = GGX[c] * UU[c];
    double FYP = A(GGY, I, J1, K) * A(VV, I, J1, K), FYM = GGY[c] * VV[c];
    double FZP = A(GGZ, I, J, K1) * A(WW, I, J, K1), FZM = GGZ[c] * WW[c];
    if (NF0 == 5) A(WW, I, J, K1) = (FZM - ZZ_(2, K) * (XX_(4, I) * (FXP - FXM) + YY_(4, J) * (FYP - FYM))) / A(GGZ, I, J, K1);
    else if (NF0 == 6) WW[c] = (FZP + ZZ_(2, K) * (XX_(4, I) * (FXP - FXM) + YY_(4, J) * (FYP - FYM))) / GGZ[c];
    else if (NF0 == 3) A(VV, I, J1, K) = (FYM - YY_(2, J) * (XX_(4, I) * (FXP - FXM) + ZZ_(4, K) * (FZP - FZM))) / A(GGY, I, J1, K);
    else if (NF0 == 4) VV[c] = (FYP + YY_(2, J) * (XX_(4, I) * (FXP - FXM) + ZZ_(4, K) * (FZP - FZM))) / GGY[c];
    else if (NF0 == 1) A(UU, I1, J, K) = (FXM - XX_(2, I) * (YY_(4, J) * (FYP - FYM) + ZZ_(4, K) * (FZP - FZM))) / A(GGX, I1, J, K);
    else if (NF0 == 2) UU[c] = (FXP + XX_(2, I) * (YY_(4, J) * (FYP - FYM) + ZZ_(4, K) * (FZP - FZM))) / GGX[c];
  }
  ROW_LOOP_END
}

// ----------------------------------------------------------- VF_BSUWN3
__device__ __forceinline__ void lat(const Geo &g, const int *NF, long long a, long long b, int &is,
                                    double &d, double &v, double dv, double vv) {
  if (NF[a] == 0 || NF[b] == 0)
    if (NF[a] != -1 && NF[b] != -1) { is = 1; d = dv; v = vv; }
}

__global__ void __launch_bounds__(ROW_THREADS, 3) k_bsuwn3(Geo g, Fld f, Prm p) {
  const int S0 = (p.ibsuw0 == 0);
  const int *NF = f.nf;
  double *UU = f.uu, *VV = f.vv, *WW = f.ww;
  ROW_LOOP_BEGIN(g)
  const long long c = cid(g, I, J, K);
  const int NF0 = NF[c];
  if (NF0 >= 1 && NF0 <= 6 && surf_interior(g, I, J, K)) {
    int IS1 = 0, IS2 = 0, IS3 = 0, IS4 = 0;
    double D0, V0, D1 = 0, V1 = 0, D2 = 0, V2 = 0, D3 = 0, V3 = 0, D4 = 0, V4 = 0;
    long long out;
    double vx;  // extrapolation result when no lateral neighbour qualifies
    if (NF0 == 5) {
      D0 = ZZ_(2, K); V0 = WW[c]; const int L1 = K + 1;
      lat(g, NF, cid(g, I - 1, J, K), cid(g, I - 1, J, L1), IS1, D1, V1, XX_(3, I), A(WW, I - 1, J, L1));
      lat(g, NF, cid(g, I + 1, J, K), cid(g, I + 1, J, L1), IS2, D2, V2, XX_(3, I + 1), A(WW, I + 1, J, L1));
      lat(g, NF, cid(g, I, J - 1, K), cid(g, I, J - 1, L1), IS3, D3, V3, YY_(3, J), A(WW, I, J - 1, L1));
      lat(g, NF, cid(g, I, J + 1, K), cid(g, I, J + 1, L1), IS4, D4, V4, YY_(3, J + 1), A(WW, I, J + 1, L1));
      out = cid(g, I, J, K + 1);
      vx = V0;
      if (S0 && K - 2 >= 1 && A(NF, I, J, K - 2) == 0) vx = V0 + (V0 - A(WW, I, J, K - 1)) * ZZ_(2, K) / ZZ_(2, K - 1);
    } else if (NF0 == 6) {
      D0 = ZZ_(2, K); V0 = A(WW, I, J, K + 1); const int L1 = K - 1;
      lat(g, NF, cid(g, I - 1, J, K), cid(g, I - 1, J, L1), IS1, D1, V1, XX_(3, I), A(WW, I - 1, J, K));
      lat(g, NF, cid(g, I + 1, J, K), cid(g, I + 1, J, L1), IS2, D2, V2, XX_(3, I + 1), A(WW, I + 1, J, K));
      lat(g, NF, cid(g, I, J - 1, K), cid(g, I, J - 1, L1), IS3, D3, V3, YY_(3, J), A(WW, I, J - 1, K));
      lat(g, NF, cid(g, I, J + 1, K), cid(g, I, J + 1, L1), IS4, D4, V4, YY_(3, J + 1), A(WW, I, J + 1, K));
      out = c;
      vx = V0;
      if (S0 && K + 2 <= g.NK && A(NF, I, J, K + 2) == 0) vx = V0 + (V0 - A(WW, I, J, K + 2)) * ZZ_(2, K) / ZZ_(2, K + 1);
    } else if (NF0 == 3) {
      D0 = YY_(2, J); V0 = VV[c]; const int L1 = J + 1;
      lat(g, NF, cid(g, I - 1, J, K), cid(g, I - 1, L1, K), IS1, D1, V1, XX_(3, I), A(VV, I - 1, L1, K));
      lat(g, NF, cid(g, I + 1, J, K), cid(g, I + 1, L1, K), IS2, D2, V2, XX_(3, I + 1), A(VV, I + 1, L1, K));
      lat(g, NF, cid(g, I, J, K - 1), cid(g, I, L1, K - 1), IS3, D3, V3, ZZ_(3, K), A(VV, I, L1, K - 1));
      lat(g, NF, cid(g, I, J, K + 1), cid(g, I, L1, K + 1), IS4, D4, V4, ZZ_(3, K + 1), A(VV, I, L1, K + 1));
      out = cid(g, I, J + 1, K);
      vx = V0;
      if (S0 && J - 2 >= 1 && A(NF, I, J - 2, K) == 0) vx = V0 + (V0 - A(VV, I, J - 1, K)) * YY_(2, J) / YY_(2, J - 1);
    } else if (NF0 == 4) {
      D0 = YY_(2, J); V0 = A(VV, I, J + 1, K); const int L1 = J - 1;
      lat(g, NF, cid(g, I - 1, J, K), cid(g, I - 1, L1, K), IS1, D1, V1, XX_(3, I), A(VV, I - 1, J, K));
      lat(g, NF, cid(g, I + 1, J, K), cid(g, I + 1, L1, K), IS2, D2, V2, XX_(3, I + 1), A(VV, I + 1, J, K));
      lat(g, NF, cid(g, I, J, K - 1), cid(g, I, L1, K - 1), IS3, D3, V3, ZZ_(3, K), A(VV, I, J, K - 1));
      lat(g, NF, cid(g, I, J, K + 1), cid(g, I, L1, K + 1), IS4, D4, V4, ZZ_(3, K + 1), A(VV, I, J, K + 1));
      out = c;
      vx = V0;
      if (S0 && J + 2 <= g.NJ && A(NF, I, J + 2, K) == 0) vx = V0 + (V0 - A(VV, I, J + 2, K)) * YY_(2, J) / YY_(2, J + 1);
    } else if (NF0 == 1) {
      D0 = XX_(2, I); V0 = UU[c]; const int L1 = I + 1;
      lat(g, NF, cid(g, I, J - 1, K), cid(g, L1, J - 1, K), IS1, D1, V1, YY_(3, J), A(UU, L1, J - 1, K));
      lat(g, NF, cid(g, I, J + 1, K), cid(g, L1, J + 1, K), IS2, D2, V2, YY_(3, J + 1), A(UU, L1, J + 1, K));
      lat(g, NF, cid(g, I, J, K - 1), cid(g, L1, J, K - 1), IS3, D3, V3, ZZ_(3, K), A(UU, L1, J, K - 1));
      lat(g, NF, cid(g, I, J, K + 1), cid(g, L1, J, K + 1), IS4, D4, V4, ZZ_(3, K + 1), A(UU, L1, J, K + 1));
      out = cid(g, I + 1, J, K);
      vx = V0;
      if (S0 && I - 2 >= 1 && A(NF, I - 2, J, K) == 0) vx = V0 + (V0 - A(UU, I - 1, J, K)) * XX_(2, I) / XX_(2, I - 1);
    } else {
      D0 = XX_(2, I); V0 = A(UU, I + 1, J, K); const int L1 = I - 1;
      lat(g, NF, cid(g, I, J - 1, K), cid(g, L1, J - 1, K), IS1, D1, V1, YY_(3, J), A(UU, I, J - 1, K));
      lat(g, NF, cid(g, I, J + 1, K), cid(g, L1, J + 1, K), IS2, D2, V2, YY_(3, J + 1), A(UU, I, J + 1, K));
      lat(g, NF, cid(g, I, J, K - 1), cid(g, L1, J, K - 1), IS3, D3, V3, ZZ_(3, K), A(UU, I, J, K - 1));
      lat(g, NF, cid(g, I, J, K + 1), cid(g, L1, J, K + 1), IS4, D4, V4, ZZ_(3, K + 1), A(UU, I, J, K + 1));
      out = c;
      vx = V0;
      if (S0 && I + 2 <= g.NI && A(NF, I + 2, J, K) == 0) vx = V0 + (V0 - A(UU, I + 2, J, K)) * XX_(2, I) / XX_(2, I + 1);
    }
    const int ISS = IS1 + IS2 + IS3 + IS4;
    double val;
    if (ISS <= 0) {
      val = vx;
    } else {
      double DS = D0 + D1 + D2 + D3 + D4;
      val = ((DS - D0) * V0 + (DS - D1) * V1 + (DS - D2) * V2 + (DS - D3) * V3 + (DS - D4) * V4) / DS / (double)ISS;
    }
    double *arr = (NF0 >= 5) ? WW : (NF0 >= 3 ? VV : UU);
    arr[out] = val;
  }
  ROW_LOOP_END
}

// ----------------------------------------------------------- VF_BSUWEM
// NLIM of each cell = number of surface neighbours for which it is a
// lateral (non-normal) neighbour (vf_bsuwem.f:55-78), as a gather.
__global__ void k_bsuwem_count(Geo g, Fld f, int *NLIM) {
  const int *NF = f.nf;
  ROW_LOOP_BEGIN(g)
  const long long c = cid(g, I, J, K);
  int n = 0;
  if (I >= 2 && I <= g.NI - 1 && J >= 2 && J <= g.NJ - 1 && K >= 2 && K <= g.NK - 1) {
    int s;
    s = A(NF, I - 1, J, K); if (s >= 3 && s <= 6) n++;
    s = A(NF, I + 1, J, K); if (s >= 3 && s <= 6) n++;
    s = A(NF, I, J - 1, K); if (s == 5 || s == 6 || s == 1 || s == 2) n++;
    s = A(NF, I, J + 1, K); if (s == 5 || s == 6 || s == 1 || s == 2) n++;
    s = A(NF, I, J, K - 1); if (s >= 1 && s <= 4) n++;
    s = A(NF, I, J, K + 1); if (s >= 1 && s <= 4) n++;
  }
  NLIM[c] = n;
  ROW_LOOP_END
}

__global__ void k_bsuwem_fix(Geo g, Fld f, const int *NLIM) {
  const int *NF = f.nf;
  double *UU = f.uu, *VV = f.vv, *WW = f.ww;
  ROW_LOOP_BEGIN(g)
  const long long c = cid(g, I, J, K);
  if (surf_interior(g, I, J, K) && NLIM[c] >= 2 && NF[c] == 8) {
    if (A(NF, I - 1, J, K) == 8 && A(NLIM, I - 1, J, K) < 2)
      if (A(NF, I + 1, J, K) != 8) UU[c] = A(UU, I + 1, J, K);
    if (A(NF, I + 1, J, K) == 8 && A(NLIM, I + 1, J, K) < 2)
      if (A(NF, I - 1, J, K) != 8) A(UU, I + 1, J, K) = UU[c];
    if (A(NF, I, J - 1, K) == 8 && A(NLIM, I, J - 1, K) < 2)
      if (A(NF, I, J + 1, K) != 8) VV[c] = A(VV, I, J + 1, K);
    if (A(NF, I, J + 1, K) == 8 && A(NLIM, I, J + 1, K) < 2)
      if (A(NF, I, J - 1, K) != 8) A(VV, I, J + 1, K) = VV[c];
    if (A(NF, I, J, K - 1) == 8 && A(NLIM, I, J, K - 1) < 2)
      if (A(NF, I, J, K + 1) != 8) WW[c] = A(WW, I, J, K + 1);
    if (A(NF, I, J, K + 1) == 8 && A(NLIM, I, J, K + 1) < 2)
      if (A(NF, I, J, K - 1) != 8) A(WW, I, J, K + 1) = WW[c];
  }
  ROW_LOOP_END
}

// ------------------------------------------------------------- VF_BSPP
__global__ void k_bspp(Geo g, Fld f) {
  const double PPS = 0.0;
  double *PP = f.pp;
  const double *FF = f.ff;
  ROW_LOOP_BEGIN(g)
  const long long c = cid(g, I, J, K);
  if (surf_interior(g, I, J, K)) {
    const int n = f.nf[c];
    double PSI;
    if (n == 8) PP[c] = 0.0;
    else if (n == 5) { PSI = ZZ_(3, K) / (0.5 * ZZ_(2, K - 1) + FF[c] * ZZ_(2, K)); PP[c] = (1.0 - PSI) * A(PP, I, J, K - 1) + PSI * PPS; }
    else if (n == 6) { PSI = ZZ_(3, K + 1) / (0.5 * ZZ_(2, K + 1) + FF[c] * ZZ_(2, K)); PP[c] = (1.0 - PSI) * A(PP, I, J, K + 1) + PSI * PPS; }
    else if (n == 3) { PSI = YY_(3, J) / (0.5 * YY_(2, J - 1) + FF[c] * YY_(2, J)); PP[c] = (1.0 - PSI) * A(PP, I, J - 1, K) + PSI * PPS; }
    else if (n == 4) { PSI = YY_(3, J + 1) / (0.5 * YY_(2, J + 1) + FF[c] * YY_(2, J)); PP[c] = (1.0 - PSI) * A(PP, I, J + 1, K) + PSI * PPS; }
    else if (n == 1) { PSI = XX_(3, I) / (0.5 * XX_(2, I - 1) + FF[c] * XX_(2, I)); PP[c] = (1.0 - PSI) * A(PP, I - 1, J, K) + PSI * PPS; }
    else if (n == 2) { PSI = XX_(3, I + 1) / (0.5 * XX_(2, I + 1) + FF[c] * XX_(2, I)); PP[c] = (1.0 - PSI) * A(PP, I + 1, J, K) + PSI * PPS; }
  }
  ROW_LOOP_END
}

// ---------------------------------------------------- boundary-list rules
// VF_BWUWT (vf_bwuwt.f:41-181): tangential boundary values.  Slip and free
// faces take the adjacent cell's averages; log-law (6) and rough (8) faces
// take them reduced by the wall shear, V (1 - DL u*^2 / (ANU VA)), with the
// friction velocity u* of VF_CLOGLW or VF_CLOGKS.
__global__ void k_bwuwt(Geo g, Fld f, Prm p, int *err) {
  int L = blockIdx.x * blockDim.x + threadIdx.x + 1;
  if (L > g.NB) return;
  int I, J, K;
  decode(g, indb(f, 1, L), I, J, K);
  const int NS = indb(f, 2, L), IB = indb(f, 3, L);
  const double *UU = f.uu, *VV = f.vv, *WW = f.ww;
  if (IB == 6 || IB == 8) {
    double V1, V2, DL, AN;
    if (NS == 1) {
      V1 = (A(VV, I, J, K) + A(VV, I, J + 1, K)) * 0.5; V2 = (A(WW, I, J, K) + A(WW, I, J, K + 1)) * 0.5;
      DL = XX_(2, I) * 0.5; AN = A(f.anu, I, J, K);
    } else if (NS == 2) {
      V1 = (A(VV, I - 1, J, K) + A(VV, I - 1, J + 1, K)) * 0.5; V2 = (A(WW, I - 1, J, K) + A(WW, I - 1, J, K + 1)) * 0.5;
      DL = XX_(2, I - 1) * 0.5; AN = A(f.anu, I - 1, J, K);
    } else if (NS == 3) {
      V1 = (A(UU, I, J, K) + A(UU, I + 1, J, K)) * 0.5; V2 = (A(WW, I, J, K) + A(WW, I, J, K + 1)) * 0.5;
      DL = YY_(2, J) * 0.5; AN = A(f.anu, I, J, K);
    } else if (NS == 4) {
      V1 = (A(UU, I, J - 1, K) + A(UU, I + 1, J - 1, K)) * 0.5; V2 = (A(WW, I, J - 1, K) + A(WW, I, J - 1, K + 1)) * 0.5;
      DL = YY_(2, J - 1) * 0.5; AN = A(f.anu, I, J - 1, K);
    } else if (NS == 5) {
      V1 = (A(UU, I, J, K) + A(UU, I + 1, J, K)) * 0.5; V2 = (A(VV, I, J, K) + A(VV, I, J + 1, K)) * 0.5;
      DL = ZZ_(2, K) * 0.5; AN = A(f.anu, I, J, K);
    } else {
      V1 = (A(UU, I, J, K - 1) + A(UU, I + 1, J, K - 1)) * 0.5; V2 = (A(VV, I, J, K - 1) + A(VV, I, J + 1, K - 1)) * 0.5;
      DL = ZZ_(2, K - 1) * 0.5; AN = A(f.anu, I, J, K - 1);
    }
    const double ZERO = 1.0e-20;
    double VA = sqrt(V1 * V1 + V2 * V2), VT;
    if (VA < ZERO || AN < ZERO) {
      V1 = 0.0; V2 = 0.0; DL = 1.0; AN = 1.0; VA = 1.0; VT = 1.0;
    } else if (IB == 6) {
      if (!cloglw(DL, VA, p.anu0, p.akk0, p.aka0, VT)) atomicOr(err, ERR_NOTCONV);
    } else {
      VT = clogks(DL, VA, f.bcvi[L - 1], p.anu0, p.akk0, p.aka0);
    }
    VA = DL / AN * VT * VT / VA;
    V1 = V1 - VA * V1;
    V2 = V2 - VA * V2;
    if (NS == 1 || NS == 2) { f.bcv[L - 1] = V1; f.bcw[L - 1] = V2; }
    else if (NS == 3 || NS == 4) { f.bcu[L - 1] = V1; f.bcw[L - 1] = V2; }
    else { f.bcu[L - 1] = V1; f.bcv[L - 1] = V2; }
  } else if (IB == 1 || IB == 4 || (IB == 5 && fixlvl_face(g, p, NS, I, J))) {
    if (NS == 1) { f.bcv[L - 1] = (A(VV, I, J, K) + A(VV, I, J + 1, K)) * 0.5; f.bcw[L - 1] = (A(WW, I, J, K) + A(WW, I, J, K + 1)) * 0.5; }
    else if (NS == 2) { f.bcv[L - 1] = (A(VV, I - 1, J, K) + A(VV, I - 1, J + 1, K)) * 0.5; f.bcw[L - 1] = (A(WW, I - 1, J, K) + A(WW, I - 1, J, K + 1)) * 0.5; }
    else if (NS == 3) { f.bcu[L - 1] = (A(UU, I, J, K) + A(UU, I + 1, J, K)) * 0.5; f.bcw[L - 1] = (A(WW, I, J, K) + A(WW, I, J, K + 1)) * 0.5; }
    else if (NS == 4) { f.bcu[L - 1] = (A(UU, I, J - 1, K) + A(UU, I + 1, J - 1, K)) * 0.5; f.bcw[L - 1] = (A(WW, I, J - 1, K) + A(WW, I, J - 1, K + 1)) * 0.5; }
    else if (NS == 5) { f.bcu[L - 1] = (A(UU, I, J, K) + A(UU, I + 1, J, K)) * 0.5; f.bcv[L - 1] = (A(VV, I, J, K) + A(VV, I, J + 1, K)) * 0.5; }
    else if (NS == 6) { f.bcu[L - 1] = (A(UU, I, J, K - 1) + A(UU, I + 1, J, K - 1)) * 0.5; f.bcv[L - 1] = (A(VV, I, J, K - 1) + A(VV, I, J + 1, K - 1)) * 0.5; }
  }
}

__global__ void k_bwpp(Geo g, Fld f) {
  int L = blockIdx.x * blockDim.x + threadIdx.x + 1;
  if (L > g.NB) return;
  int I, J, K;
  decode(g, indb(f, 1, L), I, J, K);
  const int NS = indb(f, 2, L);
  const double *PP = f.pp;
  double v = 0.0;
  if (NS == 1) v = A(PP, I, J, K);
  else if (NS == 2) v = A(PP, I - 1, J, K);
  else if (NS == 3) v = A(PP, I, J, K);
  else if (NS == 4) v = A(PP, I, J - 1, K);
  else if (NS == 5) v = A(PP, I, J, K);
  else if (NS == 6) v = A(PP, I, J, K - 1);
  else return;
  f.bcp[L - 1] = v;
}

__global__ void k_bwff(Geo g, Fld f, int *err) {
  int L = blockIdx.x * blockDim.x + threadIdx.x + 1;
  if (L > g.NB) return;
  int I, J, K;
  decode(g, indb(f, 1, L), I, J, K);
  const int NS = indb(f, 2, L), IB = indb(f, 4, L);
  const double *FF = f.ff;
  if (IB == 1) return;
  if (IB == 2 || IB == 5 || IB == 7) {
    if (NS == 1) f.bcf[L - 1] = A(FF, I, J, K);
    else if (NS == 2) f.bcf[L - 1] = A(FF, I - 1, J, K);
    else if (NS == 3) f.bcf[L - 1] = A(FF, I, J, K);
    else if (NS == 4) f.bcf[L - 1] = A(FF, I, J - 1, K);
    else if (IB == 2 && NS == 5) f.bcf[L - 1] = A(FF, I, J, K);
    else if (IB == 2 && NS == 6) f.bcf[L - 1] = A(FF, I, J, K - 1);
    else atomicOr(err, ERR_PG);
  } else {
    atomicOr(err, ERR_PG);
  }
}

// ----------------------------------------------------------- VF_CDIV00
__global__ void k_cdiv(Geo g, Fld f, double *rb) {
  double s = 0.0;
  const long long nrows = (long long)g.NJ * g.NK;
  ROW_LOOP_BEGIN(g)
  const long long c = cid(g, I, J, K);
  if (surf_interior(g, I, J, K) && f.indc[c] != -1) {
    double VD = YY_(2, J) * ZZ_(2, K) * (A(f.ggx, I + 1, J, K) * A(f.uu, I + 1, J, K) - f.ggx[c] * f.uu[c]) +
                XX_(2, I) * ZZ_(2, K) * (A(f.ggy, I, J + 1, K) * A(f.vv, I, J + 1, K) - f.ggy[c] * f.vv[c]) +
                XX_(2, I) * YY_(2, J) * (A(f.ggz, I, J, K + 1) * A(f.ww, I, J, K + 1) - f.ggz[c] * f.ww[c]);
    s = s + VD * VD;
  }
  ROW_LOOP_END
  const long long row = (long long)blockIdx.x * ROWS_PER_BLOCK + (threadIdx.x >> 5);
  row_store(s, rb, row, nrows);
}

// ----------------------------------------------------------- VF_CDTCAL
// The time-step limits of vf_cdtcal.f:107-141 per cell with NF != -1: the
// advective limit V/max|flux| (a boundary face of a dry cell and dry
// boundary value does not count) and the diffusive limit
// 0.5/(1/dx^2+1/dy^2+1/dz^2)/ANU.  The reference folds them into a running
// DT = V/MAX(FL1..FL6, V/DT) in K,J,I order, which in exact arithmetic is
// the minimum of the limits; here each limit is computed with the same
// roundings and the minimum is taken directly (order-free), the form the
// oracle's GPU order restates.  Row minima go to rb (+inf for none).
__device__ __forceinline__ double dmin_ne(double a, double b) { return b < a ? b : a; }
__global__ void k_cdtcal(Geo g, Fld f, double *rb) {
  double m = __longlong_as_double(0x7ff0000000000000LL);  // +inf
  const long long nrows = (long long)g.NJ * g.NK;
  ROW_LOOP_BEGIN(g)
  if (I >= 2 && I <= g.NI - 1 && J >= 2 && J <= g.NJ - 1 && K >= 2 && K <= g.NK - 1) {
    const long long c = cid(g, I, J, K);
    if (f.nf[c] != -1) {
      const double DX = XX_(2, I), DY = YY_(2, J), DZ = ZZ_(2, K);
      const double DXY = DX * DY, DXZ = DX * DZ, DYZ = DY * DZ, FC = f.ff[c];
      const double V = f.ggv[c] * DX * DY * DZ;
      double FL[6] = {fabs(DYZ * f.ggx[c] * f.uu[c]), fabs(DYZ * A(f.ggx, I + 1, J, K) * A(f.uu, I + 1, J, K)),
                      fabs(DXZ * f.ggy[c] * f.vv[c]), fabs(DXZ * A(f.ggy, I, J + 1, K) * A(f.vv, I, J + 1, K)),
                      fabs(DXY * f.ggz[c] * f.ww[c]), fabs(DXY * A(f.ggz, I, J, K + 1) * A(f.ww, I, J, K + 1))};
      const int ind[6] = {f.indx[c], A(f.indx, I + 1, J, K), f.indy[c], A(f.indy, I, J + 1, K), f.indz[c],
                          A(f.indz, I, J, K + 1)};
#pragma unroll
      for (int q = 0; q < 6; ++q)
        if (ind[q] >= 1 && dmax(FC, f.bcf[ind[q] - 1]) <= 0.0) FL[q] = 0.0;
      double FM = FL[0];
#pragma unroll
      for (int q = 1; q < 6; ++q) FM = dmax(FM, FL[q]);
      if (FM > 0.0) m = dmin_ne(m, V / FM);
      const double V2 = 0.5 / (1.0 / (DX * DX) + 1.0 / (DY * DY) + 1.0 / (DZ * DZ));
      if (f.anu[c] > 0.0) m = dmin_ne(m, V2 / f.anu[c]);
    }
  }
  ROW_LOOP_END
  for (int off = 16; off >= 1; off >>= 1) m = dmin_ne(m, __shfl_down_sync(0xffffffffu, m, off));
  const long long row = (long long)blockIdx.x * ROWS_PER_BLOCK + (threadIdx.x >> 5);
  if ((threadIdx.x & 31) == 0 && row < nrows) rb[row] = m;
}
// vf_cdtcal.f:46, 142-147: DT = MAX(MIN(min(DTMAX/DTSAFE, limits)*DTSAFE,
// 1.2*W), DTMIN) with W = DTNOW, or DTINIT at NNOW = 0.
__global__ void k_cdtcal_fin(const double *rb, long long nrows, double dt0, double dtsafe, double w, double dtmin,
                             double *out) {
  __shared__ double wm[32];
  double m = dt0;
  for (long long r = threadIdx.x; r < nrows; r += blockDim.x) m = dmin_ne(m, rb[r]);
  for (int off = 16; off >= 1; off >>= 1) m = dmin_ne(m, __shfl_down_sync(0xffffffffu, m, off));
  if ((threadIdx.x & 31) == 0) wm[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    double DT = wm[0];
    for (int q = 1; q < (int)(blockDim.x >> 5); ++q) DT = dmin_ne(DT, wm[q]);
    *out = dmax(dmin(DT * dtsafe, 1.20 * w), dtmin);
  }
}

#undef A
#undef XX_
#undef YY_
#undef ZZ_

// ------------------------------------------------------------ launchers
#define RL(kern, ...) (kern<<<row_blocks(g), ROW_THREADS, 0, s>>>(__VA_ARGS__), count_launch())
#define BL(kern, ...) if (g.NB > 0) (kern<<<(g.NB + 255) / 256, 256, 0, s>>>(__VA_ARGS__), count_launch())
void launch_bsuwt(cudaStream_t s, const Geo &g, const Fld &f, const Prm &p) { RL(k_bsuwt, g, f, p); }
void launch_bsuwt2(cudaStream_t s, const Geo &g, const Fld &f) { RL(k_bsuwt2, g, f); }
// Wave-source part of VF_BSUWN (vf_bsuwn.f:81-118): on the source's line,
// the first surface cell of each column from the bottom (obstacle, fluid
// and gas cells skipped) passes the source flow 2 XX(4,I) SRCUV (or
// YY(4,J)) through its face toward the gas.  One thread per column.  A
// column writes a face whose other cell is fluid or gas at that height
// (the surface cell's orientation, VF_FNFPRV), never a face another
// column of the line writes at the same height.
__global__ void k_bsuwn_src(Geo g, Fld f, Prm p) {
  const bool xs = p.iws != 0;
  const int IJ = 2 + (int)(blockIdx.x * blockDim.x + threadIdx.x);
  if (IJ > (xs ? g.NJ : g.NI) - 1) return;
  const int I = xs ? p.iws : IJ, J = xs ? IJ : p.jws;
  for (int K = 2; K <= g.NK - 1; ++K) {
    const long long c = cid(g, I, J, K);
    const int N = f.nf[c];
    if (N == -1 || N == 0 || N == 8) continue;
    const double Q = xs ? 2.0 * gx(g, 4, I) * f.srcuv[(J - 1) + (long long)g.NJ * (K - 1)]
                        : 2.0 * gy(g, 4, J) * f.srcuv[(I - 1) + (long long)g.NI * (K - 1)];
    if (N == 1) {
      const long long d = cid(g, I + 1, J, K);
      f.uu[d] = f.uu[d] + gx(g, 2, I) * Q / f.ggx[d];
    } else if (N == 2) {
      f.uu[c] = f.uu[c] - gx(g, 2, I) * Q / f.ggx[c];
    } else if (N == 3) {
      const long long d = cid(g, I, J + 1, K);
      f.vv[d] = f.vv[d] + gy(g, 2, J) * Q / f.ggy[d];
    } else if (N == 4) {
      f.vv[c] = f.vv[c] - gy(g, 2, J) * Q / f.ggy[c];
    } else if (N == 5) {
      const long long d = cid(g, I, J, K + 1);
      f.ww[d] = f.ww[d] + gz(g, 2, K) * Q / f.ggz[d];
    } else if (N == 6) {
      f.ww[c] = f.ww[c] - gz(g, 2, K) * Q / f.ggz[c];
    }
    break;
  }
}

void launch_bsuwn(cudaStream_t s, const Geo &g, const Fld &f) { RL(k_bsuwn, g, f); }
void launch_bsuwn_src(cudaStream_t s, const Geo &g, const Fld &f, const Prm &p) {
  const int n = (p.iws != 0 ? g.NJ : g.NI) - 2;
  k_bsuwn_src<<<(n + 127) / 128, 128, 0, s>>>(g, f, p);
  count_launch();
}
void launch_bsuwn3(cudaStream_t s, const Geo &g, const Fld &f, const Prm &p) { RL(k_bsuwn3, g, f, p); }
void launch_bsuwem(cudaStream_t s, const Geo &g, const Fld &f, int *nlim) {
  RL(k_bsuwem_count, g, f, nlim);
  RL(k_bsuwem_fix, g, f, nlim);
}
void launch_bspp(cudaStream_t s, const Geo &g, const Fld &f) { RL(k_bspp, g, f); }
// VF_BWFFSF (vf_bwffsf.f:48-128): F of the column next to a fixed-water-
// level side from the level wl = WVLVL + the table's level, per cell
// height; obstacle cells keep theirs.  One thread per cell of the column.
__global__ void k_bwffsf(Geo g, Fld f, int side, int first, int last, double WL) {
  const int n = first + (int)(blockIdx.x * blockDim.x + threadIdx.x);
  const int K = 2 + (int)blockIdx.y;
  if (n > last || K > g.NK - 1) return;
  double VAL;
  if (gz(g, 1, K) > WL) VAL = 0.0;
  else if (gz(g, 1, K + 1) < WL) VAL = 1.0;
  else VAL = (WL - gz(g, 1, K)) / (gz(g, 1, K + 1) - gz(g, 1, K));
  long long c;
  if (side <= 2) c = cid(g, side == 1 ? 2 : g.NI - 1, n, K);
  else c = cid(g, n, side == 3 ? 2 : g.NJ - 1, K);
  if (f.nf[c] != -1) f.ff[c] = VAL;
}
void launch_bwffsf(cudaStream_t s, const Geo &g, const Fld &f, int side, int first, int last, double wl) {
  const int n = last - first + 1;
  if (n <= 0 || g.NK <= 2) return;
  k_bwffsf<<<dim3((n + 127) / 128, g.NK - 2), 128, 0, s>>>(g, f, side, first, last, wl);
  count_launch();
}
void launch_bwuwt(cudaStream_t s, const Geo &g, const Fld &f, const Prm &p, int *err) { BL(k_bwuwt, g, f, p, err); }
void launch_bwpp(cudaStream_t s, const Geo &g, const Fld &f) { BL(k_bwpp, g, f); }
void launch_bwff(cudaStream_t s, const Geo &g, const Fld &f, int *err) { BL(k_bwff, g, f, err); }
void launch_cdiv(cudaStream_t s, const Geo &g, const Fld &f, double *rb) { RL(k_cdiv, g, f, rb); }
void launch_cdtcal(cudaStream_t s, const Geo &g, const Fld &f, double *rb, double dt0, double dtsafe, double w,
                   double dtmin, double *out) {
  RL(k_cdtcal, g, f, rb);
  k_cdtcal_fin<<<1, 1024, 0, s>>>(rb, (long long)g.NJ * g.NK, dt0, dtsafe, w, dtmin, out);
  count_launch();
}
#undef RL
#undef BL

}  // namespace cadmas
