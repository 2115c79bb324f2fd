// k_momentum.cu -- porous momentum predictor of VF_V1CAL (vf_v1cal.f:118-230).
//
//   k_flux     VF_VFLXDU/DV/DW  (vf_vflxdu.f:62-347, vf_vflxdv.f, vf_vflxdw.f)
//              all nine face fluxes of one cell index in one pass
//   k_predict  VF_VGENE + VF_VEULER (vf_vgene.f:84-332, vf_veuler.f:115-284)
//              sources and provisional velocity fused; reads the old
//              velocities and writes the new ones to the other buffer, so
//              the interpolated neighbour velocities of the drag term are
//              the values before the update, as in the reference
//   k_bwuwn    VF_BWUWN boundary-list loop (vf_bwuwn.f:93-160)
//
// Roofline: HBM bound.  k_flux reads u,v,w,ANU,GLX..Z,GGX..Z,NF,INDX..Z,INDC
// once (plus cached neighbours) and writes 9 flux arrays; k_predict reads
// the 9 fluxes, u,v,w,p,GGV,GLV,CD0,GGX..Z,NF,INDX..Z and writes u,v,w.
#include "cadmas_dev.cuh"
#include "kernels.h"

namespace cadmas {

// ------------------------------------------------------------- fluxes
// The "special" branch of the cross fluxes takes the tangential velocity on
// a boundary face from the face's type (vf_vflxdu.f:128-156).
__device__ __forceinline__ double bnd_tan(const Fld &f, int IS, int nsFirst, double vFirst,
                                          double vSecond, const double *bc) {
  int t = indb(f, 3, IS);
  if (t == 1 || t == 4) return (indb(f, 2, IS) == nsFirst) ? vFirst : vSecond;
  return bc[IS - 1];
}

__global__ void __launch_bounds__(ROW_THREADS, 3) k_flux(Geo g, Fld f, Prm p, double *FLUU, double *FLUV, double *FLUW,
                       double *FLVU, double *FLVV, double *FLVW, double *FLWU, double *FLWV,
                       double *FLWW) {
  const double SU = p.scmvp, SC = 1.0 - p.scmvp;
  const double *UU = f.uu, *VV = f.vv, *WW = f.ww, *ANU = f.anu;
  const int *NF = f.nf;
  ROW_LOOP_BEGIN(g)
  const long long c = cid(g, I, J, K);
  const int NI = g.NI, NJ = g.NJ, NK = g.NK;
#define A(a, i, j, k) a[cid(g, i, j, k)]
#define XX_(m, i) gx(g, m, i)
#define YY_(m, j) gy(g, m, j)
#define ZZ_(m, k) gz(g, m, k)
  // ---------------- FLUU (Gx*u)*u, Gx*Nu*2du/dx   vf_vflxdu.f:71-91
  {
    double F = 0.0;
    if (K >= 2 && K <= NK - 1 && J >= 2 && J <= NJ - 1 && I >= 2 && I <= NI - 1 && f.indc[c] != -1) {
      double WIN = (A(f.glx, I, J, K) * A(UU, I, J, K) + A(f.glx, I + 1, J, K) * A(UU, I + 1, J, K)) * 0.5;
      double FG = WIN * (A(UU, I, J, K) + A(UU, I + 1, J, K)) * 0.5;
      F = F - SU * (dmax(WIN, 0.0) * A(UU, I, J, K) - dmax(-WIN, 0.0) * A(UU, I + 1, J, K)) - SC * FG;
      F = F + (A(f.ggx, I, J, K) + A(f.ggx, I + 1, J, K)) * A(ANU, I, J, K) * XX_(4, I) *
                  (A(UU, I + 1, J, K) - A(UU, I, J, K));
    }
    FLUU[c] = F;
  }
  // ---------------- FLUV (Gy*v)*u   vf_vflxdu.f:93-213
  {
    double F = 0.0;
    if (K >= 2 && J >= 2 && I >= 3 && I <= NI - 1) {
      int IC = A(NF, I - 1, J - 1, K) * A(NF, I, J - 1, K) * A(NF, I - 1, J, K) * A(NF, I, J, K);
      int IT = A(f.indx, I, J, K), IB = A(f.indx, I, J - 1, K);
      if (IC != 0 || (IT != 0 && IB != 0)) {
      } else if (IT == 0 && IB == 0) {
        double WIN = XX_(6, I) * (XX_(2, I - 1) * A(f.gly, I, J, K) * A(VV, I, J, K) +
                                  XX_(2, I) * A(f.gly, I - 1, J, K) * A(VV, I - 1, J, K));
        double FG = WIN * YY_(6, J) * (YY_(2, J - 1) * A(UU, I, J, K) + YY_(2, J) * A(UU, I, J - 1, K));
        F = F - SU * (dmax(WIN, 0.0) * A(UU, I, J - 1, K) - dmax(-WIN, 0.0) * A(UU, I, J, K)) - SC * FG;
        double GG = XX_(6, I) * (XX_(2, I - 1) * A(f.ggy, I, J, K) + XX_(2, I) * A(f.ggy, I - 1, J, K));
        double ANR = YY_(6, J) * (YY_(2, J - 1) * A(ANU, I, J, K) + YY_(2, J) * A(ANU, I, J - 1, K));
        double ANL = YY_(6, J) * (YY_(2, J - 1) * A(ANU, I - 1, J, K) + YY_(2, J) * A(ANU, I - 1, J - 1, K));
        double AN = XX_(6, I) * (XX_(2, I - 1) * ANR + XX_(2, I) * ANL);
        double D1 = YY_(5, J) * (A(UU, I, J, K) - A(UU, I, J - 1, K));
        double D2 = XX_(5, I) * (A(VV, I, J, K) - A(VV, I - 1, J, K));
        F = F + GG * AN * (D1 + D2);
      } else {
        double BR, BL;
        int IS = A(f.indy, I, J, K);
        if (IS >= 1) BR = bnd_tan(f, IS, 3, A(UU, I, J, K), A(UU, I, J - 1, K), f.bcu);
        else BR = YY_(6, J) * (YY_(2, J - 1) * (A(UU, I, J, K) + A(UU, I + 1, J, K)) +
                               YY_(2, J) * (A(UU, I, J - 1, K) + A(UU, I + 1, J - 1, K))) * 0.5;
        IS = A(f.indy, I - 1, J, K);
        if (IS >= 1) BL = bnd_tan(f, IS, 3, A(UU, I, J, K), A(UU, I, J - 1, K), f.bcu);
        else BL = YY_(6, J) * (YY_(2, J - 1) * (A(UU, I, J, K) + A(UU, I - 1, J, K)) +
                               YY_(2, J) * (A(UU, I, J - 1, K) + A(UU, I - 1, J - 1, K))) * 0.5;
        double WIN = XX_(6, I) * (XX_(2, I - 1) * A(f.gly, I, J, K) * A(VV, I, J, K) +
                                  XX_(2, I) * A(f.gly, I - 1, J, K) * A(VV, I - 1, J, K));
        double FG = XX_(6, I) * (XX_(2, I) * A(f.gly, I, J, K) * A(VV, I, J, K) * BR +
                                 XX_(2, I - 1) * A(f.gly, I - 1, J, K) * A(VV, I - 1, J, K) * BL);
        if (IT == 0 && WIN < 0.0) F = F - SU * WIN * A(UU, I, J, K) - SC * FG;
        else if (IB == 0 && WIN > 0.0) F = F - SU * WIN * A(UU, I, J - 1, K) - SC * FG;
        else F = F - FG;
        double GG = XX_(6, I) * (XX_(2, I - 1) * A(f.ggy, I, J, K) + XX_(2, I) * A(f.ggy, I - 1, J, K));
        FG = XX_(6, I) * (XX_(2, I) * BR + XX_(2, I - 1) * BL);
        double ANR, ANL;
        if (A(NF, I, J, K) == -1) ANR = A(ANU, I, J - 1, K);
        else if (A(NF, I, J - 1, K) == -1) ANR = A(ANU, I, J, K);
        else ANR = YY_(6, J) * (YY_(2, J - 1) * A(ANU, I, J, K) + YY_(2, J) * A(ANU, I, J - 1, K));
        if (A(NF, I - 1, J, K) == -1) ANL = A(ANU, I - 1, J - 1, K);
        else if (A(NF, I - 1, J - 1, K) == -1) ANL = A(ANU, I - 1, J, K);
        else ANL = YY_(6, J) * (YY_(2, J - 1) * A(ANU, I - 1, J, K) + YY_(2, J) * A(ANU, I - 1, J - 1, K));
        double AN = XX_(6, I) * (XX_(2, I - 1) * ANR + XX_(2, I) * ANL);
        double D1 = (IT == 0) ? YY_(4, J) * (A(UU, I, J, K) - FG) * 2.0 : YY_(4, J - 1) * (FG - A(UU, I, J - 1, K)) * 2.0;
        double D2 = XX_(5, I) * (A(VV, I, J, K) - A(VV, I - 1, J, K));
        F = F + GG * AN * (D1 + D2);
      }
    }
    FLUV[c] = F;
  }
  // ---------------- FLUW (Gz*w)*u   vf_vflxdu.f:215-345
  {
    double F = 0.0;
    if (K >= 2 && J >= 2 && J <= NJ - 1 && I >= 3 && I <= NI - 1) {
      int IC = A(NF, I - 1, J, K - 1) * A(NF, I, J, K - 1) * A(NF, I - 1, J, K) * A(NF, I, J, K);
      int IT = A(f.indx, I, J, K), IB = A(f.indx, I, J, K - 1);
      if (IC != 0 || (IT != 0 && IB != 0)) {
      } else if (IT == 0 && IB == 0) {
        double WIN = XX_(6, I) * (XX_(2, I - 1) * A(f.glz, I, J, K) * A(WW, I, J, K) +
                                  XX_(2, I) * A(f.glz, I - 1, J, K) * A(WW, I - 1, J, K));
        double FG = WIN * ZZ_(6, K) * (ZZ_(2, K - 1) * A(UU, I, J, K) + ZZ_(2, K) * A(UU, I, J, K - 1));
        F = F - SU * (dmax(WIN, 0.0) * A(UU, I, J, K - 1) - dmax(-WIN, 0.0) * A(UU, I, J, K)) - SC * FG;
        double GG = XX_(6, I) * (XX_(2, I - 1) * A(f.ggz, I, J, K) + XX_(2, I) * A(f.ggz, I - 1, J, K));
        double ANR = ZZ_(6, K) * (ZZ_(2, K - 1) * A(ANU, I, J, K) + ZZ_(2, K) * A(ANU, I, J, K - 1));
        double ANL = ZZ_(6, K) * (ZZ_(2, K - 1) * A(ANU, I - 1, J, K) + ZZ_(2, K) * A(ANU, I - 1, J, K - 1));
        double AN = XX_(6, I) * (XX_(2, I - 1) * ANR + XX_(2, I) * ANL);
        double D1 = ZZ_(5, K) * (A(UU, I, J, K) - A(UU, I, J, K - 1));
        double D2 = XX_(5, I) * (A(WW, I, J, K) - A(WW, I - 1, J, K));
        F = F + GG * AN * (D1 + D2);
      } else {
        double BR, BL;
        int IS = A(f.indz, I, J, K);
        if (IS >= 1) BR = bnd_tan(f, IS, 5, A(UU, I, J, K), A(UU, I, J, K - 1), f.bcu);
        else BR = ZZ_(6, K) * (ZZ_(2, K - 1) * (A(UU, I, J, K) + A(UU, I + 1, J, K)) +
                               ZZ_(2, K) * (A(UU, I, J, K - 1) + A(UU, I + 1, J, K - 1))) * 0.5;
        IS = A(f.indz, I - 1, J, K);
        if (IS >= 1) BL = bnd_tan(f, IS, 5, A(UU, I, J, K), A(UU, I, J, K - 1), f.bcu);
        else BL = ZZ_(6, K) * (ZZ_(2, K - 1) * (A(UU, I, J, K) + A(UU, I - 1, J, K)) +
                               ZZ_(2, K) * (A(UU, I, J, K - 1) + A(UU, I - 1, J, K - 1))) * 0.5;
        double WIN = XX_(6, I) * (XX_(2, I - 1) * A(f.glz, I, J, K) * A(WW, I, J, K) +
                                  XX_(2, I) * A(f.glz, I - 1, J, K) * A(WW, I - 1, J, K));
        double FG = XX_(6, I) * (XX_(2, I) * A(f.glz, I, J, K) * A(WW, I, J, K) * BR +
                                 XX_(2, I - 1) * A(f.glz, I - 1, J, K) * A(WW, I - 1, J, K) * BL);
        if (IT == 0 && WIN < 0.0) F = F - SU * WIN * A(UU, I, J, K) - SC * FG;
        else if (IB == 0 && WIN > 0.0) F = F - SU * WIN * A(UU, I, J, K - 1) - SC * FG;
        else F = F - FG;
        double GG = XX_(6, I) * (XX_(2, I - 1) * A(f.ggz, I, J, K) + XX_(2, I) * A(f.ggz, I - 1, J, K));
        FG = XX_(6, I) * (XX_(2, I) * BR + XX_(2, I - 1) * BL);
        double ANR, ANL;
        if (A(NF, I, J, K) == -1) ANR = A(ANU, I, J, K - 1);
        else if (A(NF, I, J, K - 1) == -1) ANR = A(ANU, I, J, K);
        else ANR = ZZ_(6, K) * (ZZ_(2, K - 1) * A(ANU, I, J, K) + ZZ_(2, K) * A(ANU, I, J, K - 1));
        if (A(NF, I - 1, J, K) == -1) ANL = A(ANU, I - 1, J, K - 1);
        else if (A(NF, I - 1, J, K - 1) == -1) ANL = A(ANU, I - 1, J, K);
        else ANL = ZZ_(6, K) * (ZZ_(2, K - 1) * A(ANU, I - 1, J, K) + ZZ_(2, K) * A(ANU, I - 1, J, K - 1));
        double AN = XX_(6, I) * (XX_(2, I - 1) * ANR + XX_(2, I) * ANL);
        double D1 = (IT == 0) ? ZZ_(4, K) * (A(UU, I, J, K) - FG) * 2.0 : ZZ_(4, K - 1) * (FG - A(UU, I, J, K - 1)) * 2.0;
        double D2 = XX_(5, I) * (A(WW, I, J, K) - A(WW, I - 1, J, K));
        F = F + GG * AN * (D1 + D2);
      }
    }
    FLUW[c] = F;
  }
  // ---------------- FLVV (Gy*v)*v   vf_vflxdv.f:71-91
  {
    double F = 0.0;
    if (K >= 2 && K <= NK - 1 && J >= 2 && J <= NJ - 1 && I >= 2 && I <= NI - 1 && f.indc[c] != -1) {
      double WIN = (A(f.gly, I, J, K) * A(VV, I, J, K) + A(f.gly, I, J + 1, K) * A(VV, I, J + 1, K)) * 0.5;
      double FG = WIN * (A(VV, I, J, K) + A(VV, I, J + 1, K)) * 0.5;
      F = F - SU * (dmax(WIN, 0.0) * A(VV, I, J, K) - dmax(-WIN, 0.0) * A(VV, I, J + 1, K)) - SC * FG;
      F = F + (A(f.ggy, I, J, K) + A(f.ggy, I, J + 1, K)) * A(ANU, I, J, K) * YY_(4, J) *
                  (A(VV, I, J + 1, K) - A(VV, I, J, K));
    }
    FLVV[c] = F;
  }
  // ---------------- FLVU (Gx*u)*v   vf_vflxdv.f:93-213
  {
    double F = 0.0;
    if (K >= 2 && J >= 3 && J <= NJ - 1 && I >= 2) {
      int IC = A(NF, I - 1, J - 1, K) * A(NF, I - 1, J, K) * A(NF, I, J - 1, K) * A(NF, I, J, K);
      int IT = A(f.indy, I, J, K), IB = A(f.indy, I - 1, J, K);
      if (IC != 0 || (IT != 0 && IB != 0)) {
      } else if (IT == 0 && IB == 0) {
        double WIN = YY_(6, J) * (YY_(2, J - 1) * A(f.glx, I, J, K) * A(UU, I, J, K) +
                                  YY_(2, J) * A(f.glx, I, J - 1, K) * A(UU, I, J - 1, K));
        double FG = WIN * XX_(6, I) * (XX_(2, I - 1) * A(VV, I, J, K) + XX_(2, I) * A(VV, I - 1, J, K));
        F = F - SU * (dmax(WIN, 0.0) * A(VV, I - 1, J, K) - dmax(-WIN, 0.0) * A(VV, I, J, K)) - SC * FG;
        double GG = YY_(6, J) * (YY_(2, J - 1) * A(f.ggx, I, J, K) + YY_(2, J) * A(f.ggx, I, J - 1, K));
        double ANR = XX_(6, I) * (XX_(2, I - 1) * A(ANU, I, J, K) + XX_(2, I) * A(ANU, I - 1, J, K));
        double ANL = XX_(6, I) * (XX_(2, I - 1) * A(ANU, I, J - 1, K) + XX_(2, I) * A(ANU, I - 1, J - 1, K));
        double AN = YY_(6, J) * (YY_(2, J - 1) * ANR + YY_(2, J) * ANL);
        double D1 = XX_(5, I) * (A(VV, I, J, K) - A(VV, I - 1, J, K));
        double D2 = YY_(5, J) * (A(UU, I, J, K) - A(UU, I, J - 1, K));
        F = F + GG * AN * (D1 + D2);
      } else {
        double BR, BL;
        int IS = A(f.indx, I, J, K);
        if (IS >= 1) BR = bnd_tan(f, IS, 1, A(VV, I, J, K), A(VV, I - 1, J, K), f.bcv);
        else BR = XX_(6, I) * (XX_(2, I - 1) * (A(VV, I, J, K) + A(VV, I, J + 1, K)) +
                               XX_(2, I) * (A(VV, I - 1, J, K) + A(VV, I - 1, J + 1, K))) * 0.5;
        IS = A(f.indx, I, J - 1, K);
        if (IS >= 1) BL = bnd_tan(f, IS, 1, A(VV, I, J, K), A(VV, I - 1, J, K), f.bcv);
        else BL = XX_(6, I) * (XX_(2, I - 1) * (A(VV, I, J, K) + A(VV, I, J - 1, K)) +
                               XX_(2, I) * (A(VV, I - 1, J, K) + A(VV, I - 1, J - 1, K))) * 0.5;
        double WIN = YY_(6, J) * (YY_(2, J - 1) * A(f.glx, I, J, K) * A(UU, I, J, K) +
                                  YY_(2, J) * A(f.glx, I, J - 1, K) * A(UU, I, J - 1, K));
        double FG = YY_(6, J) * (YY_(2, J) * A(f.glx, I, J, K) * A(UU, I, J, K) * BR +
                                 YY_(2, J - 1) * A(f.glx, I, J - 1, K) * A(UU, I, J - 1, K) * BL);
        if (IT == 0 && WIN < 0.0) F = F - SU * WIN * A(VV, I, J, K) - SC * FG;
        else if (IB == 0 && WIN > 0.0) F = F - SU * WIN * A(VV, I - 1, J, K) - SC * FG;
        else F = F - FG;
        double GG = YY_(6, J) * (YY_(2, J - 1) * A(f.ggx, I, J, K) + YY_(2, J) * A(f.ggx, I, J - 1, K));
        FG = YY_(6, J) * (YY_(2, J) * BR + YY_(2, J - 1) * BL);
        double ANR, ANL;
        if (A(NF, I, J, K) == -1) ANR = A(ANU, I - 1, J, K);
        else if (A(NF, I - 1, J, K) == -1) ANR = A(ANU, I, J, K);
        else ANR = XX_(6, I) * (XX_(2, I - 1) * A(ANU, I, J, K) + XX_(2, I) * A(ANU, I - 1, J, K));
        if (A(NF, I, J - 1, K) == -1) ANL = A(ANU, I - 1, J - 1, K);
        else if (A(NF, I - 1, J - 1, K) == -1) ANL = A(ANU, I, J - 1, K);
        else ANL = XX_(6, I) * (XX_(2, I - 1) * A(ANU, I, J - 1, K) + XX_(2, I) * A(ANU, I - 1, J - 1, K));
        double AN = YY_(6, J) * (YY_(2, J - 1) * ANR + YY_(2, J) * ANL);
        double D1 = (IT == 0) ? XX_(4, I) * (A(VV, I, J, K) - FG) * 2.0 : XX_(4, I - 1) * (FG - A(VV, I - 1, J, K)) * 2.0;
        double D2 = YY_(5, J) * (A(UU, I, J, K) - A(UU, I, J - 1, K));
        F = F + GG * AN * (D1 + D2);
      }
    }
    FLVU[c] = F;
  }
  // ---------------- FLVW (Gz*w)*v   vf_vflxdv.f:215-345
  {
    double F = 0.0;
    if (K >= 2 && J >= 3 && J <= NJ - 1 && I >= 2 && I <= NI - 1) {
      int IC = A(NF, I, J - 1, K - 1) * A(NF, I, J, K - 1) * A(NF, I, J - 1, K) * A(NF, I, J, K);
      int IT = A(f.indy, I, J, K), IB = A(f.indy, I, J, K - 1);
      if (IC != 0 || (IT != 0 && IB != 0)) {
      } else if (IT == 0 && IB == 0) {
        double WIN = YY_(6, J) * (YY_(2, J - 1) * A(f.glz, I, J, K) * A(WW, I, J, K) +
                                  YY_(2, J) * A(f.glz, I, J - 1, K) * A(WW, I, J - 1, K));
        double FG = WIN * ZZ_(6, K) * (ZZ_(2, K - 1) * A(VV, I, J, K) + ZZ_(2, K) * A(VV, I, J, K - 1));
        F = F - SU * (dmax(WIN, 0.0) * A(VV, I, J, K - 1) - dmax(-WIN, 0.0) * A(VV, I, J, K)) - SC * FG;
        double GG = YY_(6, J) * (YY_(2, J - 1) * A(f.ggz, I, J, K) + YY_(2, J) * A(f.ggz, I, J - 1, K));
        double ANR = ZZ_(6, K) * (ZZ_(2, K - 1) * A(ANU, I, J, K) + ZZ_(2, K) * A(ANU, I, J, K - 1));
        double ANL = ZZ_(6, K) * (ZZ_(2, K - 1) * A(ANU, I, J - 1, K) + ZZ_(2, K) * A(ANU, I, J - 1, K - 1));
        double AN = YY_(6, J) * (YY_(2, J - 1) * ANR + YY_(2, J) * ANL);
        double D1 = ZZ_(5, K) * (A(VV, I, J, K) - A(VV, I, J, K - 1));
        double D2 = YY_(5, J) * (A(WW, I, J, K) - A(WW, I, J - 1, K));
        F = F + GG * AN * (D1 + D2);
      } else {
        double BR, BL;
        int IS = A(f.indz, I, J, K);
        if (IS >= 1) BR = bnd_tan(f, IS, 5, A(VV, I, J, K), A(VV, I, J, K - 1), f.bcv);
        else BR = ZZ_(6, K) * (ZZ_(2, K - 1) * (A(VV, I, J, K) + A(VV, I, J + 1, K)) +
                               ZZ_(2, K) * (A(VV, I, J, K - 1) + A(VV, I, J + 1, K - 1))) * 0.5;
        IS = A(f.indz, I, J - 1, K);
        if (IS >= 1) BL = bnd_tan(f, IS, 5, A(VV, I, J, K), A(VV, I, J, K - 1), f.bcv);
        else BL = ZZ_(6, K) * (ZZ_(2, K - 1) * (A(VV, I, J, K) + A(VV, I, J - 1, K)) +
                               ZZ_(2, K) * (A(VV, I, J, K - 1) + A(VV, I, J - 1, K - 1))) * 0.5;
        double WIN = YY_(6, J) * (YY_(2, J - 1) * A(f.glz, I, J, K) * A(WW, I, J, K) +
                                  YY_(2, J) * A(f.glz, I, J - 1, K) * A(WW, I, J - 1, K));
        double FG = YY_(6, J) * (YY_(2, J) * A(f.glz, I, J, K) * A(WW, I, J, K) * BR +
                                 YY_(2, J - 1) * A(f.glz, I, J - 1, K) * A(WW, I, J - 1, K) * BL);
        if (IT == 0 && WIN < 0.0) F = F - SU * WIN * A(VV, I, J, K) - SC * FG;
        else if (IB == 0 && WIN > 0.0) F = F - SU * WIN * A(VV, I, J, K - 1) - SC * FG;
        else F = F - FG;
        double GG = YY_(6, J) * (YY_(2, J - 1) * A(f.ggz, I, J, K) + YY_(2, J) * A(f.ggz, I, J - 1, K));
        FG = YY_(6, J) * (YY_(2, J) * BR + YY_(2, J - 1) * BL);
        double ANR, ANL;
        if (A(NF, I, J, K) == -1) ANR = A(ANU, I, J, K - 1);
        else if (A(NF, I, J, K - 1) == -1) ANR = A(ANU, I, J, K);
        else ANR = ZZ_(6, K) * (ZZ_(2, K - 1) * A(ANU, I, J, K) + ZZ_(2, K) * A(ANU, I, J, K - 1));
        if (A(NF, I, J - 1, K) == -1) ANL = A(ANU, I, J - 1, K - 1);
        else if (A(NF, I, J - 1, K - 1) == -1) ANL = A(ANU, I, J - 1, K);
        else ANL = ZZ_(6, K) * (ZZ_(2, K - 1) * A(ANU, I, J - 1, K) + ZZ_(2, K) * A(ANU, I, J - 1, K - 1));
        double AN = YY_(6, J) * (YY_(2, J - 1) * ANR + YY_(2, J) * ANL);
        double D1 = (IT == 0) ? ZZ_(4, K) * (A(VV, I, J, K) - FG) * 2.0 : ZZ_(4, K - 1) * (FG - A(VV, I, J, K - 1)) * 2.0;
        double D2 = YY_(5, J) * (A(WW, I, J, K) - A(WW, I, J - 1, K));
        F = F + GG * AN * (D1 + D2);
      }
    }
    FLVW[c] = F;
  }
  // ---------------- FLWW (Gz*w)*w   vf_vflxdw.f:62-82
  {
    double F = 0.0;
    if (K >= 2 && K <= NK - 1 && J >= 2 && J <= NJ - 1 && I >= 2 && I <= NI - 1 && f.indc[c] != -1) {
      double WIN = (A(f.glz, I, J, K) * A(WW, I, J, K) + A(f.glz, I, J, K + 1) * A(WW, I, J, K + 1)) * 0.5;
      double FG = WIN * (A(WW, I, J, K) + A(WW, I, J, K + 1)) * 0.5;
      F = F - SU * (dmax(WIN, 0.0) * A(WW, I, J, K) - dmax(-WIN, 0.0) * A(WW, I, J, K + 1)) - SC * FG;
      F = F + (A(f.ggz, I, J, K) + A(f.ggz, I, J, K + 1)) * A(ANU, I, J, K) * ZZ_(4, K) *
                  (A(WW, I, J, K + 1) - A(WW, I, J, K));
    }
    FLWW[c] = F;
  }
  // ---------------- FLWU (Gx*u)*w   vf_vflxdw.f:84-204
  {
    double F = 0.0;
    if (K >= 3 && K <= NK - 1 && J >= 2 && J <= NJ - 1 && I >= 2) {
      int IC = A(NF, I - 1, J, K - 1) * A(NF, I - 1, J, K) * A(NF, I, J, K - 1) * A(NF, I, J, K);
      int IT = A(f.indz, I, J, K), IB = A(f.indz, I - 1, J, K);
      if (IC != 0 || (IT != 0 && IB != 0)) {
      } else if (IT == 0 && IB == 0) {
        double WIN = ZZ_(6, K) * (ZZ_(2, K - 1) * A(f.glx, I, J, K) * A(UU, I, J, K) +
                                  ZZ_(2, K) * A(f.glx, I, J, K - 1) * A(UU, I, J, K - 1));
        double FG = WIN * XX_(6, I) * (XX_(2, I - 1) * A(WW, I, J, K) + XX_(2, I) * A(WW, I - 1, J, K));
        F = F - SU * (dmax(WIN, 0.0) * A(WW, I - 1, J, K) - dmax(-WIN, 0.0) * A(WW, I, J, K)) - SC * FG;
        double GG = ZZ_(6, K) * (ZZ_(2, K - 1) * A(f.ggx, I, J, K) + ZZ_(2, K) * A(f.ggx, I, J, K - 1));
        double ANR = XX_(6, I) * (XX_(2, I - 1) * A(ANU, I, J, K) + XX_(2, I) * A(ANU, I - 1, J, K));
        double ANL = XX_(6, I) * (XX_(2, I - 1) * A(ANU, I, J, K - 1) + XX_(2, I) * A(ANU, I - 1, J, K - 1));
        double AN = ZZ_(6, K) * (ZZ_(2, K - 1) * ANR + ZZ_(2, K) * ANL);
        double D1 = XX_(5, I) * (A(WW, I, J, K) - A(WW, I - 1, J, K));
        double D2 = ZZ_(5, K) * (A(UU, I, J, K) - A(UU, I, J, K - 1));
        F = F + GG * AN * (D1 + D2);
      } else {
        double BR, BL;
        int IS = A(f.indx, I, J, K);
        if (IS >= 1) BR = bnd_tan(f, IS, 1, A(WW, I, J, K), A(WW, I - 1, J, K), f.bcw);
        else BR = XX_(6, I) * (XX_(2, I - 1) * (A(WW, I, J, K) + A(WW, I, J, K + 1)) +
                               XX_(2, I) * (A(WW, I - 1, J, K) + A(WW, I - 1, J, K + 1))) * 0.5;
        IS = A(f.indx, I, J, K - 1);
        if (IS >= 1) BL = bnd_tan(f, IS, 1, A(WW, I, J, K), A(WW, I - 1, J, K), f.bcw);
        else BL = XX_(6, I) * (XX_(2, I - 1) * (A(WW, I, J, K) + A(WW, I, J, K - 1)) +
                               XX_(2, I) * (A(WW, I - 1, J, K) + A(WW, I - 1, J, K - 1))) * 0.5;
        double WIN = ZZ_(6, K) * (ZZ_(2, K - 1) * A(f.glx, I, J, K) * A(UU, I, J, K) +
                                  ZZ_(2, K) * A(f.glx, I, J, K - 1) * A(UU, I, J, K - 1));
        double FG = ZZ_(6, K) * (ZZ_(2, K) * A(f.glx, I, J, K) * A(UU, I, J, K) * BR +
                                 ZZ_(2, K - 1) * A(f.glx, I, J, K - 1) * A(UU, I, J, K - 1) * BL);
        if (IT == 0 && WIN < 0.0) F = F - SU * WIN * A(WW, I, J, K) - SC * FG;
        else if (IB == 0 && WIN > 0.0) F = F - SU * WIN * A(WW, I - 1, J, K) - SC * FG;
        else F = F - FG;
        double GG = ZZ_(6, K) * (ZZ_(2, K - 1) * A(f.ggx, I, J, K) + ZZ_(2, K) * A(f.ggx, I, J, K - 1));
        FG = ZZ_(6, K) * (ZZ_(2, K) * BR + ZZ_(2, K - 1) * BL);
        double ANR, ANL;
        if (A(NF, I, J, K) == -1) ANR = A(ANU, I - 1, J, K);
        else if (A(NF, I - 1, J, K) == -1) ANR = A(ANU, I, J, K);
        else ANR = XX_(6, I) * (XX_(2, I - 1) * A(ANU, I, J, K) + XX_(2, I) * A(ANU, I - 1, J, K));
        if (A(NF, I, J, K - 1) == -1) ANL = A(ANU, I - 1, J, K - 1);
        else if (A(NF, I - 1, J, K - 1) == -1) ANL = A(ANU, I, J, K - 1);
        else ANL = XX_(6, I) * (XX_(2, I - 1) * A(ANU, I, J, K - 1) + XX_(2, I) * A(ANU, I - 1, J, K - 1));
        double AN = ZZ_(6, K) * (ZZ_(2, K - 1) * ANR + ZZ_(2, K) * ANL);
        double D1 = (IT == 0) ? XX_(4, I) * (A(WW, I, J, K) - FG) * 2.0 : XX_(4, I - 1) * (FG - A(WW, I - 1, J, K)) * 2.0;
        double D2 = ZZ_(5, K) * (A(UU, I, J, K) - A(UU, I, J, K - 1));
        F = F + GG * AN * (D1 + D2);
      }
    }
    FLWU[c] = F;
  }
  // ---------------- FLWV (Gy*v)*w   vf_vflxdw.f:206-340
  {
    double F = 0.0;
    if (K >= 3 && K <= NK - 1 && J >= 2 && I >= 2 && I <= NI - 1) {
      int IC = A(NF, I, J - 1, K - 1) * A(NF, I, J - 1, K) * A(NF, I, J, K - 1) * A(NF, I, J, K);
      int IT = A(f.indz, I, J, K), IB = A(f.indz, I, J - 1, K);
      if (IC != 0 || (IT != 0 && IB != 0)) {
      } else if (IT == 0 && IB == 0) {
        double WIN = ZZ_(6, K) * (ZZ_(2, K - 1) * A(f.gly, I, J, K) * A(VV, I, J, K) +
                                  ZZ_(2, K) * A(f.gly, I, J, K - 1) * A(VV, I, J, K - 1));
        double FG = WIN * YY_(6, J) * (YY_(2, J - 1) * A(WW, I, J, K) + YY_(2, J) * A(WW, I, J - 1, K));
        F = F - SU * (dmax(WIN, 0.0) * A(WW, I, J - 1, K) - dmax(-WIN, 0.0) * A(WW, I, J, K)) - SC * FG;
        double GG = ZZ_(6, K) * (ZZ_(2, K - 1) * A(f.ggy, I, J, K) + ZZ_(2, K) * A(f.ggy, I, J, K - 1));
        double ANR = YY_(6, J) * (YY_(2, J - 1) * A(ANU, I, J, K) + YY_(2, J) * A(ANU, I, J - 1, K));
        double ANL = YY_(6, J) * (YY_(2, J - 1) * A(ANU, I, J, K - 1) + YY_(2, J) * A(ANU, I, J - 1, K - 1));
        double AN = ZZ_(6, K) * (ZZ_(2, K - 1) * ANR + ZZ_(2, K) * ANL);
        double D1 = YY_(5, J) * (A(WW, I, J, K) - A(WW, I, J - 1, K));
        double D2 = ZZ_(5, K) * (A(VV, I, J, K) - A(VV, I, J, K - 1));
        F = F + GG * AN * (D1 + D2);
      } else {
        double BR, BL;
        int IS = A(f.indy, I, J, K);
        if (IS >= 1) BR = bnd_tan(f, IS, 3, A(WW, I, J, K), A(WW, I, J - 1, K), f.bcw);
        else BR = YY_(6, J) * (YY_(2, J - 1) * (A(WW, I, J, K) + A(WW, I, J, K + 1)) +
                               YY_(2, J) * (A(WW, I, J - 1, K) + A(WW, I, J - 1, K + 1))) * 0.5;
        IS = A(f.indy, I, J, K - 1);
        if (IS >= 1) BL = bnd_tan(f, IS, 3, A(WW, I, J, K), A(WW, I, J - 1, K), f.bcw);
        else BL = YY_(6, J) * (YY_(2, J - 1) * (A(WW, I, J, K) + A(WW, I, J, K - 1)) +
                               YY_(2, J) * (A(WW, I, J - 1, K) + A(WW, I, J - 1, K - 1))) * 0.5;
        double WIN = ZZ_(6, K) * (ZZ_(2, K - 1) * A(f.gly, I, J, K) * A(VV, I, J, K) +
                                  ZZ_(2, K) * A(f.gly, I, J, K - 1) * A(VV, I, J, K - 1));
        double FG = ZZ_(6, K) * (ZZ_(2, K) * A(f.gly, I, J, K) * A(VV, I, J, K) * BR +
                                 ZZ_(2, K - 1) * A(f.gly, I, J, K - 1) * A(VV, I, J, K - 1) * BL);
        if (IT == 0 && WIN < 0.0) F = F - SU * WIN * A(WW, I, J, K) - SC * FG;
        else if (IB == 0 && WIN > 0.0) F = F - SU * WIN * A(WW, I, J - 1, K) - SC * FG;
        else F = F - FG;
        double GG = ZZ_(6, K) * (ZZ_(2, K - 1) * A(f.ggy, I, J, K) + ZZ_(2, K) * A(f.ggy, I, J, K - 1));
        FG = ZZ_(6, K) * (ZZ_(2, K) * BR + ZZ_(2, K - 1) * BL);
        double ANR, ANL;
        if (A(NF, I, J, K) == -1) ANR = A(ANU, I, J - 1, K);
        else if (A(NF, I, J - 1, K) == -1) ANR = A(ANU, I, J, K);
        else ANR = YY_(6, J) * (YY_(2, J - 1) * A(ANU, I, J, K) + YY_(2, J) * A(ANU, I, J - 1, K));
        if (A(NF, I, J, K - 1) == -1) ANL = A(ANU, I, J - 1, K - 1);
        else if (A(NF, I, J - 1, K - 1) == -1) ANL = A(ANU, I, J, K - 1);
        else ANL = YY_(6, J) * (YY_(2, J - 1) * A(ANU, I, J, K - 1) + YY_(2, J) * A(ANU, I, J - 1, K - 1));
        double AN = ZZ_(6, K) * (ZZ_(2, K - 1) * ANR + ZZ_(2, K) * ANL);
        double D1 = (IT == 0) ? YY_(4, J) * (A(WW, I, J, K) - FG) * 2.0 : YY_(4, J - 1) * (FG - A(WW, I, J - 1, K)) * 2.0;
        double D2 = ZZ_(5, K) * (A(VV, I, J, K) - A(VV, I, J, K - 1));
        F = F + GG * AN * (D1 + D2);
      }
    }
    FLWV[c] = F;
  }
#undef A
#undef XX_
#undef YY_
#undef ZZ_
  ROW_LOOP_END
}

// ----------------------------------------------------- sources + update
__device__ __forceinline__ double sponge_dmax(const Prm &p, double X, double Y, bool z) {
  double DMAX = 0.0, D;
  const double *PX = z ? p.spz : p.spx;
  if (p.ip[0] >= 0) { D = X - p.glxmin; if (D <= p.sw[0]) { D = PX[0] * ipow(1.0 - D / p.sw[0], p.ip[0]); if (D > DMAX) DMAX = D; } }
  if (p.ip[1] >= 0) { D = p.glxmax - X; if (D <= p.sw[1]) { D = PX[1] * ipow(1.0 - D / p.sw[1], p.ip[1]); if (D > DMAX) DMAX = D; } }
  if (p.ip[2] >= 0) { D = Y - p.glymin; if (D <= p.sw[2]) { D = PX[2] * ipow(1.0 - D / p.sw[2], p.ip[2]); if (D > DMAX) DMAX = D; } }
  if (p.ip[3] >= 0) { D = p.glymax - Y; if (D <= p.sw[3]) { D = PX[3] * ipow(1.0 - D / p.sw[3], p.ip[3]); if (D > DMAX) DMAX = D; } }
  return DMAX;
}

__global__ void __launch_bounds__(ROW_THREADS, 3) k_predict(Geo g, Fld f, Prm p, const double *FLUU, const double *FLUV,
                          const double *FLUW, const double *FLVU, const double *FLVV,
                          const double *FLVW, const double *FLWU, const double *FLWV,
                          const double *FLWW, double *UN, double *VN, double *WN) {
  const double *UU = f.uu, *VV = f.vv, *WW = f.ww, *PP = f.pp, *GGV = f.ggv, *GLV = f.glv,
               *CD0 = f.cd0;
  const int *NF = f.nf;
  const double RI = 1.0 / p.rho0, DT = p.dtnow, VM = p.vvmax;
  ROW_LOOP_BEGIN(g)
  const long long c = cid(g, I, J, K);
  const int NI = g.NI, NJ = g.NJ, NK = g.NK;
#define A(a, i, j, k) a[cid(g, i, j, k)]
#define XX_(m, i) gx(g, m, i)
#define YY_(m, j) gy(g, m, j)
#define ZZ_(m, k) gz(g, m, k)
  // ------------------------------------------------ x velocity
  {
    double U = UU[c];
    if (K >= 2 && K <= NK - 1 && J >= 2 && J <= NJ - 1 && I >= 3 && I <= NI - 1 &&
        f.indx[c] == 0 && A(NF, I - 1, J, K) * A(NF, I, J, K) == 0) {
      const int I1 = I - 1;
      // VF_VGENE vf_vgene.f:94-110
      double GVg = XX_(6, I) * (XX_(2, I) * GGV[c] + XX_(2, I1) * A(GGV, I1, J, K));
      double CD = XX_(6, I) * (XX_(2, I) * CD0[c] + XX_(2, I1) * A(CD0, I1, J, K));
      double Q = 0.0;
      Q = Q + GVg * RI * XX_(5, I) * (A(PP, I1, J, K) - PP[c]);
      double Uc = UU[c];
      double V = XX_(6, I) * (XX_(2, I1) * (A(VV, I, J, K) + A(VV, I, J + 1, K)) +
                              XX_(2, I) * (A(VV, I1, J, K) + A(VV, I1, J + 1, K))) * 0.5;
      double W = XX_(6, I) * (XX_(2, I1) * (A(WW, I, J, K) + A(WW, I, J, K + 1)) +
                              XX_(2, I) * (A(WW, I1, J, K) + A(WW, I1, J, K + 1))) * 0.5;
      double UVW = sqrt(Uc * Uc + V * V + W * W);
      Q = Q - 0.5 * CD * XX_(5, I) * (1.0 - f.ggx[c]) * Uc * UVW;
      // wave source of an x line (vf_vgene.f:149-152)
      if (p.iws != 0 && (p.iws == I || p.iws + 1 == I)) {
        const double QS = 2.0 * XX_(4, p.iws) * f.srcuv[(J - 1) + (long long)NJ * (K - 1)];
        Q = Q + UU[c] * QS * XX_(2, p.iws) * XX_(5, I) * 0.5;
      }
      // VF_VEULER vf_veuler.f:119-128
      double GV = XX_(6, I) * (XX_(2, I) * GLV[c] + XX_(2, I - 1) * A(GLV, I - 1, J, K));
      double GV0 = XX_(6, I) * (XX_(2, I) * GLV[c] + XX_(2, I - 1) * A(GLV, I - 1, J, K));
      double DU = (XX_(5, I) * (FLUU[c] - A(FLUU, I - 1, J, K)) + YY_(4, J) * (A(FLUV, I, J + 1, K) - FLUV[c]) +
                   ZZ_(4, K) * (A(FLUW, I, J, K + 1) - FLUW[c]) + Q);
      U = (GV * U + DT * DU) / GV0;
      if (U > VM) U = VM;
      if (U < -VM) U = -VM;
      if (p.ipa != 0) {
        double X = XX_(1, I), Y = (YY_(1, J) + YY_(1, J + 1)) * 0.5;
        double DMAX = sponge_dmax(p, X, Y, false);
        double G = XX_(6, I) * (XX_(2, I) * GGV[c] + XX_(2, I - 1) * A(GGV, I - 1, J, K));
        double D = GV0 / (GV0 + DT * G * DMAX);
        U = U * D;
      }
    }
    UN[c] = U;
  }
  // ------------------------------------------------ y velocity
  {
    double V = VV[c];
    if (K >= 2 && K <= NK - 1 && J >= 3 && J <= NJ - 1 && I >= 2 && I <= NI - 1 &&
        f.indy[c] == 0 && A(NF, I, J - 1, K) * A(NF, I, J, K) == 0) {
      const int J1 = J - 1;
      double GVg = YY_(6, J) * (YY_(2, J) * GGV[c] + YY_(2, J1) * A(GGV, I, J1, K));
      double CD = YY_(6, J) * (YY_(2, J) * CD0[c] + YY_(2, J1) * A(CD0, I, J1, K));
      double Q = 0.0;
      Q = Q + GVg * RI * YY_(5, J) * (A(PP, I, J1, K) - PP[c]);
      double U = YY_(6, J) * (YY_(2, J1) * (A(UU, I, J, K) + A(UU, I + 1, J, K)) +
                              YY_(2, J) * (A(UU, I, J1, K) + A(UU, I + 1, J1, K))) * 0.5;
      double Vc = VV[c];
      double W = YY_(6, J) * (YY_(2, J1) * (A(WW, I, J, K) + A(WW, I, J, K + 1)) +
                              YY_(2, J) * (A(WW, I, J1, K) + A(WW, I, J1, K + 1))) * 0.5;
      double UVW = sqrt(U * U + Vc * Vc + W * W);
      Q = Q - 0.5 * CD * YY_(5, J) * (1.0 - f.ggy[c]) * Vc * UVW;
      // wave source of a y line (vf_vgene.f:225-228)
      if (p.jws != 0 && (p.jws == J || p.jws + 1 == J)) {
        const double QS = 2.0 * YY_(4, p.jws) * f.srcuv[(I - 1) + (long long)NI * (K - 1)];
        Q = Q + VV[c] * QS * YY_(2, p.jws) * YY_(5, J) * 0.5;
      }
      double GV = YY_(6, J) * (YY_(2, J) * GLV[c] + YY_(2, J - 1) * A(GLV, I, J - 1, K));
      double GV0 = YY_(6, J) * (YY_(2, J) * GLV[c] + YY_(2, J - 1) * A(GLV, I, J - 1, K));
      double DV = (XX_(4, I) * (A(FLVU, I + 1, J, K) - FLVU[c]) + YY_(5, J) * (FLVV[c] - A(FLVV, I, J - 1, K)) +
                   ZZ_(4, K) * (A(FLVW, I, J, K + 1) - FLVW[c]) + Q);
      V = (GV * V + DT * DV) / GV0;
      if (V > VM) V = VM;
      if (V < -VM) V = -VM;
      if (p.ipa != 0) {
        double X = (XX_(1, I) + XX_(1, I + 1)) * 0.5, Y = YY_(1, J);
        double DMAX = sponge_dmax(p, X, Y, false);
        double G = YY_(6, J) * (YY_(2, J) * GGV[c] + YY_(2, J - 1) * A(GGV, I, J - 1, K));
        double D = GV0 / (GV0 + DT * G * DMAX);
        V = V * D;
      }
    }
    VN[c] = V;
  }
  // ------------------------------------------------ z velocity
  {
    double W = WW[c];
    if (K >= 3 && K <= NK - 1 && J >= 2 && J <= NJ - 1 && I >= 2 && I <= NI - 1 &&
        f.indz[c] == 0 && A(NF, I, J, K - 1) * A(NF, I, J, K) == 0) {
      const int K1 = K - 1;
      double GVg = ZZ_(6, K) * (ZZ_(2, K) * GGV[c] + ZZ_(2, K1) * A(GGV, I, J, K1));
      double CD = ZZ_(6, K) * (ZZ_(2, K) * CD0[c] + ZZ_(2, K1) * A(CD0, I, J, K1));
      double Q = 0.0;
      Q = Q + GVg * RI * ZZ_(5, K) * (A(PP, I, J, K1) - PP[c]);
      double U = ZZ_(6, K) * (ZZ_(2, K1) * (A(UU, I, J, K) + A(UU, I + 1, J, K)) +
                              ZZ_(2, K) * (A(UU, I, J, K1) + A(UU, I + 1, J, K1))) * 0.5;
      double V = ZZ_(6, K) * (ZZ_(2, K1) * (A(VV, I, J, K) + A(VV, I, J + 1, K)) +
                              ZZ_(2, K) * (A(VV, I, J, K1) + A(VV, I, J + 1, K1))) * 0.5;
      double Wc = WW[c];
      double UVW = sqrt(U * U + V * V + Wc * Wc);
      Q = Q - 0.5 * CD * ZZ_(5, K) * (1.0 - f.ggz[c]) * Wc * UVW;
      Q = Q - GVg * p.grz0;
      // wave source (vf_vgene.f:304-315)
      if (p.iws == I) {
        const double Q1 = 2.0 * XX_(4, I) * f.srcuv[(J - 1) + (long long)NJ * (K - 2)];
        const double Q2 = 2.0 * XX_(4, I) * f.srcuv[(J - 1) + (long long)NJ * (K - 1)];
        Q = Q + ZZ_(5, K) * (Q2 - Q1) * p.anu0 / 3.0;
        Q = Q + WW[c] * (Q1 + Q2) * 0.5;
      }
      if (p.jws == J) {
        const double Q1 = 2.0 * YY_(4, J) * f.srcuv[(I - 1) + (long long)NI * (K - 2)];
        const double Q2 = 2.0 * YY_(4, J) * f.srcuv[(I - 1) + (long long)NI * (K - 1)];
        Q = Q + ZZ_(5, K) * (Q2 - Q1) * p.anu0 / 3.0;
        Q = Q + WW[c] * (Q1 + Q2) * 0.5;
      }
      double DR = 0.0;
      Q = Q - GVg * p.grz0 * DR / p.rho0;
      double GV = ZZ_(6, K) * (ZZ_(2, K) * GLV[c] + ZZ_(2, K - 1) * A(GLV, I, J, K - 1));
      double GV0 = ZZ_(6, K) * (ZZ_(2, K) * GLV[c] + ZZ_(2, K - 1) * A(GLV, I, J, K - 1));
      double DW = (XX_(4, I) * (A(FLWU, I + 1, J, K) - FLWU[c]) + YY_(4, J) * (A(FLWV, I, J + 1, K) - FLWV[c]) +
                   ZZ_(5, K) * (FLWW[c] - A(FLWW, I, J, K - 1)) + Q);
      W = (GV * W + DT * DW) / GV0;
      if (W > VM) W = VM;
      if (W < -VM) W = -VM;
      if (p.ipa != 0) {
        double X = (XX_(1, I) + XX_(1, I + 1)) * 0.5, Y = (YY_(1, J) + YY_(1, J + 1)) * 0.5;
        double DMAX = sponge_dmax(p, X, Y, true);
        double G = ZZ_(6, K) * (ZZ_(2, K) * GGV[c] + ZZ_(2, K - 1) * A(GGV, I, J, K - 1));
        double D = GV0 / (GV0 + DT * G * DMAX);
        W = W * D;
      }
    }
    WN[c] = W;
  }
#undef A
#undef XX_
#undef YY_
#undef ZZ_
  ROW_LOOP_END
}

// ------------------------------------------------------------ VF_BWUWN
__global__ void k_bwuwn(Geo g, Fld f, Prm p, int *err) {
  int L = blockIdx.x * blockDim.x + threadIdx.x + 1;
  if (L > g.NB) return;
  int I, J, K;
  decode(g, indb(f, 1, L), I, J, K);
  int NS = indb(f, 2, L), IB = indb(f, 3, L);
  double *UU = f.uu, *VV = f.vv, *WW = f.ww;
  if (IB == 1) {
    if (NS == 1 || NS == 2) { f.bcu[L - 1] = 0.0; UU[cid(g, I, J, K)] = 0.0; }
    else if (NS == 3 || NS == 4) { f.bcv[L - 1] = 0.0; VV[cid(g, I, J, K)] = 0.0; }
    else { f.bcw[L - 1] = 0.0; WW[cid(g, I, J, K)] = 0.0; }
  } else if (IB == 2) {
    f.bcu[L - 1] = 0.0; f.bcv[L - 1] = 0.0; f.bcw[L - 1] = 0.0;
    if (NS == 1 || NS == 2) UU[cid(g, I, J, K)] = f.bcu[L - 1];
    else if (NS == 3 || NS == 4) VV[cid(g, I, J, K)] = f.bcv[L - 1];
    else WW[cid(g, I, J, K)] = f.bcw[L - 1];
  } else if (IB == 3) {
    if (NS == 1 || NS == 2) UU[cid(g, I, J, K)] = f.bcu[L - 1];
    else if (NS == 3 || NS == 4) VV[cid(g, I, J, K)] = f.bcv[L - 1];
    else WW[cid(g, I, J, K)] = f.bcw[L - 1];
  } else if (IB == 4) {
    // Free faces copy the neighbouring interior face; two free faces of a
    // one-cell gap would read each other (sequential order in the
    // reference), which the configurations here do not contain.
    double VAL;
    if (NS == 1) { VAL = UU[cid(g, I + 1, J, K)]; f.bcu[L - 1] = VAL; UU[cid(g, I, J, K)] = VAL; }
    else if (NS == 2) { VAL = UU[cid(g, I - 1, J, K)]; f.bcu[L - 1] = VAL; UU[cid(g, I, J, K)] = VAL; }
    else if (NS == 3) { VAL = VV[cid(g, I, J + 1, K)]; f.bcv[L - 1] = VAL; VV[cid(g, I, J, K)] = VAL; }
    else if (NS == 4) { VAL = VV[cid(g, I, J - 1, K)]; f.bcv[L - 1] = VAL; VV[cid(g, I, J, K)] = VAL; }
    else if (NS == 5) { VAL = WW[cid(g, I, J, K + 1)]; f.bcw[L - 1] = VAL; WW[cid(g, I, J, K)] = VAL; }
    else if (NS == 6) { VAL = WW[cid(g, I, J, K - 1)]; f.bcw[L - 1] = VAL; WW[cid(g, I, J, K)] = VAL; }
  } else if (IB == 6 || IB == 8) {  // log-law and rough walls (vf_bwuwn.f:237-249)
    if (NS == 1 || NS == 2) { f.bcu[L - 1] = 0.0; UU[cid(g, I, J, K)] = 0.0; }
    else if (NS == 3 || NS == 4) { f.bcv[L - 1] = 0.0; VV[cid(g, I, J, K)] = 0.0; }
    else { f.bcw[L - 1] = 0.0; WW[cid(g, I, J, K)] = 0.0; }
  } else if (IB == 5) {
    // wave-maker faces: set by k_wave after this pass (vf_bwuwn.f:259-470);
    // on a fixed-water-level side (MTBTYP 3) they copy the face inside
    // as free faces do (vf_bwuwn.f:161-216)
    if (fixlvl_face(g, p, NS, I, J)) {
      double VAL;
      if (NS == 1) { VAL = UU[cid(g, I + 1, J, K)]; f.bcu[L - 1] = VAL; UU[cid(g, I, J, K)] = VAL; }
      else if (NS == 2) { VAL = UU[cid(g, I - 1, J, K)]; f.bcu[L - 1] = VAL; UU[cid(g, I, J, K)] = VAL; }
      else if (NS == 3) { VAL = VV[cid(g, I, J + 1, K)]; f.bcv[L - 1] = VAL; VV[cid(g, I, J, K)] = VAL; }
      else { VAL = VV[cid(g, I, J - 1, K)]; f.bcv[L - 1] = VAL; VV[cid(g, I, J, K)] = VAL; }
    } else if (NS > 4) {
      atomicOr(err, ERR_PG);
    }
  } else if (IB == 7) {
    // open (radiation) faces: set by k_open after this pass
    // (vf_bwuwn.f:234-235, 481-598)
  } else {
    atomicOr(err, ERR_PG);
  }
}

// ------------------------------------------------------- VF_CWMSRC
// The wave source's velocity SRCUV(IJ,K) of every line IJ = 2..NUMIJ-1
// (vf_cwmsrc.f:100-143) from the matrix table or a wave theory: the
// column's water level scales the heights (a theory, or MTBTYP 1), then
// VF_CWMTB2's height interpolation between the rows the host chose (phase
// weights wt1/wt2 at row mtbnow) or the theory's velocity at the phase
// (VF_CWMAK2), times the fade-in AW.  One thread per line.
__global__ void k_srcuv(Geo g, Fld f, WaveDev w, double *SRCUV, int *err) {
  const int IJ = 2 + (int)(blockIdx.x * blockDim.x + threadIdx.x);
  const bool xs = (w.side > 0);  // x source at I = side, y source at J = -side
  const int NIJ = xs ? g.NJ : g.NI, NK = g.NK;
  if (IJ > NIJ - 1) return;
  const int I = xs ? w.side : IJ, J = xs ? IJ : -w.side;
  double VWS;
  if (w.mtbtyp == 1) {
    double VAL = 0.0;
    for (int K = 2; K <= NK - 1; ++K) {
      const int NW = f.nf[cid(g, I, J, K)];
      if (NW == -1) {
        VAL = VAL + gz(g, 2, K) * 1.0;
      } else if (NW == 0) {
        VAL = VAL + gz(g, 2, K) * f.ff[cid(g, I, J, K)];
      } else if (NW != 8) {
        VAL = VAL + gz(g, 2, K) * f.ff[cid(g, I, J, K)];
        break;
      }
    }
    VAL = VAL - (w.wvlvl - gz(g, 1, 2));
    VWS = (w.wvz + w.d) / (VAL + w.d);
  } else {
    VWS = 1.0;
  }
  int KM = 1;
  const int nz = w.nzz;
  for (int K = 2; K <= NK - 1; ++K) {
    double ZC = (gz(g, 1, K) + gz(g, 1, K + 1)) * 0.5 - w.wvlvl;
    ZC = VWS * (ZC + w.d) - w.d;
    if (w.theory) {  // VF_CWMAK2 of the wave theory (wavetheory.cuh)
      double UN, UT;
      wt_velocity(w.ph, ZC, UN, UT);
      SRCUV[(IJ - 1) + (long long)NIJ * (K - 1)] = UN * VWS * w.aw;
      continue;
    }
    double W1, W2;
    if (ZC <= w.zz[0]) {
      KM = 1; W1 = 1.0; W2 = 0.0;
    } else if (ZC >= w.zz[nz - 1]) {
      KM = nz - 1; W1 = 0.0; W2 = 1.0;
    } else {
      int KP = 0;
      W1 = 0.0; W2 = 0.0;
      for (int k = KM; k <= nz - 1; ++k) {
        if (w.zz[k - 1] <= ZC && ZC <= w.zz[k]) {
          KP = k;
          W2 = 1.0 / (w.zz[k] - w.zz[k - 1]);
          W1 = (w.zz[k] - ZC) * W2;
          W2 = (ZC - w.zz[k - 1]) * W2;
          break;
        }
      }
      if (KP == 0) { atomicOr(err, ERR_PG); return; }
      KM = KP;
    }
    const long long i0 = (long long)nz * (w.mtbnow - 1), i1 = i0 + nz;
    const double P1 = W1 * w.un[i0 + KM - 1] + W2 * w.un[i0 + KM];
    const double P2 = W1 * w.un[i1 + KM - 1] + W2 * w.un[i1 + KM];
    const double UN = w.wt1 * P1 + w.wt2 * P2;
    SRCUV[(IJ - 1) + (long long)NIJ * (K - 1)] = UN * VWS * w.aw;
  }
}

// ------------------------------------------------- VF_BWUWN, wave maker
// Wave-maker faces of one side (vf_bwuwn.f:330-470), one thread per
// boundary line (J on the X sides, I on the Y sides), from the matrix
// table (VF_CWMTB2, vf_cwmtb2.f) or a wave theory (VF_CWMAK2).  The host
// has done the time part: phase, fade-in AW, VF_CWMTB1's weights and row
// MTBNOW or the theory's level and phase part, one per line under oblique
// incidence.
__global__ void k_wave(Geo g, Fld f, WaveDev w, int *err) {
  const int n = w.first + (int)(blockIdx.x * blockDim.x + threadIdx.x);
  if (n > w.last) return;
  const int NI = g.NI, NJ = g.NJ, NK = g.NK;
  const bool xs = (w.side <= 2);
  int I, J, IC, JC;
  if (xs) {
    J = n; JC = n;
    if (J < 2 || J > NJ - 1) return;
    I = (w.side == 1) ? 2 : NI;
    IC = (w.side == 1) ? 2 : NI - 1;
  } else {
    I = n; IC = n;
    if (I < 2 || I > NI - 1) return;
    J = (w.side == 3) ? 2 : NJ;
    JC = (w.side == 3) ? 2 : NJ - 1;
  }
  // oblique incidence: this line's level and phase (vf_bwuwn.f:345-356)
  const WavePhase &ph = w.col ? w.col[n - w.first].ph : w.ph;
  const double WVZ = w.col ? w.col[n - w.first].wvz : w.wvz;
  // current water level of the column next to the boundary, scaling
  double VWS;
  if (w.mtbtyp != 1) {
    VWS = 1.0;
  } else {
    double VAL = 0.0;
    for (int K = 2; K <= NK - 1; ++K) {
      const int NW = f.nf[cid(g, IC, JC, K)];
      if (NW == -1) {
        VAL = VAL + gz(g, 2, K) * 1.0;
      } else if (NW == 0) {
        VAL = VAL + gz(g, 2, K) * f.ff[cid(g, IC, JC, K)];
      } else if (NW != 8) {
        VAL = VAL + gz(g, 2, K) * f.ff[cid(g, IC, JC, K)];
        break;
      }
    }
    VAL = VAL - (w.wvlvl - gz(g, 1, 2));
    VWS = (WVZ + w.d) / (VAL + w.d);
  }
  // boundary values face by face; the height search starts where the face
  // below found its interval
  int KM = 1;
  const int nz = w.nzz;
  for (int K = 2; K <= NK - 1; ++K) {
    const long long c = cid(g, I, J, K);
    const int L = xs ? f.indx[c] : f.indy[c];
    if (L < 1) continue;
    double ZC = (gz(g, 1, K) + gz(g, 1, K + 1)) * 0.5 - w.wvlvl;
    ZC = VWS * (ZC + w.d) - w.d;
    if (w.theory) {  // VF_CWMAK2 of the wave theory (wavetheory.cuh)
      double UN, UT;
      wt_velocity(ph, ZC, UN, UT);
      f.bcu[L - 1] = UN * VWS * w.aw * w.sa;
      f.bcv[L - 1] = UN * VWS * w.aw * w.sb;
      f.bcw[L - 1] = UT * VWS * w.aw;
      if (xs) f.uu[c] = f.bcu[L - 1];
      else f.vv[c] = f.bcv[L - 1];
      continue;
    }
    double W1, W2;
    if (ZC <= w.zz[0]) {
      KM = 1; W1 = 1.0; W2 = 0.0;
    } else if (ZC >= w.zz[nz - 1]) {
      KM = nz - 1; W1 = 0.0; W2 = 1.0;
    } else {
      int KP = 0;
      W1 = 0.0; W2 = 0.0;
      for (int k = KM; k <= nz - 1; ++k) {
        if (w.zz[k - 1] <= ZC && ZC <= w.zz[k]) {
          KP = k;
          W2 = 1.0 / (w.zz[k] - w.zz[k - 1]);
          W1 = (w.zz[k] - ZC) * W2;
          W2 = (ZC - w.zz[k - 1]) * W2;
          break;
        }
      }
      if (KP == 0) { atomicOr(err, ERR_PG); return; }
      KM = KP;
    }
    const long long i0 = (long long)nz * (w.mtbnow - 1), i1 = i0 + nz;  // columns MTBNOW, MTBNOW+1
    double P1 = W1 * w.un[i0 + KM - 1] + W2 * w.un[i0 + KM];
    double P2 = W1 * w.un[i1 + KM - 1] + W2 * w.un[i1 + KM];
    const double UN = w.wt1 * P1 + w.wt2 * P2;
    P1 = W1 * w.ut[i0 + KM - 1] + W2 * w.ut[i0 + KM];
    P2 = W1 * w.ut[i1 + KM - 1] + W2 * w.ut[i1 + KM];
    const double UT = w.wt1 * P1 + w.wt2 * P2;
    f.bcu[L - 1] = UN * VWS * w.aw * w.sa;
    f.bcv[L - 1] = UN * VWS * w.aw * w.sb;
    f.bcw[L - 1] = UT * VWS * w.aw;
    if (xs) f.uu[c] = f.bcu[L - 1];
    else f.vv[c] = f.bcv[L - 1];
  }
}

// ------------------------------------------------- VF_BWUWN, open boundary
// Radiation faces of one side (vf_bwuwn.f:481-598), one thread per
// boundary line (J on the X sides, I on the Y sides), its faces in the
// reference's K order.  A face next to a fluid cell blends its stored
// value toward the interior of the step's start: the normal component
// toward the face one cell inside with ALN = min(C DTNOW / DX, 1), the
// tangential ones toward the cell-centre averages with ALT = min(2 ALN, 1)
// (both 1 at NNOW = 0); a face next to any other cell gets zero.  Then the
// faces of surface cells open downward (NF 5) or upward (NF 6) copy the
// face below or above; the upward ones leave the normal velocity 0 on the
// X sides and the copied value on the Y sides, as the reference does.
__global__ void k_open(Geo g, Fld f, OpenDev o, const double *UB, const double *VB, const double *WB, int *err) {
  const int n = 2 + (int)(blockIdx.x * blockDim.x + threadIdx.x);
  const int NI = g.NI, NJ = g.NJ, NK = g.NK;
  const bool xs = (o.side <= 2);
  if (n > (xs ? NJ - 1 : NI - 1)) return;
  int I, J, IC, JC, I2, J2;
  if (xs) {
    J = n; JC = n; J2 = n;
    I = (o.side == 1) ? 2 : NI;
    IC = (o.side == 1) ? 2 : NI - 1;
    I2 = (o.side == 1) ? 3 : IC;
  } else {
    I = n; IC = n; I2 = n;
    J = (o.side == 3) ? 2 : NJ;
    JC = (o.side == 3) ? 2 : NJ - 1;
    J2 = (o.side == 3) ? 3 : JC;
  }
  double ALN = 1.0, ALT = 1.0;
  if (o.nnow != 0) {
    const double a = o.c * o.dtnow / (xs ? gx(g, 2, IC) : gy(g, 2, JC));
    ALN = (a < 1.0) ? a : 1.0;
    const double b = ALN * 2.0;
    ALT = (b < 1.0) ? b : 1.0;
  }
  const int *ind = xs ? f.indx : f.indy;
  for (int K = 2; K <= NK - 1; ++K) {
    const long long c = cid(g, I, J, K);
    const int L = ind[c];
    if (L < 1) continue;
    const long long cc = cid(g, IC, JC, K);
    double &BU = f.bcu[L - 1], &BV = f.bcv[L - 1], &BW = f.bcw[L - 1];
    if (f.nf[cc] == 0) {
      const double WC = (WB[cc] + WB[cid(g, IC, JC, K + 1)]) * 0.5;
      if (xs) {
        const double VC = (VB[cc] + VB[cid(g, IC, JC + 1, K)]) * 0.5;
        BU = (1.0 - ALN) * BU + ALN * UB[cid(g, I2, J, K)];
        BV = (1.0 - ALT) * BV + ALT * VC;
        BW = (1.0 - ALT) * BW + ALT * WC;
        f.uu[c] = BU;
      } else {
        const double UC = (UB[cc] + UB[cid(g, IC + 1, JC, K)]) * 0.5;
        BU = (1.0 - ALT) * BU + ALT * UC;
        BV = (1.0 - ALN) * BV + ALN * VB[cid(g, I, J2, K)];
        BW = (1.0 - ALT) * BW + ALT * WC;
        f.vv[c] = BV;
      }
    } else {
      BU = 0.0; BV = 0.0; BW = 0.0;
      if (xs) f.uu[c] = 0.0;
      else f.vv[c] = 0.0;
    }
  }
  for (int K = 2; K <= NK - 1; ++K) {
    const long long c = cid(g, I, J, K);
    const int L = ind[c];
    if (L < 1) continue;
    const int NW = f.nf[cid(g, IC, JC, K)];
    if (NW != 5 && NW != 6) continue;
    const int L2 = ind[cid(g, I, J, NW == 5 ? K - 1 : K + 1)];
    if (L2 < 1) { atomicOr(err, ERR_PG); return; }
    f.bcu[L - 1] = f.bcu[L2 - 1];
    f.bcv[L - 1] = f.bcv[L2 - 1];
    f.bcw[L - 1] = f.bcw[L2 - 1];
    if (xs) f.uu[c] = (NW == 5) ? f.bcu[L - 1] : 0.0;
    else f.vv[c] = f.bcv[L - 1];
  }
}

// ------------------------------------------------------------ launchers
void launch_wave(cudaStream_t s, const Geo &g, const Fld &f, const WaveDev &w, int *err) {
  const int n = w.last - w.first + 1;
  if (n <= 0) return;
  k_wave<<<(n + 127) / 128, 128, 0, s>>>(g, f, w, err);
  count_launch();
}
void launch_srcuv(cudaStream_t s, const Geo &g, const Fld &f, const WaveDev &w, double *srcuv, int *err) {
  const int n = (w.side > 0 ? g.NJ : g.NI) - 2;
  k_srcuv<<<(n + 127) / 128, 128, 0, s>>>(g, f, w, srcuv, err);
  count_launch();
}
void launch_open(cudaStream_t s, const Geo &g, const Fld &f, const OpenDev &o, const double *ub,
                 const double *vb, const double *wb, int *err) {
  const int n = ((o.side <= 2) ? g.NJ : g.NI) - 2;
  if (n <= 0) return;
  k_open<<<(n + 127) / 128, 128, 0, s>>>(g, f, o, ub, vb, wb, err);
  count_launch();
}
void launch_flux(cudaStream_t s, const Geo &g, const Fld &f, const Prm &p, double *const *fl) {
  k_flux<<<row_blocks(g), ROW_THREADS, 0, s>>>(g, f, p, fl[0], fl[1], fl[2], fl[3], fl[4], fl[5],
                                                fl[6], fl[7], fl[8]);
  count_launch();
}
void launch_predict(cudaStream_t s, const Geo &g, const Fld &f, const Prm &p,
                    double *const *fl, double *un, double *vn, double *wn) {
  k_predict<<<row_blocks(g), ROW_THREADS, 0, s>>>(g, f, p, fl[0], fl[1], fl[2], fl[3], fl[4],
                                                   fl[5], fl[6], fl[7], fl[8], un, vn, wn);
  count_launch();
}
void launch_bwuwn(cudaStream_t s, const Geo &g, const Fld &f, const Prm &p, int *err) {
  if (g.NB <= 0) return;
  k_bwuwn<<<(g.NB + 255) / 256, 256, 0, s>>>(g, f, p, err);
  count_launch();
}

}  // namespace cadmas
