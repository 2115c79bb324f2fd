// vof_face.cuh -- the donor-acceptor flux of one face, VF_FCONV
// (vf_fconv.f:73-99); VF_FCONVS (vf_fconvs.f:417-444) uses the same
// expression for the faces it does not treat by slope.
#pragma once
#include "cadmas_dev.cuh"

namespace cadmas {

// DT_G_U = DTNOW*G*U of the face; N, FDv the donor's NF and F; ndm, FDMv
// those of the cell behind the donor; Vd the donor's width times GGV, Vo
// its width; bcfv the boundary F when the donor is an obstacle (N = -1);
// na, FAv the acceptor's NF and F; d1..d4 the surface orientations whose
// donor takes its own F (the other two axes); FL = FLOWER.
__device__ __forceinline__ double fconv_face(double DT_G_U, int N, double FDv, int ndm, double FDMv,
                                             double Vd, double Vo, double bcfv, int na, double FAv,
                                             int d1, int d2, int d3, int d4, double FL) {
  double C = DT_G_U;
  double AC = fabs(C), FD, FDMW, V, FA;
  if (N != -1) { FD = FDv; FDMW = 1.0; if (ndm != -1) FDMW = FDMv; V = Vd; }
  else { FD = bcfv; FDMW = 1.0; V = Vo; }
  FA = (na != -1) ? FAv : FD;
  double FAD = FA;
  if (N == -1 || N == d1 || N == d2 || N == d3 || N == d4)
    if (FDMW != 0.0 && FA != 0.0) FAD = FD;
  double FDM = dmax(FDMW, FD);
  if (FDMW < FL && FA < FL) FDM = dmax(FDM, 0.1);
  double CFX = dmax((FDM - FAD) * AC - (FDM - FD) * V, 0.0);
  double FVX = FAD * AC + CFX;
  double FVM = FD * V;
  return dmin(FVX, FVM);
}

}  // namespace cadmas
