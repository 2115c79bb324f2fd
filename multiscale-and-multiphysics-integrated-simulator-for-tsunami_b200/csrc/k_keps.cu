// k_keps.cu -- the k-epsilon model of CADMAS-SURF/3D (LEQK != 0):
// VF_K1CAL between VF_V1CAL and VF_F1CAL and the updates after VF_F1CAL
// (vf_a1main.f:1093-1127), and its part of VF_CINIT.
//
//   k_kstep   VF_K1CAL (vf_k1cal.f:84-153) for each fluid cell at once:
//             the donor-cell and diffusive fluxes of k and e through its
//             six faces (VF_SCONVD, VF_SDIFF), production and dissipation
//             (VF_KGENE), the Euler step (VF_SEULER) and the cut-off, into
//             a second buffer; every other cell is copied.  A face's flux
//             is the same expression whichever of its two cells evaluates
//             it, so the sequence of face loops then cell loop of the
//             reference gives the same values as this cell-centred form.
//   k_kbsss   VF_BSSS (vf_bsss.f:27-66) on k and e; with NUT also VF_CNUT0
//             and VF_CNU00 (vf_cnut0.f:37-49, vf_cnu00.f:52-61) on the same
//             cell.  A surface cell reads only fluid neighbours, which the
//             pass does not write, so it runs in place.
//   k_bwke    VF_BWKE (vf_bwke.f:33-108), one thread per boundary face.
//   k_kinit   vf_cinit.f:295-315 and 359-364: k, e from AKINIK, AKINIE on
//             INDC != -1 cells, then ANUT and ANU.
//
// VF_BWKELG acts on log-law and rough walls only (IB 6 and 8), which
// cadmas_create refuses, so it is not built.
#include "cadmas_dev.cuh"
#include "kernels.h"
#include "loglaw.cuh"

namespace cadmas {

#define A(a, i, j, k) a[cid(g, i, j, k)]
#define XX_(m, i) gx(g, m, i)
#define YY_(m, j) gy(g, m, j)
#define ZZ_(m, k) gz(g, m, k)

__device__ __forceinline__ bool kint(const Geo &g, int I, int J, int K) {
  return I >= 2 && I <= g.NI - 1 && J >= 2 && J <= g.NJ - 1 && K >= 2 && K <= g.NK - 1;
}

// WKNU of VF_K1CAL (vf_k1cal.f:114-120): ANU0 + ANUT*W on interior cells
// with NF != -1, else the 0 it was cleared to.
__device__ __forceinline__ double kdiffusivity(const Geo &g, const Fld &f, const KeArrays &t, double anu0,
                                               double W, int I, int J, int K, long long c) {
  return (kint(g, I, J, K) && f.nf[c] != -1) ? anu0 + t.anut[c] * W : 0.0;
}

// The flux of CC through the face between cell m (minus side) and cell c
// (plus side) on axis AX, with face index IND, area ratio G, velocity U:
// VF_SCONVD (vf_sconvd.f:49-83) then VF_SDIFF (vf_sdiff.f:58-86) on the
// same face, starting from the cleared 0.  w6, wm, wc: metric 6 of the
// face and the widths of cells m and c; w5 metric 5 of the face; w4c, w4m
// metric 4 of cells c and m; Dc, Dm the two cells' diffusivities.
__device__ __forceinline__ double kface(const Fld &f, const int NB, long long c, long long m, double G, double U,
                                        int IND, const double *CC, const double *BCC, const int *INDBC, double SU,
                                        double SC, double w6, double wm, double wc, double w5, double w4c,
                                        double w4m, double Dc, double Dm, int *err) {
  double FL = 0.0;
  const int nc = f.nf[c], nm = f.nf[m];
  if (nm * nc != 0) return FL;
  const double WIN = G * U;
  const bool bnd = IND >= 1 && IND <= NB;
  if (IND != 0 && !bnd) { atomicOr(err, ERR_PG); return FL; }
  if (IND == 0) {
    double FLC = WIN * w6 * (wm * CC[c] + wc * CC[m]);
    FL = FL - SU * (dmax(WIN, 0.0) * CC[m] - dmax(-WIN, 0.0) * CC[c]) - SC * FLC;
  } else if (INDBC[IND - 1] >= 1) {
    double FLC = WIN * BCC[IND - 1];
    if (nc == 0) {
      if (WIN >= 0.0) FL = FL - FLC;
      else FL = FL - SU * WIN * CC[c] - SC * FLC;
    } else {
      if (WIN <= 0.0) FL = FL - FLC;
      else FL = FL - SU * WIN * CC[m] - SC * FLC;
    }
  }
  const double AL = 1.0;
  if (IND == 0) {
    double D = w6 * (wm * Dc + wc * Dm);
    D = D * AL;
    FL = FL + G * D * w5 * (CC[c] - CC[m]);
  } else {
    double CW = BCC[IND - 1];
    if (nc == 0) {
      double D = Dc * AL;
      FL = FL + G * D * w4c * (CC[c] - CW) * 2.0;
    } else {
      double D = Dm * AL;
      FL = FL + G * D * w4m * (CW - CC[m]) * 2.0;
    }
  }
  return FL;
}

// VF_BWKELG (vf_bwkelg.f:30-160) on fluid cell (I,J,K): when one of its
// six faces is a log-law (6) or rough (8) wall, k and e become the
// averages over those faces of u*^2/sqrt(C_mu) and u*^3/(kappa DL), u* the
// friction velocity of the cell-centre speed along the face (VF_CLOGLW,
// VF_CLOGKS) and DL half the cell width.  As in the reference, two z
// log-law faces count once unless the cell's two y faces are log-law.
// Returns false (k, e untouched) for a cell with no such face.
__device__ bool bwkelg_cell(const Geo &g, const Fld &f, const Prm &p, double akcmu, long long c, int I, int J, int K,
                            double &AK, double &AE, int *err) {
  const int LXM = f.indx[c], LXP = f.indx[cid(g, I + 1, J, K)];
  const int LYM = f.indy[c], LYP = f.indy[cid(g, I, J + 1, K)];
  const int LZM = f.indz[c], LZP = f.indz[cid(g, I, J, K + 1)];
  const int IXM = LXM >= 1 ? indb(f, 3, LXM) : 0, IXP = LXP >= 1 ? indb(f, 3, LXP) : 0;
  const int IYM = LYM >= 1 ? indb(f, 3, LYM) : 0, IYP = LYP >= 1 ? indb(f, 3, LYP) : 0;
  const int IZM = LZM >= 1 ? indb(f, 3, LZM) : 0, IZP = LZP >= 1 ? indb(f, 3, LZP) : 0;
  auto wall = [](int t) { return t == 6 || t == 8; };
  if (!(wall(IXM) || wall(IXP) || wall(IYM) || wall(IYP) || wall(IZM) || wall(IZP))) return false;
  const double ZERO = 1.0e-20;
  const double CMR = 1.0 / sqrt(akcmu), CKR = 1.0 / p.akk0;
  const double UC = (f.uu[c] + f.uu[cid(g, I + 1, J, K)]) * 0.5;
  const double VC = (f.vv[c] + f.vv[cid(g, I, J + 1, K)]) * 0.5;
  const double WC = (f.ww[c] + f.ww[cid(g, I, J, K + 1)]) * 0.5;
  const double VX = sqrt(VC * VC + WC * WC), VY = sqrt(UC * UC + WC * WC), VZ = sqrt(UC * UC + VC * VC);
  const double DX = XX_(2, I) * 0.5, DY = YY_(2, J) * 0.5, DZ = ZZ_(2, K) * 0.5;
  auto lw = [&](double D, double V, double &T) {
    if (V >= ZERO && p.anu0 >= ZERO && !cloglw(D, V, p.anu0, p.akk0, p.aka0, T)) atomicOr(err, ERR_NOTCONV);
  };
  double SX = 0.0, UT = 0.0, SY = 0.0, VT = 0.0, SZ = 0.0, WT = 0.0;
  if (IXM == 6 || IXP == 6) { lw(DX, VX, UT); SX = 1.0; if (IXM == 6 && IXP == 6) SX = 2.0; }
  if (IYM == 6 || IYP == 6) { lw(DY, VY, VT); SY = 1.0; if (IYM == 6 && IYP == 6) SY = 2.0; }
  if (IZM == 6 || IZP == 6) { lw(DZ, VZ, WT); SZ = 1.0; if (IYM == 6 && IYP == 6) SZ = 2.0; }
  auto ks = [&](double D, double V, int L) { return (V >= ZERO) ? clogks(D, V, f.bcvi[L - 1], p.anu0, p.akk0, p.aka0) : 0.0; };
  double SXM = 0.0, UTM = 0.0, SXP = 0.0, UTP = 0.0, SYM = 0.0, VTM = 0.0, SYP = 0.0, VTP = 0.0;
  double SZM = 0.0, WTM = 0.0, SZP = 0.0, WTP = 0.0;
  if (IXM == 8) { UTM = ks(DX, VX, LXM); SXM = 1.0; }
  if (IXP == 8) { UTP = ks(DX, VX, LXP); SXP = 1.0; }
  if (IYM == 8) { VTM = ks(DY, VY, LYM); SYM = 1.0; }
  if (IYP == 8) { VTP = ks(DY, VY, LYP); SYP = 1.0; }
  if (IZM == 8) { WTM = ks(DZ, VZ, LZM); SZM = 1.0; }
  if (IZP == 8) { WTP = ks(DZ, VZ, LZP); SZP = 1.0; }
  const double SR = 1.0 / (SX + SY + SZ + SXM + SXP + SYM + SYP + SZM + SZP);
  AK = CMR * (UT * UT * SX + VT * VT * SY + WT * WT * SZ + UTM * UTM * SXM + UTP * UTP * SXP + VTM * VTM * SYM +
              VTP * VTP * SYP + WTM * WTM * SZM + WTP * WTP * SZP) * SR;
  AE = CKR * (UT * UT * UT / DX * SX + VT * VT * VT / DY * SY + WT * WT * WT / DZ * SZ + UTM * UTM * UTM / DX * SXM +
              UTP * UTP * UTP / DX * SXP + VTM * VTM * VTM / DY * SYM + VTP * VTP * VTP / DY * SYP +
              WTM * WTM * WTM / DZ * SZM + WTP * WTP * WTP / DZ * SZP) * SR;
  return true;
}

// VF_BWKELG after VF_F1CAL (vf_a1main.f:1120): k and e in place on the
// fluid cells (new NF) next to log-law or rough walls.
__global__ void k_bwkelg(Geo g, Fld f, Prm p, KeConst kc, double *AK, double *AE, int *err) {
  ROW_LOOP_BEGIN(g)
  const long long c = cid(g, I, J, K);
  if (kint(g, I, J, K) && f.nf[c] == 0) {
    double ak, ae;
    if (bwkelg_cell(g, f, p, kc.akcmu, c, I, J, K, ak, ae, err)) { AK[c] = ak; AE[c] = ae; }
  }
  ROW_LOOP_END
}

__global__ void k_kstep(Geo g, Fld f, Prm p, KeConst kc, KeArrays t, double *AKN, double *AEN, int *err) {
  ROW_LOOP_BEGIN(g)
  const long long c = cid(g, I, J, K);
  double akn = t.ak[c], aen = t.ae[c];
  if (kint(g, I, J, K) && f.nf[c] == 0) {
    const int NB = g.NB;
    const long long sJ = g.NI, sK = (long long)g.NI * g.NJ;
    const double *UU = f.uu, *VV = f.vv, *WW = f.ww;
    const double Wk = 1.0 / kc.aksgk, We = 1.0 / kc.aksge;
    // the six faces: x at I and I+1, y at J and J+1, z at K and K+1
    double FK[6], FE[6];
#pragma unroll
    for (int s = 0; s < 6; ++s) {
      const int ax = s >> 1, up = s & 1;
      const int Ic = I + (ax == 0 ? up : 0), Jc = J + (ax == 1 ? up : 0), Kc = K + (ax == 2 ? up : 0);
      const long long cc = cid(g, Ic, Jc, Kc);
      const long long mm = cc - (ax == 0 ? 1 : ax == 1 ? sJ : sK);
      const int Im = Ic - (ax == 0), Jm = Jc - (ax == 1), Km = Kc - (ax == 2);
      double G, U, w6, wm, wc, w5, w4c, w4m;
      int IND;
      if (ax == 0) { G = f.ggx[cc]; U = UU[cc]; IND = f.indx[cc]; w6 = XX_(6, Ic); wm = XX_(2, Ic - 1); wc = XX_(2, Ic); w5 = XX_(5, Ic); w4c = XX_(4, Ic); w4m = XX_(4, Ic - 1); }
      else if (ax == 1) { G = f.ggy[cc]; U = VV[cc]; IND = f.indy[cc]; w6 = YY_(6, Jc); wm = YY_(2, Jc - 1); wc = YY_(2, Jc); w5 = YY_(5, Jc); w4c = YY_(4, Jc); w4m = YY_(4, Jc - 1); }
      else { G = f.ggz[cc]; U = WW[cc]; IND = f.indz[cc]; w6 = ZZ_(6, Kc); wm = ZZ_(2, Kc - 1); wc = ZZ_(2, Kc); w5 = ZZ_(5, Kc); w4c = ZZ_(4, Kc); w4m = ZZ_(4, Kc - 1); }
      const double Dkc = kdiffusivity(g, f, t, kc.anu0, Wk, Ic, Jc, Kc, cc), Dkm = kdiffusivity(g, f, t, kc.anu0, Wk, Im, Jm, Km, mm);
      const double Dec = kdiffusivity(g, f, t, kc.anu0, We, Ic, Jc, Kc, cc), Dem = kdiffusivity(g, f, t, kc.anu0, We, Im, Jm, Km, mm);
      FK[s] = kface(f, NB, cc, mm, G, U, IND, t.ak, t.bck, t.indbk, kc.scmk, 1.0 - kc.scmk, w6, wm, wc, w5, w4c, w4m, Dkc, Dkm, err);
      FE[s] = kface(f, NB, cc, mm, G, U, IND, t.ae, t.bce, t.indbe, kc.scmk, 1.0 - kc.scmk, w6, wm, wc, w5, w4c, w4m, Dec, Dem, err);
    }
    // VF_KGENE (vf_kgene.f:55-178)
    const int IM = I - 1, IP = I + 1, JM = J - 1, JP = J + 1, KM = K - 1, KP = K + 1;
    auto bc = [&](const double *a, int l) -> double {
      if (l < 1 || l > NB) { atomicOr(err, ERR_PG); return 0.0; }
      return a[l - 1];
    };
    double UXM = A(UU, I, J, K), UXP = A(UU, IP, J, K);
    double VYM = A(VV, I, J, K), VYP = A(VV, I, JP, K);
    double WZM = A(WW, I, J, K), WZP = A(WW, I, J, KP);
    double VXM, WXM, VXP, WXP, UYM, WYM, UYP, WYP, UZM, VZM, UZP, VZP;
    int IND = A(f.indx, I, J, K);
    if (IND == 0) {
      VXM = 0.5 * XX_(6, I) * (XX_(2, IM) * (A(VV, I, J, K) + A(VV, I, JP, K)) + XX_(2, I) * (A(VV, IM, J, K) + A(VV, IM, JP, K)));
      WXM = 0.5 * XX_(6, I) * (XX_(2, IM) * (A(WW, I, J, K) + A(WW, I, J, KP)) + XX_(2, I) * (A(WW, IM, J, K) + A(WW, IM, J, KP)));
    } else { VXM = bc(f.bcv, IND); WXM = bc(f.bcw, IND); }
    IND = A(f.indx, IP, J, K);
    if (IND == 0) {
      VXP = 0.5 * XX_(6, IP) * (XX_(2, I) * (A(VV, IP, J, K) + A(VV, IP, JP, K)) + XX_(2, IP) * (A(VV, I, J, K) + A(VV, I, JP, K)));
      WXP = 0.5 * XX_(6, IP) * (XX_(2, I) * (A(WW, IP, J, K) + A(WW, IP, J, KP)) + XX_(2, IP) * (A(WW, I, J, K) + A(WW, I, J, KP)));
    } else { VXP = bc(f.bcv, IND); WXP = bc(f.bcw, IND); }
    IND = A(f.indy, I, J, K);
    if (IND == 0) {
      UYM = 0.5 * YY_(6, J) * (YY_(2, JM) * (A(UU, I, J, K) + A(UU, IP, J, K)) + YY_(2, J) * (A(UU, I, JM, K) + A(UU, IP, JM, K)));
      WYM = 0.5 * YY_(6, J) * (YY_(2, JM) * (A(WW, I, J, K) + A(WW, I, J, KP)) + YY_(2, J) * (A(WW, I, JM, K) + A(WW, I, JM, KP)));
    } else { UYM = bc(f.bcu, IND); WYM = bc(f.bcw, IND); }
    IND = A(f.indy, I, JP, K);
    if (IND == 0) {
      UYP = 0.5 * YY_(6, JP) * (YY_(2, J) * (A(UU, I, JP, K) + A(UU, IP, JP, K)) + YY_(2, JP) * (A(UU, I, J, K) + A(UU, IP, J, K)));
      WYP = 0.5 * YY_(6, JP) * (YY_(2, J) * (A(WW, I, JP, K) + A(WW, I, JP, KP)) + YY_(2, JP) * (A(WW, I, J, K) + A(WW, I, J, KP)));
    } else { UYP = bc(f.bcu, IND); WYP = bc(f.bcw, IND); }
    IND = A(f.indz, I, J, K);
    if (IND == 0) {
      UZM = 0.5 * ZZ_(6, K) * (ZZ_(2, KM) * (A(UU, I, J, K) + A(UU, IP, J, K)) + ZZ_(2, K) * (A(UU, I, J, KM) + A(UU, IP, J, KM)));
      VZM = 0.5 * ZZ_(6, K) * (ZZ_(2, KM) * (A(VV, I, J, K) + A(VV, I, JP, K)) + ZZ_(2, K) * (A(VV, I, J, KM) + A(VV, I, JP, KM)));
    } else { UZM = bc(f.bcu, IND); VZM = bc(f.bcv, IND); }
    IND = A(f.indz, I, J, KP);
    if (IND == 0) {
      UZP = 0.5 * ZZ_(6, KP) * (ZZ_(2, K) * (A(UU, I, J, KP) + A(UU, IP, J, KP)) + ZZ_(2, KP) * (A(UU, I, J, K) + A(UU, IP, J, K)));
      VZP = 0.5 * ZZ_(6, KP) * (ZZ_(2, K) * (A(VV, I, J, KP) + A(VV, I, JP, KP)) + ZZ_(2, KP) * (A(VV, I, J, K) + A(VV, I, JP, K)));
    } else { UZP = bc(f.bcu, IND); VZP = bc(f.bcv, IND); }
    double DLR = XX_(4, I);
    const double DUDX = DLR * (UXP - UXM), DVDX = DLR * (VXP - VXM), DWDX = DLR * (WXP - WXM);
    DLR = YY_(4, J);
    const double DUDY = DLR * (UYP - UYM), DVDY = DLR * (VYP - VYM), DWDY = DLR * (WYP - WYM);
    DLR = ZZ_(4, K);
    const double DUDZ = DLR * (UZP - UZM), DVDZ = DLR * (VZP - VZM), DWDZ = DLR * (WZP - WZM);
    const double GS = t.anut[c] * (2.0 * (DUDX * DUDX + DVDY * DVDY + DWDZ * DWDZ) + ipow(DUDY + DVDX, 2) +
                                   ipow(DVDZ + DWDY, 2) + ipow(DWDX + DUDZ, 2));
    const double GT = 0.0;
    const double GST = GS + GT;
    const double RF = -GT / dmax(GST, 1.0e-20);
    const double AK0 = dmax(t.ak[c], kc.akmink);
    const double AE0 = t.ae[c];
    const double AEK = AE0 / AK0;
    const double GG = f.ggv[c];
    const double QK = 0.0 + GG * (GST - AE0);
    const double QE = 0.0 + GG * (kc.akc1 * AEK * GST * (1.0 + kc.akc3 * RF) - kc.akc2 * AEK * AE0);
    // VF_SEULER (vf_seuler.f:43-52), GGV0 = GGV
    const double G0 = GG - (GG - GG) * 1.0;
    const double DSK = (XX_(4, I) * (FK[1] - FK[0]) + YY_(4, J) * (FK[3] - FK[2]) + ZZ_(4, K) * (FK[5] - FK[4]) + QK);
    const double DSE = (XX_(4, I) * (FE[1] - FE[0]) + YY_(4, J) * (FE[3] - FE[2]) + ZZ_(4, K) * (FE[5] - FE[4]) + QE);
    akn = (G0 * akn + p.dtnow * DSK) / GG;
    aen = (G0 * aen + p.dtnow * DSE) / GG;
    // VF_BWKELG (vf_k1cal.f:147-149)
    if (p.loglaw) bwkelg_cell(g, f, p, kc.akcmu, c, I, J, K, akn, aen, err);
    // cut-off (vf_k1cal.f:155-167)
    if (aen < kc.akmine) { akn = kc.akmink; aen = kc.akmine; }
    else if (akn < kc.akmink) akn = kc.akmink;
  }
  AKN[c] = akn;
  AEN[c] = aen;
  ROW_LOOP_END
}

// BS: VF_BSSS on k and e; NUT: then VF_CNUT0 and VF_CNU00 on the same cell.
template <bool BS, bool NUT>
__global__ void k_kbsss(Geo g, Fld f, KeConst kc, double *AK, double *AE, double *ANUT, double *ANU) {
  ROW_LOOP_BEGIN(g)
  if (kint(g, I, J, K)) {
    const long long c = cid(g, I, J, K);
    const int n = f.nf[c];
    double ak = AK[c], ae = AE[c];
    if (!BS) {
    } else if (n == 8) { ak = 0.0; ae = 0.0; AK[c] = ak; AE[c] = ae; }
    else if (n >= 1) {
      const long long sJ = g.NI, sK = (long long)g.NI * g.NJ;
      const long long nb[6] = {c - 1, c + 1, c - sJ, c + sJ, c - sK, c + sK};
      int N = 0;
      double SK = 0.0, SE = 0.0;
#pragma unroll
      for (int q = 0; q < 6; ++q)
        if (f.nf[nb[q]] == 0) { N = N + 1; SK = SK + AK[nb[q]]; SE = SE + AE[nb[q]]; }
      ak = SK / (double)N;
      ae = SE / (double)N;
      AK[c] = ak; AE[c] = ae;
    }
    if (NUT) {
      double nut = 0.0;
      if (n != -1) {
        const double W = dmax(ae, kc.akmine);
        nut = kc.akcmu * ak * ak / W;
      }
      ANUT[c] = nut;
      ANU[c] = (n != -1) ? kc.anu0 + nut : 0.0;
    }
  }
  ROW_LOOP_END
}

__global__ void k_bwke(Geo g, Fld f, KeArrays t, int *err) {
  const int L = blockIdx.x * blockDim.x + threadIdx.x + 1;
  if (L > g.NB) return;
  int I, J, K;
  decode(g, indb(f, 1, L), I, J, K);
  const int NS = indb(f, 2, L);
  const int IBK = abs(t.indbk[L - 1]), IBE = abs(t.indbe[L - 1]);
  long long c;
  if (NS == 2) c = cid(g, I - 1, J, K);
  else if (NS == 4) c = cid(g, I, J - 1, K);
  else if (NS == 6) c = cid(g, I, J, K - 1);
  else c = cid(g, I, J, K);
  if (IBK == 2 || IBK == 6 || IBK == 8) t.bck[L - 1] = t.ak[c];
  else if (IBK != 1) atomicOr(err, ERR_PG);
  if (IBE == 2 || IBE == 6 || IBE == 8) t.bce[L - 1] = t.ae[c];
  else if (IBE != 1) atomicOr(err, ERR_PG);
}

__global__ void k_kinit(Geo g, Fld f, KeConst kc, double *AK, double *AE, double *ANUT, double *ANU) {
  ROW_LOOP_BEGIN(g)
  const long long c = cid(g, I, J, K);
  double ak = 0.0, ae = 0.0, nut = 0.0, nu = 0.0;
  if (kint(g, I, J, K)) {
    if (f.indc[c] != -1) { ak = kc.akinik; ae = kc.akinie; }
    const int n = f.nf[c];
    if (n != -1) {
      const double W = dmax(ae, kc.akmine);
      nut = kc.akcmu * ak * ak / W;
      nu = kc.anu0 + nut;
    }
  }
  AK[c] = ak; AE[c] = ae; ANUT[c] = nut; ANU[c] = nu;
  ROW_LOOP_END
}

#undef A
#undef XX_
#undef YY_
#undef ZZ_

#define RL(kern, ...) (kern<<<row_blocks(g), ROW_THREADS, 0, s>>>(__VA_ARGS__), count_launch())
void launch_bwkelg(cudaStream_t s, const Geo &g, const Fld &f, const Prm &p, const KeConst &kc, double *ak, double *ae,
                   int *err) {
  k_bwkelg<<<row_blocks(g), ROW_THREADS, 0, s>>>(g, f, p, kc, ak, ae, err);
  count_launch();
}
void launch_kstep(cudaStream_t s, const Geo &g, const Fld &f, const Prm &p, const KeConst &kc, const KeArrays &t,
                  double *akn, double *aen, int *err) {
  RL(k_kstep, g, f, p, kc, t, akn, aen, err);
}
void launch_kbsss(cudaStream_t s, const Geo &g, const Fld &f, const KeConst &kc, double *ak, double *ae, double *anut,
                  double *anu, bool bsss, bool nut) {
  if (bsss && nut) RL((k_kbsss<true, true>), g, f, kc, ak, ae, anut, anu);
  else if (bsss) RL((k_kbsss<true, false>), g, f, kc, ak, ae, anut, anu);
  else if (nut) RL((k_kbsss<false, true>), g, f, kc, ak, ae, anut, anu);
}
void launch_bwke(cudaStream_t s, const Geo &g, const Fld &f, const KeArrays &t, int *err) {
  if (g.NB <= 0) return;
  k_bwke<<<(g.NB + 255) / 256, 256, 0, s>>>(g, f, t, err);
  count_launch();
}
void launch_kinit(cudaStream_t s, const Geo &g, const Fld &f, const KeConst &kc, double *ak, double *ae, double *anut,
                  double *anu) {
  RL(k_kinit, g, f, kc, ak, ae, anut, anu);
}

}  // namespace cadmas
