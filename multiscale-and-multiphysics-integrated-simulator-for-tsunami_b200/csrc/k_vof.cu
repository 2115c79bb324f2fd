// k_vof.cu -- donor-acceptor VOF advection and surface-cell flagging of
// VF_F1CAL (vf_f1cal.f:121-230).
//
//   k_fconv        VF_FCONV  (vf_fconv.f:56-206)  three face fluxes per cell
//   k_feuler       VF_FEULER (vf_feuler.f:43-56)
//   k_fmod1_*      VF_FMOD1  (vf_fmod1.f:37-200) as gathers:
//                    count  - NLIM of each fluid/gas cell = surface cells
//                             whose donor (F) or acceptor (E) it is
//                    redist - loop 300 per surface cell; the E/F cells it
//                             writes have NLIM = 1, i.e. belong to it alone
//                    target - loop 400 for E/F cells: the over/under-fill of
//                             the surface neighbours added in ascending
//                             linear index, the order of the INDS list
//                    clamp  - loop 400 for the surface cells themselves
//   k_fcut         VF_FCUT01 (vf_fcut01.f:34-56) cut-off + FSUM/FCUT partials
//   k_fnf_*        VF_FNFINI (vf_fnfini.f:36-197), one pass per sweep of
//                  the reference; the fixed-point loop is driven by the host
//                  with a device change counter
//   k_fbubup       VF_FBUBUP (vf_fbubup.f:35-51) one thread per column
//   k_fnfprv       VF_FNFPRV (vf_fnfprv.f:34-225)
//   k_cindc        VF_CINDC  (vf_cindc.f:35-53), also counts NUMS
//   k_bsppfl       VF_BSPPFL (vf_bsppfl.f:40-67) into a second buffer
//
// The surface list INDS of the reference is not kept: every loop over it
// is a pass over the grid that acts on cells with NF in 1..6 (or 7).  The
// loops are free of ordering effects because FNFPRV gives each surface
// cell a fluid neighbour (NF=0) on its fluid side and a gas neighbour
// (NF=8) on the other, so the cells one surface cell writes are never
// read by another in the same loop; the one scatter-add (loop 400 of
// FMOD1) is done as an ordered gather.
#include "cadmas_dev.cuh"
#include "kernels.h"
#include "vof_face.cuh"

namespace cadmas {

#define A(a, i, j, k) a[cid(g, i, j, k)]
#define XX_(m, i) gx(g, m, i)
#define YY_(m, j) gy(g, m, j)
#define ZZ_(m, k) gz(g, m, k)

// ------------------------------------------------------------ VF_FCONV
__global__ void k_fconv(Geo g, Fld f, Prm p, double *FLFU, double *FLFV, double *FLFW) {
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
    int N = A(NF, LD, J, K);
    int ndm = (N != -1) ? A(NF, LDM, J, K) : -1;
    double fdm = (N != -1 && ndm != -1) ? A(FF, LDM, J, K) : 0.0;
    double vd = (N != -1) ? XX_(2, LD) * A(GGV, LD, J, K) : 0.0;
    double bcf = (N == -1) ? f.bcf[f.indx[c] - 1] : 0.0;
    int na = A(NF, LA, J, K);
    double fl = fconv_face(C, N, (N != -1) ? A(FF, LD, J, K) : 0.0, ndm, fdm, vd, XX_(2, LD), bcf, na,
                           (na != -1) ? A(FF, LA, J, K) : 0.0, 3, 4, 5, 6, FL);
    fu = 0.0 - (double)LSN * fl;
  }
  if (K >= 2 && K <= NK - 1 && J >= 2 && I >= 2 && I <= NI - 1 && f.indy[c] != -1) {
    double C = DT * f.ggy[c] * f.vv[c];
    int LSN, LA, LD, LDM;
    if (C >= 0.0) { LSN = 1; LA = J; LD = J - 1; LDM = J - 2; } else { LSN = -1; LA = J - 1; LD = J; LDM = J + 1; }
    int N = A(NF, I, LD, K);
    int ndm = (N != -1) ? A(NF, I, LDM, K) : -1;
    double fdm = (N != -1 && ndm != -1) ? A(FF, I, LDM, K) : 0.0;
    double vd = (N != -1) ? YY_(2, LD) * A(GGV, I, LD, K) : 0.0;
    double bcf = (N == -1) ? f.bcf[f.indy[c] - 1] : 0.0;
    int na = A(NF, I, LA, K);
    double fl = fconv_face(C, N, (N != -1) ? A(FF, I, LD, K) : 0.0, ndm, fdm, vd, YY_(2, LD), bcf, na,
                           (na != -1) ? A(FF, I, LA, K) : 0.0, 1, 2, 5, 6, FL);
    fv = 0.0 - (double)LSN * fl;
  }
  if (K >= 2 && J >= 2 && J <= NJ - 1 && I >= 2 && I <= NI - 1 && f.indz[c] != -1) {
    double C = DT * f.ggz[c] * f.ww[c];
    int LSN, LA, LD, LDM;
    if (C >= 0.0) { LSN = 1; LA = K; LD = K - 1; LDM = K - 2; } else { LSN = -1; LA = K - 1; LD = K; LDM = K + 1; }
    int N = A(NF, I, J, LD);
    int ndm = (N != -1) ? A(NF, I, J, LDM) : -1;
    double fdm = (N != -1 && ndm != -1) ? A(FF, I, J, LDM) : 0.0;
    double vd = (N != -1) ? ZZ_(2, LD) * A(GGV, I, J, LD) : 0.0;
    double bcf = (N == -1) ? f.bcf[f.indz[c] - 1] : 0.0;
    int na = A(NF, I, J, LA);
    double fl = fconv_face(C, N, (N != -1) ? A(FF, I, J, LD) : 0.0, ndm, fdm, vd, ZZ_(2, LD), bcf, na,
                           (na != -1) ? A(FF, I, J, LA) : 0.0, 1, 2, 3, 4, FL);
    fw = 0.0 - (double)LSN * fl;
  }
  FLFU[c] = fu; FLFV[c] = fv; FLFW[c] = fw;
  ROW_LOOP_END
}

// ----------------------------------------------------------- VF_FEULER
__global__ void k_feuler(Geo g, Fld f, Prm p, const double *FLFU, const double *FLFV, const double *FLFW) {
  ROW_LOOP_BEGIN(g)
  if (I >= 2 && I <= g.NI - 1 && J >= 2 && J <= g.NJ - 1 && K >= 2 && K <= g.NK - 1) {
    const long long c = cid(g, I, J, K);
    if (f.nf[c] != -1) {
      double G = f.ggv[c];
      double G0 = G - (G - G) * 1.0;
      // QF of VF_FGENE (vf_fgene.f:42-70): on the wave source's line, the
      // fluid cells up to and the first surface cell of the column (gas
      // cells below it skipped) gain F * 2 XX(4,I) SRCUV (or YY(4,J))
      double QF = 0.0;
      if ((p.iws == I || p.jws == J) && f.nf[c] != 8) {
        bool below = true;  // no surface cell under this one
        for (int K2 = 2; K2 < K; ++K2) {
          const int n2 = A(f.nf, I, J, K2);
          if (n2 != -1 && n2 != 0 && n2 != 8) { below = false; break; }
        }
        if (below) {
          if (p.iws == I) QF = QF + f.ff[c] * (2.0 * XX_(4, I) * f.srcuv[(J - 1) + (long long)g.NJ * (K - 1)]);
          if (p.jws == J) QF = QF + f.ff[c] * (2.0 * YY_(4, J) * f.srcuv[(I - 1) + (long long)g.NI * (K - 1)]);
        }
      }
      double DF = (XX_(4, I) * (A(FLFU, I + 1, J, K) - FLFU[c]) + YY_(4, J) * (A(FLFV, I, J + 1, K) - FLFV[c]) +
                   ZZ_(4, K) * (A(FLFW, I, J, K + 1) - FLFW[c]) + p.dtnow * QF);
      f.ff[c] = (G0 * f.ff[c] + DF) / G;
    }
  }
  ROW_LOOP_END
}

// ------------------------------------------------------------ VF_FMOD1
// E (acceptor, gas side) and F (donor, fluid side) cells of a surface cell.
__device__ __forceinline__ void fmod_ends(int N, int I, int J, int K, int &IE, int &JE, int &KE, int &IF,
                                          int &JF, int &KF) {
  IE = I; JE = J; KE = K; IF = I; JF = J; KF = K;
  if (N == 5) { KE = K + 1; KF = K - 1; }
  else if (N == 6) { KE = K - 1; KF = K + 1; }
  else if (N == 3) { JE = J + 1; JF = J - 1; }
  else if (N == 4) { JE = J - 1; JF = J + 1; }
  else if (N == 1) { IE = I + 1; IF = I - 1; }
  else if (N == 2) { IE = I - 1; IF = I + 1; }
}
__device__ __forceinline__ bool is_surf(int n) { return n >= 1 && n <= 6; }

// Neighbour offsets in ascending linear-index order and the NF value a
// surface cell at that offset must have for this cell to be its E or F.
// Offset (-K): the cell below; it points up at us if it is NF=5 (fluid
// below it, so we are its E) or NF=6 (we are its F).
struct NbSel { int di, dj, dk, nE, nF; };
__constant__ NbSel c_nb[6] = {
    {0, 0, -1, 5, 6}, {0, -1, 0, 3, 4}, {-1, 0, 0, 1, 2},
    {1, 0, 0, 2, 1},  {0, 1, 0, 4, 3},  {0, 0, 1, 6, 5}};

__global__ void k_fmod1_count(Geo g, Fld f, int *NLIM) {
  ROW_LOOP_BEGIN(g)
  const long long c = cid(g, I, J, K);
  int n = 0;
  if (I >= 2 && I <= g.NI - 1 && J >= 2 && J <= g.NJ - 1 && K >= 2 && K <= g.NK - 1) {
#pragma unroll
    for (int q = 0; q < 6; ++q) {
      int nb = A(f.nf, I + c_nb[q].di, J + c_nb[q].dj, K + c_nb[q].dk);
      if (nb == c_nb[q].nE || nb == c_nb[q].nF) n++;
    }
  }
  NLIM[c] = n;
  ROW_LOOP_END
}

__device__ __forceinline__ double cellvol(const Geo &g, const double *GGV, int I, int J, int K) {
  return gx(g, 2, I) * gy(g, 2, J) * gz(g, 2, K) * GGV[cid(g, I, J, K)];
}

__global__ void k_fmod1_redist(Geo g, Fld f, const int *NLIM) {
  double *FF = f.ff;
  ROW_LOOP_BEGIN(g)
  const long long s = cid(g, I, J, K);
  int N = f.nf[s];
  if (is_surf(N) && I >= 2 && I <= g.NI - 1 && J >= 2 && J <= g.NJ - 1 && K >= 2 && K <= g.NK - 1) {
    int IE, JE, KE, IF, JF, KF;
    fmod_ends(N, I, J, K, IE, JE, KE, IF, JF, KF);
    const long long e = cid(g, IE, JE, KE), fc = cid(g, IF, JF, KF);
    double VE = cellvol(g, f.ggv, IE, JE, KE), VS = cellvol(g, f.ggv, I, J, K), VF = cellvol(g, f.ggv, IF, JF, KF);
    double SS = VS * FF[s];
    if (NLIM[e] == 1) SS = SS + VE * FF[e];
    if (NLIM[fc] == 1) SS = SS + VF * FF[fc];
    double DS;
    if (NLIM[fc] == 1) { DS = dmin(VF, SS); SS = SS - DS; FF[fc] = DS / VF; }
    DS = dmin(VS, SS); SS = SS - DS; FF[s] = DS / VS;
    if (NLIM[e] == 1) { DS = dmin(VE, SS); SS = SS - DS; FF[e] = DS / VE; }
    if (SS > 0.0) {
      if (NLIM[e] == 1) FF[e] = FF[e] + SS / VE;
      else FF[s] = FF[s] + SS / VS;
    }
  }
  ROW_LOOP_END
}

// Loop 400 for E/F cells (non-surface), gathering from surface neighbours.
__global__ void k_fmod1_target(Geo g, Fld f) {
  double *FF = f.ff;
  ROW_LOOP_BEGIN(g)
  const long long c = cid(g, I, J, K);
  if (!is_surf(f.nf[c]) && I >= 2 && I <= g.NI - 1 && J >= 2 && J <= g.NJ - 1 && K >= 2 && K <= g.NK - 1) {
    double v = FF[c];
    bool touched = false;
#pragma unroll
    for (int q = 0; q < 6; ++q) {
      const int Is = I + c_nb[q].di, Js = J + c_nb[q].dj, Ks = K + c_nb[q].dk;
      const long long s = cid(g, Is, Js, Ks);
      const int n = f.nf[s];
      if (n == c_nb[q].nE) {            // we are the E cell of s
        double fs = FF[s];
        if (fs > 1.0) {
          double VS = cellvol(g, f.ggv, Is, Js, Ks), VE = cellvol(g, f.ggv, I, J, K);
          v = v + VS * (fs - 1.0) / VE;
          touched = true;
        }
      } else if (n == c_nb[q].nF) {     // we are the F cell of s
        double fs = FF[s];
        if (!(fs > 1.0) && fs < 0.0) {
          double VS = cellvol(g, f.ggv, Is, Js, Ks), VF = cellvol(g, f.ggv, I, J, K);
          v = v + VS * fs / VF;
          touched = true;
        }
      }
    }
    if (touched) FF[c] = v;
  }
  ROW_LOOP_END
}

__global__ void k_fmod1_clamp(Geo g, Fld f) {
  ROW_LOOP_BEGIN(g)
  const long long s = cid(g, I, J, K);
  if (is_surf(f.nf[s]) && I >= 2 && I <= g.NI - 1 && J >= 2 && J <= g.NJ - 1 && K >= 2 && K <= g.NK - 1) {
    double v = f.ff[s];
    if (v > 1.0) v = 1.0;
    else if (v < 0.0) v = 0.0;
    f.ff[s] = v;
  }
  ROW_LOOP_END
}

// ----------------------------------------------------------- VF_FCUT01
__global__ void k_fcut(Geo g, Fld f, Prm p, double *rb_sum, double *rb_cut) {
  double ssum = 0.0, scut = 0.0;
  const long long nrows = (long long)g.NJ * g.NK;
  ROW_LOOP_BEGIN(g)
  if (I >= 2 && I <= g.NI - 1 && J >= 2 && J <= g.NJ - 1 && K >= 2 && K <= g.NK - 1) {
    const long long c = cid(g, I, J, K);
    if (f.nf[c] != -1) {
      double V = XX_(2, I) * YY_(2, J) * ZZ_(2, K) * f.ggv[c];
      double F = f.ff[c];
      if (F > p.fupper) { scut = scut + (F - 1.0) * V; F = 1.0; f.ff[c] = F; }
      else if (F < p.flower) { scut = scut + (F - 0.0) * V; F = 0.0; f.ff[c] = F; }
      ssum = ssum + F * V;
    }
  }
  ROW_LOOP_END
  const long long row = (long long)blockIdx.x * ROWS_PER_BLOCK + (threadIdx.x >> 5);
  row_store(ssum, rb_sum, row, nrows);
  row_store(scut, rb_cut, row, nrows);
}

// ----------------------------------------------------------- VF_FNFINI
// Phase 1+2: non-obstacle cells to fluid, then gas where F < FLOWER and no
// neighbour face carries F > FUPPER (vf_fnfini.f:39-103).
__global__ void k_fnf_init(Geo g, Fld f, Prm p) {
  const double FU = p.fupper;
  const double *FF = f.ff;
  ROW_LOOP_BEGIN(g)
  const long long c = cid(g, I, J, K);
  if (K >= 2 && K <= g.NK - 1) {
    int n = f.nf[c];
    if (n != -1) {
      n = 0;
      if (I >= 2 && I <= g.NI - 1 && J >= 2 && J <= g.NJ - 1 && FF[c] < p.flower) {
        int IX1 = f.indx[c], IX2 = A(f.indx, I + 1, J, K), IY1 = f.indy[c], IY2 = A(f.indy, I, J + 1, K);
        int IZ1 = f.indz[c], IZ2 = A(f.indz, I, J, K + 1);
        double FX1 = IX1 >= 1 ? f.bcf[IX1 - 1] : A(FF, I - 1, J, K);
        double FX2 = IX2 >= 1 ? f.bcf[IX2 - 1] : A(FF, I + 1, J, K);
        double FY1 = IY1 >= 1 ? f.bcf[IY1 - 1] : A(FF, I, J - 1, K);
        double FY2 = IY2 >= 1 ? f.bcf[IY2 - 1] : A(FF, I, J + 1, K);
        double FZ1 = IZ1 >= 1 ? f.bcf[IZ1 - 1] : A(FF, I, J, K - 1);
        double FZ2 = IZ2 >= 1 ? f.bcf[IZ2 - 1] : A(FF, I, J, K + 1);
        if (!(FZ1 > FU && IZ1 == 0) && !(FY1 > FU && IY1 == 0) && !(FY2 > FU && IY2 == 0) &&
            !(FX1 > FU && IX1 == 0) && !(FX2 > FU && IX2 == 0) && !(FZ2 > FU && IZ2 == 0))
          n = 8;
      }
      f.nf[c] = n;
    }
  }
  ROW_LOOP_END
}

__device__ __forceinline__ bool interior3(const Geo &g, int I, int J, int K) {
  return I >= 2 && I <= g.NI - 1 && J >= 2 && J <= g.NJ - 1 && K >= 2 && K <= g.NK - 1;
}

// loop 1100: cells next to gas become surface (7)
__global__ void k_fnf_mark7(Geo g, int *NF, const int *done) {
  if (*done) return;
  ROW_LOOP_BEGIN(g)
  const long long c = cid(g, I, J, K);
  if (interior3(g, I, J, K)) {
    int n = NF[c];
    if (n != -1 && n != 8) {
      if (A(NF, I, J, K + 1) == 8 || A(NF, I, J + 1, K) == 8 || A(NF, I, J - 1, K) == 8 ||
          A(NF, I + 1, J, K) == 8 || A(NF, I - 1, J, K) == 8 || A(NF, I, J, K - 1) == 8)
        NF[c] = 7;
    }
  }
  ROW_LOOP_END
}
// loop 1200: surface cells without a fluid neighbour become gas
__global__ void k_fnf_to8(Geo g, int *NF, const int *done) {
  if (*done) return;
  ROW_LOOP_BEGIN(g)
  const long long c = cid(g, I, J, K);
  if (interior3(g, I, J, K) && NF[c] == 7) {
    if (A(NF, I, J, K + 1) != 0 && A(NF, I, J + 1, K) != 0 && A(NF, I, J - 1, K) != 0 &&
        A(NF, I + 1, J, K) != 0 && A(NF, I - 1, J, K) != 0 && A(NF, I, J, K - 1) != 0)
      NF[c] = 8;
  }
  ROW_LOOP_END
}
// loop 1300: surface cells not between fluid and gas along any axis -> -7
__global__ void k_fnf_markm7(Geo g, int *NF, int *nch, const int *done) {
  if (*done) return;
  int cnt = 0;
  ROW_LOOP_BEGIN(g)
  const long long c = cid(g, I, J, K);
  if (interior3(g, I, J, K) && NF[c] == 7) {
    if (A(NF, I, J, K - 1) != 0 || A(NF, I, J, K + 1) != 8)
      if (A(NF, I - 1, J, K) != 0 || A(NF, I + 1, J, K) != 8)
        if (A(NF, I + 1, J, K) != 0 || A(NF, I - 1, J, K) != 8)
          if (A(NF, I, J - 1, K) != 0 || A(NF, I, J + 1, K) != 8)
            if (A(NF, I, J + 1, K) != 0 || A(NF, I, J - 1, K) != 8)
              if (A(NF, I, J, K + 1) != 0 || A(NF, I, J, K - 1) != 8) { NF[c] = -7; cnt++; }
  }
  ROW_LOOP_END
  if (cnt) atomicAdd(nch, cnt);
}
// loop exit test: NCH = 0 ends the iteration; the counter is cleared for
// the next sweep.  Capped so that no input can keep the loop running.
__global__ void k_fnf_check(int *nch, int *done, int *iter, int cap, int *err) {
  if (*done) return;
  int n = *nch;
  *nch = 0;
  *iter = *iter + 1;
  if (n <= 0) *done = 1;
  else if (*iter >= cap) { *done = 1; atomicOr(err, ERR_CAP); }
}
// loop 1400: -7 -> gas
__global__ void k_fnf_m7to8(Geo g, int *NF, const int *done) {
  if (*done) return;
  ROW_LOOP_BEGIN(g)
  const long long c = cid(g, I, J, K);
  if (NF[c] == -7) NF[c] = 8;
  ROW_LOOP_END
}

// ----------------------------------------------------------- VF_FBUBUP
// One thread per (I,J) column walks K = NK-2 .. 2 over the levels whose
// timer fired (active[K] != 0, decided on the host from TBUB and TNOW).
__global__ void k_fbubup(Geo g, Fld f, Prm p, const unsigned char *active) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  int ni = g.NI - 2, nj = g.NJ - 2;
  if (t >= ni * nj) return;
  const int I = 2 + t % ni, J = 2 + t / ni;
  double *FF = f.ff;
  for (int K = g.NK - 2; K >= 2; --K) {
    if (!active[K]) continue;
    const int K1 = K + 1;
    const long long c = cid(g, I, J, K), u = cid(g, I, J, K1);
    if (FF[c] < p.fupper && f.nf[c] == 0 && f.nf[u] != -1) {
      double V0 = ZZ_(2, K) * f.ggv[c], V1 = ZZ_(2, K1) * f.ggv[u];
      double FMOVE = dmin((1.0 - FF[c]) * V0, FF[u] * V1);
      FF[u] = FF[u] - FMOVE / V1;
      FF[c] = FF[c] + FMOVE / V0;
    }
  }
}

// ----------------------------------------------------------- VF_FNFPRV
__device__ __forceinline__ double bcf_or(const Fld &f, int ind, double v) { return ind >= 1 ? f.bcf[ind - 1] : v; }

__global__ void __launch_bounds__(ROW_THREADS, 3) k_fnfprv(Geo g, Fld f, int *err) {
  const double *FF = f.ff;
  int *NF = f.nf;
  ROW_LOOP_BEGIN(g)
  const long long c = cid(g, I, J, K);
  if (interior3(g, I, J, K) && NF[c] == 7) {
    double FM = -1.0, FS;
    int res = 7;
    int KB = K - 1;
    if (A(NF, I, J, KB) == 0 && A(NF, I, J, K + 1) == 8) {
      FS = 2.0 * A(FF, I, J, KB);
      FS = FS + bcf_or(f, A(f.indx, I, J, KB), A(FF, I - 1, J, KB));
      FS = FS + bcf_or(f, A(f.indx, I + 1, J, KB), A(FF, I + 1, J, KB));
      FS = FS + bcf_or(f, A(f.indy, I, J, KB), A(FF, I, J - 1, KB));
      FS = FS + bcf_or(f, A(f.indy, I, J + 1, KB), A(FF, I, J + 1, KB));
      if (FS > FM) { res = 5; FM = FS; }
    }
    KB = K + 1;
    if (A(NF, I, J, KB) == 0 && A(NF, I, J, K - 1) == 8) {
      FS = 2.0 * A(FF, I, J, KB);
      FS = FS + bcf_or(f, A(f.indx, I, J, KB), A(FF, I - 1, J, KB));
      FS = FS + bcf_or(f, A(f.indx, I + 1, J, KB), A(FF, I + 1, J, KB));
      FS = FS + bcf_or(f, A(f.indy, I, J, KB), A(FF, I, J - 1, KB));
      FS = FS + bcf_or(f, A(f.indy, I, J + 1, KB), A(FF, I, J + 1, KB));
      if (FS > FM) { res = 6; FM = FS; }
    }
    int JB = J - 1;
    if (A(NF, I, JB, K) == 0 && A(NF, I, J + 1, K) == 8) {
      FS = 2.0 * A(FF, I, JB, K);
      FS = FS + bcf_or(f, A(f.indx, I, JB, K), A(FF, I - 1, JB, K));
      FS = FS + bcf_or(f, A(f.indx, I + 1, JB, K), A(FF, I + 1, JB, K));
      FS = FS + bcf_or(f, A(f.indz, I, JB, K), A(FF, I, JB, K - 1));
      FS = FS + bcf_or(f, A(f.indz, I, JB, K + 1), A(FF, I, JB, K + 1));
      if (FS > FM) { res = 3; FM = FS; }
    }
    JB = J + 1;
    if (A(NF, I, JB, K) == 0 && A(NF, I, J - 1, K) == 8) {
      FS = 2.0 * A(FF, I, JB, K);
      FS = FS + bcf_or(f, A(f.indx, I, JB, K), A(FF, I - 1, JB, K));
      FS = FS + bcf_or(f, A(f.indx, I + 1, JB, K), A(FF, I + 1, JB, K));
      FS = FS + bcf_or(f, A(f.indz, I, JB, K), A(FF, I, JB, K - 1));
      FS = FS + bcf_or(f, A(f.indz, I, JB, K + 1), A(FF, I, JB, K + 1));
      if (FS > FM) { res = 4; FM = FS; }
    }
    int IB = I - 1;
    if (A(NF, IB, J, K) == 0 && A(NF, I + 1, J, K) == 8) {
      FS = 2.0 * A(FF, IB, J, K);
      FS = FS + bcf_or(f, A(f.indy, IB, J, K), A(FF, IB, J - 1, K));
      FS = FS + bcf_or(f, A(f.indy, IB, J + 1, K), A(FF, IB, J + 1, K));
      FS = FS + bcf_or(f, A(f.indz, IB, J, K), A(FF, IB, J, K - 1));
      FS = FS + bcf_or(f, A(f.indz, IB, J, K + 1), A(FF, IB, J, K + 1));
      if (FS > FM) { res = 1; FM = FS; }
    }
    IB = I + 1;
    if (A(NF, IB, J, K) == 0 && A(NF, I - 1, J, K) == 8) {
      FS = 2.0 * A(FF, IB, J, K);
      FS = FS + bcf_or(f, A(f.indy, IB, J, K), A(FF, IB, J - 1, K));
      FS = FS + bcf_or(f, A(f.indy, IB, J + 1, K), A(FF, IB, J + 1, K));
      FS = FS + bcf_or(f, A(f.indz, IB, J, K), A(FF, IB, J, K - 1));
      FS = FS + bcf_or(f, A(f.indz, IB, J, K + 1), A(FF, IB, J, K + 1));
      if (FS > FM) { res = 2; FM = FS; }
    }
    NF[c] = res;
    if (res == 7) atomicOr(err, ERR_PG);
  }
  ROW_LOOP_END
}

// ------------------------------------------------------------ VF_CINDC
__global__ void k_cindc(Geo g, Fld f, int *nums) {
  int cnt = 0;
  ROW_LOOP_BEGIN(g)
  if (interior3(g, I, J, K)) {
    const long long c = cid(g, I, J, K);
    int n = f.nf[c];
    f.indc[c] = (n == 8 || n == -1) ? -1 : 0;
    if (n >= 1 && n <= 7) cnt++;
  }
  ROW_LOOP_END
  if (cnt) atomicAdd(nums, cnt);
}

// ----------------------------------------------------------- VF_BSPPFL
__global__ void k_bsppfl(Geo g, Fld f, const double *PP0, double *PPN) {
  ROW_LOOP_BEGIN(g)
  const long long c = cid(g, I, J, K);
  double v = PP0[c];
  if (interior3(g, I, J, K) && f.nf[c] == 0 && f.nf0[c] == 8) {
    double SUMF = 0.0, SUMP = 0.0;
    for (int KP = -1; KP <= 1; ++KP)
      for (int JP = -1; JP <= 1; ++JP)
        for (int IP = -1; IP <= 1; ++IP) {
          const long long q = cid(g, I + IP, J + JP, K + KP);
          if (f.nf[q] == 0) { double F = f.ff[q]; SUMF = SUMF + F; SUMP = SUMP + F * PP0[q]; }
        }
    v = (SUMF < 1.0e-20) ? 0.0 : SUMP / SUMF;
  }
  PPN[c] = v;
  ROW_LOOP_END
}

#undef A
#undef XX_
#undef YY_
#undef ZZ_

// ------------------------------------------------------------ launchers
#define RL(kern, ...) (kern<<<row_blocks(g), ROW_THREADS, 0, s>>>(__VA_ARGS__), count_launch())
void launch_fconv(cudaStream_t s, const Geo &g, const Fld &f, const Prm &p, double *a, double *b, double *c) { RL(k_fconv, g, f, p, a, b, c); }
void launch_feuler(cudaStream_t s, const Geo &g, const Fld &f, const Prm &p, const double *a, const double *b, const double *c) { RL(k_feuler, g, f, p, a, b, c); }
void launch_fmod1(cudaStream_t s, const Geo &g, const Fld &f, int *nlim) {
  RL(k_fmod1_count, g, f, nlim);
  RL(k_fmod1_redist, g, f, nlim);
  RL(k_fmod1_target, g, f);
  RL(k_fmod1_clamp, g, f);
}
void launch_fcut(cudaStream_t s, const Geo &g, const Fld &f, const Prm &p, double *rbs, double *rbc) { RL(k_fcut, g, f, p, rbs, rbc); }
void launch_fnf_init(cudaStream_t s, const Geo &g, const Fld &f, const Prm &p) { RL(k_fnf_init, g, f, p); }
void launch_fnf_sweep(cudaStream_t s, const Geo &g, int *nf, int *nch, int *done, int *iter, int cap, int *err) {
  RL(k_fnf_mark7, g, nf, done);
  RL(k_fnf_to8, g, nf, done);
  RL(k_fnf_markm7, g, nf, nch, done);
  k_fnf_check<<<1, 1, 0, s>>>(nch, done, iter, cap, err);
  count_launch();
  RL(k_fnf_m7to8, g, nf, done);
}
void launch_fbubup(cudaStream_t s, const Geo &g, const Fld &f, const Prm &p, const unsigned char *active) {
  int n = (g.NI - 2) * (g.NJ - 2);
  k_fbubup<<<(n + 255) / 256, 256, 0, s>>>(g, f, p, active);
  count_launch();
}
void launch_fnfprv(cudaStream_t s, const Geo &g, const Fld &f, int *err) { RL(k_fnfprv, g, f, err); }
void launch_cindc(cudaStream_t s, const Geo &g, const Fld &f, int *nums) { RL(k_cindc, g, f, nums); }
void launch_bsppfl(cudaStream_t s, const Geo &g, const Fld &f, const double *pp0, double *ppn) { RL(k_bsppfl, g, f, pp0, ppn); }
#undef RL

}  // namespace cadmas
