// k_poisson.cu -- pressure-Poisson assembly, MILU-BiCGSTAB and correction.
//
//   k_vpcoef            VF_VPCOEF (vf_vpcoef.f:117-437)
//   k_dcmp  (tile)      VF_MZDCMP (vf_mzdcmp.f:53-67)
//   k_fwd   (tile)      VF_MZFRWD (vf_mzfrwd.f:37-48), optionally fused with
//                       the SpMV VF_MZAX (vf_mzax.f:42-56) of its input
//   k_bwd   (tile)      VF_MZBKWD (vf_mzbkwd.f:37-47)
//   row kernels         the vector updates and VF_MZIP dot products of
//                       VF_M1BCGS (vf_m1bcgs.f:76-266)
//   k_vmodif            VF_VMODIF (vf_vmodif.f:58-215)
//
// MILU is a lexicographic recurrence.  A tile of TI x TJ z-columns is one
// thread block; thread (ti,tj) owns column (is+ti, js+tj) and at wavefront
// step s processes k = 2 + s - ti - tj, so X(i-1,j,k) and X(i,j-1,k) were
// produced by the neighbouring threads at step s-1 and X(i,j,k-1) by the
// thread itself.  Every cell is evaluated with exactly the expression and
// operand order of the sequential loop, so a single tile covering the
// interior reproduces the serial reference bit for bit.  Several tiles form
// the block-Jacobi preconditioner that the reference itself applies when it
// runs on NPI x NPJ MPI ranks (each rank factors and sweeps its own x-y
// block; neighbour terms outside the block are coef*0*0 because the rank's
// halo DD and coefficients are zero).
#include "cadmas_dev.cuh"
#include "kernels.h"

namespace cadmas {

#define A(a, i, j, k) a[cid(g, i, j, k)]
#define XX_(m, i) gx(g, m, i)
#define YY_(m, j) gy(g, m, j)
#define ZZ_(m, k) gz(g, m, k)

// ------------------------------------------------------------- VF_VPCOEF
__global__ void k_vpcoef(Geo g, Fld f, Prm p, SysPtr A_, int *err) {
  const double DTI = 1.0 / p.dtnow, TR = p.dtnow / p.rho0, PPS = 0.0;
  const double *GGV = f.ggv, *GLV = f.glv, *FF = f.ff, *PP = f.pp;
  ROW_LOOP_BEGIN(g)
  const long long c = cid(g, I, J, K);
  double AD = 0.0, ALI = 0.0, ALJ = 0.0, ALK = 0.0, AUI = 0.0, AUJ = 0.0, AUK = 0.0, BB = 0.0;
  int N = f.nf[c];
  if (f.indc[c] == -1) {
    AD = 1.0;
  } else if (N == 0) {
    const int IM = I - 1, IP = I + 1, JM = J - 1, JP = J + 1, KM = K - 1, KP = K + 1;
    double AXY = XX_(2, I) * YY_(2, J), AXZ = XX_(2, I) * ZZ_(2, K), AYZ = YY_(2, J) * ZZ_(2, K);
    double AVL = XX_(2, I) * YY_(2, J) * ZZ_(2, K);
    double AIM, AIP, AJM, AJP, AKM, AKP, GV;
    int IS = f.indx[c];
    if (IS == 0) {
      GV = XX_(6, I) * (XX_(2, I) * GGV[c] / GLV[c] + XX_(2, IM) * A(GGV, IM, J, K) / A(GLV, IM, J, K));
      AIM = AYZ * XX_(5, I) * f.ggx[c] * GV; ALI = -AIM;
    } else if (IS >= 1) {
      if (indb(f, 3, IS) == 4) AIM = 2.0 * AYZ * XX_(4, I) * f.ggx[c] * GGV[c] / GLV[c];
      else AIM = 0.0;
    } else { AIM = 0.0; atomicOr(err, ERR_PG); }
    IS = A(f.indx, IP, J, K);
    if (IS == 0) {
      GV = XX_(6, IP) * (XX_(2, IP) * A(GGV, IP, J, K) / A(GLV, IP, J, K) + XX_(2, I) * GGV[c] / GLV[c]);
      AIP = AYZ * XX_(5, IP) * A(f.ggx, IP, J, K) * GV; AUI = -AIP;
    } else if (IS >= 1) {
      if (indb(f, 3, IS) == 4) AIP = 2.0 * AYZ * XX_(4, I) * A(f.ggx, IP, J, K) * GGV[c] / GLV[c];
      else AIP = 0.0;
    } else { AIP = 0.0; atomicOr(err, ERR_PG); }
    IS = f.indy[c];
    if (IS == 0) {
      GV = YY_(6, J) * (YY_(2, J) * GGV[c] / GLV[c] + YY_(2, JM) * A(GGV, I, JM, K) / A(GLV, I, JM, K));
      AJM = AXZ * YY_(5, J) * f.ggy[c] * GV; ALJ = -AJM;
    } else if (IS >= 1) {
      if (indb(f, 3, IS) == 4) AJM = 2.0 * AXZ * YY_(4, J) * f.ggy[c] * GGV[c] / GLV[c];
      else AJM = 0.0;
    } else { AJM = 0.0; atomicOr(err, ERR_PG); }
    IS = A(f.indy, I, JP, K);
    if (IS == 0) {
      GV = YY_(6, JP) * (YY_(2, JP) * A(GGV, I, JP, K) / A(GLV, I, JP, K) + YY_(2, J) * GGV[c] / GLV[c]);
      AJP = AXZ * YY_(5, JP) * A(f.ggy, I, JP, K) * GV; AUJ = -AJP;
    } else if (IS >= 1) {
      if (indb(f, 3, IS) == 4) AJP = 2.0 * AXZ * YY_(4, J) * A(f.ggy, I, JP, K) * GGV[c] / GLV[c];
      else AJP = 0.0;
    } else { AJP = 0.0; atomicOr(err, ERR_PG); }
    IS = f.indz[c];
    if (IS == 0) {
      GV = ZZ_(6, K) * (ZZ_(2, K) * GGV[c] / GLV[c] + ZZ_(2, KM) * A(GGV, I, J, KM) / A(GLV, I, J, KM));
      AKM = AXY * ZZ_(5, K) * f.ggz[c] * GV; ALK = -AKM;
    } else if (IS >= 1) {
      if (indb(f, 3, IS) != 4) AKM = 0.0;
      else AKM = 2.0 * AXY * ZZ_(4, K) * f.ggz[c] * GGV[c] / GLV[c];
    } else { AKM = 0.0; atomicOr(err, ERR_PG); }
    IS = A(f.indz, I, J, KP);
    if (IS == 0) {
      GV = ZZ_(6, KP) * (ZZ_(2, KP) * A(GGV, I, J, KP) / A(GLV, I, J, KP) + ZZ_(2, K) * GGV[c] / GLV[c]);
      AKP = AXY * ZZ_(5, KP) * A(f.ggz, I, J, KP) * GV; AUK = -AKP;
    } else if (IS >= 1) {
      if (indb(f, 3, IS) != 4) AKP = 0.0;
      else AKP = 2.0 * AXY * ZZ_(4, K) * A(f.ggz, I, J, KP) * GGV[c] / GLV[c];
    } else { AKP = 0.0; atomicOr(err, ERR_PG); }
    AD = AKM + AJM + AIM + AIP + AJP + AKP;
    double VD = AYZ * (A(f.ggx, IP, J, K) * A(f.uu, IP, J, K) - f.ggx[c] * f.uu[c]) +
                AXZ * (A(f.ggy, I, JP, K) * A(f.vv, I, JP, K) - f.ggy[c] * f.vv[c]) +
                AXY * (A(f.ggz, I, J, KP) * A(f.ww, I, J, KP) - f.ggz[c] * f.ww[c]);
    double VQ = -(GGV[c] - GGV[c]) * DTI * AVL;
    BB = VD - VQ;
  } else if (N == 5) {
    double PSI = ZZ_(3, K) / (0.5 * ZZ_(2, K - 1) + FF[c] * ZZ_(2, K));
    AD = 1.0; ALK = PSI - 1.0;
    BB = -TR * ((1.0 - PSI) * A(PP, I, J, K - 1) + PSI * PPS - PP[c]);
  } else if (N == 6) {
    double PSI = ZZ_(3, K + 1) / (0.5 * ZZ_(2, K + 1) + FF[c] * ZZ_(2, K));
    AD = 1.0; AUK = PSI - 1.0;
    BB = -TR * ((1.0 - PSI) * A(PP, I, J, K + 1) + PSI * PPS - PP[c]);
  } else if (N == 3) {
    double PSI = YY_(3, J) / (0.5 * YY_(2, J - 1) + FF[c] * YY_(2, J));
    AD = 1.0; ALJ = PSI - 1.0;
    BB = -TR * ((1.0 - PSI) * A(PP, I, J - 1, K) + PSI * PPS - PP[c]);
  } else if (N == 4) {
    double PSI = YY_(3, J + 1) / (0.5 * YY_(2, J + 1) + FF[c] * YY_(2, J));
    AD = 1.0; AUJ = PSI - 1.0;
    BB = -TR * ((1.0 - PSI) * A(PP, I, J + 1, K) + PSI * PPS - PP[c]);
  } else if (N == 1) {
    double PSI = XX_(3, I) / (0.5 * XX_(2, I - 1) + FF[c] * XX_(2, I));
    AD = 1.0; ALI = PSI - 1.0;
    BB = -TR * ((1.0 - PSI) * A(PP, I - 1, J, K) + PSI * PPS - PP[c]);
  } else if (N == 2) {
    double PSI = XX_(3, I + 1) / (0.5 * XX_(2, I + 1) + FF[c] * XX_(2, I));
    AD = 1.0; AUI = PSI - 1.0;
    BB = -TR * ((1.0 - PSI) * A(PP, I + 1, J, K) + PSI * PPS - PP[c]);
  } else {
    atomicOr(err, ERR_PG);
  }
  A_.ad[c] = AD; A_.ali[c] = ALI; A_.alj[c] = ALJ; A_.alk[c] = ALK;
  A_.aui[c] = AUI; A_.auj[c] = AUJ; A_.auk[c] = AUK; A_.bb[c] = BB;
  ROW_LOOP_END
}

// ----------------------------------------------------------- tile sweeps
struct TileGeo {
  int is, js, wi, wj;  // tile origin and width in cells
  int ti, tj;          // thread coordinates
  bool valid;
};
__device__ __forceinline__ TileGeo tile_geo(const Geo &g, int TI, int TJ) {
  TileGeo t;
  t.is = 2 + blockIdx.x * TI;
  t.js = 2 + blockIdx.y * TJ;
  t.wi = min(TI, g.NI - t.is);  // interior cells is..NI-1
  t.wj = min(TJ, g.NJ - t.js);
  t.ti = threadIdx.x % TI;
  t.tj = threadIdx.x / TI;
  t.valid = (t.ti < t.wi) && (t.tj < t.wj);
  return t;
}

// VF_MZDCMP over one tile.  Shared: DD of the previous step.
__global__ void k_dcmp(Geo g, int TI, int TJ, double U, SysPtr A_, const int *INDC, double *DD,
                       int *pivot_bad) {
  extern __shared__ double sm[];
  const int T = TI * TJ;
  double *ds = sm;  // [2][T]
  TileGeo t = tile_geo(g, TI, TJ);
  const int I = t.is + t.ti, J = t.js + t.tj;
  const int nsteps = (g.NK - 2) + (t.wi - 1) + (t.wj - 1);
  double dk1 = 0.0, au3 = 0.0;  // DD(i,j,k-1) and its AU3; k-1 = 1 is the zero ghost layer
  bool bad = false;
  for (int s = 0; s < nsteps; ++s) {
    const int k = 2 + s - t.ti - t.tj;
    const int cur = s & 1, prv = cur ^ 1;
    if (t.valid && k >= 2 && k <= g.NK - 1) {
      const long long c = cid(g, I, J, k);
      double dd = 0.0;
      if (INDC[c] != -1) {
        double d1 = 0.0, a1, d2 = 0.0, a2;
        if (t.ti > 0) {
          const long long n = c - 1;
          d1 = ds[prv * T + threadIdx.x - 1];
          a1 = A_.aui[n] + U * (A_.auj[n] + A_.auk[n]);
        } else {
          a1 = 0.0 + U * (0.0 + 0.0);
        }
        if (t.tj > 0) {
          const long long n = c - g.NI;
          d2 = ds[prv * T + threadIdx.x - TI];
          a2 = A_.auj[n] + U * (A_.aui[n] + A_.auk[n]);
        } else {
          a2 = 0.0 + U * (0.0 + 0.0);
        }
        dd = 1.0 / (A_.ad[c] - A_.ali[c] * d1 * a1 - A_.alj[c] * d2 * a2 - A_.alk[c] * dk1 * au3);
        if (dd <= 0.0) bad = true;
      }
      DD[c] = dd;
      ds[cur * T + threadIdx.x] = dd;
      dk1 = dd;
      au3 = A_.auk[c] + U * (A_.aui[c] + A_.auj[c]);
    }
    __syncthreads();
  }
  if (bad) atomicOr(pivot_bad, 1);
}

// Forward sweep (L D^-1 + I) X = Y.  When spmv_x is non-null the input is
// Y = A * spmv_x computed on the fly (VF_MZAX then VF_MZFRWD); otherwise
// Y is read from y.  Either way X is written for every column cell (0 on
// INDC=-1 cells, where the reference leaves its zero-initialised value).
__global__ void k_fwd(Geo g, int TI, int TJ, SysPtr A_, const int *INDC, const double *DD,
                      const double *y, const double *spmv_x, double *X, const SolveState *st) {
  if (st && st->done) return;
  extern __shared__ double sm[];
  const int T = TI * TJ;
  double *xs = sm, *ds = sm + 2 * T;
  TileGeo t = tile_geo(g, TI, TJ);
  const int I = t.is + t.ti, J = t.js + t.tj;
  const int nsteps = (g.NK - 2) + (t.wi - 1) + (t.wj - 1);
  double xk1 = 0.0, dk1 = 0.0;
  for (int s = 0; s < nsteps; ++s) {
    const int k = 2 + s - t.ti - t.tj;
    const int cur = s & 1, prv = cur ^ 1;
    if (t.valid && k >= 2 && k <= g.NK - 1) {
      const long long c = cid(g, I, J, k);
      double x = 0.0, d = DD[c];
      if (INDC[c] != -1) {
        double yv;
        if (spmv_x) {
          const double *P = spmv_x;
          yv = A_.ad[c] * P[c] + A_.ali[c] * P[c - 1] + A_.alj[c] * P[c - g.NI] +
               A_.alk[c] * P[c - (long long)g.NI * g.NJ] + A_.aui[c] * P[c + 1] +
               A_.auj[c] * P[c + g.NI] + A_.auk[c] * P[c + (long long)g.NI * g.NJ];
        } else {
          yv = y[c];
        }
        double d1 = 0.0, x1 = 0.0, d2 = 0.0, x2 = 0.0;
        if (t.ti > 0) { d1 = ds[prv * T + threadIdx.x - 1]; x1 = xs[prv * T + threadIdx.x - 1]; }
        if (t.tj > 0) { d2 = ds[prv * T + threadIdx.x - TI]; x2 = xs[prv * T + threadIdx.x - TI]; }
        x = yv - A_.ali[c] * d1 * x1 - A_.alj[c] * d2 * x2 - A_.alk[c] * dk1 * xk1;
      }
      X[c] = x;
      xs[cur * T + threadIdx.x] = x;
      ds[cur * T + threadIdx.x] = d;
      xk1 = x;
      dk1 = d;
    }
    __syncthreads();
  }
}

// Backward sweep (D + U) X = Tin, reversed loop order.
__global__ void k_bwd(Geo g, int TI, int TJ, SysPtr A_, const int *INDC, const double *DD,
                      const double *Tin, double *X, const SolveState *st) {
  if (st && st->done) return;
  extern __shared__ double sm[];
  const int T = TI * TJ;
  double *xs = sm;
  TileGeo t = tile_geo(g, TI, TJ);
  const int I = t.is + t.ti, J = t.js + t.tj;
  const int ri = t.wi - 1 - t.ti, rj = t.wj - 1 - t.tj;  // distance from the far corner
  const int nsteps = (g.NK - 2) + (t.wi - 1) + (t.wj - 1);
  double xk1 = 0.0;  // X(i,j,k+1); k+1 = NK is the zero ghost layer
  for (int s = 0; s < nsteps; ++s) {
    const int k = (g.NK - 1) - (s - ri - rj);
    const int cur = s & 1, prv = cur ^ 1;
    if (t.valid && k >= 2 && k <= g.NK - 1) {
      const long long c = cid(g, I, J, k);
      double x = 0.0;
      if (INDC[c] != -1) {
        double x1 = (ri > 0) ? xs[prv * T + threadIdx.x + 1] : 0.0;
        double x2 = (rj > 0) ? xs[prv * T + threadIdx.x + TI] : 0.0;
        x = (Tin[c] - A_.aui[c] * x1 - A_.auj[c] * x2 - A_.auk[c] * xk1) * DD[c];
      }
      X[c] = x;
      xs[cur * T + threadIdx.x] = x;
      xk1 = x;
    }
    __syncthreads();
  }
}

// ------------------------------------------------------------ row kernels
__device__ __forceinline__ bool interior(const Geo &g, int I, int J, int K) {
  return I >= 2 && I <= g.NI - 1 && J >= 2 && J <= g.NJ - 1 && K >= 2 && K <= g.NK - 1;
}

// Y = A X on INDC != -1 (VF_MZAX); Y untouched elsewhere.
__global__ void k_spmv(Geo g, SysPtr A_, const int *INDC, const double *X, double *Y,
                       const SolveState *st) {
  if (st && st->done) return;
  ROW_LOOP_BEGIN(g)
  const long long c = cid(g, I, J, K);
  if (INDC[c] != -1) {
    Y[c] = A_.ad[c] * X[c] + A_.ali[c] * X[c - 1] + A_.alj[c] * X[c - g.NI] +
           A_.alk[c] * X[c - (long long)g.NI * g.NJ] + A_.aui[c] * X[c + 1] +
           A_.auj[c] * X[c + g.NI] + A_.auk[c] * X[c + (long long)g.NI * g.NJ];
  }
  ROW_LOOP_END
}

// Y = B - Y on INDC != -1 (vf_m1bcgs.f:124-132)
__global__ void k_bmy(Geo g, const int *INDC, const double *B, double *Y, const SolveState *st) {
  if (st->done) return;
  ROW_LOOP_BEGIN(g)
  const long long c = cid(g, I, J, K);
  if (INDC[c] != -1) Y[c] = B[c] - Y[c];
  ROW_LOOP_END
}

// Row partials of up to two dot products (VF_MZIP).
__global__ void k_dot(Geo g, const int *INDC, const double *x0, const double *y0, const double *x1,
                      const double *y1, double *rb0, double *rb1, const SolveState *st) {
  if (st && st->done) return;
  double s0 = 0.0, s1 = 0.0;
  const long long nrows = (long long)g.NJ * g.NK;
  ROW_LOOP_BEGIN(g)
  const long long c = cid(g, I, J, K);
  if (INDC[c] != -1) {
    s0 = s0 + x0[c] * y0[c];
    if (x1) s1 = s1 + x1[c] * y1[c];
  }
  ROW_LOOP_END
  const long long row = (long long)blockIdx.x * ROWS_PER_BLOCK + (threadIdx.x >> 5);
  row_store(s0, rb0, row, nrows);
  if (x1) row_store(s1, rb1, row, nrows);
}

// RR = R0, PP = R0
__global__ void k_copy2(Geo g, const int *INDC, const double *R0, double *RR, double *PP,
                        const SolveState *st) {
  if (st->done) return;
  ROW_LOOP_BEGIN(g)
  const long long c = cid(g, I, J, K);
  if (INDC[c] != -1) { RR[c] = R0[c]; PP[c] = R0[c]; }
  ROW_LOOP_END
}

// RR = RR - ALPHA*AP (vf_m1bcgs.f:181-189)
__global__ void k_axpy_rr(Geo g, const int *INDC, const double *AP, double *RR, const SolveState *st) {
  if (st->done) return;
  const double alpha = st->alpha;
  ROW_LOOP_BEGIN(g)
  const long long c = cid(g, I, J, K);
  if (INDC[c] != -1) RR[c] = RR[c] - alpha * AP[c];
  ROW_LOOP_END
}

// XW = XW + (ALPHA*PP + OMEGA*RR); RR = RR - OMEGA*AE; row partials of
// (RR,RR) and (R0,RR) on the updated RR (vf_m1bcgs.f:206-225).
__global__ void k_upd_xr(Geo g, const int *INDC, const double *PP, const double *AE, const double *R0,
                         double *XW, double *RR, double *rb0, double *rb1, const SolveState *st) {
  if (st->done) return;
  const double alpha = st->alpha, omega = st->omega;
  double s0 = 0.0, s1 = 0.0;
  const long long nrows = (long long)g.NJ * g.NK;
  ROW_LOOP_BEGIN(g)
  const long long c = cid(g, I, J, K);
  if (INDC[c] != -1) {
    XW[c] = XW[c] + (alpha * PP[c] + omega * RR[c]);
    double r = RR[c] - omega * AE[c];
    RR[c] = r;
    s0 = s0 + r * r;
    s1 = s1 + R0[c] * r;
  }
  ROW_LOOP_END
  const long long row = (long long)blockIdx.x * ROWS_PER_BLOCK + (threadIdx.x >> 5);
  row_store(s0, rb0, row, nrows);
  row_store(s1, rb1, row, nrows);
}

// PP = RR + BETA*(PP - OMEGA*AP) (vf_m1bcgs.f:229-238)
__global__ void k_upd_p(Geo g, const int *INDC, const double *RR, const double *AP, double *PP,
                        const SolveState *st) {
  if (st->done) return;
  const double beta = st->beta, omega = st->omega;
  ROW_LOOP_BEGIN(g)
  const long long c = cid(g, I, J, K);
  if (INDC[c] != -1) PP[c] = RR[c] + beta * (PP[c] - omega * AP[c]);
  ROW_LOOP_END
}

// X0 = XW on INDC != -1 when ITER >= 0 (vf_m1bcgs.f:251-261)
__global__ void k_x0(Geo g, const int *INDC, const double *XW, double *X0, const SolveState *st) {
  if (st->iter < 0) return;
  ROW_LOOP_BEGIN(g)
  const long long c = cid(g, I, J, K);
  if (INDC[c] != -1) X0[c] = XW[c];
  ROW_LOOP_END
}

// ||b-Ax||^2 and ||b||^2 row partials (diagnostic of the metric)
__global__ void k_relres(Geo g, SysPtr A_, const int *INDC, const double *X, double *rb0,
                         double *rb1) {
  double s0 = 0.0, s1 = 0.0;
  const long long nrows = (long long)g.NJ * g.NK;
  ROW_LOOP_BEGIN(g)
  const long long c = cid(g, I, J, K);
  if (interior(g, I, J, K) && INDC[c] != -1) {
    double ax = A_.ad[c] * X[c] + A_.ali[c] * X[c - 1] + A_.alj[c] * X[c - g.NI] +
                A_.alk[c] * X[c - (long long)g.NI * g.NJ] + A_.aui[c] * X[c + 1] +
                A_.auj[c] * X[c + g.NI] + A_.auk[c] * X[c + (long long)g.NI * g.NJ];
    double r = A_.bb[c] - ax;
    s0 = s0 + r * r;
    s1 = s1 + A_.bb[c] * A_.bb[c];
  }
  ROW_LOOP_END
  const long long row = (long long)blockIdx.x * ROWS_PER_BLOCK + (threadIdx.x >> 5);
  row_store(s0, rb0, row, nrows);
  row_store(s1, rb1, row, nrows);
}

// ------------------------------------------------------------- finalisers
// One block of 1024 threads: reduce the row partials and advance the
// BiCGSTAB scalars exactly as the host code of vf_m1bcgs.f would.
__global__ void k_fin(int mode, const double *rb0, const double *rb1, long long nrows,
                      SolveState *st, double *out, double epsa2, double epsr2, double div2,
                      int icgmax) {
  if (mode < FIN_ALPHA && mode != FIN_STORE && mode != FIN_RELRES && st->done) return;
  if (mode >= FIN_ALPHA && st->done) return;
  double a = block_final(rb0, nrows);
  double b = (rb1 ? block_final(rb1, nrows) : 0.0);
  if (threadIdx.x != 0) return;
  switch (mode) {
    case FIN_BNORM:
      st->bnorm = a;
      break;
    case FIN_START:  // S=(R0,R0), first convergence test (vf_m1bcgs.f:140-144)
      st->S = a;
      st->xnorm = a;
      st->iter = 0;
      if (st->xnorm <= st->bnorm * epsr2 + epsa2) { st->done = 1; st->status = 0; }
      else {
        st->iter = 1;
        if (st->iter > icgmax) { st->done = 1; }
      }
      break;
    case FIN_ALPHA:
      st->w1 = a;
      st->alpha = st->S / a;
      break;
    case FIN_OMEGA:
      st->w1 = a;
      st->w2 = b;
      st->omega = a / b;
      break;
    case FIN_CONV: {  // vf_m1bcgs.f:218-241
      st->xnorm = a;
      if (st->xnorm <= st->bnorm * epsr2 + epsa2) { st->done = 1; break; }
      if (st->xnorm > div2) { st->iter = -2; st->done = 1; break; }
      double W1 = b;
      st->beta = W1 * st->alpha / (st->S * st->omega);
      st->S = W1;
      st->iter = st->iter + 1;
      if (st->iter > icgmax) st->done = 1;
    } break;
    case FIN_RELRES:
      st->rn = a;
      st->bn = b;
      break;
    case FIN_STORE:
      out[0] = a;
      out[1] = b;
      break;
    default:
      break;
  }
}

// Factorisation failure ends the solve with ITER = -1 (vf_m1bcgs.f:101-102).
__global__ void k_pivot_check(SolveState *st) {
  if (st->pivot_bad) { st->iter = -1; st->done = 1; }
}

// ------------------------------------------------------------- VF_VMODIF
__global__ void k_vmodif(Geo g, Fld f, Prm p, const double *PT) {
  const double *GGV = f.ggv, *GLV = f.glv;
  const int *NF = f.nf;
  const double RT = p.rho0 / p.dtnow;
  ROW_LOOP_BEGIN(g)
  const long long c = cid(g, I, J, K);
  const int NI = g.NI, NJ = g.NJ, NK = g.NK;
  if (K >= 2 && K <= NK - 1 && J >= 2 && J <= NJ - 1 && I >= 2 && A(NF, I - 1, J, K) * NF[c] == 0) {
    int IS = f.indx[c];
    if (IS == 0) {
      double GV = XX_(6, I) * (XX_(2, I) * GGV[c] / GLV[c] + XX_(2, I - 1) * A(GGV, I - 1, J, K) / A(GLV, I - 1, J, K));
      f.uu[c] = f.uu[c] + XX_(5, I) * GV * (PT[c] - A(PT, I - 1, J, K));
    } else if (IS > 0 && indb(f, 3, IS) == 4) {
      if (indb(f, 2, IS) == 1) f.uu[c] = f.uu[c] + 2.0 * XX_(4, I) * GGV[c] / GLV[c] * PT[c];
      else f.uu[c] = f.uu[c] - 2.0 * XX_(4, I - 1) * A(GGV, I - 1, J, K) / A(GLV, I - 1, J, K) * A(PT, I - 1, J, K);
      f.bcu[IS - 1] = f.uu[c];
    }
  }
  if (K >= 2 && K <= NK - 1 && J >= 2 && I >= 2 && I <= NI - 1 && A(NF, I, J - 1, K) * NF[c] == 0) {
    int IS = f.indy[c];
    if (IS == 0) {
      double GV = YY_(6, J) * (YY_(2, J) * GGV[c] / GLV[c] + YY_(2, J - 1) * A(GGV, I, J - 1, K) / A(GLV, I, J - 1, K));
      f.vv[c] = f.vv[c] + YY_(5, J) * GV * (PT[c] - A(PT, I, J - 1, K));
    } else if (IS > 0 && indb(f, 3, IS) == 4) {
      if (indb(f, 2, IS) == 3) f.vv[c] = f.vv[c] + 2.0 * YY_(4, J) * GGV[c] / GLV[c] * PT[c];
      else f.vv[c] = f.vv[c] - 2.0 * YY_(4, J - 1) * A(GGV, I, J - 1, K) / A(GLV, I, J - 1, K) * A(PT, I, J - 1, K);
      f.bcv[IS - 1] = f.vv[c];
    }
  }
  if (K >= 2 && J >= 2 && J <= NJ - 1 && I >= 2 && I <= NI - 1 && A(NF, I, J, K - 1) * NF[c] == 0) {
    int IS = f.indz[c];
    if (IS == 0) {
      double GV = ZZ_(6, K) * (ZZ_(2, K) * GGV[c] / GLV[c] + ZZ_(2, K - 1) * A(GGV, I, J, K - 1) / A(GLV, I, J, K - 1));
      f.ww[c] = f.ww[c] + ZZ_(5, K) * GV * (PT[c] - A(PT, I, J, K - 1));
    } else if (IS > 0 && indb(f, 3, IS) == 4) {
      if (indb(f, 2, IS) == 5) f.ww[c] = f.ww[c] + 2.0 * ZZ_(4, K) * GGV[c] / GLV[c] * PT[c];
      else f.ww[c] = f.ww[c] - 2.0 * ZZ_(4, K - 1) * A(GGV, I, J, K - 1) / A(GLV, I, J, K - 1) * A(PT, I, J, K - 1);
      f.bcw[IS - 1] = f.ww[c];
    }
  }
  if (interior(g, I, J, K) && f.indc[c] != -1) f.pp[c] = f.pp[c] - RT * PT[c];
  ROW_LOOP_END
}

#undef A
#undef XX_
#undef YY_
#undef ZZ_

// ------------------------------------------------------------- launchers
void launch_vpcoef(cudaStream_t s, const Geo &g, const Fld &f, const Prm &p, const SysPtr &a, int *err) {
  k_vpcoef<<<row_blocks(g), ROW_THREADS, 0, s>>>(g, f, p, a, err);
  count_launch();
}
static inline dim3 tile_grid(const Geo &g, int TI, int TJ) {
  return dim3((unsigned)((g.NI - 2 + TI - 1) / TI), (unsigned)((g.NJ - 2 + TJ - 1) / TJ));
}
void launch_dcmp(cudaStream_t s, const Geo &g, int TI, int TJ, double U, const SysPtr &a,
                 const int *indc, double *dd, int *pivot_bad) {
  k_dcmp<<<tile_grid(g, TI, TJ), TI * TJ, 2 * TI * TJ * sizeof(double), s>>>(g, TI, TJ, U, a, indc, dd, pivot_bad);
  count_launch();
}
void launch_fwd(cudaStream_t s, const Geo &g, int TI, int TJ, const SysPtr &a, const int *indc,
                const double *dd, const double *y, const double *spmv_x, double *x, const SolveState *st) {
  k_fwd<<<tile_grid(g, TI, TJ), TI * TJ, 4 * TI * TJ * sizeof(double), s>>>(g, TI, TJ, a, indc, dd, y, spmv_x, x, st);
  count_launch();
}
void launch_bwd(cudaStream_t s, const Geo &g, int TI, int TJ, const SysPtr &a, const int *indc,
                const double *dd, const double *t, double *x, const SolveState *st) {
  k_bwd<<<tile_grid(g, TI, TJ), TI * TJ, 2 * TI * TJ * sizeof(double), s>>>(g, TI, TJ, a, indc, dd, t, x, st);
  count_launch();
}
void launch_spmv(cudaStream_t s, const Geo &g, const SysPtr &a, const int *indc, const double *x, double *y,
                 const SolveState *st) {
  k_spmv<<<row_blocks(g), ROW_THREADS, 0, s>>>(g, a, indc, x, y, st);
  count_launch();
}
void launch_bmy(cudaStream_t s, const Geo &g, const int *indc, const double *b, double *y,
                const SolveState *st) {
  k_bmy<<<row_blocks(g), ROW_THREADS, 0, s>>>(g, indc, b, y, st);
  count_launch();
}
void launch_dot(cudaStream_t s, const Geo &g, const int *indc, const double *x0, const double *y0,
                const double *x1, const double *y1, double *rb0, double *rb1, const SolveState *st) {
  k_dot<<<row_blocks(g), ROW_THREADS, 0, s>>>(g, indc, x0, y0, x1, y1, rb0, rb1, st);
  count_launch();
}
void launch_copy2(cudaStream_t s, const Geo &g, const int *indc, const double *r0, double *rr,
                  double *pp, const SolveState *st) {
  k_copy2<<<row_blocks(g), ROW_THREADS, 0, s>>>(g, indc, r0, rr, pp, st);
  count_launch();
}
void launch_axpy_rr(cudaStream_t s, const Geo &g, const int *indc, const double *ap, double *rr,
                    const SolveState *st) {
  k_axpy_rr<<<row_blocks(g), ROW_THREADS, 0, s>>>(g, indc, ap, rr, st);
  count_launch();
}
void launch_upd_xr(cudaStream_t s, const Geo &g, const int *indc, const double *pp, const double *ae,
                   const double *r0, double *xw, double *rr, double *rb0, double *rb1, const SolveState *st) {
  k_upd_xr<<<row_blocks(g), ROW_THREADS, 0, s>>>(g, indc, pp, ae, r0, xw, rr, rb0, rb1, st);
  count_launch();
}
void launch_upd_p(cudaStream_t s, const Geo &g, const int *indc, const double *rr, const double *ap,
                  double *pp, const SolveState *st) {
  k_upd_p<<<row_blocks(g), ROW_THREADS, 0, s>>>(g, indc, rr, ap, pp, st);
  count_launch();
}
void launch_x0(cudaStream_t s, const Geo &g, const int *indc, const double *xw, double *x0,
               const SolveState *st) {
  k_x0<<<row_blocks(g), ROW_THREADS, 0, s>>>(g, indc, xw, x0, st);
  count_launch();
}
void launch_relres(cudaStream_t s, const Geo &g, const SysPtr &a, const int *indc, const double *x,
                   double *rb0, double *rb1) {
  k_relres<<<row_blocks(g), ROW_THREADS, 0, s>>>(g, a, indc, x, rb0, rb1);
  count_launch();
}
void launch_fin(cudaStream_t s, int mode, const double *rb0, const double *rb1, long long nrows,
                SolveState *st, double *out, double epsa2, double epsr2, double div2, int icgmax) {
  k_fin<<<1, 1024, 0, s>>>(mode, rb0, rb1, nrows, st, out, epsa2, epsr2, div2, icgmax);
  count_launch();
}
void launch_pivot_check(cudaStream_t s, SolveState *st) {
  k_pivot_check<<<1, 1, 0, s>>>(st);
  count_launch();
}
void launch_vmodif(cudaStream_t s, const Geo &g, const Fld &f, const Prm &p, const double *pt) {
  k_vmodif<<<row_blocks(g), ROW_THREADS, 0, s>>>(g, f, p, pt);
  count_launch();
}

}  // namespace cadmas
