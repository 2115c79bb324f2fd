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
#include <algorithm>

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

// ---------------------------------------------------------------------------
// Column prefetch.  Each thread streams its own column through a ring of R
// shared-memory slots with cp.async, D wavefront steps ahead of use, so a
// step only waits for shared memory and one barrier.  Values of the
// neighbouring columns at the same plane are read from the neighbours' ring
// slots: the left/lower neighbour handled plane k one step earlier (slot
// s-1), the right/upper one handles it one step later (slot s+1, prefetched
// long before).  R = D+3: at step s a thread refills slot s+D before the
// step's barrier, while a slower neighbour may still read slot s-2.
__device__ __forceinline__ void cp_async8(void *smem, const void *gmem) {
  unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async4(void *smem, const void *gmem) {
  unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Ring layout in dynamic shared memory: double r[R][NV][T], int ri[R][T],
// then the exchange buffers double xb[2][T].
template <int NV> struct Ring {
  double *r;
  int *ri;
  double *xb;
  int T, R;
  __device__ __forceinline__ double &v(int slot, int q, int t) const { return r[((slot * NV) + q) * T + t]; }
  __device__ __forceinline__ int &ind(int slot, int t) const { return ri[slot * T + t]; }
};
template <int NV> __device__ __forceinline__ Ring<NV> ring_setup(int T, int R) {
  extern __shared__ double sm[];
  Ring<NV> g;
  g.T = T; g.R = R;
  g.r = sm;
  g.xb = sm + (size_t)R * NV * T;
  g.ri = (int *)(g.xb + 2 * T);
  return g;
}
inline size_t ring_bytes(int NV, int T, int R) {
  return (size_t)R * NV * T * sizeof(double) + 2 * (size_t)T * sizeof(double) + (size_t)R * T * sizeof(int);
}

// ----------------------------------------------------- tile-skewed layout
// The MILU kernels visit, at wavefront step s, cell (is+ti, js+tj,
// k = 2+s-ti-tj) with thread t = ti + TI*tj.  The arrays that stay constant
// through a solve (7 coefficients, DD, INDC) and the forward-sweep result
// are stored tile by tile in that visiting order,
//     sl(b, w, t) = (b*W + w)*T + t,   w = (k-2) + ti + tj,
// b = tile index, W = (NK-2) + (TI-1) + (TJ-1), so the T values a block
// needs at one step are contiguous and every load of the sweep coalesces.
__device__ __forceinline__ long long sl_index(const SkewGeo &q, int b, int w, int t) {
  return ((long long)b * q.W + w) * q.T + t;
}

// Copy the Poisson system (7 coefficients) and INDC into the skewed layout.
// Entries outside the tile or the interior get 0 (INDC -1).
__global__ void k_to_skew(Geo g, SkewGeo q, SysPtr A_, const int *INDC, SkewSys S, const double *X0,
                          double *bsl, double *xsl) {
  const long long n = (long long)q.nb * q.W * q.T;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
    const int t = (int)(e % q.T);
    const long long bw = e / q.T;
    const int w = (int)(bw % q.W), b = (int)(bw / q.W);
    const int ti = t % q.TI, tj = t / q.TI;
    const int I = 2 + (b % q.ntx) * q.TI + ti, J = 2 + (b / q.ntx) * q.TJ + tj, k = 2 + w - ti - tj;
    double v[7] = {0, 0, 0, 0, 0, 0, 0}, bv = 0.0, xv = 0.0;
    int ic = -1;
    if (I <= g.NI - 1 && J <= g.NJ - 1 && k >= 2 && k <= g.NK - 1) {
      const long long c = cid(g, I, J, k);
      v[0] = A_.ad[c]; v[1] = A_.ali[c]; v[2] = A_.alj[c]; v[3] = A_.alk[c];
      v[4] = A_.aui[c]; v[5] = A_.auj[c]; v[6] = A_.auk[c];
      ic = INDC[c];
      bv = A_.bb[c];
      xv = X0[c];
    }
    S.ad[e] = v[0]; S.ali[e] = v[1]; S.alj[e] = v[2]; S.alk[e] = v[3];
    S.aui[e] = v[4]; S.auj[e] = v[5]; S.auk[e] = v[6]; S.indc[e] = ic;
    bsl[e] = bv;
    xsl[e] = xv;
  }
}

// Value of a skewed vector at the cell (ti,tj,k) of tile (bx,by), where ti
// and tj may step one past the tile into the neighbouring tile; cells
// outside the interior are the zero ghost layer of the reference vectors.
__device__ __forceinline__ long long skew_nb(const Geo &g, const SkewGeo &q, int bx, int by, int ti, int tj,
                                             int k) {
  if (ti < 0) { bx -= 1; ti += q.TI; } else if (ti >= q.TI) { bx += 1; ti -= q.TI; }
  if (tj < 0) { by -= 1; tj += q.TJ; } else if (tj >= q.TJ) { by += 1; tj -= q.TJ; }
  const int I = 2 + bx * q.TI + ti, J = 2 + by * q.TJ + tj;
  if (bx < 0 || by < 0 || I > g.NI - 1 || J > g.NJ - 1 || k < 2 || k > g.NK - 1) return -1;
  return sl_index(q, bx + q.ntx * by, (k - 2) + ti + tj, ti + q.TI * tj);
}
__device__ __forceinline__ double skew_at(const Geo &g, const SkewGeo &q, const double *X, int bx, int by,
                                          int ti, int tj, int k) {
  const long long e = skew_nb(g, q, bx, by, ti, tj, k);
  return e < 0 ? 0.0 : X[e];
}
// Asynchronous copy of a neighbour value into shared memory (0 for ghosts).
__device__ __forceinline__ void skew_fetch(double *dst, const Geo &g, const SkewGeo &q, const double *X, int bx,
                                           int by, int ti, int tj, int k) {
  const long long e = skew_nb(g, q, bx, by, ti, tj, k);
  if (e < 0) *dst = 0.0;
  else cp_async8(dst, X + e);
}

// ------------------------------------------------------------ VF_MZDCMP
// ring values: 0 AD, 1 ALI, 2 ALJ, 3 ALK, 4 AUI, 5 AUJ, 6 AUK; DD is
// written in the skewed layout.
template <int D>
__global__ void k_dcmp(Geo g, SkewGeo q, double U, SkewSys S, int *pivot_bad) {
  constexpr int NV = 7, R = D + 3;
  const int TI = q.TI, T = q.T;
  Ring<NV> rg = ring_setup<NV>(T, R);
  TileGeo t = tile_geo(g, TI, q.TJ);
  const int tid = threadIdx.x, b = blockIdx.x + q.ntx * blockIdx.y;
  const int nsteps = (g.NK - 2) + (t.wi - 1) + (t.wj - 1);
  auto prefetch = [&](int s) {
    const int k = 2 + s - t.ti - t.tj;
    if (t.valid && k >= 2 && k <= g.NK - 1) {
      const long long e = sl_index(q, b, s, tid);
      const int sl = s % R;
      cp_async8(&rg.v(sl, 0, tid), S.ad + e);  cp_async8(&rg.v(sl, 1, tid), S.ali + e);
      cp_async8(&rg.v(sl, 2, tid), S.alj + e); cp_async8(&rg.v(sl, 3, tid), S.alk + e);
      cp_async8(&rg.v(sl, 4, tid), S.aui + e); cp_async8(&rg.v(sl, 5, tid), S.auj + e);
      cp_async8(&rg.v(sl, 6, tid), S.auk + e); cp_async4(&rg.ind(sl, tid), S.indc + e);
    }
    cp_commit();
  };
#pragma unroll 1
  for (int s = 0; s < D; ++s) prefetch(s);
  double dk1 = 0.0, au3 = 0.0;  // DD(i,j,k-1) and AU3 of (i,j,k-1); k-1 = 1 is the zero ghost layer
  bool bad = false;
  for (int s = 0; s < nsteps; ++s) {
    prefetch(s + D);
    cp_wait<D - 1>();
    __syncthreads();
    const int k = 2 + s - t.ti - t.tj;
    const int sl = s % R, slp = (s + R - 1) % R, cur = s & 1, prv = cur ^ 1;
    if (t.valid && k >= 2 && k <= g.NK - 1) {
      double dd = 0.0;
      if (rg.ind(sl, tid) != -1) {
        double d1 = 0.0, a1, d2 = 0.0, a2;
        if (t.ti > 0) {
          d1 = rg.xb[prv * T + tid - 1];
          a1 = rg.v(slp, 4, tid - 1) + U * (rg.v(slp, 5, tid - 1) + rg.v(slp, 6, tid - 1));
        } else {
          a1 = 0.0 + U * (0.0 + 0.0);
        }
        if (t.tj > 0) {
          d2 = rg.xb[prv * T + tid - TI];
          a2 = rg.v(slp, 5, tid - TI) + U * (rg.v(slp, 4, tid - TI) + rg.v(slp, 6, tid - TI));
        } else {
          a2 = 0.0 + U * (0.0 + 0.0);
        }
        dd = 1.0 / (rg.v(sl, 0, tid) - rg.v(sl, 1, tid) * d1 * a1 - rg.v(sl, 2, tid) * d2 * a2 -
                    rg.v(sl, 3, tid) * dk1 * au3);
        if (dd <= 0.0) bad = true;
      }
      S.dd[sl_index(q, b, s, tid)] = dd;
      rg.xb[cur * T + tid] = dd;
      dk1 = dd;
      au3 = rg.v(sl, 6, tid) + U * (rg.v(sl, 4, tid) + rg.v(sl, 5, tid));
    }
  }
  cp_wait<0>();
  if (bad) atomicOr(pivot_bad, 1);
}

// ------------------------------------------------------- VF_MZFRWD (+MZAX)
// FUSED: the input is Y = A*P computed on the fly (VF_MZAX then VF_MZFRWD).
// Ring values, fused:  0 AD, 1 ALI, 2 ALJ, 3 ALK, 4 AUI, 5 AUJ, 6 AUK, 7 DD
//                      (skewed), 8 P, 9 P(i-1), 10 P(i+1), 11 P(j-1),
//                      12 P(j+1) (P in the standard layout; 9..12 only on
//                      tile-edge threads)
// Ring values, plain:  0 Y (standard layout), 1 ALI, 2 ALJ, 3 ALK, 4 DD
// The result is written in the skewed layout for k_bwd.
template <int D, bool FUSED>
__global__ void k_fwd(Geo g, SkewGeo q, SkewSys S, const double *y, const double *P, double *Tout,
                      const SolveState *st) {
  if (st && st->done) return;
  constexpr int NV = FUSED ? 13 : 5, R = D + 3;
  constexpr int QDD = FUSED ? 7 : 4;
  const int TI = q.TI, T = q.T;
  Ring<NV> rg = ring_setup<NV>(T, R);
  TileGeo t = tile_geo(g, TI, q.TJ);
  const int tid = threadIdx.x, b = blockIdx.x + q.ntx * blockIdx.y;
  const int bx = blockIdx.x, by = blockIdx.y;
  const int nsteps = (g.NK - 2) + (t.wi - 1) + (t.wj - 1);
  const bool ex0 = (t.ti == 0), ex1 = (t.ti == t.wi - 1), ey0 = (t.tj == 0), ey1 = (t.tj == t.wj - 1);
  auto prefetch = [&](int s) {
    const int k = 2 + s - t.ti - t.tj;
    if (t.valid && k >= 2 && k <= g.NK - 1) {
      const long long e = sl_index(q, b, s, tid);
      const int sl = s % R;
      if (FUSED) {
        cp_async8(&rg.v(sl, 0, tid), S.ad + e);  cp_async8(&rg.v(sl, 1, tid), S.ali + e);
        cp_async8(&rg.v(sl, 2, tid), S.alj + e); cp_async8(&rg.v(sl, 3, tid), S.alk + e);
        cp_async8(&rg.v(sl, 4, tid), S.aui + e); cp_async8(&rg.v(sl, 5, tid), S.auj + e);
        cp_async8(&rg.v(sl, 6, tid), S.auk + e); cp_async8(&rg.v(sl, 7, tid), S.dd + e);
        cp_async8(&rg.v(sl, 8, tid), P + e);
        // values of the neighbouring tiles (or the zero ghost layer)
        if (ex0) skew_fetch(&rg.v(sl, 9, tid), g, q, P, bx, by, t.ti - 1, t.tj, k);
        if (ex1) skew_fetch(&rg.v(sl, 10, tid), g, q, P, bx, by, t.ti + 1, t.tj, k);
        if (ey0) skew_fetch(&rg.v(sl, 11, tid), g, q, P, bx, by, t.ti, t.tj - 1, k);
        if (ey1) skew_fetch(&rg.v(sl, 12, tid), g, q, P, bx, by, t.ti, t.tj + 1, k);
      } else {
        cp_async8(&rg.v(sl, 0, tid), y + e);      cp_async8(&rg.v(sl, 1, tid), S.ali + e);
        cp_async8(&rg.v(sl, 2, tid), S.alj + e);  cp_async8(&rg.v(sl, 3, tid), S.alk + e);
        cp_async8(&rg.v(sl, 4, tid), S.dd + e);
      }
      cp_async4(&rg.ind(sl, tid), S.indc + e);
    }
    cp_commit();
  };
#pragma unroll 1
  for (int s = 0; s < D; ++s) prefetch(s);
  double xk1 = 0.0, dk1 = 0.0;  // X and DD at (i,j,k-1); k-1 = 1 is the zero ghost layer
  for (int s = 0; s < nsteps; ++s) {
    prefetch(s + D);
    cp_wait<D - 1>();
    __syncthreads();
    const int k = 2 + s - t.ti - t.tj;
    const int sl = s % R, slp = (s + R - 1) % R, sln = (s + 1) % R, cur = s & 1, prv = cur ^ 1;
    if (t.valid && k >= 2 && k <= g.NK - 1) {
      double x = 0.0;
      const double d = rg.v(sl, QDD, tid);
      if (rg.ind(sl, tid) != -1) {
        double yv;
        if (FUSED) {
          const double pc = rg.v(sl, 8, tid);
          const double pxm = ex0 ? rg.v(sl, 9, tid) : rg.v(slp, 8, tid - 1);
          const double pym = ey0 ? rg.v(sl, 11, tid) : rg.v(slp, 8, tid - TI);
          const double pzm = (k > 2) ? rg.v(slp, 8, tid) : 0.0;
          const double pxp = ex1 ? rg.v(sl, 10, tid) : rg.v(sln, 8, tid + 1);
          const double pyp = ey1 ? rg.v(sl, 12, tid) : rg.v(sln, 8, tid + TI);
          const double pzp = (k < g.NK - 1) ? rg.v(sln, 8, tid) : 0.0;
          yv = rg.v(sl, 0, tid) * pc + rg.v(sl, 1, tid) * pxm + rg.v(sl, 2, tid) * pym +
               rg.v(sl, 3, tid) * pzm + rg.v(sl, 4, tid) * pxp + rg.v(sl, 5, tid) * pyp +
               rg.v(sl, 6, tid) * pzp;
        } else {
          yv = rg.v(sl, 0, tid);
        }
        double d1 = 0.0, x1 = 0.0, d2 = 0.0, x2 = 0.0;
        if (t.ti > 0) { d1 = rg.v(slp, QDD, tid - 1); x1 = rg.xb[prv * T + tid - 1]; }
        if (t.tj > 0) { d2 = rg.v(slp, QDD, tid - TI); x2 = rg.xb[prv * T + tid - TI]; }
        x = yv - rg.v(sl, 1, tid) * d1 * x1 - rg.v(sl, 2, tid) * d2 * x2 - rg.v(sl, 3, tid) * dk1 * xk1;
      }
      Tout[sl_index(q, b, s, tid)] = x;
      rg.xb[cur * T + tid] = x;
      xk1 = x;
      dk1 = d;
    }
  }
  cp_wait<0>();
}

// ------------------------------------------------------------ VF_MZBKWD
// ring values: 0 T, 1 AUI, 2 AUJ, 3 AUK, 4 DD (all skewed); reversed loop
// order; X written in the standard layout.
template <int D>
__global__ void k_bwd(Geo g, SkewGeo q, SkewSys S, const double *Tin, double *X, const SolveState *st) {
  if (st && st->done) return;
  constexpr int NV = 5, R = D + 3;
  const int TI = q.TI, T = q.T;
  Ring<NV> rg = ring_setup<NV>(T, R);
  TileGeo t = tile_geo(g, TI, q.TJ);
  const int I = t.is + t.ti, J = t.js + t.tj, tid = threadIdx.x, b = blockIdx.x + q.ntx * blockIdx.y;
  const int ri = t.wi - 1 - t.ti, rj = t.wj - 1 - t.tj;  // distance from the far corner
  const int nsteps = (g.NK - 2) + (t.wi - 1) + (t.wj - 1);
  auto prefetch = [&](int s) {
    const int k = (g.NK - 1) - (s - ri - rj);
    if (t.valid && k >= 2 && k <= g.NK - 1) {
      const long long e = sl_index(q, b, (k - 2) + t.ti + t.tj, tid);
      const int sl = s % R;
      cp_async8(&rg.v(sl, 0, tid), Tin + e);      cp_async8(&rg.v(sl, 1, tid), S.aui + e);
      cp_async8(&rg.v(sl, 2, tid), S.auj + e);    cp_async8(&rg.v(sl, 3, tid), S.auk + e);
      cp_async8(&rg.v(sl, 4, tid), S.dd + e);     cp_async4(&rg.ind(sl, tid), S.indc + e);
    }
    cp_commit();
  };
#pragma unroll 1
  for (int s = 0; s < D; ++s) prefetch(s);
  double xk1 = 0.0;  // X(i,j,k+1); k+1 = NK is the zero ghost layer
  for (int s = 0; s < nsteps; ++s) {
    prefetch(s + D);
    cp_wait<D - 1>();
    __syncthreads();
    const int k = (g.NK - 1) - (s - ri - rj);
    const int sl = s % R, cur = s & 1, prv = cur ^ 1;
    if (t.valid && k >= 2 && k <= g.NK - 1) {
      double x = 0.0;
      if (rg.ind(sl, tid) != -1) {
        const double x1 = (ri > 0) ? rg.xb[prv * T + tid + 1] : 0.0;
        const double x2 = (rj > 0) ? rg.xb[prv * T + tid + TI] : 0.0;
        x = (rg.v(sl, 0, tid) - rg.v(sl, 1, tid) * x1 - rg.v(sl, 2, tid) * x2 - rg.v(sl, 3, tid) * xk1) *
            rg.v(sl, 4, tid);
      }
      X[sl_index(q, b, (k - 2) + t.ti + t.tj, tid)] = x;
      rg.xb[cur * T + tid] = x;
      xk1 = x;
    }
  }
  cp_wait<0>();
  (void)I; (void)J;
}

// ------------------------------------------------------------ slab kernels
// The BiCGSTAB vectors live in the skewed layout; a vector kernel maps one
// warp to one slab (b,w) of T entries and lets lane l visit t = l, l+32, ...
// The dot products (VF_MZIP) sum in that order: lane partials, warp tree
// per slab, then the 1024-thread tree over the slab partials (block_final).
// Padding entries carry INDC = -1 and are skipped like non-computed cells.
#define SLAB_LOOP_BEGIN(q)                                                          \
  const int lane_ = threadIdx.x & 31;                                               \
  const long long slab_ = (long long)blockIdx.x * ROWS_PER_BLOCK + (threadIdx.x >> 5); \
  if (slab_ < (long long)(q).nb * (q).W) {                                          \
    for (int t_ = lane_; t_ < (q).T; t_ += 32) {                                    \
      const long long e = slab_ * (q).T + t_;
#define SLAB_LOOP_END \
    }                 \
  }
#define SLAB_ROW ((long long)blockIdx.x * ROWS_PER_BLOCK + (threadIdx.x >> 5))

__device__ __forceinline__ bool interior(const Geo &g, int I, int J, int K) {
  return I >= 2 && I <= g.NI - 1 && J >= 2 && J <= g.NJ - 1 && K >= 2 && K <= g.NK - 1;
}

// A*X at skewed entry e (VF_MZAX expression, vf_mzax.f:46-53).
__device__ __forceinline__ double skew_ax(const Geo &g, const SkewGeo &q, const SkewSys &S, const double *X,
                                          long long e) {
  const int t = (int)(e % q.T);
  const long long bw = e / q.T;
  const int w = (int)(bw % q.W), b = (int)(bw / q.W);
  const int ti = t % q.TI, tj = t / q.TI, bx = b % q.ntx, by = b / q.ntx, k = 2 + w - ti - tj;
  return S.ad[e] * X[e] + S.ali[e] * skew_at(g, q, X, bx, by, ti - 1, tj, k) +
         S.alj[e] * skew_at(g, q, X, bx, by, ti, tj - 1, k) + S.alk[e] * skew_at(g, q, X, bx, by, ti, tj, k - 1) +
         S.aui[e] * skew_at(g, q, X, bx, by, ti + 1, tj, k) + S.auj[e] * skew_at(g, q, X, bx, by, ti, tj + 1, k) +
         S.auk[e] * skew_at(g, q, X, bx, by, ti, tj, k + 1);
}

// Y = A X on INDC != -1 (VF_MZAX); Y untouched elsewhere.
__global__ void k_spmv(Geo g, SkewGeo q, SkewSys S, const double *X, double *Y, const SolveState *st) {
  if (st && st->done) return;
  SLAB_LOOP_BEGIN(q)
  if (S.indc[e] != -1) Y[e] = skew_ax(g, q, S, X, e);
  SLAB_LOOP_END
}

// Y = B - Y on INDC != -1 (vf_m1bcgs.f:124-132)
__global__ void k_bmy(SkewGeo q, const int *INDC, const double *B, double *Y, const SolveState *st) {
  if (st->done) return;
  SLAB_LOOP_BEGIN(q)
  if (INDC[e] != -1) Y[e] = B[e] - Y[e];
  SLAB_LOOP_END
}

// Slab partials of up to two dot products (VF_MZIP).
__global__ void k_dot(SkewGeo q, const int *INDC, const double *x0, const double *y0, const double *x1,
                      const double *y1, double *rb0, double *rb1, const SolveState *st) {
  if (st && st->done) return;
  double s0 = 0.0, s1 = 0.0;
  const long long nslab = (long long)q.nb * q.W;
  SLAB_LOOP_BEGIN(q)
  if (INDC[e] != -1) {
    s0 = s0 + x0[e] * y0[e];
    if (x1) s1 = s1 + x1[e] * y1[e];
  }
  SLAB_LOOP_END
  row_store(s0, rb0, SLAB_ROW, nslab);
  if (x1) row_store(s1, rb1, SLAB_ROW, nslab);
}

// RR = R0, PP = R0
__global__ void k_copy2(SkewGeo q, const int *INDC, const double *R0, double *RR, double *PP,
                        const SolveState *st) {
  if (st->done) return;
  SLAB_LOOP_BEGIN(q)
  if (INDC[e] != -1) { RR[e] = R0[e]; PP[e] = R0[e]; }
  SLAB_LOOP_END
}

// RR = RR - ALPHA*AP (vf_m1bcgs.f:181-189)
__global__ void k_axpy_rr(SkewGeo q, const int *INDC, const double *AP, double *RR, const SolveState *st) {
  if (st->done) return;
  const double alpha = st->alpha;
  SLAB_LOOP_BEGIN(q)
  if (INDC[e] != -1) RR[e] = RR[e] - alpha * AP[e];
  SLAB_LOOP_END
}

// XW = XW + (ALPHA*PP + OMEGA*RR); RR = RR - OMEGA*AE; slab partials of
// (RR,RR) and (R0,RR) on the updated RR (vf_m1bcgs.f:206-225).
__global__ void k_upd_xr(SkewGeo q, const int *INDC, const double *PP, const double *AE, const double *R0,
                         double *XW, double *RR, double *rb0, double *rb1, const SolveState *st) {
  if (st->done) return;
  const double alpha = st->alpha, omega = st->omega;
  double s0 = 0.0, s1 = 0.0;
  const long long nslab = (long long)q.nb * q.W;
  SLAB_LOOP_BEGIN(q)
  if (INDC[e] != -1) {
    XW[e] = XW[e] + (alpha * PP[e] + omega * RR[e]);
    double r = RR[e] - omega * AE[e];
    RR[e] = r;
    s0 = s0 + r * r;
    s1 = s1 + R0[e] * r;
  }
  SLAB_LOOP_END
  row_store(s0, rb0, SLAB_ROW, nslab);
  row_store(s1, rb1, SLAB_ROW, nslab);
}

// PP = RR + BETA*(PP - OMEGA*AP) (vf_m1bcgs.f:229-238)
__global__ void k_upd_p(SkewGeo q, const int *INDC, const double *RR, const double *AP, double *PP,
                        const SolveState *st) {
  if (st->done) return;
  const double beta = st->beta, omega = st->omega;
  SLAB_LOOP_BEGIN(q)
  if (INDC[e] != -1) PP[e] = RR[e] + beta * (PP[e] - omega * AP[e]);
  SLAB_LOOP_END
}

// X0 = XW on INDC != -1 when ITER >= 0 (vf_m1bcgs.f:251-261), back to the
// standard layout.
__global__ void k_x0(Geo g, SkewGeo q, const int *INDC, const double *XW, double *X0, const SolveState *st) {
  if (st->iter < 0) return;
  SLAB_LOOP_BEGIN(q)
  if (INDC[e] != -1) {
    const int ti = t_ % q.TI, tj = t_ / q.TI;
    const int w = (int)(slab_ % q.W), b = (int)(slab_ / q.W);
    const int I = 2 + (b % q.ntx) * q.TI + ti, J = 2 + (b / q.ntx) * q.TJ + tj, k = 2 + w - ti - tj;
    X0[cid(g, I, J, k)] = XW[e];
  }
  SLAB_LOOP_END
}

// ||b-Ax||^2 and ||b||^2 slab partials (diagnostic of the metric)
__global__ void k_relres(Geo g, SkewGeo q, SkewSys S, const double *B, const double *X, double *rb0,
                         double *rb1) {
  double s0 = 0.0, s1 = 0.0;
  const long long nslab = (long long)q.nb * q.W;
  SLAB_LOOP_BEGIN(q)
  if (S.indc[e] != -1) {
    double r = B[e] - skew_ax(g, q, S, X, e);
    s0 = s0 + r * r;
    s1 = s1 + B[e] * B[e];
  }
  SLAB_LOOP_END
  row_store(s0, rb0, SLAB_ROW, nslab);
  row_store(s1, rb1, SLAB_ROW, nslab);
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
// Prefetch depth: the largest of 8, 4, 2, 1 whose ring fits the shared
// memory a block may use (200 KB here).
static int ring_depth(int NV, int T) {
  const size_t cap = 200 * 1024;
  for (int d : {8, 4, 2, 1})
    if (ring_bytes(NV, T, d + 3) <= cap) return d;
  return 0;
}
template <class K> static void set_smem(K kern, size_t bytes) {
  cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

static inline dim3 skew_grid(const SkewGeo &q) { return dim3((unsigned)q.ntx, (unsigned)(q.nb / q.ntx)); }
#define RING_LAUNCH2(KER, NV, ...)                                                             \
  do {                                                                                        \
    const int T_ = q.T, d_ = ring_depth(NV, T_);                                              \
    const size_t b_ = ring_bytes(NV, T_, d_ + 3);                                             \
    switch (d_) {                                                                             \
      case 8: set_smem(KER<8 RING_EXTRA>, b_); KER<8 RING_EXTRA><<<skew_grid(q), T_, b_, s>>>(__VA_ARGS__); break; \
      case 4: set_smem(KER<4 RING_EXTRA>, b_); KER<4 RING_EXTRA><<<skew_grid(q), T_, b_, s>>>(__VA_ARGS__); break; \
      case 2: set_smem(KER<2 RING_EXTRA>, b_); KER<2 RING_EXTRA><<<skew_grid(q), T_, b_, s>>>(__VA_ARGS__); break; \
      default: set_smem(KER<1 RING_EXTRA>, b_); KER<1 RING_EXTRA><<<skew_grid(q), T_, b_, s>>>(__VA_ARGS__); break; \
    }                                                                                         \
    count_launch();                                                                           \
  } while (0)

void launch_to_skew(cudaStream_t s, const Geo &g, const SkewGeo &q, const SysPtr &a, const int *indc,
                    const SkewSys &S, const double *x0, double *bsl, double *xsl) {
  const long long n = (long long)q.nb * q.W * q.T;
  const int blocks = (int)std::min<long long>((n + 255) / 256, 148LL * 16);
  k_to_skew<<<blocks, 256, 0, s>>>(g, q, a, indc, S, x0, bsl, xsl);
  count_launch();
}
void launch_dcmp(cudaStream_t s, const Geo &g, const SkewGeo &q, double U, const SkewSys &S, int *pivot_bad) {
#define RING_EXTRA
  RING_LAUNCH2(k_dcmp, 7, g, q, U, S, pivot_bad);
#undef RING_EXTRA
}
void launch_fwd(cudaStream_t s, const Geo &g, const SkewGeo &q, const SkewSys &S, const double *y,
                const double *spmv_x, double *tout, const SolveState *st, double *ybuf) {
  if (spmv_x && ring_depth(13, q.T) == 0) {
    // Ring of the fused kernel too large for this tile: SpMV first.
    launch_spmv(s, g, q, S, spmv_x, ybuf, st);
    y = ybuf;
    spmv_x = nullptr;
  }
  if (spmv_x) {
#define RING_EXTRA , true
    RING_LAUNCH2(k_fwd, 13, g, q, S, y, spmv_x, tout, st);
#undef RING_EXTRA
  } else {
#define RING_EXTRA , false
    RING_LAUNCH2(k_fwd, 5, g, q, S, y, spmv_x, tout, st);
#undef RING_EXTRA
  }
}
void launch_bwd(cudaStream_t s, const Geo &g, const SkewGeo &q, const SkewSys &S, const double *tin,
                double *x, const SolveState *st) {
#define RING_EXTRA
  RING_LAUNCH2(k_bwd, 5, g, q, S, tin, x, st);
#undef RING_EXTRA
}
static inline unsigned slab_blocks(const SkewGeo &q) {
  return (unsigned)(((long long)q.nb * q.W + ROWS_PER_BLOCK - 1) / ROWS_PER_BLOCK);
}
#define SL(kern, ...) (kern<<<slab_blocks(q), ROW_THREADS, 0, s>>>(__VA_ARGS__), count_launch())
void launch_spmv(cudaStream_t s, const Geo &g, const SkewGeo &q, const SkewSys &S, const double *x, double *y,
                 const SolveState *st) { SL(k_spmv, g, q, S, x, y, st); }
void launch_bmy(cudaStream_t s, const SkewGeo &q, const int *indc, const double *b, double *y,
                const SolveState *st) { SL(k_bmy, q, indc, b, y, st); }
void launch_dot(cudaStream_t s, const SkewGeo &q, const int *indc, const double *x0, const double *y0,
                const double *x1, const double *y1, double *rb0, double *rb1, const SolveState *st) {
  SL(k_dot, q, indc, x0, y0, x1, y1, rb0, rb1, st);
}
void launch_copy2(cudaStream_t s, const SkewGeo &q, const int *indc, const double *r0, double *rr, double *pp,
                  const SolveState *st) { SL(k_copy2, q, indc, r0, rr, pp, st); }
void launch_axpy_rr(cudaStream_t s, const SkewGeo &q, const int *indc, const double *ap, double *rr,
                    const SolveState *st) { SL(k_axpy_rr, q, indc, ap, rr, st); }
void launch_upd_xr(cudaStream_t s, const SkewGeo &q, const int *indc, const double *pp, const double *ae,
                   const double *r0, double *xw, double *rr, double *rb0, double *rb1, const SolveState *st) {
  SL(k_upd_xr, q, indc, pp, ae, r0, xw, rr, rb0, rb1, st);
}
void launch_upd_p(cudaStream_t s, const SkewGeo &q, const int *indc, const double *rr, const double *ap,
                  double *pp, const SolveState *st) { SL(k_upd_p, q, indc, rr, ap, pp, st); }
void launch_x0(cudaStream_t s, const Geo &g, const SkewGeo &q, const int *indc, const double *xw, double *x0,
               const SolveState *st) { SL(k_x0, g, q, indc, xw, x0, st); }
void launch_relres(cudaStream_t s, const Geo &g, const SkewGeo &q, const SkewSys &S, const double *b,
                   const double *x, double *rb0, double *rb1) { SL(k_relres, g, q, S, b, x, rb0, rb1); }
#undef SL
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
