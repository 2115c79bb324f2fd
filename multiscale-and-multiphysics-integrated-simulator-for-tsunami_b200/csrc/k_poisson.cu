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
#include <mutex>
#include "cadmas_dev.cuh"
#include "kernels.h"
#include <algorithm>

namespace cadmas {

#define A(a, i, j, k) a[cid(g, i, j, k)]
#define XX_(m, i) gx(g, m, i)
#define YY_(m, j) gy(g, m, j)
#define ZZ_(m, k) gz(g, m, k)

// ------------------------------------------------------------- VF_VPCOEF
__global__ void __launch_bounds__(ROW_THREADS, 3) k_vpcoef(Geo g, Fld f, Prm p, SysPtr A_, int *err) {
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
      if (indb(f, 3, IS) == 4 || (indb(f, 3, IS) == 5 && I == 2 && p.fixlvl[0]))  // vf_vpcoef.f:158-175
        AIM = 2.0 * AYZ * XX_(4, I) * f.ggx[c] * GGV[c] / GLV[c];
      else AIM = 0.0;
    } else { AIM = 0.0; atomicOr(err, ERR_PG); }
    IS = A(f.indx, IP, J, K);
    if (IS == 0) {
      GV = XX_(6, IP) * (XX_(2, IP) * A(GGV, IP, J, K) / A(GLV, IP, J, K) + XX_(2, I) * GGV[c] / GLV[c]);
      AIP = AYZ * XX_(5, IP) * A(f.ggx, IP, J, K) * GV; AUI = -AIP;
    } else if (IS >= 1) {
      if (indb(f, 3, IS) == 4 || (indb(f, 3, IS) == 5 && IP == g.NI && p.fixlvl[1]))
        AIP = 2.0 * AYZ * XX_(4, I) * A(f.ggx, IP, J, K) * GGV[c] / GLV[c];
      else AIP = 0.0;
    } else { AIP = 0.0; atomicOr(err, ERR_PG); }
    IS = f.indy[c];
    if (IS == 0) {
      GV = YY_(6, J) * (YY_(2, J) * GGV[c] / GLV[c] + YY_(2, JM) * A(GGV, I, JM, K) / A(GLV, I, JM, K));
      AJM = AXZ * YY_(5, J) * f.ggy[c] * GV; ALJ = -AJM;
    } else if (IS >= 1) {
      if (indb(f, 3, IS) == 4 || (indb(f, 3, IS) == 5 && J == 2 && p.fixlvl[2]))
        AJM = 2.0 * AXZ * YY_(4, J) * f.ggy[c] * GGV[c] / GLV[c];
      else AJM = 0.0;
    } else { AJM = 0.0; atomicOr(err, ERR_PG); }
    IS = A(f.indy, I, JP, K);
    if (IS == 0) {
      GV = YY_(6, JP) * (YY_(2, JP) * A(GGV, I, JP, K) / A(GLV, I, JP, K) + YY_(2, J) * GGV[c] / GLV[c]);
      AJP = AXZ * YY_(5, JP) * A(f.ggy, I, JP, K) * GV; AUJ = -AJP;
    } else if (IS >= 1) {
      if (indb(f, 3, IS) == 4 || (indb(f, 3, IS) == 5 && JP == g.NJ && p.fixlvl[3]))
        AJP = 2.0 * AXZ * YY_(4, J) * A(f.ggy, I, JP, K) * GGV[c] / GLV[c];
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
    // wave source line (vf_vpcoef.f:349-350)
    if (p.iws == I) VQ = 2.0 * ZZ_(2, K) * f.srcuv[(J - 1) + (long long)g.NJ * (K - 1)] * YY_(2, J);
    if (p.jws == J) VQ = 2.0 * ZZ_(2, K) * f.srcuv[(I - 1) + (long long)g.NI * (K - 1)] * XX_(2, I);
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
__device__ __forceinline__ TileGeo tile_geo(const Geo &g, const SkewGeo &q, int bx, int by) {
  TileGeo t;
  t.is = 2 + bx * q.TI;
  t.js = 2 + by * q.TJ;
  t.wi = min(q.TI, g.NI - t.is);  // interior cells is..NI-1
  t.wj = min(q.TJ, g.NJ - t.js);
  t.ti = threadIdx.x % q.TIp;
  t.tj = threadIdx.x / q.TIp;
  t.valid = (t.ti < t.wi) && (t.tj < t.wj);  // also false on the padding column ti = TI
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

template <typename V> __device__ __forceinline__ void cp_async_v(V *smem, const V *gmem) {
  if (sizeof(V) == 8) cp_async8(smem, gmem);
  else cp_async4(smem, gmem);
}

// Ring layout in dynamic shared memory: V r[R][NV][T], then the exchange
// buffers V xb[2][T], then int ri[R][T].
template <int NV, typename V> struct Ring {
  V *r;
  int *ri;
  V *xb;
  int T, R;
  __device__ __forceinline__ V &v(int slot, int q, int t) const { return r[((slot * NV) + q) * T + t]; }
  __device__ __forceinline__ int &ind(int slot, int t) const { return ri[slot * T + t]; }
};
template <int NV, typename V> __device__ __forceinline__ Ring<NV, V> ring_setup(int T, int R) {
  extern __shared__ __align__(16) double sm[];
  Ring<NV, V> g;
  g.T = T; g.R = R;
  g.r = reinterpret_cast<V *>(sm);
  g.xb = g.r + (size_t)R * NV * T;
  g.ri = (int *)(g.xb + 2 * T);
  return g;
}
inline size_t ring_bytes(int NV, int T, int R, size_t es = sizeof(double)) {
  return (size_t)R * NV * T * es + 2 * (size_t)T * es + (size_t)R * T * sizeof(int);
}

// ----------------------------------------------------- tile-skewed layout
// The MILU kernels visit, at wavefront step s, cell (is+ti, js+tj,
// k = 2+s-ti-tj) with thread t = ti + TIp*tj.  The arrays that stay constant
// through a solve (7 coefficients, DD, INDC), the right-hand side and the
// BiCGSTAB vectors are stored tile by tile in that visiting order,
//     sl(b, w, t) = (b*W + w)*T + t,   w = (k-2) + ti + tj,
// b = tile index, W = (NK-2) + (TI-1) + (TJ-1), so the T values a block
// needs at one step are contiguous and every load of the sweep coalesces.
__device__ __forceinline__ long long sl_index(const SkewGeo &q, int b, int w, int t) {
  return ((long long)b * q.W + w) * q.T + t;
}

// Copy the Poisson system (7 coefficients, interleaved per slab; DD set to
// 0 for MZDCMP to fill), INDC, BB and X0 into the skewed layout.  Entries
// outside the tile or the interior get 0 (INDC -1).  warm: keep the
// previous solution already in xsl as the initial guess (0 where INDC is
// now -1) instead of X0.
__device__ __forceinline__ void to_skew_elem(const Geo &g, const SkewGeo &q, const SysPtr &A_, const int *INDC,
                                             const SkewSys &S, const double *X0, double *bsl, double *xsl, int warm,
                                             long long e) {
  {
    const int t = (int)(e % q.T);
    const long long bw = e / q.T;
    const int w = (int)(bw % q.W), b = (int)(bw / q.W);
    const int ti = t % q.TIp, tj = t / q.TIp;
    const int I = 2 + (b % q.ntx) * q.TI + ti, J = 2 + (b / q.ntx) * q.TJ + tj, k = 2 + w - ti - tj;
    double v[7] = {0, 0, 0, 0, 0, 0, 0}, bv = 0.0, xv = 0.0;
    int ic = -1;
    if (ti < q.TI && I <= g.NI - 1 && J <= g.NJ - 1 && k >= 2 && k <= g.NK - 1) {
      const long long c = cid(g, I, J, k);
      v[0] = A_.ad[c]; v[1] = A_.ali[c]; v[2] = A_.alj[c]; v[3] = A_.alk[c];
      v[4] = A_.aui[c]; v[5] = A_.auj[c]; v[6] = A_.auk[c];
      ic = INDC[c];
      bv = A_.bb[c];
      xv = warm ? (ic != -1 ? xsl[e] : 0.0) : X0[c];
    }
    constexpr int cs[7] = {SYS_AD, SYS_ALI, SYS_ALJ, SYS_ALK, SYS_AUI, SYS_AUJ, SYS_AUK};
#pragma unroll
    for (int c = 0; c < 7; ++c) S.sys[sys_at(bw, cs[c], q.T, t)] = v[c];
    S.sys[sys_at(bw, SYS_DD, q.T, t)] = 0.0;
    S.sys[sys_at(bw, SYS_T, q.T, t)] = 0.0;
    S.indc[e] = ic;
    bsl[e] = bv;
    xsl[e] = xv;
  }
}
__global__ void k_to_skew(Geo g, SkewGeo q, SysPtr A_, const int *INDC, SkewSys S, const double *X0,
                          double *bsl, double *xsl, int warm) {
  pdl_enter();
  const long long n = (long long)q.nb * q.W * q.T;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x)
    to_skew_elem(g, q, A_, INDC, S, X0, bsl, xsl, warm, e);
}

// The same conversion, one block per row tj of a layout tile b: the row's
// interior cells of all layers, (NK-2) x TI values of one array at a time,
// are staged in shared memory with coalesced loads and then written slab
// by slab (TIp consecutive entries of a slab per row).  Same values as
// to_skew_elem; used when a panel fits in shared memory.
__global__ void k_to_skew_rows(Geo g, SkewGeo q, SysPtr A_, const int *INDC, SkewSys S, const double *X0,
                               double *bsl, double *xsl, int warm) {
  extern __shared__ __align__(16) double pan[];  // [(NK-2) * TI]
  pdl_enter();
  const int b = blockIdx.x / q.TJ, tj = blockIdx.x % q.TJ;
  const int TI = q.TI, TIp = q.TIp, T = q.T, W = q.W, nk = g.NK - 2;
  const int is = 2 + (b % q.ntx) * TI, J = 2 + (b / q.ntx) * q.TJ + tj;
  const int wi = (J <= g.NJ - 1) ? min(TI, g.NI - is) : 0;  // columns of the row inside the interior
  const int npan = nk * TI, nent = W * TIp;
  const long long slab0 = (long long)b * W;
  int *ipan = reinterpret_cast<int *>(pan);
  // INDC, then DD = T = 0, INDC and the warm guess
#pragma unroll 4
  for (int x = threadIdx.x; x < npan; x += blockDim.x) {
    const int k = 2 + x / TI, ti = x % TI;
    ipan[x] = ti < wi ? INDC[cid(g, is + ti, J, k)] : -1;
  }
  __syncthreads();
  for (int x = threadIdx.x; x < nent; x += blockDim.x) {
    const int w = x / TIp, ti = x % TIp, k = 2 + w - ti - tj, t = ti + TIp * tj;
    const int ic = (ti < TI && k >= 2 && k <= g.NK - 1) ? ipan[(k - 2) * TI + ti] : -1;
    const long long e = (slab0 + w) * T + t;
    S.indc[e] = ic;
    S.sys[sys_at(slab0 + w, SYS_DD, T, t)] = 0.0;
    S.sys[sys_at(slab0 + w, SYS_T, T, t)] = 0.0;
    if (warm) xsl[e] = ic != -1 ? xsl[e] : 0.0;
  }
  // AD, ALI, ALJ, ALK, AUI, AUJ, AUK, BB and (not warm) X0
  const double *src[9] = {A_.ad, A_.ali, A_.alj, A_.alk, A_.aui, A_.auj, A_.auk, A_.bb, X0};
  constexpr int cs[7] = {SYS_AD, SYS_ALI, SYS_ALJ, SYS_ALK, SYS_AUI, SYS_AUJ, SYS_AUK};
  const int na = warm ? 8 : 9;
#pragma unroll 1
  for (int a = 0; a < na; ++a) {
    __syncthreads();
    const double *sa = src[a];
#pragma unroll 4
    for (int x = threadIdx.x; x < npan; x += blockDim.x) {
      const int k = 2 + x / TI, ti = x % TI;
      pan[x] = ti < wi ? sa[cid(g, is + ti, J, k)] : 0.0;
    }
    __syncthreads();
    for (int x = threadIdx.x; x < nent; x += blockDim.x) {
      const int w = x / TIp, ti = x % TIp, k = 2 + w - ti - tj, t = ti + TIp * tj;
      const double v = (ti < TI && k >= 2 && k <= g.NK - 1) ? pan[(k - 2) * TI + ti] : 0.0;
      if (a < 7) S.sys[sys_at(slab0 + w, cs[a], T, t)] = v;
      else if (a == 7) bsl[(slab0 + w) * T + t] = v;
      else xsl[(slab0 + w) * T + t] = v;
    }
  }
}
// Shared memory of k_to_skew_rows (0: the panel does not fit, k_to_skew).
static size_t to_skew_rows_bytes(const Geo &g, const SkewGeo &q) {
  const size_t b = (size_t)(g.NK - 2) * q.TI * sizeof(double);
  return b <= 64 * 1024 ? b : 0;
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
  return sl_index(q, bx + q.ntx * by, (k - 2) + ti + tj, ti + q.TIp * tj);
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
// One thread block per preconditioner block (TI x TJ*split columns; with
// split = 2 the block's columns live in two layout tiles), one thread per
// column, wavefront step s at k = 2+s-ti-tj.  Ring values: 0 AD, 1 ALI,
// 2 ALJ, 3 ALK, 4 AUI, 5 AUJ, 6 AUK; DD is written in the skewed layout.
template <int D, typename V>
__device__ __forceinline__ void dcmp_body(const Geo &g, const SkewGeo &q, V U, const SkewSysT<V> &S, int *pivot_bad,
                                          int bx, int by) {
  constexpr int NV = 7, R = D + 3;
  const int TIp = q.TIp, TJl = q.TJ, Tl = q.T;      // layout tile
  const int TJb = TJl * q.split, Tb = TIp * TJb;    // preconditioner block
  Ring<NV, V> rg = ring_setup<NV, V>(Tb, R);
  const int tid = threadIdx.x;
  const int ti = tid % TIp, tj = tid / TIp;
  const int is = 2 + bx * q.TI, js = 2 + by * TJb;
  const int wi = min(q.TI, g.NI - is), wj = min(TJb, g.NJ - js);
  const bool valid = ti < wi && tj < wj;
  const int r = tj / TJl, tjl = tj % TJl;
  const long long bl = bx + (long long)q.ntx * (by * q.split + r);  // layout tile
  // slab of step s: w = (k-2) + ti + tjl = s - r*TJl
  const long long slab0 = bl * q.W - (long long)r * TJl;
  const int tl = ti + TIp * tjl;
  const int nsteps = (g.NK - 2) + (wi - 1) + (wj - 1);
  auto prefetch = [&](int s) {
    const int k = 2 + s - ti - tj;
    if (valid && k >= 2 && k <= g.NK - 1) {
      const long long slab = slab0 + s, e = slab * Tl + tl;
      const V *sy = S.sys + sys_at(slab, 0, Tl, tl);
      const int sl = s % R;
      constexpr int cs[7] = {SYS_AD, SYS_ALI, SYS_ALJ, SYS_ALK, SYS_AUI, SYS_AUJ, SYS_AUK};
#pragma unroll
      for (int c = 0; c < 7; ++c) cp_async_v(&rg.v(sl, c, tid), sy + (long long)cs[c] * Tl);
      cp_async4(&rg.ind(sl, tid), S.indc + e);
    }
    cp_commit();
  };
#pragma unroll 1
  for (int s = 0; s < D; ++s) prefetch(s);
  V dk1 = V(0), au3 = V(0);  // DD(i,j,k-1) and AU3 of (i,j,k-1); k-1 = 1 is the zero ghost layer
  const V z = V(0), one = V(1);
  bool bad = false;
  const int T = Tb;
  for (int s = 0; s < nsteps; ++s) {
    prefetch(s + D);
    cp_wait<D - 1>();
    __syncthreads();
    const int k = 2 + s - ti - tj;
    const int sl = s % R, slp = (s + R - 1) % R, cur = s & 1, prv = cur ^ 1;
    if (valid && k >= 2 && k <= g.NK - 1) {
      V dd = z;
      if (rg.ind(sl, tid) != -1) {
        V d1 = z, a1, d2 = z, a2;
        if (ti > 0) {
          d1 = rg.xb[prv * T + tid - 1];
          a1 = rg.v(slp, 4, tid - 1) + U * (rg.v(slp, 5, tid - 1) + rg.v(slp, 6, tid - 1));
        } else {
          a1 = z + U * (z + z);
        }
        if (tj > 0) {
          d2 = rg.xb[prv * T + tid - TIp];
          a2 = rg.v(slp, 5, tid - TIp) + U * (rg.v(slp, 4, tid - TIp) + rg.v(slp, 6, tid - TIp));
        } else {
          a2 = z + U * (z + z);
        }
        dd = one / (rg.v(sl, 0, tid) - rg.v(sl, 1, tid) * d1 * a1 - rg.v(sl, 2, tid) * d2 * a2 -
                    rg.v(sl, 3, tid) * dk1 * au3);
        if (dd <= z) bad = true;
      }
      S.sys[sys_at(slab0 + s, SYS_DD, Tl, tl)] = dd;
      rg.xb[cur * T + tid] = dd;
      dk1 = dd;
      au3 = rg.v(sl, 6, tid) + U * (rg.v(sl, 4, tid) + rg.v(sl, 5, tid));
    }
  }
  cp_wait<0>();
  if (bad) atomicOr(pivot_bad, 1);
}
template <int D, typename V>
__global__ void k_dcmp(Geo g, SkewGeo q, V U, SkewSysT<V> S, int *pivot_bad) {
  pdl_enter();
  dcmp_body<D, V>(g, q, U, S, pivot_bad, (int)blockIdx.x, (int)blockIdx.y);
}

// ------------------------------------------------ bulk-copy slab pipeline
// The sweeps read, at every wavefront step, one contiguous slab of T
// values from each of 5 or 9 skewed arrays.  A producer warp moves those
// slabs into a ring of R = D+2 shared-memory slots with cp.async.bulk, D
// steps ahead, each slot completing on its own mbarrier (transaction
// count); the T consumer threads wait on the mbarrier of the step they
// need and then work purely from shared memory.  One block barrier per
// step orders the exchange of the sweep values between neighbouring
// columns and frees the slot of step s-2 for the producer.
__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(unsigned bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try(unsigned bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ void bulk_load(unsigned dst, const void *src, unsigned bytes, unsigned bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;\n" : "=l"(t));
  return t;
}
// Wait for the phase `parity` of an mbarrier, giving up after limit_ns.
__device__ __noinline__ bool mbar_wait_slow(unsigned bar, unsigned parity, unsigned long long limit_ns) {
  const unsigned long long t0 = global_ns();
  for (;;) {
    for (int i = 0; i < 64; ++i)
      if (mbar_try(bar, parity)) return true;
    if (global_ns() - t0 > limit_ns) return false;
  }
}
// Non-blocking test of a phase: its latency overlaps the instructions that
// follow until the predicate is used.
__device__ __forceinline__ bool mbar_test(unsigned bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}
// The limit comes from the solve state, read only once a wait has to
// spin, so that it occupies no register in the sweeps' step loop.
__device__ __noinline__ bool mbar_wait_st(unsigned bar, unsigned parity, const SolveState *st) {
  return mbar_wait_slow(bar, parity, (unsigned long long)st->wait_ns);
}
__device__ __forceinline__ bool mbar_wait(unsigned bar, unsigned parity, const SolveState *st) {
  return mbar_try(bar, parity) || mbar_wait_st(bar, parity, st);
}

// ------------------------------------- cluster exchange (precond_split 2)
__device__ __forceinline__ unsigned cluster_rank() {
  unsigned r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;\n" : "=r"(r));
  return r;
}
// Address of the same shared-memory location in CTA `rank` of the cluster.
__device__ __forceinline__ unsigned mapa(unsigned addr, unsigned rank) {
  unsigned r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;\n" : "=r"(r) : "r"(addr), "r"(rank));
  return r;
}
// Store into another CTA of the cluster and credit the stored bytes to an
// mbarrier there (transaction count); no release of earlier stores.
__device__ __forceinline__ void st_async(unsigned addr, double v, unsigned mbar) {
  asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.f64 [%0], %1, [%2];\n" ::"r"(addr), "d"(v),
               "r"(mbar)
               : "memory");
}
__device__ __forceinline__ void st_async(unsigned addr, float v, unsigned mbar) {
  asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.f32 [%0], %1, [%2];\n" ::"r"(addr), "f"(v),
               "r"(mbar)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_cluster(unsigned bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait (limit_ns) acquiring what other CTAs of the cluster released.
__device__ __noinline__ bool mbar_wait_cluster_slow(unsigned bar, unsigned parity, unsigned long long limit_ns) {
  const unsigned long long t0 = global_ns();
  for (;;) {
    for (int i = 0; i < 64; ++i)
      if (mbar_try_cluster(bar, parity)) return true;
    if (global_ns() - t0 > limit_ns) return false;
  }
}
__device__ __noinline__ bool mbar_wait_cluster_st(unsigned bar, unsigned parity, const SolveState *st) {
  return mbar_wait_cluster_slow(bar, parity, (unsigned long long)st->wait_ns);
}
__device__ __forceinline__ bool mbar_wait_cluster(unsigned bar, unsigned parity, const SolveState *st) {
  return mbar_try_cluster(bar, parity) || mbar_wait_cluster_st(bar, parity, st);
}
__device__ __forceinline__ void cluster_barrier() {
  asm volatile("barrier.cluster.arrive.release;\nbarrier.cluster.wait.acquire;\n" ::: "memory");
}

// ------------------------------------ VF_MZFRWD (+VF_MZAX) and VF_MZBKWD
// One block per tile: T consumer threads (thread t = ti + TIp*tj owns
// column (ti,tj)) and one producer warp.  MODE (SweepMode):
//   SWEEP_FWD     T = MINV_L * Y, Y given (skewed);  vf_mzfrwd.f
//   SWEEP_FWD_AX  T = MINV_L * (A*P), A*P formed on the fly (VF_MZAX
//                 then VF_MZFRWD: vf_mzax.f:46-53, vf_mzfrwd.f)
//   SWEEP_BWD     X = MINV_U * T;  vf_mzbkwd.f
// The forward sweeps write T into the system block (SYS_T), where the
// backward sweep's one bulk copy per step finds it with AUI..DD; the
// backward sweep writes X in the skewed layout.  Forward step s visits
// k = 2+s-ti-tj, backward step s visits k = NK-1-(s-ri-rj) (ri, rj the
// distances from the far corner), so step s of every thread is one slab.
// A cell is computed where DD != 0: MZDCMP gives DD = 0 exactly on
// INDC = -1 and a positive (or NaN) DD elsewhere, and a zero or negative
// pivot ends the solve before any sweep runs.
//
// Only the recurrence sits between two block barriers: the neighbours'
// results of step s-1 are read, combined in five dependent operations and
// published.  Everything that does not depend on step s-1 -- the ring
// loads, the 7-term product A*P and the products ALI*DD(i-1) etc. of the
// recurrence -- is prepared for step s+1 after the result of step s is
// published, while the other warps reach the barrier.  The expressions
// and their evaluation order are those of the reference loops, so the
// results do not change.  The step loop is unrolled by the ring length so
// slot addresses and mbarrier phases are constants.
// CT, CTIP: the layout tile's T and TIp at compile time (0: from q), so
// that the slot offsets of a common tile shape are immediates and take no
// registers.
template <int D, int MODE, typename V, int CS, int CT = 0, int CTIP = 0>
__device__ __forceinline__ void sweep_body(const Geo &g, const SkewGeo &q_, const SkewSysT<V> &S, const V *vin,
                                           V *vout, SolveState *st, const V *vin2, double *rb, int bx, int by) {
  constexpr bool BWD = MODE >= SWEEP_BWD;
  constexpr int NDOT = sweep_ndot(MODE);
  SkewGeo q = q_;
  if (CT > 0) {
    q.T = CT;
    q.TIp = CTIP;
    q.TJ = CT / (CTIP > 0 ? CTIP : 1);
  }
  // CS = 2: the thread blocks of a cluster are the two layout tiles of one
  // preconditioner block; every block of a cluster runs through the two
  // cluster barriers below, so none returns early.
  const bool skip = st->done || (CS == 2 && by >= q.nb / q.ntx);
  if (CS == 1 && skip) return;
  if (CS == 2 && skip) {
    cluster_barrier();
    cluster_barrier();
    return;
  }
  constexpr int R = D + 2;
  constexpr int AHEAD = (MODE == SWEEP_FWD_AX) ? 2 : 1;  // preparing step s+1 reads the slot of step s+AHEAD
  extern __shared__ __align__(16) double sm[];
  const int T = q.T, TIp = q.TIp;
  const int Tc = (T + 31) & ~31;
  constexpr int ES = (int)sizeof(V);
  const int SS = sweep_slot(q, MODE, ES);
  // slot offsets of the system arrays
  constexpr int SF = sweep_sys_first(MODE) - sweep_sys_dst(MODE);
  const int oDD = (SYS_DD - SF) * T, oAD = (SYS_AD - SF) * T, oALI = (SYS_ALI - SF) * T,
            oALJ = (SYS_ALJ - SF) * T, oALK = (SYS_ALK - SF) * T, oAUI = (SYS_AUI - SF) * T,
            oAUJ = (SYS_AUJ - SF) * T, oAUK = (SYS_AUK - SF) * T;
  unsigned long long *bar = reinterpret_cast<unsigned long long *>(sm);
  V *ring = reinterpret_cast<V *>(sm + ((R + 1) & ~1));
  V *xb = ring + (size_t)R * SS;
  const int tid = threadIdx.x, b = bx + q.ntx * by;
  TileGeo t = tile_geo(g, q, bx, by);
  const int nsteps = (g.NK - 2) + (t.wi - 1) + (t.wj - 1);
  const bool producer = tid >= Tc;
  const int lane = tid & 31;

  // Cluster exchange (CS = 2).  The forward sweeps need, on row 0 of the
  // upper tile, the result and DD of row TJ-1 of the lower tile at the
  // same k; the backward sweep needs the reverse.  The sending row stores
  // its values of step u into slot u of the receiver's xin/din with
  // st.async, each store crediting its bytes to the receiver's xfull[u],
  // which the receiver armed at start-up for one full row (TIp values of x,
  // and of DD for the forward sweeps); a slot is written once per sweep.
  const int NX = q.W;                                   // slots: steps of a tile at most
  unsigned long long *xfull = reinterpret_cast<unsigned long long *>(xb + 2 * T);
  V *xin = reinterpret_cast<V *>(xfull + NX);
  V *din = xin + (size_t)NX * TIp;
  const int crank = (CS == 2) ? (by & 1) : 0;
  const int nty = q.nb / q.ntx;
  const bool has_up = CS == 2 && crank == 0 && by + 1 < nty;
  const bool has_lo = CS == 2 && crank == 1;
  const bool recv = BWD ? has_up : has_lo;
  const bool send = BWD ? has_lo : has_up;
  const bool srow = send && (BWD ? t.tj == 0 : t.tj == q.TJ - 1) && !producer;
  const bool rrow = recv && (BWD ? t.tj == t.wj - 1 : t.tj == 0) && !producer;
  // receiver's step lag: rows of the sending tile minus one
  const int lag = BWD ? min(q.TJ, g.NJ - (2 + (by + 1) * q.TJ)) - 1 : q.TJ - 1;
  unsigned r_xin = 0, r_din = 0, r_full = 0;            // the partner's xin, din, xfull
  if (CS == 2 && send) {
    const unsigned peer = cluster_rank() ^ 1u;
    r_xin = mapa(smem_u32(xin), peer);
    r_din = mapa(smem_u32(din), peer);
    r_full = mapa(smem_u32(xfull), peer);
  }

  // s_abort[c & 1]: a wait of some thread ran out of time during ring
  // cycle c.  Written during a cycle, read after its last barrier; the two
  // entries keep those reads apart from the writes of the next cycle.
  __shared__ int s_abort[2];
  if (tid == 0) {
    for (int r = 0; r < R; ++r) mbar_init(smem_u32(bar + r), 1);
    s_abort[0] = s_abort[1] = 0;
  }
  if (CS == 2 && recv) {
    const unsigned row_bytes = (unsigned)(TIp * ES * (BWD ? 1 : 2));
    for (int u = tid; u < NX; u += blockDim.x) {
      mbar_init(smem_u32(xfull + u), 1u);
      mbar_expect_tx(smem_u32(xfull + u), row_bytes);
    }
  }
  if (MODE == SWEEP_FWD_AX) {  // halo values of absent neighbours stay 0 (ghost layer)
    const int nh = 2 * halo_span(q, ES) + 2 * TIp;
    for (int r = 0; r < R; ++r)
      for (int i = tid; i < nh; i += blockDim.x) ring[(size_t)r * SS + halo_left(q, ES) + i] = V(0);
  }
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
  if (CS == 2) cluster_barrier();  // partner's barriers initialised before any remote arrival
  else __syncthreads();

  // Producer: lane l issues copy l of every step (at most 6); its fixed
  // part is worked out once here.
  const V *src0 = nullptr;
  SweepLane l0;
  l0.dlo = 1; l0.dhi = 0; l0.bytes = 0; l0.dst = 0; l0.wstride = 0;  // empty range: no copy
  if (producer && lane < sweep_ncopy(q, MODE) && sweep_lane(q, MODE, b, lane, l0, ES))
    src0 = (l0.arr == 0 ? S.sys : (l0.arr == 1 ? vin : vin2)) + l0.base;
  else { l0.dlo = 1; l0.dhi = 0; l0.bytes = 0; }
  const unsigned bar0 = smem_u32(bar), ring0 = smem_u32(ring);
  const int stall_from = producer ? st->stall_from : 0;  // read by the producer warp only
  auto issue = [&](int u, int slot) {
    if (u >= nsteps || u >= stall_from) return;
    const int w = BWD ? nsteps - 1 - u : u;
    const unsigned bslot = bar0 + 8u * slot;
    const unsigned dslot = ring0 + (unsigned)ES * (unsigned)(slot * SS);
    const bool v0 = (w >= l0.dlo && w <= l0.dhi);
    const unsigned bytes = __reduce_add_sync(0xffffffffu, v0 ? l0.bytes : 0);
    if (lane == 0) mbar_expect_tx(bslot, bytes);
    __syncwarp();
    if (v0) bulk_load(dslot + (unsigned)ES * l0.dst, src0 + (long long)w * l0.wstride, l0.bytes, bslot);
  };
  // data of step u sits in slot u % R, phase (u / R) & 1
  auto wait_data = [&](int u, int slot, unsigned parity) -> bool {
    return u >= nsteps || mbar_wait(bar0 + 8u * slot, parity, st);
  };

  if (producer) {
#pragma unroll 1
    for (int u = 0; u < D; ++u) issue(u, u % R);
  }

  // Column geometry: active steps slo..shi (k inside 2..NK-1).
  const int ri = t.wi - 1 - t.ti, rj = t.wj - 1 - t.tj;
  const bool ex0 = (t.ti == 0), ex1 = (t.ti == t.wi - 1), ey0 = (t.tj == 0), ey1 = (t.tj == t.wj - 1);
  const int slo = BWD ? ri + rj : t.ti + t.tj, shi = slo + g.NK - 3;
  const bool col = t.valid && !producer;
  const int hl = halo_left(q, ES) + TIp * t.tj + halo_lofs(q, ES), hr = halo_right(q, ES) + TIp * t.tj,
            hd = halo_down(q, ES) + t.ti, hu = halo_up(q, ES) + t.ti;
  // forward: T into the system block; backward: X
  V *vp = BWD ? vout + ((long long)b * q.W + nsteps - 1) * T + tid
                              : S.sys + sys_at((long long)b * q.W, SYS_T, T, tid);
  const long long vstep = BWD ? -(long long)T : (long long)SYS_N * T;

  // Prepared values of the next step.
  bool act = false;             // the column has a cell at this step
  V dd = V(0);              // DD of the cell (0: not computed)
  V y0 = V(0);              // FWD: Y or A*P;  BWD: T
  V c1 = V(0), c2 = V(0), c3 = V(0);  // FWD: ALI*DD(i-1), ALJ*DD(j-1), ALK*DD(k-1); BWD: AUI, AUJ, AUK
  V dk1 = V(0), pk1 = V(0);  // DD and P of this column at the previous step (FWD)
  V xk1 = V(0);             // result of this column at the previous step
  V q0 = V(0), q1 = V(0);   // NDOT: R0 and RR of the cell
  double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0, a4 = 0.0;  // NDOT: this column's sums
  // Prepare step s: cs = slot of s, ps = slot of s-1, ns = slot of s+1.
  auto prepare = [&](int s, const V *cs, const V *ps, const V *ns) {
    act = col && s >= slo && s <= shi;
    if (!act) return;
    if (MODE == SWEEP_FWD_AX) {
      const int k = 2 + s - t.ti - t.tj;
      const V d = cs[oDD + tid], pc = cs[8 * T + tid];
      if (d != V(0)) {
        const V pxm = ex0 ? cs[hl] : ps[8 * T + tid - 1];
        const V pym = ey0 ? cs[hd] : ps[8 * T + tid - TIp];
        const V pzm = (k > 2) ? pk1 : V(0);
        const V pxp = ex1 ? cs[hr] : ns[8 * T + tid + 1];
        const V pyp = ey1 ? cs[hu] : ns[8 * T + tid + TIp];
        const V pzp = (k < g.NK - 1) ? ns[8 * T + tid] : V(0);
        y0 = cs[oAD + tid] * pc + cs[oALI + tid] * pxm + cs[oALJ + tid] * pym + cs[oALK + tid] * pzm +
             cs[oAUI + tid] * pxp + cs[oAUJ + tid] * pyp + cs[oAUK + tid] * pzp;
        const V d1 = (t.ti > 0) ? ps[oDD + tid - 1] : V(0);
        const V d2 = (t.tj > 0) ? ps[oDD + tid - TIp] : (rrow ? din[(size_t)(s + lag) * TIp + t.ti] : V(0));
        c1 = cs[oALI + tid] * d1;
        c2 = cs[oALJ + tid] * d2;
        c3 = cs[oALK + tid] * dk1;
      }
      dd = d; dk1 = d; pk1 = pc;
    } else if (MODE == SWEEP_FWD) {
      const V d = cs[oDD + tid];
      if (d != V(0)) {
        const V d1 = (t.ti > 0) ? ps[oDD + tid - 1] : V(0);
        const V d2 = (t.tj > 0) ? ps[oDD + tid - TIp] : (rrow ? din[(size_t)(s + lag) * TIp + t.ti] : V(0));
        y0 = cs[tid];
        c1 = cs[oALI + tid] * d1;
        c2 = cs[oALJ + tid] * d2;
        c3 = cs[oALK + tid] * dk1;
      }
      dd = d; dk1 = d;
    } else {
      dd = cs[oDD + tid];
      if (dd != V(0)) { y0 = cs[tid]; c1 = cs[oAUI + tid]; c2 = cs[oAUJ + tid]; c3 = cs[oAUK + tid]; }
      if (NDOT > 0) q0 = cs[5 * T + tid];
      if (NDOT == 5) q1 = cs[6 * T + tid];
    }
  };
  auto slot_ptr = [&](int r) -> const V * { return ring + (size_t)r * SS; };

  bool ok = true;
  if (!producer) {
    for (int u = 0; u < AHEAD; ++u) if (ok) ok = wait_data(u, u % R, (unsigned)((u / R) & 1));
    if (CS == 2 && ok && rrow && col && 0 >= slo && 0 <= shi) ok = mbar_wait_cluster(smem_u32(xfull + lag), 0u, st);
    if (ok) prepare(0, slot_ptr(0), slot_ptr(R - 1), slot_ptr(1 % R));
    else s_abort[0] = 1;
  }
  bool aborted = false;
  int issued = min(min(D, nsteps), stall_from) - 1;  // last step whose copies were issued (producer)
  unsigned ph = 0;                  // (s0 / R) & 1, also the ring cycle's s_abort entry
#pragma unroll 1
  for (int s0 = 0; s0 < nsteps && !aborted; s0 += R, ph ^= 1u) {
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int s = s0 + r;
      if (s >= nsteps) break;
      if (producer) {
        issue(s + D, (r + D) % R);
        if (s + D < nsteps && s + D < stall_from) issued = s + D;
      } else {
        // Test the data of the step to prepare next now, so the test's
        // latency overlaps the recurrence; wait only if it is not there.
        const int u = s + AHEAD;  // newest data that preparing s+1 reads
        const unsigned ubar = bar0 + 8u * ((r + AHEAD) % R), upar = ph ^ (unsigned)((r + AHEAD) / R);
        const bool ready = !ok || u >= nsteps || mbar_test(ubar, upar);
        // the recurrence of step s
        V xcur = V(0);
        if (act && ok) {
          const int cur = (s & 1) * T, prv = T - cur;
          V x = V(0);
          if (dd != V(0)) {
            const V xr = rrow ? xin[(size_t)(s + lag) * TIp + t.ti] : V(0);  // partner tile's row
            if (BWD) {
              const V x1 = (ri > 0) ? xb[prv + tid + 1] : V(0);
              const V x2 = (rj > 0) ? xb[prv + tid + TIp] : xr;
              x = (y0 - c1 * x1 - c2 * x2 - c3 * xk1) * dd;
            } else {
              const V x1 = (t.ti > 0) ? xb[prv + tid - 1] : V(0);
              const V x2 = (t.tj > 0) ? xb[prv + tid - TIp] : xr;
              x = y0 - c1 * x1 - c2 * x2 - c3 * xk1;
            }
          }
          xb[cur + tid] = x;
          *vp = x;
          xk1 = x;
          xcur = x;
          // products of two single-precision values are exact in double
          if (NDOT == 1) a0 += (double)q0 * (double)x;
          if (NDOT == 5) {
            const double r = (double)q1, e = (double)x, z = (double)q0;
            a0 += r * e;
            a1 += e * e;
            a2 += r * r;
            a3 += z * r;
            a4 += z * e;
          }
        }
        vp += vstep;
        if (CS == 2 && srow) {  // this step's boundary-row values to the partner tile
          const unsigned off = (unsigned)(((size_t)s * TIp + t.ti) * ES), fb = r_full + 8u * (unsigned)s;
          st_async(r_xin + off, xcur, fb);
          if (!BWD) st_async(r_din + off, act ? dd : V(0), fb);
        }
        // prepare step s+1
        if (!ready) {
          ok = mbar_wait_st(ubar, upar, st);
          if (!ok) s_abort[ph] = 1;
        }
        if (CS == 2 && ok && rrow && col && s + 1 >= slo && s + 1 <= shi) {
          ok = mbar_wait_cluster(smem_u32(xfull + (s + 1 + lag)), 0u, st);
          if (!ok) s_abort[ph] = 1;
        }
        if (ok && s + 1 < nsteps) prepare(s + 1, slot_ptr((r + 1) % R), slot_ptr(r), slot_ptr((r + 2) % R));
      }
      __syncthreads();
    }
    // A timed-out wait stops the sweep at the end of this ring cycle; the
    // threads that gave up skip their remaining waits and work meanwhile.
    if (s_abort[ph]) aborted = true;
  }
  if (aborted && producer) {
    // Let the copies already issued land (bounded) before the block exits.
    if (lane == 0)
      for (int u = max(0, issued - R + 1); u <= issued; ++u)
        mbar_wait_slow(bar0 + 8u * (u % R), (unsigned)((u / R) & 1), 100000000ull);
    if (lane == 0) { st->timeout = 1; st->done = 1; }
  }
  if (NDOT > 0) {
    // the tile's sums: warps by a butterfly, then the warps' partials by
    // warp 0, in a fixed order; one partial per tile into rb[c*nb + b]
    __shared__ double s_red[5][32];
    double a[5] = {a0, a1, a2, a3, a4};
#pragma unroll
    for (int c = 0; c < NDOT; ++c) {
      double v = a[c];
#pragma unroll
      for (int o = 16; o >= 1; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      if (lane == 0) s_red[c][tid >> 5] = v;
    }
    __syncthreads();
    if (tid < 32) {
      const int nw = (int)(blockDim.x >> 5);
#pragma unroll
      for (int c = 0; c < NDOT; ++c) {
        double v = (tid < nw) ? s_red[c][tid] : 0.0;
#pragma unroll
        for (int o = 16; o >= 1; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (tid == 0) rb[(long long)c * q.nb + b] = v;
      }
    }
  }
  if (CS == 2) cluster_barrier();  // the partner may still write into this block's shared memory
}
template <int D, int MODE, int MAXT, typename V, int CS, int MINB = 1, int CT = 0, int CTIP = 0>
__global__ void __launch_bounds__(MAXT, MINB)
    k_sweep(Geo g, SkewGeo q, SkewSysT<V> S, const V *vin, V *vout, SolveState *st, const V *vin2, double *rb) {
  pdl_enter();
  sweep_body<D, MODE, V, CS, CT, CTIP>(g, q, S, vin, vout, st, vin2, rb, (int)blockIdx.x, (int)blockIdx.y);
}

// ------------------------------------------------------------ slab kernels
// The BiCGSTAB vectors live in the skewed layout; a vector kernel maps one
// warp to one slab (b,w) of T entries and lets lane l visit t = l, l+32, ...
// The dot products (VF_MZIP) sum in that order: lane partials, warp tree
// per slab, then the 1024-thread tree over the slab partials (block_final).
// Padding entries carry INDC = -1 and are skipped like non-computed cells.
// The hot kernels load every operand of an entry before testing its INDC
// (all entries of the layout are allocated), so the unrolled loop keeps
// several entries' loads in flight.
#define SLAB_LOOP_BEGIN(q)                                                          \
  const int lane_ = threadIdx.x & 31;                                               \
  const long long slab_ = (long long)BX_ * ROWS_PER_BLOCK + (threadIdx.x >> 5);      \
  if (slab_ < (long long)(q).nb * (q).W) {                                          \
    _Pragma("unroll 4")                                                             \
    for (int t_ = lane_; t_ < (q).T; t_ += 32) {                                    \
      const long long e = slab_ * (q).T + t_;
#define SLAB_LOOP_END \
    }                 \
  }
// Partial of one block of a slab sum: each warp's slab sum (warp tree),
// then the block's ROWS_PER_BLOCK slabs added in slab order by thread 0,
// into rb[bx] (bx the block's index).  The finaliser then reduces one
// partial per block (nslab / 8 of them) instead of one per slab.  Every
// thread of the block calls it (it holds block barriers).
__device__ __forceinline__ void slab_store(double s, double *rb, long long nslab, unsigned bx) {
  __shared__ double ws[ROWS_PER_BLOCK];
  s = warp_tree(s);
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    const long long first = (long long)bx * ROWS_PER_BLOCK;
    double t = 0.0;
    for (int i = 0; i < ROWS_PER_BLOCK; ++i)
      if (first + i < nslab) t = t + ws[i];
    rb[bx] = t;
  }
  __syncthreads();
}

__device__ __forceinline__ bool interior(const Geo &g, int I, int J, int K) {
  return I >= 2 && I <= g.NI - 1 && J >= 2 && J <= g.NJ - 1 && K >= 2 && K <= g.NK - 1;
}

// A*X at skewed entry e (VF_MZAX expression, vf_mzax.f:46-53).
template <typename V>
__device__ __forceinline__ V skew_ax(const Geo &g, const SkewGeo &q, const SkewSysT<V> &S, const V *X,
                                     long long e) {
  const int t = (int)(e % q.T);
  const long long bw = e / q.T;
  const int w = (int)(bw % q.W), b = (int)(bw / q.W);
  const int ti = t % q.TIp, tj = t / q.TIp, bx = b % q.ntx, by = b / q.ntx, k = 2 + w - ti - tj;
  const V *a = S.sys + sys_at(bw, 0, q.T, t);
  const long long T = q.T;
  auto at = [&](int di, int dj, int dk) -> V {
    const long long n = skew_nb(g, q, bx, by, ti + di, tj + dj, k + dk);
    return n < 0 ? V(0) : X[n];
  };
  return a[SYS_AD * T] * X[e] + a[SYS_ALI * T] * at(-1, 0, 0) + a[SYS_ALJ * T] * at(0, -1, 0) +
         a[SYS_ALK * T] * at(0, 0, -1) + a[SYS_AUI * T] * at(1, 0, 0) + a[SYS_AUJ * T] * at(0, 1, 0) +
         a[SYS_AUK * T] * at(0, 0, 1);
}

// Y = A X on INDC != -1 (VF_MZAX); Y untouched elsewhere.
template <typename V>
__device__ __forceinline__ void spmv_body(Geo g, SkewGeo q, SkewSysT<V> S, const V *X, V *Y, const SolveState *st, unsigned BX_) {
  if (st && st->done) return;
  SLAB_LOOP_BEGIN(q)
  if (S.indc[e] != -1) Y[e] = skew_ax(g, q, S, X, e);
  SLAB_LOOP_END
}
template <typename V>
__global__ void k_spmv(Geo g, SkewGeo q, SkewSysT<V> S, const V *X, V *Y, const SolveState *st) {
  pdl_enter();
  spmv_body<V>(g, q, S, X, Y, st, blockIdx.x);
}

// Y = B - Y on INDC != -1 (vf_m1bcgs.f:124-132)
__device__ __forceinline__ void bmy_body(SkewGeo q, const int *INDC, const double *B, double *Y, const SolveState *st, unsigned BX_) {
  if (st && st->done) return;
  SLAB_LOOP_BEGIN(q)
  if (INDC[e] != -1) Y[e] = B[e] - Y[e];
  SLAB_LOOP_END
}
__global__ void k_bmy(SkewGeo q, const int *INDC, const double *B, double *Y, const SolveState *st) {
  pdl_enter();
  bmy_body(q, INDC, B, Y, st, blockIdx.x);
}

// The BiCGSTAB vector kernels below serve the FP64 solve (V = double) and
// the FP32 inner solves of the mixed solver (V = float).  With float
// vectors the arithmetic runs in double (the scalars are double) and is
// rounded once on the store; dot products always accumulate in double.

// Slab partials of up to two dot products (VF_MZIP).
template <typename V>
__device__ __forceinline__ void dot_body(SkewGeo q, const int *INDC, const V *x0, const V *y0, const V *x1, const V *y1,
                      double *rb0, double *rb1, const SolveState *st, unsigned BX_) {
  if (st && st->done) return;
  double s0 = 0.0, s1 = 0.0;
  const long long nslab = (long long)q.nb * q.W;
  SLAB_LOOP_BEGIN(q)
  const int ic = INDC[e];
  const double a0 = (double)x0[e] * (double)y0[e];
  const double a1 = x1 ? (double)x1[e] * (double)y1[e] : 0.0;
  if (ic != -1) {
    s0 = s0 + a0;
    if (x1) s1 = s1 + a1;
  }
  SLAB_LOOP_END
  slab_store(s0, rb0, nslab, BX_);
  if (x1) slab_store(s1, rb1, nslab, BX_);
}
template <typename V>
__global__ void k_dot(SkewGeo q, const int *INDC, const V *x0, const V *y0, const V *x1, const V *y1,
                      double *rb0, double *rb1, const SolveState *st) {
  pdl_enter();
  dot_body<V>(q, INDC, x0, y0, x1, y1, rb0, rb1, st, blockIdx.x);
}

// RR = R0, PP = R0
template <typename V>
__device__ __forceinline__ void copy2_body(SkewGeo q, const int *INDC, const V *R0, V *RR, V *PP, const SolveState *st, unsigned BX_) {
  if (st->done) return;
  SLAB_LOOP_BEGIN(q)
  if (INDC[e] != -1) { RR[e] = R0[e]; PP[e] = R0[e]; }
  SLAB_LOOP_END
}
template <typename V>
__global__ void k_copy2(SkewGeo q, const int *INDC, const V *R0, V *RR, V *PP, const SolveState *st) {
  pdl_enter();
  copy2_body<V>(q, INDC, R0, RR, PP, st, blockIdx.x);
}

// RR = RR - ALPHA*AP (vf_m1bcgs.f:181-189)
template <typename V>
__global__ void k_axpy_rr(SkewGeo q, const int *INDC, const V *AP, V *RR, const SolveState *st) {
  pdl_enter();
  const unsigned BX_ = blockIdx.x;
  if (st->done) return;
  const double alpha = st->alpha;
  SLAB_LOOP_BEGIN(q)
  const int ic = INDC[e];
  const V r = RR[e], a = AP[e];
  if (ic != -1) RR[e] = (V)(r - alpha * a);
  SLAB_LOOP_END
}

// XW = XW + (ALPHA*PP + OMEGA*RR); RR = RR - OMEGA*AE; slab partials of
// (RR,RR) and (R0,RR) on the updated RR (vf_m1bcgs.f:206-225).
template <typename V>
__global__ void k_upd_xr(SkewGeo q, const int *INDC, const V *PP, const V *AE, const V *R0, V *XW, V *RR,
                         double *rb0, double *rb1, const SolveState *st) {
  pdl_enter();
  const unsigned BX_ = blockIdx.x;
  if (st->done) return;
  const double alpha = st->alpha, omega = st->omega;
  double s0 = 0.0, s1 = 0.0;
  const long long nslab = (long long)q.nb * q.W;
  SLAB_LOOP_BEGIN(q)
  const int ic = INDC[e];
  const V xw = XW[e], pp = PP[e], rr = RR[e], ae = AE[e], r0 = R0[e];
  if (ic != -1) {
    XW[e] = (V)(xw + (alpha * pp + omega * rr));
    const V r = (V)(rr - omega * ae);
    RR[e] = r;
    s0 = s0 + (double)r * (double)r;
    s1 = s1 + (double)r0 * (double)r;
  }
  SLAB_LOOP_END
  slab_store(s0, rb0, nslab, BX_);
  slab_store(s1, rb1, nslab, BX_);
}

// PP = RR + BETA*(PP - OMEGA*AP) (vf_m1bcgs.f:229-238)
template <typename V>
__global__ void k_upd_p(SkewGeo q, const int *INDC, const V *RR, const V *AP, V *PP, const SolveState *st) {
  pdl_enter();
  const unsigned BX_ = blockIdx.x;
  if (st->done) return;
  const double beta = st->beta, omega = st->omega;
  SLAB_LOOP_BEGIN(q)
  const int ic = INDC[e];
  const V rr = RR[e], pp = PP[e], ap = AP[e];
  if (ic != -1) PP[e] = (V)(rr + beta * (pp - omega * ap));
  SLAB_LOOP_END
}

// --------------------------------- FP32 inner solves of the mixed solver
// The inner BiCGSTAB of the mixed solver (V = float) runs a regrouped
// iteration with fewer passes over the vectors; it is the same method and
// ends on the same criterion, but its sums are not those of VF_M1BCGS,
// whose FP64 form (above) keeps the reference's order.
//   * Every vector is zero wherever INDC = -1 and on the layout's padding
//     (zeroed at the start of a solve and never written there: the
//     sweeps write 0 for non-computed cells), so these kernels read no
//     INDC: an update leaves a zero entry zero and adds nothing to a sum.
//   * One lane moves 4 consecutive entries (16-byte loads; T is a multiple
//     of 4 and every slab starts on a 16-byte boundary).
//   * After the second sweep pair one pass forms the five sums (RR,AE),
//     (AE,AE), (RR,RR), (R0,RR), (R0,AE); OMEGA, the new |RR|^2 =
//     (RR,RR) - 2 OMEGA (RR,AE) + OMEGA^2 (AE,AE), the new (R0,RR) =
//     (R0,RR) - OMEGA (R0,AE), the convergence test and BETA follow from
//     them (k_fin5), and one pass updates XW, RR and PP together (k_upd3f).
//     Per iteration a sum drops by about 25 times, so the expansion loses
//     nothing to cancellation at the tolerances used (FP64 sums).
#define SLAB4_LOOP_BEGIN(q)                                                         \
  const int lane_ = threadIdx.x & 31;                                               \
  const long long slab_ = (long long)BX_ * ROWS_PER_BLOCK + (threadIdx.x >> 5);      \
  if (slab_ < (long long)(q).nb * (q).W) {                                          \
    const int T4_ = (q).T >> 2;                                                     \
    _Pragma("unroll 2")                                                             \
    for (int t_ = lane_; t_ < T4_; t_ += 32) {                                      \
      const long long e4 = slab_ * T4_ + t_;
#define SLAB4_LOOP_END \
    }                  \
  }
__device__ __forceinline__ double dot4(const float4 &a, const float4 &b) {
  return (double)a.x * (double)b.x + (double)a.y * (double)b.y + (double)a.z * (double)b.z +
         (double)a.w * (double)b.w;
}
// slab partials of (R0,AP)
__global__ void k_dot2f(SkewGeo q, const float *R0, const float *AP, double *rb, const SolveState *st) {
  pdl_enter();
  const unsigned BX_ = blockIdx.x;
  if (st->done) return;
  const float4 *r0 = reinterpret_cast<const float4 *>(R0), *ap = reinterpret_cast<const float4 *>(AP);
  double s0 = 0.0;
  const long long nslab = (long long)q.nb * q.W;
  SLAB4_LOOP_BEGIN(q)
  s0 += dot4(r0[e4], ap[e4]);
  SLAB4_LOOP_END
  slab_store(s0, rb, nslab, BX_);
}
// RR = RR - ALPHA*AP
__device__ __forceinline__ void axpyf_body(SkewGeo q, const float *AP, float *RR, const SolveState *st, unsigned BX_) {
  if (st->done) return;
  const double alpha = st->alpha;
  const float4 *ap = reinterpret_cast<const float4 *>(AP);
  float4 *rr = reinterpret_cast<float4 *>(RR);
  SLAB4_LOOP_BEGIN(q)
  const float4 a = ap[e4];
  float4 r = rr[e4];
  r.x = (float)(r.x - alpha * a.x); r.y = (float)(r.y - alpha * a.y);
  r.z = (float)(r.z - alpha * a.z); r.w = (float)(r.w - alpha * a.w);
  rr[e4] = r;
  SLAB4_LOOP_END
}
__global__ void k_axpyf(SkewGeo q, const float *AP, float *RR, const SolveState *st) {
  pdl_enter();
  axpyf_body(q, AP, RR, st, blockIdx.x);
}
// block partials of (RR,AE), (AE,AE), (RR,RR), (R0,RR), (R0,AE) into
// rb + c*nrb, c = 0..4 (nrb = blocks of the launch)
__global__ void k_dot5f(SkewGeo q, const float *R0, const float *RR, const float *AE, double *rb,
                        const SolveState *st) {
  pdl_enter();
  const unsigned BX_ = blockIdx.x;
  if (st->done) return;
  const float4 *r0 = reinterpret_cast<const float4 *>(R0), *rr = reinterpret_cast<const float4 *>(RR),
               *ae = reinterpret_cast<const float4 *>(AE);
  double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0, s4 = 0.0;
  const long long nslab = (long long)q.nb * q.W;
  SLAB4_LOOP_BEGIN(q)
  const float4 a = r0[e4], r = rr[e4], e = ae[e4];
  s0 += dot4(r, e);
  s1 += dot4(e, e);
  s2 += dot4(r, r);
  s3 += dot4(a, r);
  s4 += dot4(a, e);
  SLAB4_LOOP_END
  const long long nrb = gridDim.x;  // block partials of each sum
  slab_store(s0, rb, nslab, BX_);
  slab_store(s1, rb + nrb, nslab, BX_);
  slab_store(s2, rb + 2 * nrb, nslab, BX_);
  slab_store(s3, rb + 3 * nrb, nslab, BX_);
  slab_store(s4, rb + 4 * nrb, nslab, BX_);
}
// XW = XW + (ALPHA*PP + OMEGA*RR); RR' = RR - OMEGA*AE;
// PP = RR' + BETA*(PP - OMEGA*AP); RR = RR'
__device__ __forceinline__ void upd3f_body(SkewGeo q, const float *AE, const float *AP, float *XW, float *RR, float *PP,
                        const SolveState *st, unsigned BX_) {
  if (st->done) return;
  const double alpha = st->alpha, omega = st->omega, beta = st->beta;
  const float4 *ae = reinterpret_cast<const float4 *>(AE), *ap = reinterpret_cast<const float4 *>(AP);
  float4 *xw = reinterpret_cast<float4 *>(XW), *rr = reinterpret_cast<float4 *>(RR),
         *pp = reinterpret_cast<float4 *>(PP);
  SLAB4_LOOP_BEGIN(q)
  const float4 e = ae[e4], a = ap[e4], r = rr[e4], p = pp[e4];
  float4 x = xw[e4], rn, pn;
#define UPD3_(c)                                                   \
  x.c = (float)(x.c + (alpha * p.c + omega * r.c));                \
  rn.c = (float)(r.c - omega * e.c);                               \
  pn.c = (float)(rn.c + beta * (p.c - omega * a.c));
  UPD3_(x) UPD3_(y) UPD3_(z) UPD3_(w)
#undef UPD3_
  xw[e4] = x;
  rr[e4] = rn;
  pp[e4] = pn;
  SLAB4_LOOP_END
}
__global__ void k_upd3f(SkewGeo q, const float *AE, const float *AP, float *XW, float *RR, float *PP,
                        const SolveState *st) {
  pdl_enter();
  upd3f_body(q, AE, AP, XW, RR, PP, st, blockIdx.x);
}
// OMEGA, the new |RR|^2 and (R0,RR), convergence and BETA from the five
// sums (vf_m1bcgs.f:196-241 regrouped).  A finished solve sets `stop`;
// k_commit turns it into `done` once the last update has run.
__device__ __forceinline__ void fin5_body(const double *rb, long long nrows, SolveState *st, double epsa2,
                                          double epsr2, double div2, int icgmax) {
  if (st->done) return;
  const double rae = block_final(rb, nrows), aeae = block_final(rb + nrows, nrows),
               rrrr = block_final(rb + 2 * nrows, nrows), r0rr = block_final(rb + 3 * nrows, nrows),
               r0ae = block_final(rb + 4 * nrows, nrows);
  if (threadIdx.x != 0) return;
  const double omega = rae / aeae;
  st->omega = omega;
  st->w1 = rae;
  st->w2 = aeae;
  const double xn = rrrr - 2.0 * omega * rae + omega * omega * aeae;
  st->xnorm = xn;
  if (xn <= st->bnorm * epsr2 + epsa2) { st->stop = 1; st->beta = 0.0; return; }
  if (xn > div2) { st->iter = -2; st->stop = 1; st->beta = 0.0; return; }
  const double W1 = r0rr - omega * r0ae;
  st->beta = W1 * st->alpha / (st->S * omega);
  st->S = W1;
  st->iter = st->iter + 1;
  if (st->iter > icgmax) st->stop = 1;
}
__global__ void k_fin5(const double *rb, long long nrows, SolveState *st, double epsa2, double epsr2, double div2,
                       int icgmax) {
  pdl_enter();
  fin5_body(rb, nrows, st, epsa2, epsr2, div2, icgmax);
}
__global__ void k_commit(SolveState *st) {
  pdl_enter();
  if (st->stop) st->done = 1;
}

// ------------------------------------------- mixed-precision conversions
// FP32 copy of the 7 coefficients (DD comes from the FP32 factorisation,
// T from the FP32 forward sweeps).
__device__ __forceinline__ void sys_to_f_elem(const SkewGeo &q, const double *sys, float *sysf, long long e) {
  const long long slab = e / q.T;
  const int t = (int)(e - slab * q.T);
  constexpr int cs[7] = {SYS_AD, SYS_ALI, SYS_ALJ, SYS_ALK, SYS_AUI, SYS_AUJ, SYS_AUK};
#pragma unroll
  for (int c = 0; c < 7; ++c) sysf[sys_at(slab, cs[c], q.T, t)] = (float)sys[sys_at(slab, cs[c], q.T, t)];
}
__global__ void k_sys_to_f(SkewGeo q, const double *sys, float *sysf) {
  pdl_enter();
  const long long n = (long long)q.nb * q.W * q.T;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x)
    sys_to_f_elem(q, sys, sysf, e);
}
// RF = R * scale on INDC != -1 (the right-hand side of an inner solve)
__device__ __forceinline__ void scale_to_f_body(SkewGeo q, const int *INDC, const double *R, double scale, float *RF, unsigned BX_) {
  SLAB_LOOP_BEGIN(q)
  if (INDC[e] != -1) RF[e] = (float)(R[e] * scale);
  SLAB_LOOP_END
}
__global__ void k_scale_to_f(SkewGeo q, const int *INDC, const double *R, double scale, float *RF) {
  pdl_enter();
  scale_to_f_body(q, INDC, R, scale, RF, blockIdx.x);
}
// X = X + D * inv_scale on INDC != -1 (the correction of an inner solve)
__device__ __forceinline__ void add_f_body(SkewGeo q, const int *INDC, const float *D, double inv_scale, double *X, unsigned BX_) {
  SLAB_LOOP_BEGIN(q)
  if (INDC[e] != -1) X[e] = X[e] + (double)D[e] * inv_scale;
  SLAB_LOOP_END
}
__global__ void k_add_f(SkewGeo q, const int *INDC, const float *D, double inv_scale, double *X) {
  pdl_enter();
  add_f_body(q, INDC, D, inv_scale, X, blockIdx.x);
}

// X0 = XW on INDC != -1 when ITER >= 0 (vf_m1bcgs.f:251-261), back to the
// standard layout.
__device__ __forceinline__ void x0_body(Geo g, SkewGeo q, const int *INDC, const double *XW, double *X0, const SolveState *st, unsigned BX_) {
  if (st->iter < 0) return;
  SLAB_LOOP_BEGIN(q)
  if (INDC[e] != -1) {
    const int ti = t_ % q.TIp, tj = t_ / q.TIp;
    const int w = (int)(slab_ % q.W), b = (int)(slab_ / q.W);
    const int I = 2 + (b % q.ntx) * q.TI + ti, J = 2 + (b / q.ntx) * q.TJ + tj, k = 2 + w - ti - tj;
    X0[cid(g, I, J, k)] = XW[e];
  }
  SLAB_LOOP_END
}
__global__ void k_x0(Geo g, SkewGeo q, const int *INDC, const double *XW, double *X0, const SolveState *st) {
  pdl_enter();
  x0_body(g, q, INDC, XW, X0, st, blockIdx.x);
}

// ||b-Ax||^2 and ||b||^2 slab partials (diagnostic of the metric)
__global__ void k_relres(Geo g, SkewGeo q, SkewSys S, const double *B, const double *X, double *rb0,
                         double *rb1) {
  pdl_enter();
  const unsigned BX_ = blockIdx.x;
  double s0 = 0.0, s1 = 0.0;
  const long long nslab = (long long)q.nb * q.W;
  SLAB_LOOP_BEGIN(q)
  if (S.indc[e] != -1) {
    double r = B[e] - skew_ax(g, q, S, X, e);
    s0 = s0 + r * r;
    s1 = s1 + B[e] * B[e];
  }
  SLAB_LOOP_END
  slab_store(s0, rb0, nslab, BX_);
  slab_store(s1, rb1, nslab, BX_);
}

// ------------------------------------------------------------- finalisers
// One block of 1024 threads: reduce the row partials and advance the
// BiCGSTAB scalars exactly as the host code of vf_m1bcgs.f would.
__device__ __forceinline__ void fin_body(int mode, const double *rb0, const double *rb1, long long nrows,
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
__global__ void k_fin(int mode, const double *rb0, const double *rb1, long long nrows,
                      SolveState *st, double *out, double epsa2, double epsr2, double div2,
                      int icgmax) {
  pdl_enter();
  fin_body(mode, rb0, rb1, nrows, st, out, epsa2, epsr2, div2, icgmax);
}

// Factorisation failure ends the solve with ITER = -1 (vf_m1bcgs.f:101-102).
__global__ void k_pivot_check(SolveState *st) {
  pdl_enter();
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
    } else if (IS > 0 && (indb(f, 3, IS) == 4 || (indb(f, 3, IS) == 5 && fixlvl_face(g, p, indb(f, 2, IS), I, J)))) {
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
    } else if (IS > 0 && (indb(f, 3, IS) == 4 || (indb(f, 3, IS) == 5 && fixlvl_face(g, p, indb(f, 2, IS), I, J)))) {
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
static int ring_depth(int NV, int T, size_t es) {
  const size_t cap = 200 * 1024;
  for (int d : {8, 4, 2, 1})
    if (ring_bytes(NV, T, d + 3, es) <= cap) return d;
  return 0;
}
// Launch a kernel that starts with pdl_enter() with programmatic stream
// serialisation (cluster dimensions optional).
template <typename... KArgs, typename... Args>
static void launch_pdl(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, int cluster_y,
                       Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid; cfg.blockDim = block; cfg.dynamicSmemBytes = smem; cfg.stream = s;
  cudaLaunchAttribute at[2];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  int na = 1;
  if (cluster_y > 1) {
    at[1].id = cudaLaunchAttributeClusterDimension;
    at[1].val.clusterDim.x = 1; at[1].val.clusterDim.y = (unsigned)cluster_y; at[1].val.clusterDim.z = 1;
    na = 2;
  }
  cfg.attrs = at; cfg.numAttrs = na;
  cudaLaunchKernelEx(&cfg, kern, ((KArgs)args)...);
  count_launch();
}
// The kernel's dynamic shared-memory limit, raised to the bytes of this
// launch and never lowered: handles stepped from several host threads at
// once (cadmas_step_ensemble) with different tile shapes then never lower
// it under one another's launches.
template <class K> static void set_smem(K kern, size_t bytes) {
  raise_dynamic_smem((const void *)kern, bytes);
}

static inline dim3 skew_grid(const SkewGeo &q) { return dim3((unsigned)q.ntx, (unsigned)(q.nb / q.ntx)); }

void launch_to_skew(cudaStream_t s, const Geo &g, const SkewGeo &q, const SysPtr &a, const int *indc,
                    const SkewSys &S, const double *x0, double *bsl, double *xsl, int warm) {
  const size_t rb = to_skew_rows_bytes(g, q);
  if (rb > 0) {
    raise_dynamic_smem((const void *)k_to_skew_rows, rb);
    launch_pdl(k_to_skew_rows, dim3((unsigned)(q.nb * q.TJ)), dim3(128), rb, s, 1, g, q, a, indc, S, x0, bsl, xsl,
               warm);
    return;
  }
  const long long n = (long long)q.nb * q.W * q.T;
  const int blocks = (int)std::min<long long>((n + 255) / 256, 148LL * 16);
  launch_pdl(k_to_skew, dim3(blocks), dim3(256), 0, s, 1, g, q, a, indc, S, x0, bsl, xsl, warm);
}
template <typename V>
static void launch_dcmp_t(cudaStream_t s, const Geo &g, const SkewGeo &q, V U, const SkewSysT<V> &S, int *pivot_bad) {
  const int T = q.T * q.split, d = ring_depth(7, T, sizeof(V));  // one thread per block column
  const size_t bytes = ring_bytes(7, T, d + 3, sizeof(V));
  const int TJb = q.TJ * q.split, nby = (g.NJ - 2 + TJb - 1) / TJb;
  const dim3 grid((unsigned)q.ntx, (unsigned)nby);
  switch (d) {
#define DCMP_CASE(DD)                                                                    \
  case DD:                                                                               \
    set_smem(k_dcmp<DD, V>, bytes);                                                      \
    launch_pdl(k_dcmp<DD, V>, grid, dim3(T), bytes, s, 1, g, q, U, S, pivot_bad);              \
    break;
    DCMP_CASE(8) DCMP_CASE(4) DCMP_CASE(2)
    default: DCMP_CASE(1)
#undef DCMP_CASE
  }
}
void launch_dcmp(cudaStream_t s, const Geo &g, const SkewGeo &q, double U, const SkewSys &S, int *pivot_bad) {
  launch_dcmp_t<double>(s, g, q, U, S, pivot_bad);
}
void launch_dcmp_f(cudaStream_t s, const Geo &g, const SkewGeo &q, double U, const SkewSysF &S, int *pivot_bad) {
  launch_dcmp_t<float>(s, g, q, (float)U, S, pivot_bad);
}
// Sweeps: prefetch depth D in {8, 6, 4, 3, 2}, the largest whose ring
// (R = D+2 slots, mbarriers, exchange buffers) fits the 227 KB of shared
// memory a block may use.
static size_t sweep_bytes(const SkewGeo &q, int mode, int D, int es) {
  const int R = D + 2;
  size_t b = (size_t)((R + 1) & ~1) * 8 + (size_t)R * sweep_slot(q, mode, es) * es + 2 * (size_t)q.T * es;
  if (q.split == 2)  // cluster exchange: xfull[W] barriers, xin (and din) [W][TIp]
    b += (size_t)q.W * 8 + (size_t)q.W * q.TIp * es * (mode >= SWEEP_BWD ? 1 : 2);
  return b;
}
static int sweep_depth(const SkewGeo &q, int mode, int es) {
  if (sweep_threads(q.T) > (q.split == 2 ? 512 : 1024)) return 0;
  for (int d : {8, 6, 4, 3, 2}) {
    if (q.split == 2 && (d == 6 || d == 3)) continue;  // depths built for the cluster form
    if (sweep_bytes(q, mode, d, es) <= 227 * 1024) return d;
  }
  return 0;
}
// Two thread blocks per SM (q.occ == 2): blocks of at most SWEEP2_THREADS
// threads, registers capped for two resident blocks, and a ring that
// leaves room for the second block's (228 KB per SM, 1 KB reserved per
// block).  Two tiles' wavefronts then interleave on every SM.
// The register cap (96 for two 288-thread blocks) makes deeper rings
// spill: depths up to 3 (fused forward sweep, backward sweep with five
// sums) or 4 (the others) are used.
constexpr int SWEEP2_THREADS = 288;
static int sweep_depth2(const SkewGeo &q, int mode, int es) {
  if (q.split != 1 || sweep_threads(q.T) > SWEEP2_THREADS) return 0;
  // 16x16 tiles run the instances with the tile's constants compiled in,
  // which leave room for depth 6 everywhere (8 measured no faster for the
  // forward sweeps and slower for the backward ones)
  const bool t256 = q.T == 256 && q.TIp == 16;
  const int dmax = t256 ? 6 : ((mode == SWEEP_FWD_AX || mode == SWEEP_BWD5) ? 3 : 4);
  for (int d : {6, 4, 3, 2})
    if (d <= dmax && sweep_bytes(q, mode, d, es) <= 113 * 1024) return d;
  return 0;
}
// Four thread blocks per SM: the FP32 backward sweeps of 16x16 tiles, ring
// depth 4 and at most 56 registers, so that up to four tiles per SM run in
// one wave.  By default where the tiles fill more than two blocks per SM
// (on 512 tiles: 19.6 against 23.0 ms of backward sweeps per step of the
// mixed solver), or always with q.occ == 4; the other sweeps follow the
// default's rule then.
static bool sweep_four(const SkewGeo &q, int mode) {
  return (q.occ == 4 || (q.occ == 0 && q.nb > 2 * q.nsm)) && q.split == 1 && mode >= SWEEP_BWD && q.T == 256 &&
         q.TIp == 16 && sweep_bytes(q, mode, 4, 4) <= 55 * 1024;
}
// The default's rule for q.occ 0 and 4.
static int sweep_occ(const SkewGeo &q) { return q.occ == 4 ? 0 : q.occ; }
template <int MODE, typename V>
static void launch_sweep(cudaStream_t s, const Geo &g, const SkewGeo &q, const SkewSysT<V> &S, const V *vin,
                         V *vout, SolveState *st) {
  constexpr int ES = (int)sizeof(V);
  const V *vnull = nullptr;
  double *rnull = nullptr;
  const bool t256 = q.T == 256 && q.TIp == 16;  // 16x16 tiles: the shape's constants compiled in
  const int d = sweep_depth(q, MODE, ES);
  const size_t bytes = sweep_bytes(q, MODE, d, ES);
  const int nty = q.nb / q.ntx;
  const dim3 block((unsigned)sweep_threads(q.T));
  // The register budget follows the block size (255, 128 or 64 registers
  // for blocks of up to 256, 512 or 1024 threads).
  const int nt = sweep_threads(q.T);
  const int mt = nt <= 256 ? 256 : (nt <= 512 ? 512 : 1024);
  if (q.split == 2) {
    // one cluster of two thread blocks per preconditioner block
    const dim3 grid((unsigned)q.ntx, (unsigned)((nty + 1) & ~1));
    switch (d * 4096 + mt) {
#define SWEEP_CASE2(DD, MT)                                                             \
  case DD * 4096 + MT:                                                                  \
    set_smem(k_sweep<DD, MODE, MT, V, 2>, bytes);                                       \
    launch_pdl(k_sweep<DD, MODE, MT, V, 2>, grid, block, bytes, s, 2, g, q, S, vin, vout, st, vnull, rnull); \
    break;
      SWEEP_CASE2(8, 256) SWEEP_CASE2(4, 256) SWEEP_CASE2(2, 256)
      SWEEP_CASE2(8, 512) SWEEP_CASE2(4, 512) SWEEP_CASE2(2, 512)
#undef SWEEP_CASE2
      default: return;  // rejected by cadmas_create (sweep_supported)
    }
    return;
  }
  const dim3 grid = skew_grid(q);
  // Two blocks per SM pay where the tiles fill the SMs twice over: there
  // the sweeps' per-step latency, not the bandwidth, sets the time and a
  // second tile's wavefront fills it.  The fused FP64 forward sweep keeps
  // one block: its ring of 8 arrays needs the depth and registers.
  if constexpr (ES == 4 && MODE >= SWEEP_BWD) {
    if (sweep_four(q, MODE)) {
      const size_t b4 = sweep_bytes(q, MODE, 4, ES);
      set_smem(k_sweep<4, MODE, SWEEP2_THREADS, V, 1, 4, 256, 16>, b4);
      launch_pdl(k_sweep<4, MODE, SWEEP2_THREADS, V, 1, 4, 256, 16>, grid, block, b4, s, 1, g, q, S, vin, vout, st,
                 vnull, rnull);
      return;
    }
  }
  const int oc = sweep_occ(q);
  const bool two = oc == 2 || (oc == 0 && q.nb >= 2 * q.nsm && (ES == 4 || MODE >= SWEEP_BWD));
  if (two) {
    const int d2 = sweep_depth2(q, MODE, ES);
    if (d2 > 0) {
      const size_t bytes2 = sweep_bytes(q, MODE, d2, ES);
      switch (d2) {
#define SWEEP_CASE_OCC2(DD)                                                                            \
  case DD:                                                                                             \
    if (t256) {                                                                                        \
      set_smem(k_sweep<DD, MODE, SWEEP2_THREADS, V, 1, 2, 256, 16>, bytes2);                           \
      launch_pdl(k_sweep<DD, MODE, SWEEP2_THREADS, V, 1, 2, 256, 16>, grid, block, bytes2, s, 1, g, q, S, vin, vout, \
                 st, vnull, rnull);                                                                    \
    } else {                                                                                           \
      set_smem(k_sweep<DD, MODE, SWEEP2_THREADS, V, 1, 2>, bytes2);                                    \
      launch_pdl(k_sweep<DD, MODE, SWEEP2_THREADS, V, 1, 2>, grid, block, bytes2, s, 1, g, q, S, vin, vout, st, vnull, \
                 rnull);                                                                               \
    }                                                                                                  \
    return;
        SWEEP_CASE_OCC2(6) SWEEP_CASE_OCC2(4) SWEEP_CASE_OCC2(3) SWEEP_CASE_OCC2(2)
#undef SWEEP_CASE_OCC2
        default: break;
      }
    }
  }
  switch (d * 4096 + mt) {
#define SWEEP_CASE(DD, MT)                                                              \
  case DD * 4096 + MT:                                                                  \
    if (MT == 512 && t256) {                                                            \
      constexpr int CT_ = MT == 512 ? 256 : 0, CI_ = MT == 512 ? 16 : 0;                \
      set_smem(k_sweep<DD, MODE, MT, V, 1, 1, CT_, CI_>, bytes);                        \
      launch_pdl(k_sweep<DD, MODE, MT, V, 1, 1, CT_, CI_>, grid, block, bytes, s, 1, g, q, S, vin, vout, st, vnull, \
                 rnull);                                                                \
    } else {                                                                            \
      set_smem(k_sweep<DD, MODE, MT, V, 1>, bytes);                                     \
      launch_pdl(k_sweep<DD, MODE, MT, V, 1>, grid, block, bytes, s, 1, g, q, S, vin, vout, st, vnull, rnull); \
    }                                                                                   \
    break;
    SWEEP_CASE(8, 256) SWEEP_CASE(6, 256) SWEEP_CASE(4, 256) SWEEP_CASE(3, 256) SWEEP_CASE(2, 256)
    SWEEP_CASE(8, 512) SWEEP_CASE(6, 512) SWEEP_CASE(4, 512) SWEEP_CASE(3, 512) SWEEP_CASE(2, 512)
    SWEEP_CASE(8, 1024) SWEEP_CASE(6, 1024) SWEEP_CASE(4, 1024) SWEEP_CASE(3, 1024) SWEEP_CASE(2, 1024)
#undef SWEEP_CASE
    default: return;  // rejected by cadmas_create (sweep_supported)
  }
}
bool sweep_supported(const SkewGeo &q) {
  const int tb = q.T * q.split;  // threads of the factorisation kernel
  return sweep_depth(q, SWEEP_FWD, 8) > 0 && sweep_depth(q, SWEEP_BWD, 8) > 0 &&
         (q.split == 1 || sweep_depth(q, SWEEP_FWD_AX, 8) > 0) && tb <= 1024 && ring_depth(7, tb, 8) > 0;
}
bool sweep_supported_f(const SkewGeo &q) {
  const int tb = q.T * q.split;
  return sweep_depth(q, SWEEP_FWD, 4) > 0 && sweep_depth(q, SWEEP_BWD, 4) > 0 &&
         (q.split == 1 || sweep_depth(q, SWEEP_FWD_AX, 4) > 0) && tb <= 1024 && ring_depth(7, tb, 4) > 0;
}
template <typename V>
static void launch_fwd_t(cudaStream_t s, const Geo &g, const SkewGeo &q, const SkewSysT<V> &S, const V *y,
                         const V *spmv_x, SolveState *st, V *ybuf) {
  if (spmv_x && sweep_depth(q, SWEEP_FWD_AX, (int)sizeof(V)) == 0) {
    // Ring of the fused sweep too large for this tile: SpMV first.
    launch_spmv_t<V>(s, g, q, S, spmv_x, ybuf, st);
    y = ybuf;
    spmv_x = nullptr;
  }
  if (spmv_x) launch_sweep<SWEEP_FWD_AX, V>(s, g, q, S, spmv_x, nullptr, st);
  else launch_sweep<SWEEP_FWD, V>(s, g, q, S, y, nullptr, st);
}
void launch_fwd(cudaStream_t s, const Geo &g, const SkewGeo &q, const SkewSys &S, const double *y,
                const double *spmv_x, SolveState *st, double *ybuf) {
  launch_fwd_t<double>(s, g, q, S, y, spmv_x, st, ybuf);
}
void launch_fwd_f(cudaStream_t s, const Geo &g, const SkewGeo &q, const SkewSysF &S, const float *y,
                  const float *spmv_x, SolveState *st, float *ybuf) {
  launch_fwd_t<float>(s, g, q, S, y, spmv_x, st, ybuf);
}
void launch_bwd(cudaStream_t s, const Geo &g, const SkewGeo &q, const SkewSys &S, double *x, SolveState *st) {
  launch_sweep<SWEEP_BWD, double>(s, g, q, S, nullptr, x, st);
}
void launch_bwd_f(cudaStream_t s, const Geo &g, const SkewGeo &q, const SkewSysF &S, float *x, SolveState *st) {
  launch_sweep<SWEEP_BWD, float>(s, g, q, S, nullptr, x, st);
}
// The FP32 backward sweep with the inner products that follow it summed
// on the way (mode 3: (R0,X); mode 4: the five sums of k_dot5f), one
// partial per tile into rb (rb + c*nb for sum c).  Ring depths 2..4, one
// layout tile per preconditioner block, blocks of up to 512 threads;
// false (nothing launched) where that does not hold.
template <int MODE>
static bool launch_bwd_dots(cudaStream_t s, const Geo &g, const SkewGeo &q, const SkewSysF &S, const float *r0,
                            const float *rr, float *x, double *rb, SolveState *st) {
  constexpr int ES = 4;
  if (q.split != 1) return false;
  const bool t256 = q.T == 256 && q.TIp == 16;
  const dim3 grid = skew_grid(q), block((unsigned)sweep_threads(q.T));
  if (sweep_four(q, MODE)) {
    const size_t b4 = sweep_bytes(q, MODE, 4, ES);
    set_smem(k_sweep<4, MODE, SWEEP2_THREADS, float, 1, 4, 256, 16>, b4);
    launch_pdl(k_sweep<4, MODE, SWEEP2_THREADS, float, 1, 4, 256, 16>, grid, block, b4, s, 1, g, q, S, r0, x, st, rr,
               rb);
    return true;
  }
  const int oc = sweep_occ(q);
  const bool two = oc == 2 || (oc == 0 && q.nb >= 2 * q.nsm);
  if (two) {
    const int d2 = sweep_depth2(q, MODE, ES);
    const size_t bytes2 = sweep_bytes(q, MODE, d2, ES);
    switch (d2) {
#define DOTS_OCC2(DD)                                                                                              \
  case DD:                                                                                                         \
    if (t256) {                                                                                                    \
      set_smem(k_sweep<DD, MODE, SWEEP2_THREADS, float, 1, 2, 256, 16>, bytes2);                                   \
      launch_pdl(k_sweep<DD, MODE, SWEEP2_THREADS, float, 1, 2, 256, 16>, grid, block, bytes2, s, 1, g, q, S, r0, x, \
                 st, rr, rb);                                                                                      \
    } else {                                                                                                       \
      set_smem(k_sweep<DD, MODE, SWEEP2_THREADS, float, 1, 2>, bytes2);                                            \
      launch_pdl(k_sweep<DD, MODE, SWEEP2_THREADS, float, 1, 2>, grid, block, bytes2, s, 1, g, q, S, r0, x, st, rr, rb); \
    }                                                                                                              \
    return true;
      DOTS_OCC2(6) DOTS_OCC2(4) DOTS_OCC2(3) DOTS_OCC2(2)
#undef DOTS_OCC2
      default: break;
    }
  }
  const int d = std::min(sweep_depth(q, MODE, ES), 4), nt = sweep_threads(q.T);
  const int mt = nt <= 256 ? 256 : (nt <= 512 ? 512 : 0);
  if (mt == 0 || d < 2) return false;
  const size_t bytes = sweep_bytes(q, MODE, d, ES);
  switch (d * 4096 + mt) {
#define DOTS_CASE(DD, MT)                                                                            \
  case DD * 4096 + MT:                                                                               \
    if (MT == 512 && t256) {                                                                         \
      constexpr int CT_ = MT == 512 ? 256 : 0, CI_ = MT == 512 ? 16 : 0;                             \
      set_smem(k_sweep<DD, MODE, MT, float, 1, 1, CT_, CI_>, bytes);                                 \
      launch_pdl(k_sweep<DD, MODE, MT, float, 1, 1, CT_, CI_>, grid, block, bytes, s, 1, g, q, S, r0, x, st, rr, rb); \
    } else {                                                                                         \
      set_smem(k_sweep<DD, MODE, MT, float, 1>, bytes);                                              \
      launch_pdl(k_sweep<DD, MODE, MT, float, 1>, grid, block, bytes, s, 1, g, q, S, r0, x, st, rr, rb); \
    }                                                                                                \
    return true;
    DOTS_CASE(4, 256) DOTS_CASE(3, 256) DOTS_CASE(2, 256) DOTS_CASE(4, 512) DOTS_CASE(3, 512) DOTS_CASE(2, 512)
#undef DOTS_CASE
    default: return false;
  }
}
bool launch_bwd_f_dot1(cudaStream_t s, const Geo &g, const SkewGeo &q, const SkewSysF &S, const float *r0, float *x,
                       double *rb, SolveState *st) {
  return launch_bwd_dots<SWEEP_BWD1>(s, g, q, S, r0, nullptr, x, rb, st);
}
bool launch_bwd_f_dot5(cudaStream_t s, const Geo &g, const SkewGeo &q, const SkewSysF &S, const float *r0,
                       const float *rr, float *x, double *rb, SolveState *st) {
  return launch_bwd_dots<SWEEP_BWD5>(s, g, q, S, r0, rr, x, rb, st);
}
static inline unsigned slab_blocks(const SkewGeo &q) {
  return (unsigned)(((long long)q.nb * q.W + ROWS_PER_BLOCK - 1) / ROWS_PER_BLOCK);
}
#define SL(kern, ...) launch_pdl(kern, dim3(slab_blocks(q)), dim3(ROW_THREADS), 0, s, 1, __VA_ARGS__)
template <typename V>
void launch_spmv_t(cudaStream_t s, const Geo &g, const SkewGeo &q, const SkewSysT<V> &S, const V *x, V *y,
                   const SolveState *st) { SL(k_spmv<V>, g, q, S, x, y, st); }
void launch_spmv(cudaStream_t s, const Geo &g, const SkewGeo &q, const SkewSys &S, const double *x, double *y,
                 const SolveState *st) { launch_spmv_t<double>(s, g, q, S, x, y, st); }
void launch_bmy(cudaStream_t s, const SkewGeo &q, const int *indc, const double *b, double *y,
                const SolveState *st) { SL(k_bmy, q, indc, b, y, st); }
template <typename V>
void launch_dot_t(cudaStream_t s, const SkewGeo &q, const int *indc, const V *x0, const V *y0, const V *x1,
                  const V *y1, double *rb0, double *rb1, const SolveState *st) {
  SL(k_dot<V>, q, indc, x0, y0, x1, y1, rb0, rb1, st);
}
template <typename V>
void launch_copy2_t(cudaStream_t s, const SkewGeo &q, const int *indc, const V *r0, V *rr, V *pp,
                    const SolveState *st) { SL(k_copy2<V>, q, indc, r0, rr, pp, st); }
template <typename V>
void launch_axpy_rr_t(cudaStream_t s, const SkewGeo &q, const int *indc, const V *ap, V *rr,
                      const SolveState *st) { SL(k_axpy_rr<V>, q, indc, ap, rr, st); }
template <typename V>
void launch_upd_xr_t(cudaStream_t s, const SkewGeo &q, const int *indc, const V *pp, const V *ae, const V *r0,
                     V *xw, V *rr, double *rb0, double *rb1, const SolveState *st) {
  SL(k_upd_xr<V>, q, indc, pp, ae, r0, xw, rr, rb0, rb1, st);
}
template <typename V>
void launch_upd_p_t(cudaStream_t s, const SkewGeo &q, const int *indc, const V *rr, const V *ap, V *pp,
                    const SolveState *st) { SL(k_upd_p<V>, q, indc, rr, ap, pp, st); }
template void launch_spmv_t<double>(cudaStream_t, const Geo &, const SkewGeo &, const SkewSysT<double> &,
                                    const double *, double *, const SolveState *);
template void launch_spmv_t<float>(cudaStream_t, const Geo &, const SkewGeo &, const SkewSysT<float> &,
                                   const float *, float *, const SolveState *);
template void launch_dot_t<double>(cudaStream_t, const SkewGeo &, const int *, const double *, const double *,
                                   const double *, const double *, double *, double *, const SolveState *);
template void launch_dot_t<float>(cudaStream_t, const SkewGeo &, const int *, const float *, const float *,
                                  const float *, const float *, double *, double *, const SolveState *);
template void launch_copy2_t<double>(cudaStream_t, const SkewGeo &, const int *, const double *, double *,
                                     double *, const SolveState *);
template void launch_copy2_t<float>(cudaStream_t, const SkewGeo &, const int *, const float *, float *, float *,
                                    const SolveState *);
template void launch_axpy_rr_t<double>(cudaStream_t, const SkewGeo &, const int *, const double *, double *,
                                       const SolveState *);
template void launch_axpy_rr_t<float>(cudaStream_t, const SkewGeo &, const int *, const float *, float *,
                                      const SolveState *);
template void launch_upd_xr_t<double>(cudaStream_t, const SkewGeo &, const int *, const double *, const double *,
                                      const double *, double *, double *, double *, double *, const SolveState *);
template void launch_upd_xr_t<float>(cudaStream_t, const SkewGeo &, const int *, const float *, const float *,
                                     const float *, float *, float *, double *, double *, const SolveState *);
template void launch_upd_p_t<double>(cudaStream_t, const SkewGeo &, const int *, const double *, const double *,
                                     double *, const SolveState *);
template void launch_upd_p_t<float>(cudaStream_t, const SkewGeo &, const int *, const float *, const float *,
                                    float *, const SolveState *);
void launch_dot(cudaStream_t s, const SkewGeo &q, const int *indc, const double *x0, const double *y0,
                const double *x1, const double *y1, double *rb0, double *rb1, const SolveState *st) {
  launch_dot_t<double>(s, q, indc, x0, y0, x1, y1, rb0, rb1, st);
}
void launch_copy2(cudaStream_t s, const SkewGeo &q, const int *indc, const double *r0, double *rr, double *pp,
                  const SolveState *st) { launch_copy2_t<double>(s, q, indc, r0, rr, pp, st); }
void launch_axpy_rr(cudaStream_t s, const SkewGeo &q, const int *indc, const double *ap, double *rr,
                    const SolveState *st) { launch_axpy_rr_t<double>(s, q, indc, ap, rr, st); }
void launch_upd_xr(cudaStream_t s, const SkewGeo &q, const int *indc, const double *pp, const double *ae,
                   const double *r0, double *xw, double *rr, double *rb0, double *rb1, const SolveState *st) {
  launch_upd_xr_t<double>(s, q, indc, pp, ae, r0, xw, rr, rb0, rb1, st);
}
void launch_upd_p(cudaStream_t s, const SkewGeo &q, const int *indc, const double *rr, const double *ap,
                  double *pp, const SolveState *st) { launch_upd_p_t<double>(s, q, indc, rr, ap, pp, st); }
void launch_x0(cudaStream_t s, const Geo &g, const SkewGeo &q, const int *indc, const double *xw, double *x0,
               const SolveState *st) { SL(k_x0, g, q, indc, xw, x0, st); }
void launch_relres(cudaStream_t s, const Geo &g, const SkewGeo &q, const SkewSys &S, const double *b,
                   const double *x, double *rb0, double *rb1) { SL(k_relres, g, q, S, b, x, rb0, rb1); }
void launch_dot2f(cudaStream_t s, const SkewGeo &q, const float *r0, const float *ap, double *rb,
                  const SolveState *st) { SL(k_dot2f, q, r0, ap, rb, st); }
void launch_axpyf(cudaStream_t s, const SkewGeo &q, const float *ap, float *rr, const SolveState *st) {
  SL(k_axpyf, q, ap, rr, st);
}
void launch_dot5f(cudaStream_t s, const SkewGeo &q, const float *r0, const float *rr, const float *ae, double *rb,
                  const SolveState *st) { SL(k_dot5f, q, r0, rr, ae, rb, st); }
void launch_upd3f(cudaStream_t s, const SkewGeo &q, const float *ae, const float *ap, float *xw, float *rr,
                  float *pp, const SolveState *st) { SL(k_upd3f, q, ae, ap, xw, rr, pp, st); }
void launch_fin5(cudaStream_t s, const double *rb, long long nrows, SolveState *st, double epsa2, double epsr2,
                 double div2, int icgmax) {
  launch_pdl(k_fin5, dim3(1), dim3(1024), 0, s, 1, rb, nrows, st, epsa2, epsr2, div2, icgmax);
}
void launch_commit(cudaStream_t s, SolveState *st) { launch_pdl(k_commit, dim3(1), dim3(1), 0, s, 1, st); }
void launch_sys_to_f(cudaStream_t s, const SkewGeo &q, const double *sys, float *sysf) {
  const long long n = (long long)q.nb * q.W * q.T;
  launch_pdl(k_sys_to_f, dim3((unsigned)std::min<long long>((n + 255) / 256, 148LL * 16)), dim3(256), 0, s, 1, q, sys,
             sysf);
}
void launch_scale_to_f(cudaStream_t s, const SkewGeo &q, const int *indc, const double *r, double scale,
                       float *rf) { SL(k_scale_to_f, q, indc, r, scale, rf); }
void launch_add_f(cudaStream_t s, const SkewGeo &q, const int *indc, const float *d, double inv_scale,
                  double *x) { SL(k_add_f, q, indc, d, inv_scale, x); }
#undef SL
void launch_fin(cudaStream_t s, int mode, const double *rb0, const double *rb1, long long nrows,
                SolveState *st, double *out, double epsa2, double epsr2, double div2, int icgmax) {
  launch_pdl(k_fin, dim3(1), dim3(1024), 0, s, 1, mode, rb0, rb1, nrows, st, out, epsa2, epsr2, div2, icgmax);
}
void launch_pivot_check(cudaStream_t s, SolveState *st) {
  launch_pdl(k_pivot_check, dim3(1), dim3(1), 0, s, 1, st);
}
void launch_vmodif(cudaStream_t s, const Geo &g, const Fld &f, const Prm &p, const double *pt) {
  k_vmodif<<<row_blocks(g), ROW_THREADS, 0, s>>>(g, f, p, pt);
  count_launch();
}


// ---------------------------------------------------- batched solves
// A block's member: the largest m with pre[m] <= blk (pre ascending).
__device__ __forceinline__ int batch_member(const int *pre, int nm, int blk) {
  int lo = 0, hi = nm - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (pre[mid] <= blk) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}
#define BATCH_BLOCK(range)                                                     \
  const int *pr_ = pre + (range) * (nm + 1);                                   \
  const int m_ = batch_member(pr_, nm, (int)blockIdx.x);                       \
  const BatchMember &M = bm[m_];                                               \
  const unsigned lb_ = blockIdx.x - (unsigned)pr_[m_];

__global__ void kb_to_skew(const BatchMember *bm, const int *pre, int nm) {
  pdl_enter();
  BATCH_BLOCK(BR_ELEM)
  if (!M.active) return;
  const long long e = (long long)lb_ * BATCH_ELEM + threadIdx.x;
  if (e < (long long)M.q.nb * M.q.W * M.q.T)
    to_skew_elem(M.g, M.q, M.a, M.indc, M.S, M.pt, M.vd[BD_B], M.vd[BD_X], M.warm, e);
}
__global__ void kb_sys_to_f(const BatchMember *bm, const int *pre, int nm) {
  pdl_enter();
  BATCH_BLOCK(BR_ELEM)
  if (!M.active) return;
  const long long e = (long long)lb_ * BATCH_ELEM + threadIdx.x;
  if (e < (long long)M.q.nb * M.q.W * M.q.T) sys_to_f_elem(M.q, M.S.sys, M.Sf.sys, e);
}
template <int D>
__global__ void kb_dcmp_f(const BatchMember *bm, const int *pre, int nm) {
  pdl_enter();
  BATCH_BLOCK(BR_TILE)
  if (!M.active) return;
  dcmp_body<D, float>(M.g, M.q, (float)M.U, M.Sf, M.pivot_bad, (int)(lb_ % M.q.ntx), (int)(lb_ / M.q.ntx));
}
template <int D, int MODE, int MAXT, int MINB, int CT = 0, int CTIP = 0>
__global__ void __launch_bounds__(MAXT, MINB) kb_sweep(const BatchMember *bm, const int *pre, int nm, int vin,
                                                       int vout, int vin2, int rb5) {
  pdl_enter();
  BATCH_BLOCK(BR_TILE)
  sweep_body<D, MODE, float, 1, CT, CTIP>(M.g, M.q, M.Sf, vin >= 0 ? M.vf[vin] : nullptr, vout >= 0 ? M.vf[vout] : nullptr,
                                M.st, vin2 >= 0 ? M.vf[vin2] : nullptr, rb5 ? M.rb5 : M.rb0,
                                (int)(lb_ % M.q.ntx), (int)(lb_ / M.q.ntx));
}
// the solve state of every member cleared up to the wait limit; members
// outside the pass marked done, so every solver kernel skips them
__global__ void kb_clear(const BatchMember *bm, int nm) {
  pdl_enter();
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= nm) return;
  unsigned char *p = reinterpret_cast<unsigned char *>(bm[m].st);
  for (int i = 0; i < (int)SOLVE_CLEAR_BYTES; ++i) p[i] = 0;
  bm[m].st->done = bm[m].active ? 0 : 1;
  if (bm[m].pivot_bad) *bm[m].pivot_bad = 0;
}
__global__ void kb_gather(const BatchMember *bm, int nm, double *out) {
  pdl_enter();
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= nm) return;
  const SolveState *st = bm[m].st;
  double *o = out + (long long)m * BATCH_GATHER;
  o[0] = st->done; o[1] = st->timeout; o[2] = st->iter; o[3] = st->pivot_bad;
  o[4] = bm[m].dres[6]; o[5] = bm[m].dres[7];
}
// r = b - A x in FP64 and the slab partials of (b,b) and (r,r)
__global__ void kb_residual(const BatchMember *bm, const int *pre, int nm, int part) {
  pdl_enter();
  BATCH_BLOCK(BR_SLAB)
  if (part == 0) spmv_body<double>(M.g, M.q, M.S, M.vd[BD_X], M.vd[BD_Y2], M.st, lb_);
  else if (part == 1) bmy_body(M.q, M.S.indc, M.vd[BD_B], M.vd[BD_Y2], M.st, lb_);
  else dot_body<double>(M.q, M.S.indc, M.vd[BD_B], M.vd[BD_B], M.vd[BD_Y2], M.vd[BD_Y2], M.rb0, M.rb1, M.st, lb_);
}
// one block per member: the finaliser of its sums (tile partials after a
// backward sweep with sums, slab-block partials otherwise)
__global__ void kb_fin(const BatchMember *bm, int nm, int mode, int tile_partials) {
  pdl_enter();
  const BatchMember &M = bm[blockIdx.x];
  if (mode == FIN_STORE && !M.active) return;
  const long long nrows = tile_partials ? (long long)M.q.nb : M.nrb;
  fin_body(mode, M.rb0, mode == FIN_STORE ? M.rb1 : nullptr, nrows, M.st, M.dres + 6, M.epsa2, M.eps2, M.div2,
           M.icgmax);
}
__global__ void kb_fin5(const BatchMember *bm, int nm) {
  pdl_enter();
  const BatchMember &M = bm[blockIdx.x];
  fin5_body(M.rb5, (long long)M.q.nb, M.st, M.epsa2, M.eps2, M.div2, M.icgmax);
}
__global__ void kb_commit(const BatchMember *bm, int nm) {
  pdl_enter();
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m < nm && bm[m].st->stop) bm[m].st->done = 1;
}
// the inner solve's start: BF = R/|r|, its vectors zeroed
__global__ void kb_start_f(const BatchMember *bm, const int *pre, int nm) {
  pdl_enter();
  BATCH_BLOCK(BR_SLAB)
  if (!M.active) return;
  scale_to_f_body(M.q, M.S.indc, M.vd[BD_Y2], M.scale, M.vf[BF_B], lb_);
  const long long slab = (long long)lb_ * ROWS_PER_BLOCK + (threadIdx.x >> 5);
  if (slab < (long long)M.q.nb * M.q.W) {
    const int zs[6] = {BF_X, BF_R0, BF_RR, BF_PV, BF_AP, BF_AE};
    for (int t = threadIdx.x & 31; t < M.q.T; t += 32)
      for (int c = 0; c < 6; ++c) M.vf[zs[c]][slab * M.q.T + t] = 0.0f;
  }
}
__global__ void kb_dot_r0f(const BatchMember *bm, const int *pre, int nm) {
  pdl_enter();
  BATCH_BLOCK(BR_SLAB)
  dot_body<float>(M.q, M.S.indc, M.vf[BF_R0], M.vf[BF_R0], nullptr, nullptr, M.rb0, nullptr, M.st, lb_);
}
__global__ void kb_copy2_f(const BatchMember *bm, const int *pre, int nm) {
  pdl_enter();
  BATCH_BLOCK(BR_SLAB)
  copy2_body<float>(M.q, M.S.indc, M.vf[BF_R0], M.vf[BF_RR], M.vf[BF_PV], M.st, lb_);
}
__global__ void kb_axpyf(const BatchMember *bm, const int *pre, int nm) {
  pdl_enter();
  BATCH_BLOCK(BR_SLAB)
  axpyf_body(M.q, M.vf[BF_AP], M.vf[BF_RR], M.st, lb_);
}
__global__ void kb_upd3f(const BatchMember *bm, const int *pre, int nm) {
  pdl_enter();
  BATCH_BLOCK(BR_SLAB)
  upd3f_body(M.q, M.vf[BF_AE], M.vf[BF_AP], M.vf[BF_X], M.vf[BF_RR], M.vf[BF_PV], M.st, lb_);
}
// XW += |r| D on the members whose inner solve ended within ICGMAX
__global__ void kb_add_f(const BatchMember *bm, const int *pre, int nm) {
  pdl_enter();
  BATCH_BLOCK(BR_SLAB)
  if (!M.active || M.st->iter < 0 || M.st->iter > M.icgmax) return;
  add_f_body(M.q, M.S.indc, M.vf[BF_X], M.rn, M.vd[BD_X], lb_);
}
__global__ void kb_x0(const BatchMember *bm, const int *pre, int nm) {
  pdl_enter();
  BATCH_BLOCK(BR_SLAB)
  if (!M.active) return;
  x0_body(M.g, M.q, M.S.indc, M.vd[BD_X], M.pt, M.st, lb_);
}
#undef BATCH_BLOCK

static inline dim3 bgrid(long long n) { return dim3((unsigned)n); }
void launch_b_to_skew(cudaStream_t s, const BatchMember *bm, const int *pre, int nm, long long nblk) {
  launch_pdl(kb_to_skew, bgrid(nblk), dim3(BATCH_ELEM), 0, s, 1, bm, pre, nm);
}
void launch_b_sys_to_f(cudaStream_t s, const BatchMember *bm, const int *pre, int nm, long long nblk) {
  launch_pdl(kb_sys_to_f, bgrid(nblk), dim3(BATCH_ELEM), 0, s, 1, bm, pre, nm);
}
bool launch_b_dcmp_f(cudaStream_t s, const BatchMember *bm, const int *pre, int nm, long long ntiles, int T) {
  const int d = ring_depth(7, T, sizeof(float));
  const size_t bytes = ring_bytes(7, T, d + 3, sizeof(float));
  switch (d) {
#define BDCMP(DD)                                                                          \
  case DD:                                                                                 \
    set_smem(kb_dcmp_f<DD>, bytes);                                                        \
    launch_pdl(kb_dcmp_f<DD>, bgrid(ntiles), dim3(T), bytes, s, 1, bm, pre, nm);          \
    return true;
    BDCMP(8) BDCMP(4) BDCMP(2) BDCMP(1)
#undef BDCMP
    default: return false;
  }
}
// The batched FP32 sweeps: two blocks per SM (the rule of launch_sweep,
// counted over all the members' tiles) or one, ring depths 2..4.
static int b_sweep_depth(const SkewGeo &q, int mode, bool two) {
  return two ? sweep_depth2(q, mode, 4) : std::min(sweep_depth(q, mode, 4), 4);
}
static bool b_two(const SkewGeo &q, int nsm, int occ, long long ntiles) {
  return occ == 2 || ((occ == 0 || occ == 4) && ntiles >= 2LL * nsm);
}
bool b_sweeps_supported(const SkewGeo &q, int nsm, int occ, long long ntiles) {
  if (q.split != 1 || sweep_threads(q.T) > 512) return false;
  const bool two = b_two(q, nsm, occ, ntiles) && sweep_threads(q.T) <= SWEEP2_THREADS;
  for (int mode : {(int)SWEEP_FWD, (int)SWEEP_FWD_AX, (int)SWEEP_BWD, (int)SWEEP_BWD1, (int)SWEEP_BWD5})
    if (b_sweep_depth(q, mode, two) < 2) return false;
  return true;
}
template <int MODE>
static bool launch_b_sweep_t(cudaStream_t s, const BatchMember *bm, const int *pre, int nm, long long ntiles,
                             const SkewGeo &q, int vin, int vout, int vin2, int rb5, int nsm, int occ) {
  const bool two = b_two(q, nsm, occ, ntiles) && sweep_threads(q.T) <= SWEEP2_THREADS;
  const int d = b_sweep_depth(q, MODE, two);
  if (d < 2) return false;
  const bool t256 = q.T == 256 && q.TIp == 16;
  const size_t bytes = sweep_bytes(q, MODE, d, 4);
  const dim3 block((unsigned)sweep_threads(q.T));
  switch (d * 2 + (two ? 1 : 0)) {
#define BSWEEP(DD, TWO, MT, MB)                                                                        \
  case DD * 2 + TWO:                                                                                   \
    if (t256) {                                                                                        \
      set_smem(kb_sweep<DD, MODE, MT, MB, 256, 16>, bytes);                                            \
      launch_pdl(kb_sweep<DD, MODE, MT, MB, 256, 16>, bgrid(ntiles), block, bytes, s, 1, bm, pre, nm, vin, vout, \
                 vin2, rb5);                                                                           \
    } else {                                                                                           \
      set_smem(kb_sweep<DD, MODE, MT, MB>, bytes);                                                     \
      launch_pdl(kb_sweep<DD, MODE, MT, MB>, bgrid(ntiles), block, bytes, s, 1, bm, pre, nm, vin, vout, vin2, rb5); \
    }                                                                                                  \
    return true;
    BSWEEP(2, 1, SWEEP2_THREADS, 2) BSWEEP(3, 1, SWEEP2_THREADS, 2) BSWEEP(4, 1, SWEEP2_THREADS, 2)
    BSWEEP(6, 1, SWEEP2_THREADS, 2)
    BSWEEP(2, 0, 512, 1) BSWEEP(3, 0, 512, 1) BSWEEP(4, 0, 512, 1)
#undef BSWEEP
    default: return false;
  }
}
bool launch_b_sweep(cudaStream_t s, int mode, const BatchMember *bm, const int *pre, int nm, long long ntiles,
                    const SkewGeo &q, int vin, int vout, int vin2, bool rb5, int nsm, int occ) {
  switch (mode) {
    case SWEEP_FWD: return launch_b_sweep_t<SWEEP_FWD>(s, bm, pre, nm, ntiles, q, vin, vout, vin2, rb5, nsm, occ);
    case SWEEP_FWD_AX:
      return launch_b_sweep_t<SWEEP_FWD_AX>(s, bm, pre, nm, ntiles, q, vin, vout, vin2, rb5, nsm, occ);
    case SWEEP_BWD: return launch_b_sweep_t<SWEEP_BWD>(s, bm, pre, nm, ntiles, q, vin, vout, vin2, rb5, nsm, occ);
    case SWEEP_BWD1: return launch_b_sweep_t<SWEEP_BWD1>(s, bm, pre, nm, ntiles, q, vin, vout, vin2, rb5, nsm, occ);
    case SWEEP_BWD5: return launch_b_sweep_t<SWEEP_BWD5>(s, bm, pre, nm, ntiles, q, vin, vout, vin2, rb5, nsm, occ);
    default: return false;
  }
}
// one thread per member
static inline dim3 bmem(int nm) { return dim3((unsigned)((nm + 255) / 256)); }
void launch_b_clear(cudaStream_t s, const BatchMember *bm, int nm) {
  launch_pdl(kb_clear, bmem(nm), dim3(256), 0, s, 1, bm, nm);
}
void launch_b_gather(cudaStream_t s, const BatchMember *bm, int nm, double *out) {
  launch_pdl(kb_gather, bmem(nm), dim3(256), 0, s, 1, bm, nm, out);
}
void launch_b_residual(cudaStream_t s, const BatchMember *bm, const int *pre, int nm, long long nslab) {
  for (int part = 0; part < 3; ++part)
    launch_pdl(kb_residual, bgrid(nslab), dim3(ROW_THREADS), 0, s, 1, bm, pre, nm, part);
}
void launch_b_fin(cudaStream_t s, int mode, const BatchMember *bm, int nm, bool tile_partials) {
  launch_pdl(kb_fin, dim3((unsigned)nm), dim3(1024), 0, s, 1, bm, nm, mode, tile_partials ? 1 : 0);
}
void launch_b_fin5(cudaStream_t s, const BatchMember *bm, int nm) {
  launch_pdl(kb_fin5, dim3((unsigned)nm), dim3(1024), 0, s, 1, bm, nm);
}
void launch_b_commit(cudaStream_t s, const BatchMember *bm, int nm) {
  launch_pdl(kb_commit, bmem(nm), dim3(256), 0, s, 1, bm, nm);
}
#define BSL(kern) launch_pdl(kern, bgrid(nslab), dim3(ROW_THREADS), 0, s, 1, bm, pre, nm)
void launch_b_start_f(cudaStream_t s, const BatchMember *bm, const int *pre, int nm, long long nslab) { BSL(kb_start_f); }
void launch_b_dot_r0f(cudaStream_t s, const BatchMember *bm, const int *pre, int nm, long long nslab) { BSL(kb_dot_r0f); }
void launch_b_copy2_f(cudaStream_t s, const BatchMember *bm, const int *pre, int nm, long long nslab) { BSL(kb_copy2_f); }
void launch_b_axpyf(cudaStream_t s, const BatchMember *bm, const int *pre, int nm, long long nslab) { BSL(kb_axpyf); }
void launch_b_upd3f(cudaStream_t s, const BatchMember *bm, const int *pre, int nm, long long nslab) { BSL(kb_upd3f); }
void launch_b_add_f(cudaStream_t s, const BatchMember *bm, const int *pre, int nm, long long nslab) { BSL(kb_add_f); }
void launch_b_x0(cudaStream_t s, const BatchMember *bm, const int *pre, int nm, long long nslab) { BSL(kb_x0); }
#undef BSL

}  // namespace cadmas
