// cadmas_dev.cuh -- device-side definitions shared by the kernels of
// libcadmas_gpu.so (B200, sm_100a, FP64).
//
// Arithmetic rule for the whole library: every expression is written in the
// operand order of the Fortran routine it restates and compiled with
// --fmad=false, with IEEE division and square root, so that each cell value
// is bit-identical to a sequential evaluation of the same expression.
// Global sums use one fixed tree (row_reduce below); no atomics touch a
// floating-point value.
#pragma once
#include <cstddef>
#include <cuda_runtime.h>
#include <stdint.h>
#include "../../include/cadmas_gpu.h"

namespace cadmas {

// ----------------------------------------------------------------- geometry
struct Geo {
  int NI, NJ, NK, NB;
  long long N;                 // NI*NJ*NK
  const double *XX, *YY, *ZZ;  // (6,N*) metrics
};

__device__ __forceinline__ long long cid(const Geo &g, int i, int j, int k) {
  return (long long)(i - 1) + (long long)g.NI * ((long long)(j - 1) + (long long)g.NJ * (long long)(k - 1));
}
__device__ __forceinline__ double gx(const Geo &g, int m, int i) { return g.XX[(m - 1) + 6 * (i - 1)]; }
__device__ __forceinline__ double gy(const Geo &g, int m, int j) { return g.YY[(m - 1) + 6 * (j - 1)]; }
__device__ __forceinline__ double gz(const Geo &g, int m, int k) { return g.ZZ[(m - 1) + 6 * (k - 1)]; }

// MAX/MIN with the comparison the oracle uses (first operand on ties).
__device__ __forceinline__ double dmax(double a, double b) { return (a < b) ? b : a; }
__device__ __forceinline__ double dmin(double a, double b) { return (b < a) ? b : a; }

// libgfortran's integer power (square and multiply), as x**n compiles.
__device__ __forceinline__ double ipow(double x, int n) {
  double p = 1.0;
  if (n != 0) {
    unsigned u;
    if (n < 0) { u = (unsigned)(-n); x = p / x; } else { u = (unsigned)n; }
    for (;;) {
      if (u & 1u) p *= x;
      u >>= 1;
      if (u) x *= x; else break;
    }
  }
  return p;
}

// -------------------------------------------------------------- parameters
struct Prm {
  double rho0, grz0, vvmax, cgpara, cgepsa, cgepsr, cgdiv, flower, fupper,
      plower, scmvp, wvlvl, wbub, glxmin, glxmax, glymin, glymax;
  double dtnow, tnow;
  int icgtyp, icgmax, ibsuw0;
  // sponge (vf_veuler.f:77-113), precomputed on the host
  int ipa, ip[4];
  double sw[4], spx[4], spz[4];
  // log-law and rough walls (IB 6, 8): kappa, A, ANU0; loglaw = 1 when the
  // grid has such faces
  double akk0, aka0, anu0;
  int loglaw;
  // fixlvl[JD-1] = 1: side JD is a wave side whose table fixes the water
  // level (MTBTYP 3); its faces then act as free faces
  int fixlvl[4];
  // wave source (ISCTYP(1)): IWS > 0 the x source's column I, JWS > 0 the
  // y source's row J (0: none); SRCUV in Fld::srcuv
  int iws, jws;
};

// A boundary face of a fixed-water-level side: on the domain boundary of
// the side its NS names (vf_bwuwn.f:161-216, vf_vmodif.f:89-112,
// vf_bwuwt.f:80-115).
__device__ __forceinline__ bool fixlvl_face(const Geo &g, const Prm &p, int NS, int I, int J) {
  if (NS < 1 || NS > 4 || !p.fixlvl[NS - 1]) return false;
  return NS == 1 ? I == 2 : NS == 2 ? I == g.NI : NS == 3 ? J == 2 : J == g.NJ;
}

// ---------------------------------------------------------- device arrays
struct Fld {
  // static
  const double *ggv, *ggx, *ggy, *ggz, *glv, *glx, *gly, *glz, *cd0, *anu;
  const int *indx, *indy, *indz, *indb;
  // state
  double *uu, *vv, *ww, *pp, *ff;
  int *nf, *indc, *nf0;
  double *bcu, *bcv, *bcw, *bcp, *bcf;
  const double *bcvi;  // BCVI roughness of rough-wall faces
  // SRCUV(NUMIJ,NUMK) of the wave source (NUMIJ = NUMJ for an x source,
  // NUMI for a y source); read only where Prm::iws or jws is set
  const double *srcuv;
};

// DROPTX, DROPTY, DROPTZ, DROPUU, DROPVV, DROPWW of the droplet model
struct DropArrays {
  double *tx, *ty, *tz, *uu, *vv, *ww;
};

// k-epsilon state (AK, AE, ANUT per cell; BCK, BCE and the types INDBK,
// INDBE per boundary face) and the constants of /VF_APHYSR/
struct KeArrays {
  double *ak, *ae, *anut, *bck, *bce;
  const int *indbk, *indbe;
};
struct KeConst {
  double anu0, scmk, akmink, akmine, akinik, akinie, akcmu, aksgk, aksge, akc1, akc2, akc3;
};

__device__ __forceinline__ int indb(const Fld &f, int m, int l) { return f.indb[(m - 1) + 4 * (l - 1)]; }

__device__ __forceinline__ void decode(const Geo &g, int ijk, int &i, int &j, int &k) {
  k = (ijk - 1) / (g.NI * g.NJ) + 1;
  ijk = ijk - g.NI * g.NJ * (k - 1);
  j = (ijk - 1) / g.NI + 1;
  i = ijk - g.NI * (j - 1);
}

// ------------------------------------------------------------ row kernels
// A "row kernel" maps one warp to one x-row (J,K) of the padded grid and
// lets lane l visit I = l+1, l+33, ...  Coalesced for the I-fastest layout,
// and the order in which each lane visits cells is the order of the global
// sums below.
constexpr int ROWS_PER_BLOCK = 8;
constexpr int ROW_THREADS = 32 * ROWS_PER_BLOCK;

inline unsigned row_blocks(const Geo &g) {
  long long rows = (long long)g.NJ * g.NK;
  return (unsigned)((rows + ROWS_PER_BLOCK - 1) / ROWS_PER_BLOCK);
}

#define ROW_LOOP_BEGIN(g)                                                   \
  const int lane_ = threadIdx.x & 31;                                       \
  const long long row_ = (long long)blockIdx.x * ROWS_PER_BLOCK + (threadIdx.x >> 5); \
  if (row_ < (long long)(g).NJ * (g).NK) {                                  \
    const int J = (int)(row_ % (g).NJ) + 1;                                 \
    const int K = (int)(row_ / (g).NJ) + 1;                                 \
    for (int I = lane_ + 1; I <= (g).NI; I += 32) {
#define ROW_LOOP_END \
    }                \
  }

// Programmatic dependent launch.  The solver's kernels are launched with
// programmatic stream serialisation (launch_pdl), so a kernel may be
// scheduled while the previous kernel of the stream still runs.  Each of
// them starts here: wait until the previous kernel has completed and its
// writes are visible, then let the next kernel be scheduled.  Without a
// programmatic dependency the wait returns at once.
__device__ __forceinline__ void pdl_enter() {
  asm volatile("griddepcontrol.wait;\n" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory");
}

// Warp tree: lane 0 ends with ((s0+s16)+(s8+s24))+... via shfl_down.
__device__ __forceinline__ double warp_tree(double s) {
  for (int off = 16; off >= 1; off >>= 1) s = s + __shfl_down_sync(0xffffffffu, s, off);
  return s;
}

// Store the row partial of a row kernel: call with every lane of the warp
// (lanes of an absent row store nothing).
__device__ __forceinline__ void row_store(double s, double *rowbuf, long long row, long long nrows) {
  s = warp_tree(s);
  if ((threadIdx.x & 31) == 0 && row < nrows) rowbuf[row] = s;
}

// Second stage: one block of 1024 threads sums the row partials.
__device__ __forceinline__ double block_final(const double *rowbuf, long long nrows) {
  __shared__ double w[32];
  // thread t sums rows t, t+1024, t+2048, ... in that order; the loads of
  // eight of them are issued before their additions
  double s = 0.0;
  for (long long r0 = threadIdx.x; r0 < nrows; r0 += 8 * 1024) {
    double v[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) v[j] = (r0 + j * 1024 < nrows) ? rowbuf[r0 + j * 1024] : 0.0;
#pragma unroll
    for (int j = 0; j < 8; ++j)
      if (r0 + j * 1024 < nrows) s = s + v[j];
  }
  s = warp_tree(s);
  if ((threadIdx.x & 31) == 0) w[threadIdx.x >> 5] = s;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x < 32) {
    t = w[threadIdx.x];
    t = warp_tree(t);
  }
  __syncthreads();
  return t;  // valid in thread 0
}

// -------------------------------------------------------- solver scalars
struct SolveState {
  double S, alpha, omega, beta, bnorm, xnorm, w1, w2, rn, bn;
  int iter, done, status, pivot_bad;
  int timeout;  // a bulk-copy wait of a sweep ran out of time
  int stop;     // regrouped FP32 iteration: finished, `done` after its last update
  // Set once per handle, kept when a solve clears the fields above (they
  // are read only where a sweep starts to wait, or by its producer warp,
  // so they add nothing to the sweeps' register load):
  //   wait_ns     an mbarrier wait of the sweeps gives up after this long
  //               and the solve ends with CADMAS_ETIMEOUT;
  //   stall_from  the producer warp issues no bulk copy for wavefront
  //               steps >= stall_from (failure injection for tests,
  //               cadmas_test_stall_sweeps; 2^30 otherwise).
  long long wait_ns;
  int stall_from, pad_;
};
// Bytes of SolveState that a new solve clears (everything before wait_ns).
#define SOLVE_CLEAR_BYTES offsetof(cadmas::SolveState, wait_ns)

// Error flags raised by kernels (bitmask in a device int).
enum : int {
  ERR_PG = 1,       // P.G ERROR (unexpected NF in VPCOEF, undetermined direction)
  ERR_CAP = 2,      // iteration cap
  ERR_UNSUP = 4,    // boundary type outside the implemented set
  ERR_NOTCONV = 8,  // the log-law friction velocity did not converge (VF_CLOGLW)
};

}  // namespace cadmas
