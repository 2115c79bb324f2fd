// kernels.h -- host-side launchers of the device kernels (one per file).
#pragma once
#include <cuda_runtime.h>
#include <atomic>
#include "cadmas_dev.cuh"
#include "wavetheory.cuh"

namespace cadmas {

// Kernels launched by this library in the process (cadmas_kernel_launches).
extern std::atomic<long long> g_kernel_launches;
inline void count_launch(long long n = 1) { g_kernel_launches.fetch_add(n, std::memory_order_relaxed); }
// Raise the dynamic shared-memory limit of the kernel at `kern` (on the
// current device) to at least `bytes`; it is never lowered, so handles
// stepped from several host threads at once never take it away from one
// another's launches.
void raise_dynamic_smem(const void *kern, size_t bytes);
// Record the failing CUDA call and its message as the text cadmas_strerror
// gives for CADMAS_ECUDA on this host thread.
void set_cuda_error(const char *call, cudaError_t e);

// The eight arrays of the Poisson system, WK01..WK08 of VF_V1CAL.
struct SysPtr {
  double *ad, *ali, *alj, *alk, *aui, *auj, *auk, *bb;
};

// The constant part of a solve in the tile-skewed layout of the MILU
// kernels (k_poisson.cu).  Nine arrays are interleaved slab by slab,
// sys[(slab*SYS_N + c)*T + t], so the values one wavefront step of a sweep
// needs are one contiguous run: the backward sweep's {T, AUI, AUJ, AUK,
// DD}, the fused forward sweep's {AUI .. ALK} and the plain forward
// sweep's {DD, AD, ALI, ALJ, ALK}.  SYS_T is the forward sweep's result
// T = MINV_L*Y, written by the forward sweep for the backward sweep that
// follows it.  INDC is a plain skewed array.
enum SysArray { SYS_T = 0, SYS_AUI, SYS_AUJ, SYS_AUK, SYS_DD, SYS_AD, SYS_ALI, SYS_ALJ, SYS_ALK, SYS_N };
template <typename V> struct SkewSysT {
  V *sys;
  int *indc;
};
using SkewSys = SkewSysT<double>;
using SkewSysF = SkewSysT<float>;
struct SkewGeo {
  int TI, TJ, TIp, T, W;  // layout tile TI x TJ columns (T = TIp*TJ slots), W slabs per tile
  int ntx, nb;            // layout tiles along x, tiles in total
  int split;  // layout tiles per preconditioner block along y (1 or 2)
  // Thread blocks of the sweeps per SM (k_poisson.cu): 1, 2, or 0 = by
  // the rule of launch_sweep (two for the backward sweeps and the FP32
  // sweeps when there are at least two tiles per SM); nsm = the SMs.
  int occ, nsm;
};

__host__ __device__ inline long long sys_at(long long slab, int c, int T, int t) {
  return (slab * SYS_N + c) * T + t;
}

// Bulk copies of one wavefront step of the MILU sweeps (k_sweep).  A ring
// slot holds NV slabs of T values (slab c at c*T):
// MODE 0: forward sweep of a given vector: {Y, DD, AD, ALI, ALJ, ALK}
//         (AD unused), copies: Y, system arrays DD..ALK;
// MODE 1: forward sweep fused with Y = A*P: {AUI, AUJ, AUK, DD, AD, ALI,
//         ALJ, ALK, P} plus the P values of the four neighbouring tiles at
//         the step's cells (down/up: one row of TIp; left/right: the span
//         of the neighbour's slab from its last/first column of row 0 to
//         that of row TJ-1), copies: system arrays AUI..ALK, P, down, up,
//         left, right;
// MODE 2: backward sweep: {T, AUI, AUJ, AUK, DD}, copy: system arrays
//         T..DD;
// MODE 3, 4: backward sweep that also sums products of its result with
//         given vectors (the BiCGSTAB inner products that follow it):
//         {T, AUI, AUJ, AUK, DD, R0} and {T, AUI, AUJ, AUK, DD, R0, RR},
//         copies: system arrays T..DD, R0 (and RR).
// Offsets are in elements of the sweep's type (es bytes: 8 for double, 4
// for float); `arr` 0 is the interleaved system, 1 the vector (R0 in
// modes 3 and 4), 2 the second vector (RR in mode 4).
enum SweepMode { SWEEP_FWD = 0, SWEEP_FWD_AX = 1, SWEEP_BWD = 2, SWEEP_BWD1 = 3, SWEEP_BWD5 = 4 };
// inner products a backward sweep sums (mode 3: (R0,X); mode 4: (RR,X),
// (X,X), (RR,RR), (R0,RR), (R0,X))
__host__ __device__ constexpr int sweep_ndot(int mode) {
  return mode == SWEEP_BWD1 ? 1 : (mode == SWEEP_BWD5 ? 5 : 0);
}
struct SweepCopy {
  long long src;
  int dst, bytes, arr;
};
__host__ __device__ inline int sweep_nv(int mode) {
  return mode == SWEEP_FWD_AX ? 9 : (mode == SWEEP_FWD ? 6 : 5 + (mode - SWEEP_BWD));
}
__host__ __device__ inline int sweep_ncopy(const SkewGeo &, int mode) {
  return mode == SWEEP_FWD_AX ? 6 : (mode == SWEEP_FWD ? 2 : 1 + (mode - SWEEP_BWD));
}
// First system array of a mode's slot and its position there.
__host__ __device__ constexpr int sweep_sys_first(int mode) {
  return mode == SWEEP_FWD_AX ? SYS_AUI : (mode == SWEEP_FWD ? SYS_DD : SYS_T);
}
__host__ __device__ constexpr int sweep_sys_dst(int mode) { return mode == SWEEP_FWD ? 1 : 0; }
// Elements per 16 bytes.
__host__ __device__ inline int sweep_g(int es) { return 16 / es; }
// Elements of a left/right halo span: TIp*(TJ-1) + 16 bytes.
__host__ __device__ inline int halo_span(const SkewGeo &q, int es) { return q.TIp * (q.TJ - 1) + sweep_g(es); }
// elements per ring slot (a multiple of 16 bytes, so slots stay aligned)
__host__ __device__ inline int sweep_slot(const SkewGeo &q, int mode, int es) {
  return sweep_nv(mode) * q.T + (mode == SWEEP_FWD_AX ? 2 * halo_span(q, es) + 2 * q.TIp : 0);
}
// Offsets of the halo values inside a slot (MODE 1): the value of row tj
// is at halo_left + TIp*tj + halo_lofs, halo_right + TIp*tj,
// halo_down + ti and halo_up + ti.
__host__ __device__ inline int halo_lofs(const SkewGeo &q, int es) { return (q.TI - 1) & (sweep_g(es) - 1); }
__host__ __device__ inline int halo_left(const SkewGeo &q, int) { return 9 * q.T; }
__host__ __device__ inline int halo_right(const SkewGeo &q, int es) { return 9 * q.T + halo_span(q, es); }
__host__ __device__ inline int halo_down(const SkewGeo &q, int es) { return 9 * q.T + 2 * halo_span(q, es); }
__host__ __device__ inline int halo_up(const SkewGeo &q, int es) {
  return 9 * q.T + 2 * halo_span(q, es) + q.TIp;
}
// Copy c of tile b, the part that does not change from step to step: the
// slab of step u is w = u (forward) or nsteps-1-u (backward), and the copy
// reads array `arr` at offset base + w*wstride when dlo <= w <= dhi (false
// when the copy does not exist: no neighbouring tile).  The range excludes
// the steps where the neighbour's slab lies outside 0..W-1; no cell of
// such a step uses the value (its edge cells are above or below the
// interior).
struct SweepLane {
  long long base;
  int wstride, dst, bytes, arr, dlo, dhi;
};
__host__ __device__ inline bool sweep_lane(const SkewGeo &q, int mode, int b, int c, SweepLane &l, int es) {
  const long long slab0 = (long long)b * q.W;
  l.dlo = 0; l.dhi = q.W - 1;
  const int sys_c = (mode == SWEEP_FWD) ? 1 : 0;  // copy index of the system block
  if (c == sys_c) {
    l.base = sys_at(slab0, sweep_sys_first(mode), q.T, 0);
    l.wstride = SYS_N * q.T;
    l.dst = sweep_sys_dst(mode) * q.T;
    l.bytes = (mode == SWEEP_FWD_AX ? 8 : 5) * q.T * es;
    l.arr = 0;
    return true;
  }
  if (mode >= SWEEP_BWD) {  // R0 (copy 1) at 5T, RR (copy 2) at 6T
    if (c < 1 || c >= sweep_ncopy(q, mode)) return false;
    l.base = slab0 * q.T;
    l.wstride = q.T;
    l.dst = (4 + c) * q.T;
    l.bytes = q.T * es;
    l.arr = c;
    return true;
  }
  l.wstride = q.T;
  l.arr = 1;
  if (c == 1 - sys_c) {  // the vector: Y (MODE 0) or P (MODE 1)
    l.base = slab0 * q.T;
    l.dst = (mode == SWEEP_FWD_AX) ? 8 * q.T : 0;
    l.bytes = q.T * es;
    return true;
  }
  if (mode != SWEEP_FWD_AX) return false;
  const int bx = b % q.ntx, by = b / q.ntx, nty = q.nb / q.ntx;
  int nb_tile, dw, toff;
  if (c == 2) {  // down: row tj = TJ-1 of tile b-ntx
    if (by == 0) return false;
    nb_tile = b - q.ntx; dw = q.TJ - 1; toff = q.TIp * (q.TJ - 1);
    l.dst = halo_down(q, es); l.bytes = q.TIp * es;
  } else if (c == 3) {  // up: row tj = 0 of tile b+ntx
    if (by == nty - 1) return false;
    nb_tile = b + q.ntx; dw = -(q.TJ - 1); toff = 0;
    l.dst = halo_up(q, es); l.bytes = q.TIp * es;
  } else if (c == 4) {  // left: tile b-1, from the 16 bytes holding column TI-1 of row 0 to those of row TJ-1
    if (bx == 0) return false;
    nb_tile = b - 1; dw = q.TI - 1; toff = (q.TI - 1) & ~(sweep_g(es) - 1);
    l.dst = halo_left(q, es); l.bytes = halo_span(q, es) * es;
  } else if (c == 5) {  // right: tile b+1, from column 0 of row 0 to the 16 bytes of row TJ-1
    if (bx == q.ntx - 1) return false;
    nb_tile = b + 1; dw = -(q.TI - 1); toff = 0;
    l.dst = halo_right(q, es); l.bytes = halo_span(q, es) * es;
  } else {
    return false;
  }
  l.base = ((long long)nb_tile * q.W + dw) * q.T + toff;
  l.dlo = dw < 0 ? -dw : 0;                 // 0 <= w + dw
  l.dhi = dw > 0 ? q.W - 1 - dw : q.W - 1;  // w + dw <= W-1
  return true;
}
// Copy c for wavefront step u of tile b (nsteps steps); false when it is
// not issued.
__host__ __device__ inline bool sweep_copy(const SkewGeo &q, int mode, int b, int nsteps, int u, int c,
                                           SweepCopy &cp, int es) {
  SweepLane l;
  if (!sweep_lane(q, mode, b, c, l, es)) return false;
  const int w = (mode >= SWEEP_BWD) ? nsteps - 1 - u : u;
  if (w < l.dlo || w > l.dhi) return false;
  cp.src = l.base + (long long)w * l.wstride;
  cp.dst = l.dst; cp.bytes = l.bytes; cp.arr = l.arr;
  return true;
}

// ---- batched solves of several grids (cadmas_batch_*) ----------------
// One launch of a solver kernel covers the members of a batch: its blocks
// are the members' blocks one after another (tiles for the sweeps and the
// factorisation, slab blocks for the vector kernels, blocks of 256 layout
// entries for the conversions), a block finding its member in the
// prefix table and running the member's kernel body with its block index
// inside the member.  BatchMember is a member's part of the solve.
enum BatchVecF { BF_B = 0, BF_X, BF_R0, BF_RR, BF_PV, BF_AP, BF_AE, BF_Y2, BF_N };
enum BatchVecD { BD_B = 0, BD_X, BD_Y2, BD_N };
enum BatchRange { BR_TILE = 0, BR_SLAB = 1, BR_ELEM = 2, BR_N = 3 };
constexpr int BATCH_ELEM = 256;  // layout entries per block of the conversions
struct BatchMember {
  Geo g;
  SkewGeo q;
  SkewSys S;       // FP64 system, INDC (skewed)
  SkewSysF Sf;     // FP32 system
  SysPtr a;        // the step's Poisson system (standard layout)
  const int *indc; // INDC (standard layout)
  double *pt;      // PT (standard layout): the initial guess in, the solution out
  float *vf[BF_N];
  double *vd[BD_N];
  double *rb0, *rb1, *rb5, *dres;
  SolveState *st;
  int *pivot_bad;
  long long nrb;   // slab blocks of the member (partials of its slab sums)
  double epsa2, div2, tol2;
  double scale, rn, eps2;  // the refinement pass: 1/|r|, |r|, inner tolerance squared
  double U;                // MILU relaxation (CGPARA when ICGTYP != 0)
  int icgmax, warm, active, pad;
};
// gathered per member after a kernel sequence: done, timeout, iter,
// pivot_bad, the two stored sums (dres[6], dres[7])
constexpr int BATCH_GATHER = 6;

enum FinMode { FIN_BNORM = 0, FIN_START = 1, FIN_STORE = 2, FIN_RELRES = 3,
               FIN_ALPHA = 10, FIN_OMEGA = 11, FIN_CONV = 12 };

// Time-dependent part of one wave-maker side (host side of VF_BWUWN).
struct OpenDev {
  int side, nnow;   // JD and NNOW (0: full weights ALN = ALT = 1)
  double c, dtnow;  // phase speed BCTYP(6,JD) and DTNOW
};

struct WaveDev {
  int side, first, last;  // JD and the range of boundary lines
  int mtbtyp, nzz, mtbnow;  // table type, MTBZZ, row MTBNOW (1-based)
  double d, wvz, wt1, wt2, aw, sa, sb, wvlvl;
  const double *zz, *un, *ut;  // device copies of DMTBZZ, DMTBUN, DMTBUT
  int theory;                  // 1: the wave theory of `ph` instead of the table
  WavePhase ph;
  const WaveCol *col;          // oblique incidence: level and phase part of
                               // each line first..last (device), else null
};

// wavetheory.cu: a wave theory's level at a phase (VF_CWMAK1, single
// precision as the reference's) and the phase's part of its velocities
// (VF_CWMAK2); the start phase (VF_CWZERO); the stream-function forms
void theory_phase(const cadmas_wave_theory &t, double wvt, WavePhase &ph);
double theory_eta(const cadmas_wave_theory &t, double wvt);
double theory_zero_phase(const cadmas_wave_theory &t);
void theory_from_stream(const cadmas_stream_wave &s, cadmas_wave_theory &t);
void stream_phase(const cadmas_stream_wave &s, double wvt, WavePhase &ph);
double stream_eta(const cadmas_stream_wave &s, double wvt);

// k_drop.cu: VF_FDROPF (all its passes) and the start values of its arrays
void launch_fdropf(cudaStream_t s, const Geo &g, const Fld &f, const Prm &p, const DropArrays &d);
void launch_drop_reset(cudaStream_t s, long long n, const DropArrays &d);
bool drop_supported(const Geo &g);

// k_momentum.cu
void launch_flux(cudaStream_t s, const Geo &g, const Fld &f, const Prm &p, double *const *fl);
void launch_predict(cudaStream_t s, const Geo &g, const Fld &f, const Prm &p, double *const *fl,
                    double *un, double *vn, double *wn);
void launch_bwuwn(cudaStream_t s, const Geo &g, const Fld &f, const Prm &p, int *err);
// VF_BWFFSF: F of the cells next to a fixed-water-level side set to the level wl
void launch_bwffsf(cudaStream_t s, const Geo &g, const Fld &f, int side, int first, int last, double wl);
void launch_wave(cudaStream_t s, const Geo &g, const Fld &f, const WaveDev &w, int *err);
// VF_CWMSRC: SRCUV(NUMIJ,NUMK) of the wave source from the matrix table;
// w.side = ISCTYP(1) (> 0 x source at I, < 0 y source at J = -side)
void launch_srcuv(cudaStream_t s, const Geo &g, const Fld &f, const WaveDev &w, double *srcuv, int *err);
// Open (radiation) faces of one side; ub/vb/wb the velocities the blend
// reads (the start of the step's, or a copy of the present ones at set-up)
void launch_open(cudaStream_t s, const Geo &g, const Fld &f, const OpenDev &o, const double *ub,
                 const double *vb, const double *wb, int *err);

// k_poisson.cu
void launch_vpcoef(cudaStream_t s, const Geo &g, const Fld &f, const Prm &p, const SysPtr &a, int *err);
void launch_to_skew(cudaStream_t s, const Geo &g, const SkewGeo &q, const SysPtr &a, const int *indc,
                    const SkewSys &S, const double *x0, double *bsl, double *xsl, int warm);
void launch_dcmp(cudaStream_t s, const Geo &g, const SkewGeo &q, double U, const SkewSys &S, int *pivot_bad);
// T = MINV_L*Y (Y given, or Y = A*spmv_x formed in the sweep) into the
// system block's SYS_T arrays; X = MINV_U*T from there.
void launch_fwd(cudaStream_t s, const Geo &g, const SkewGeo &q, const SkewSys &S, const double *y,
                const double *spmv_x, SolveState *st, double *ybuf);
void launch_bwd(cudaStream_t s, const Geo &g, const SkewGeo &q, const SkewSys &S, double *x, SolveState *st);
// FP32 forms for the inner solves of the mixed-precision solver.
void launch_fwd_f(cudaStream_t s, const Geo &g, const SkewGeo &q, const SkewSysF &S, const float *y,
                  const float *spmv_x, SolveState *st, float *ybuf);
void launch_bwd_f(cudaStream_t s, const Geo &g, const SkewGeo &q, const SkewSysF &S, float *x, SolveState *st);
// batched launches (k_poisson.cu); pre = the members' first blocks per
// BatchRange, (nm + 1) entries each, on the device; nblk the total blocks
void launch_b_to_skew(cudaStream_t s, const BatchMember *bm, const int *pre, int nm, long long nblk);
void launch_b_sys_to_f(cudaStream_t s, const BatchMember *bm, const int *pre, int nm, long long nblk);
bool launch_b_dcmp_f(cudaStream_t s, const BatchMember *bm, const int *pre, int nm, long long ntiles, int T);
// FP32 sweep of MODE over the members' tiles: vin, vout, vin2 select
// float vectors (-1: none), rb5 selects rb5 for the sums (else rb0)
bool launch_b_sweep(cudaStream_t s, int mode, const BatchMember *bm, const int *pre, int nm, long long ntiles,
                    const SkewGeo &qref, int vin, int vout, int vin2, bool rb5, int nsm, int occ);
bool b_sweeps_supported(const SkewGeo &qref, int nsm, int occ, long long ntiles);
void launch_b_clear(cudaStream_t s, const BatchMember *bm, int nm);
void launch_b_gather(cudaStream_t s, const BatchMember *bm, int nm, double *out);
void launch_b_residual(cudaStream_t s, const BatchMember *bm, const int *pre, int nm, long long nslab);
void launch_b_fin(cudaStream_t s, int mode, const BatchMember *bm, int nm, bool tile_partials);
void launch_b_fin5(cudaStream_t s, const BatchMember *bm, int nm);
void launch_b_commit(cudaStream_t s, const BatchMember *bm, int nm);
void launch_b_start_f(cudaStream_t s, const BatchMember *bm, const int *pre, int nm, long long nslab);
void launch_b_dot_r0f(cudaStream_t s, const BatchMember *bm, const int *pre, int nm, long long nslab);
void launch_b_copy2_f(cudaStream_t s, const BatchMember *bm, const int *pre, int nm, long long nslab);
void launch_b_axpyf(cudaStream_t s, const BatchMember *bm, const int *pre, int nm, long long nslab);
void launch_b_upd3f(cudaStream_t s, const BatchMember *bm, const int *pre, int nm, long long nslab);
void launch_b_add_f(cudaStream_t s, const BatchMember *bm, const int *pre, int nm, long long nslab);
void launch_b_x0(cudaStream_t s, const BatchMember *bm, const int *pre, int nm, long long nslab);
// the FP32 backward sweep with the inner products after it summed on the
// way, one partial per tile (rb + c*nb); false when not available for the
// layout (nothing launched)
bool launch_bwd_f_dot1(cudaStream_t s, const Geo &g, const SkewGeo &q, const SkewSysF &S, const float *r0, float *x,
                       double *rb, SolveState *st);
bool launch_bwd_f_dot5(cudaStream_t s, const Geo &g, const SkewGeo &q, const SkewSysF &S, const float *r0,
                       const float *rr, float *x, double *rb, SolveState *st);
void launch_dcmp_f(cudaStream_t s, const Geo &g, const SkewGeo &q, double U, const SkewSysF &S, int *pivot_bad);
bool sweep_supported_f(const SkewGeo &q);
// Vector kernels for both precisions (explicitly instantiated for double
// and float in k_poisson.cu).
template <typename V>
void launch_spmv_t(cudaStream_t s, const Geo &g, const SkewGeo &q, const SkewSysT<V> &S, const V *x, V *y,
                   const SolveState *st);
template <typename V>
void launch_dot_t(cudaStream_t s, const SkewGeo &q, const int *indc, const V *x0, const V *y0, const V *x1,
                  const V *y1, double *rb0, double *rb1, const SolveState *st);
template <typename V>
void launch_copy2_t(cudaStream_t s, const SkewGeo &q, const int *indc, const V *r0, V *rr, V *pp,
                    const SolveState *st);
template <typename V>
void launch_axpy_rr_t(cudaStream_t s, const SkewGeo &q, const int *indc, const V *ap, V *rr, const SolveState *st);
template <typename V>
void launch_upd_xr_t(cudaStream_t s, const SkewGeo &q, const int *indc, const V *pp, const V *ae, const V *r0,
                     V *xw, V *rr, double *rb0, double *rb1, const SolveState *st);
template <typename V>
void launch_upd_p_t(cudaStream_t s, const SkewGeo &q, const int *indc, const V *rr, const V *ap, V *pp,
                    const SolveState *st);
// Regrouped FP32 inner iteration (k_poisson.cu): vectors zero where
// INDC = -1, four entries per lane; rb5 holds 5 x nslab partials.
void launch_dot2f(cudaStream_t s, const SkewGeo &q, const float *r0, const float *ap, double *rb,
                  const SolveState *st);
void launch_axpyf(cudaStream_t s, const SkewGeo &q, const float *ap, float *rr, const SolveState *st);
void launch_dot5f(cudaStream_t s, const SkewGeo &q, const float *r0, const float *rr, const float *ae, double *rb5,
                  const SolveState *st);
// One iteration's tail: launch_dot5f, launch_fin5 (scalars; a finished
// solve sets SolveState::stop), launch_upd3f (runs while `done` is clear,
// so also in the finishing iteration), launch_commit (done = stop).
void launch_upd3f(cudaStream_t s, const SkewGeo &q, const float *ae, const float *ap, float *xw, float *rr,
                  float *pp, const SolveState *st);
void launch_fin5(cudaStream_t s, const double *rb5, long long nrows, SolveState *st, double epsa2, double epsr2,
                 double div2, int icgmax);
void launch_commit(cudaStream_t s, SolveState *st);
void launch_sys_to_f(cudaStream_t s, const SkewGeo &q, const double *sys, float *sysf);
void launch_scale_to_f(cudaStream_t s, const SkewGeo &q, const int *indc, const double *r, double scale,
                       float *rf);
void launch_add_f(cudaStream_t s, const SkewGeo &q, const int *indc, const float *d, double inv_scale, double *x);
// Thread block of the sweeps for a tile of T slab entries (T consumer
// threads rounded up to whole warps, plus the producer warp).
inline int sweep_threads(int T) { return ((T + 31) & ~31) + 32; }
// Whether the sweeps can run this tile geometry (block size, shared memory).
bool sweep_supported(const SkewGeo &q);
void launch_spmv(cudaStream_t s, const Geo &g, const SkewGeo &q, const SkewSys &S, const double *x, double *y,
                 const SolveState *st);
void launch_bmy(cudaStream_t s, const SkewGeo &q, const int *indc, const double *b, double *y,
                const SolveState *st);
void launch_dot(cudaStream_t s, const SkewGeo &q, const int *indc, const double *x0, const double *y0,
                const double *x1, const double *y1, double *rb0, double *rb1, const SolveState *st);
void launch_copy2(cudaStream_t s, const SkewGeo &q, const int *indc, const double *r0, double *rr, double *pp,
                  const SolveState *st);
void launch_axpy_rr(cudaStream_t s, const SkewGeo &q, const int *indc, const double *ap, double *rr,
                    const SolveState *st);
void launch_upd_xr(cudaStream_t s, const SkewGeo &q, const int *indc, const double *pp, const double *ae,
                   const double *r0, double *xw, double *rr, double *rb0, double *rb1, const SolveState *st);
void launch_upd_p(cudaStream_t s, const SkewGeo &q, const int *indc, const double *rr, const double *ap,
                  double *pp, const SolveState *st);
void launch_x0(cudaStream_t s, const Geo &g, const SkewGeo &q, const int *indc, const double *xw, double *x0,
               const SolveState *st);
void launch_relres(cudaStream_t s, const Geo &g, const SkewGeo &q, const SkewSys &S, const double *b,
                   const double *x, double *rb0, double *rb1);
void launch_fin(cudaStream_t s, int mode, const double *rb0, const double *rb1, long long nrows,
                SolveState *st, double *out, double epsa2, double epsr2, double div2, int icgmax);
void launch_pivot_check(cudaStream_t s, SolveState *st);
void launch_vmodif(cudaStream_t s, const Geo &g, const Fld &f, const Prm &p, const double *pt);

// k_vof.cu
void launch_fconv(cudaStream_t s, const Geo &g, const Fld &f, const Prm &p, double *a, double *b, double *c);
// learned warm start (k_unet.cu): tcgen05 implicit-GEMM 3x3x3 convolution
// (mode: BF16 out, ReLU + BF16, ReLU-backward mask + BF16, FP32 out), its
// weight gradient, and the U-Net's elementwise kernels
enum { CONV_BF16 = 0, CONV_RELU_BF16 = 1, CONV_MASK_BF16 = 2, CONV_F32 = 3 };
bool unet_kernels_configure();
size_t conv_smem_bytes(int Cin, int Cout);
size_t wgrad_smem_bytes(int Cout);
void launch_conv(cudaStream_t s, int X, int Y, int Z, int B, const void *x, int Cin, const void *w, const float *bias,
                 int Cout, int mode, const void *mask, void *y, int *err);
void launch_wgrad(cudaStream_t s, int X, int Y, int Z, int B, const void *x, int Cin, const void *dy, int Cout,
                  long long slice, float *part, float *dw, int *err);
void launch_bias_grad(cudaStream_t s, long long V, const void *dy, int C, float *part, float *db);
void launch_pool(cudaStream_t s, int Xc, int Yc, int Zc, int B, const void *f, int C, void *c);
void launch_pool_bwd(cudaStream_t s, int Xc, int Yc, int Zc, int B, const void *dc, int C, void *df, int acc);
void launch_upcat(cudaStream_t s, int X, int Y, int Z, int B, const void *c, int C1, const void *sk, int C2, void *o);
void launch_upcat_bwd(cudaStream_t s, int X, int Y, int Z, int B, const void *d, int C1, int C2, void *dc, void *dsk,
                      int acc);
void launch_relu_mask(cudaStream_t s, long long n, const void *act, void *d);
void launch_head(cudaStream_t s, long long V, const void *a, int C, const float *wh, const float *bh, float *y);
void launch_mse(cudaStream_t s, long long V, const float *y, const float *t, const float *m, float inv_n, float *dy,
                float *lpart);
void launch_head_bwd(cudaStream_t s, long long V, const float *dy, const void *a, int C, const float *wh, void *da,
                     float *part);
void launch_adam(cudaStream_t s, long long n, float *p, const float *g, float *m, float *v, float lr, float b1,
                 float b2, float eps, float c1, float c2);
void launch_wcast(cudaStream_t s, const float *w, int Cin, int Cout, void *wf, void *wt);
void launch_f32_to_bf16(cudaStream_t s, long long n, const float *a, void *b);
void launch_fill_bf16(cudaStream_t s, long long n, void *a);
void launch_pack_in(cudaStream_t s, long long V, const float *x4, void *x16);
void launch_res_fwd(cudaStream_t s, int X, int Y, int Z, int B, const float *y, const float *a7, const float *x4,
                    const float *m, float c, float *r, float *lpart);
void launch_res_bwd(cudaStream_t s, int X, int Y, int Z, int B, const float *a7, const float *r, const float *m,
                    float scale, float *dy);
void launch_bias_reduce(cudaStream_t s, const float *part, int n, int C, float *out);
// the network as a part of a solver handle (unet.cu): created on the
// handle's stream; the warm-start glue (warmstart.cu) fills its FP32
// input (4 channels per voxel), runs it and reads its output
int unet_new(int nx, int ny, int nz, int batch, cudaStream_t stream, cadmas_unet **out);
void unet_dims(const cadmas_unet *n, int &X, int &Y, int &Z);
float *unet_input(cadmas_unet *n);
const float *unet_output(const cadmas_unet *n);
const int *unet_error(const cadmas_unet *n);
void unet_run_forward(cadmas_unet *n);
int unet_error_host(cadmas_unet *n);
void launch_warm_guess(cudaStream_t s, const Geo &g, const Fld &f, const SysPtr &a, cadmas_unet *net, double *rows0,
                       double *rows1, double *scal, int *cnt, double *PT);
// k-epsilon (k_keps.cu): VF_K1CAL into akn/aen; VF_BSSS (+ VF_CNUT0 and
// VF_CNU00 with nut); VF_BWKE; the k, e, ANUT, ANU of VF_CINIT
// VF_BWKELG in place on the fluid cells next to log-law or rough walls
void launch_bwkelg(cudaStream_t s, const Geo &g, const Fld &f, const Prm &p, const KeConst &kc, double *ak, double *ae,
                   int *err);
void launch_kstep(cudaStream_t s, const Geo &g, const Fld &f, const Prm &p, const KeConst &kc, const KeArrays &t,
                  double *akn, double *aen, int *err);
void launch_kbsss(cudaStream_t s, const Geo &g, const Fld &f, const KeConst &kc, double *ak, double *ae, double *anut,
                  double *anu, bool bsss, bool nut);
void launch_bwke(cudaStream_t s, const Geo &g, const Fld &f, const KeArrays &t, int *err);
void launch_kinit(cudaStream_t s, const Geo &g, const Fld &f, const KeConst &kc, double *ak, double *ae, double *anut,
                  double *anu);
// VF_FCONVS (ISCMFF != 0): slope pass into ist/sx/sy/sz/sa (every cell
// written), then the face fluxes into flfu/flfv/flfw; ERR_PG into err
void launch_fconvs(cudaStream_t s, const Geo &g, const Fld &f, const Prm &p, int *ist, double *sx, double *sy,
                   double *sz, double *sa, double *flfu, double *flfv, double *flfw, int *err);
void launch_feuler(cudaStream_t s, const Geo &g, const Fld &f, const Prm &p, const double *a,
                   const double *b, const double *c);
void launch_fmod1(cudaStream_t s, const Geo &g, const Fld &f, int *nlim);
void launch_fcut(cudaStream_t s, const Geo &g, const Fld &f, const Prm &p, double *rbs, double *rbc);
void launch_fnf_init(cudaStream_t s, const Geo &g, const Fld &f, const Prm &p);
void launch_fnf_sweep(cudaStream_t s, const Geo &g, int *nf, int *nch, int *done, int *iter, int cap,
                      int *err);
void launch_fbubup(cudaStream_t s, const Geo &g, const Fld &f, const Prm &p, const unsigned char *active);
void launch_fnfprv(cudaStream_t s, const Geo &g, const Fld &f, int *err);
void launch_cindc(cudaStream_t s, const Geo &g, const Fld &f, int *nums);
void launch_bsppfl(cudaStream_t s, const Geo &g, const Fld &f, const double *pp0, double *ppn);

// k_bc.cu
void launch_bsuwt(cudaStream_t s, const Geo &g, const Fld &f, const Prm &p);
void launch_bsuwt2(cudaStream_t s, const Geo &g, const Fld &f);
void launch_bsuwn(cudaStream_t s, const Geo &g, const Fld &f);
// the wave source's part of VF_BSUWN (p.iws or p.jws set)
void launch_bsuwn_src(cudaStream_t s, const Geo &g, const Fld &f, const Prm &p);
void launch_bsuwn3(cudaStream_t s, const Geo &g, const Fld &f, const Prm &p);
void launch_bsuwem(cudaStream_t s, const Geo &g, const Fld &f, int *nlim);
void launch_bspp(cudaStream_t s, const Geo &g, const Fld &f);
void launch_bwuwt(cudaStream_t s, const Geo &g, const Fld &f, const Prm &p, int *err);
void launch_bwpp(cudaStream_t s, const Geo &g, const Fld &f);
void launch_bwff(cudaStream_t s, const Geo &g, const Fld &f, int *err);
void launch_cdiv(cudaStream_t s, const Geo &g, const Fld &f, double *rb);
// VF_CDTCAL: the next step's DT into *out (device)
void launch_cdtcal(cudaStream_t s, const Geo &g, const Fld &f, double *rb, double dt0, double dtsafe, double w,
                   double dtmin, double *out);

}  // namespace cadmas
