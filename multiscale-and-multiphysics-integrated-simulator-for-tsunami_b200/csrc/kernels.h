// kernels.h -- host-side launchers of the device kernels (one per file).
#pragma once
#include <cuda_runtime.h>
#include <atomic>
#include "cadmas_dev.cuh"

namespace cadmas {

// Kernels launched by this library in the process (cadmas_kernel_launches).
extern std::atomic<long long> g_kernel_launches;
inline void count_launch(long long n = 1) { g_kernel_launches.fetch_add(n, std::memory_order_relaxed); }

// The eight arrays of the Poisson system, WK01..WK08 of VF_V1CAL.
struct SysPtr {
  double *ad, *ali, *alj, *alk, *aui, *auj, *auk, *bb;
};

// The constant part of a solve in the tile-skewed layout of the MILU
// kernels (k_poisson.cu): 7 coefficients, DD and INDC.
struct SkewSys {
  double *ad, *ali, *alj, *alk, *aui, *auj, *auk, *dd;
  int *indc;
};
// Tile geometry of the skewed layout: TI x TJ columns per tile (T threads),
// W wavefront slabs per tile, ntx tiles along x, nb tiles in all.
struct SkewGeo {
  int TI, TJ, T, W, ntx, nb;
};

enum FinMode { FIN_BNORM = 0, FIN_START = 1, FIN_STORE = 2, FIN_RELRES = 3,
               FIN_ALPHA = 10, FIN_OMEGA = 11, FIN_CONV = 12 };

// k_momentum.cu
void launch_flux(cudaStream_t s, const Geo &g, const Fld &f, const Prm &p, double *const *fl);
void launch_predict(cudaStream_t s, const Geo &g, const Fld &f, const Prm &p, double *const *fl,
                    double *un, double *vn, double *wn);
void launch_bwuwn(cudaStream_t s, const Geo &g, const Fld &f, int *err);

// k_poisson.cu
void launch_vpcoef(cudaStream_t s, const Geo &g, const Fld &f, const Prm &p, const SysPtr &a, int *err);
void launch_to_skew(cudaStream_t s, const Geo &g, const SkewGeo &q, const SysPtr &a, const int *indc,
                    const SkewSys &S, const double *x0, double *bsl, double *xsl);
void launch_dcmp(cudaStream_t s, const Geo &g, const SkewGeo &q, double U, const SkewSys &S, int *pivot_bad);
void launch_fwd(cudaStream_t s, const Geo &g, const SkewGeo &q, const SkewSys &S, const double *y,
                const double *spmv_x, double *tout, const SolveState *st, double *ybuf);
void launch_bwd(cudaStream_t s, const Geo &g, const SkewGeo &q, const SkewSys &S, const double *tin,
                double *x, const SolveState *st);
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
void launch_bsuwn3(cudaStream_t s, const Geo &g, const Fld &f, const Prm &p);
void launch_bsuwem(cudaStream_t s, const Geo &g, const Fld &f, int *nlim);
void launch_bspp(cudaStream_t s, const Geo &g, const Fld &f);
void launch_bwuwt(cudaStream_t s, const Geo &g, const Fld &f);
void launch_bwpp(cudaStream_t s, const Geo &g, const Fld &f);
void launch_bwff(cudaStream_t s, const Geo &g, const Fld &f, int *err);
void launch_cdiv(cudaStream_t s, const Geo &g, const Fld &f, double *rb);

}  // namespace cadmas
