/*
 * oracle.h -- CPU restatement of the CADMAS-SURF/3D SMAC step (test infrastructure).
 *
 * THIS IS TEST INFRASTRUCTURE.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / reference arm of bench.py may load it, and only to check or
 * time the GPU library.  Nothing in the product links or calls it.
 *
 * The reference (Fortran 77 + MPI) cannot be compiled in this environment
 * (no Fortran compiler), so each routine below is restated loop by loop from
 * Simulators/CADMAS-SURF-3D/Source code/ (file:line cited at each function in
 * oracle.cpp).  The reference ships no tests or golden outputs, so parity of
 * this restatement with the Fortran program itself is UNPINNED; it is pinned
 * only by the invariants checked in tests/ (hydrostatic rest, volume balance,
 * ILU = MILU at CGPARA 0, BiCGSTAB vs a dense solve).
 *
 * Two summation orders are offered for every global sum (dot products of
 * VF_MZIP, FSUM/FCUT of VF_FCUT01, |VD| of VF_CDIV00):
 *   ORC_SUM_REF : the reference order, K,J,I sequential, per emulated rank,
 *                 ranks combined in rank order;
 *   ORC_SUM_GPU : the fixed tree order of the GPU library's reductions
 *                 (per x-row warp tree, then a 1024-thread tree over rows),
 *                 so that GPU results can be compared bit for bit.
 */
#ifndef CADMAS_ORACLE_H
#define CADMAS_ORACLE_H
#include "../include/cadmas_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_SUM_REF 0
#define ORC_SUM_GPU 1

typedef struct orc_handle orc_handle;

orc_handle *orc_create(const cadmas_dims *d, const cadmas_params *p, int sum_mode);
void orc_destroy(orc_handle *h);
int orc_upload_static(orc_handle *h, const cadmas_static *s);
int orc_set_state(orc_handle *h, const cadmas_state *s);
int orc_get_state(orc_handle *h, cadmas_state *s);
int orc_init_state(orc_handle *h, int hydrostatic);
int orc_step(orc_handle *h, double dt);
int orc_get_stats(orc_handle *h, cadmas_stats *st);
int orc_divnorm(orc_handle *h, double *val);
/* VF_M1BCGS on host arrays with the handle's decomposition and sum order. */
int orc_m1bcgs(orc_handle *h, const double *ad, const double *ali,
               const double *alj, const double *alk, const double *aui,
               const double *auj, const double *auk, const double *bb,
               double *x0, const int *indc, int *iter, double *bnorm,
               double *xnorm);
/* Read back the last Poisson system (WK01..WK08) and PT (WK09) of a step:
   which: 0 AD,1 ALI,2 ALJ,3 ALK,4 AUI,5 AUJ,6 AUK,7 BB,8 PT.               */
int orc_get_poisson(orc_handle *h, int which, double *out);
/* Wave-maker side with its matrix table (as cadmas_set_wave). */
int orc_set_wave(orc_handle *h, const cadmas_wave_bc *w, const cadmas_wave_table *t);
int orc_set_wave_source(orc_handle *h, const cadmas_wave_src *s, const cadmas_wave_table *t);
int orc_set_wave_theory(orc_handle *h, const cadmas_wave_bc *w, const cadmas_stream_wave *sw);
int orc_set_wave_func(orc_handle *h, const cadmas_wave_bc *w, const cadmas_wave_theory *th);
int orc_set_wave_angle(orc_handle *h, int side, double angle, double sx, double sy);
int orc_wave_eval(const cadmas_wave_theory *t, double phase, double z, double *eta, double *u, double *w);
int orc_set_wave_source_func(orc_handle *h, const cadmas_wave_src *src, const cadmas_wave_theory *th);
/* Open (radiation) side JD with the phase speed of depth and period (as
   cadmas_set_open); orc_open_speed is VF_COMAK0's C = L/T. */
int orc_set_open(orc_handle *h, int side, double depth, double period);
int orc_open_speed(double depth, double period, double grav, double *c);
/* Seconds spent in the last orc_step by stage: [0] momentum predictor,
   [1] assembly, [2] solve, [3] correction+BC, [4] VOF+flags.              */
int orc_get_timers(orc_handle *h, double *t5);
/* DROPTX..DROPWW of the droplet model (NULL skipped), as cadmas_get_drop. */
int orc_get_drop(orc_handle *h, double *tx, double *ty, double *tz, double *uu, double *vv, double *ww);
int orc_set_drop(orc_handle *h, const double *tx, const double *ty, const double *tz, const double *uu,
                 const double *vv, const double *ww);
/* TNOW, DTNOW, NNOW as cadmas_set_time. */
int orc_set_time(orc_handle *h, double tnow, double dtnow, int nnow);
/* VF_CDTCAL as cadmas_cdtcal (reference order: the running minimum). */
int orc_cdtcal(orc_handle *h, double dtinit, double dtmin, double dtmax, double dtsafe, double *dt);
/* The k-epsilon state as cadmas_get_turb / cadmas_set_turb. */
int orc_get_turb(orc_handle *h, double *ak, double *ae, double *anut, double *anu, double *bck, double *bce);
int orc_set_turb(orc_handle *h, const double *ak, const double *ae, const double *bck, const double *bce);
/* FF-SLOPE checks: cells of each slope type (index 0..7) seen by the
   VF_FCONVS passes so far; the elementary functions of VF_CROOT3
   (fn 0 cube root, 1 arctangent, 2 cosine); VF_FSLP2A/3A followed by
   VF_FSLP2F/3F on the same cell (dim 2 or 3); VF_CROOT3. */
int orc_slope_counts(orc_handle *h, int *counts);
double orc_slope_fn(int fn, double x);
int orc_fslp(int dim, const double *s, const double *d, double fval, double *aa, double *fback);
/* The log-law wall functions: the logarithm the oracle and the kernels
   share, VF_CLOGLW (status CADMAS_ENOTCONV when Newton did not converge)
   and VF_CLOGKS. */
double orc_ln(double x);
int orc_cloglw(double dl, double va, double anu0, double akk0, double aka0, double *vt);
double orc_clogks(double dl, double va, double ks, double anu0, double akk0, double aka0);
int orc_croot3(double a, double b, double c, double d, double *x, int *nrt);
/* Threads the oracle's parallel loops use (OpenMP). */
int orc_num_threads(void);

#ifdef __cplusplus
}
#endif
#endif
