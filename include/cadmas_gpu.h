/*
 * cadmas_gpu.h -- C ABI of the B200 SMAC time-step library (libcadmas_gpu.so).
 *
 * The library replaces the two per-step driver subroutines of CADMAS-SURF/3D:
 *   VF_V1CAL  (Simulators/CADMAS-SURF-3D/Source code/vf_v1cal.f:1-9)
 *   VF_F1CAL  (Simulators/CADMAS-SURF-3D/Source code/vf_f1cal.f:1-20)
 * which the time loop calls at vf_a1main.f:1058-1066 and :1104-1115.
 *
 * Data layout follows the Fortran program so that a Fortran or C caller can
 * pass its own arrays unchanged:
 *   - cell/face arrays are (NUMI,NUMJ,NUMK) column-major, I fastest, with one
 *     ghost layer on every side (NUMI = cells in x + 2).  Element (I,J,K),
 *     1-based, is at offset (I-1) + NUMI*((J-1) + NUMJ*(K-1));
 *   - face arrays are staggered: UU(I,J,K) is the x-face between cells I-1
 *     and I (vf_vmodif.f:74);
 *   - grid metrics XX(6,NUMI), YY(6,NUMJ), ZZ(6,NUMK) hold
 *     (coordinate, d, c, 1/d, 1/c, 1/(d_i+d_{i-1})) as built by VF_CGRID
 *     (vf_cgrid.f:44-67);
 *   - INDB(4,NUMB) is the boundary-face list of VF_CINDB (vf_cindb.f).
 *
 * Every entry point returns an int status (CADMAS_OK on success).  The
 * reference aborts the MPI job through VF_A2ERR instead (vf_a2err.f:46-49);
 * the codes below map its messages.  State lives on the GPU between calls;
 * host arrays are read or written only by the calls that name them.  A
 * handle is bound to the device that was current at cadmas_create and owns
 * one CUDA stream; calls on one handle must come from one host thread.
 */
#ifndef CADMAS_GPU_H
#define CADMAS_GPU_H
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define CADMAS_OK            0
#define CADMAS_EINVAL        1  /* bad argument or size                          */
#define CADMAS_ECUDA         2  /* CUDA runtime error                            */
#define CADMAS_ENOTCONV      3  /* 'NOT CONVERGED.'          vf_vpsol.f:71-72    */
#define CADMAS_EDIVERGE      4  /* 'INSTABILITY.'            vf_vpsol.f:73-74    */
#define CADMAS_EPIVOT        5  /* 'CAN NOT DECOMPOSITION.'  vf_vpsol.f:75-76    */
#define CADMAS_EPG           6  /* 'P.G ERROR.' (vf_vpcoef.f:433, vf_fnfprv.f:223)*/
#define CADMAS_ECAP          7  /* a device-side iteration cap was reached       */
#define CADMAS_ENOMEM        8  /* device allocation failed                      */
#define CADMAS_EUNSUPPORTED  9  /* option outside the implemented path           */
#define CADMAS_ENOSTATIC    10  /* cadmas_upload_static not called yet           */
#define CADMAS_ETIMEOUT     11  /* a device-side wait ran out of time (2 s)      */
#define CADMAS_ESCRATCH     12  /* grid larger than the static scratch of
                                   cadmas_divnorm_noalloc                       */
#define CADMAS_EIO          13  /* restart file: cannot open, read or write, or
                                   a mismatch ('INVALID NUMBER OF GRID.' etc.,
                                   vf_ir1inp.f); cadmas_strerror has the text */
#define CADMAS_EWAVE        14  /* the wave theory did not converge:
                                   '(VF_SFMB02C) NOT CONVERGED.' vf_cwmak0.f:54 */

/* ---- sizes (/VF_ANUMBI/, VF_ANUMBI.h) ----------------------------------- */
typedef struct cadmas_dims {
  int numi, numj, numk;  /* NUMI, NUMJ, NUMK: cells + 2 in each direction */
  int numb;              /* NUMB: number of boundary faces (INDB columns)  */
} cadmas_dims;

/* ---- parameters read from COMMON blocks by the reference ---------------- */
typedef struct cadmas_params {
  double rho0;           /* RHO0   /VF_APHYSR/  (default 1.0e3, vf_a2dflt.f)  */
  double grz0;           /* GRZ0   /VF_APHYSR/  gravity (default 9.8)          */
  double vvmax;          /* VVMAX  velocity clamp in VF_VEULER (default 30)     */
  double cgpara;         /* CGPARA MILU parameter (default 0.95)               */
  double cgepsa;         /* CGEPSA absolute tolerance (default 1e-15)          */
  double cgepsr;         /* CGEPSR relative tolerance (default 1e-12)          */
  double cgdiv;          /* CGDIV  divergence threshold (default 1e30)         */
  double flower;         /* FLOWER = FEPS (default 1e-6)                       */
  double fupper;         /* FUPPER = 1-FEPS                                     */
  double plower;         /* PLOWER porosity floor (default 1e-4)               */
  double scmvp;          /* SCMVP  upwind weight of momentum fluxes (1 = donor) */
  double wvlvl;          /* WVLVL  still-water level                           */
  double wbub;           /* WBUB   TimerDoor bubble rise speed; < 0 disables    */
  double glxmin, glxmax; /* GLXMIN/GLXMAX domain x extent (sponge distances)   */
  double glymin, glymax; /* GLYMIN/GLYMAX domain y extent                       */
  double damp[4][4];     /* DAMP(1..4,JD) as damp[JD-1][m-1]: PARAM-XY,
                            PARAM-Z, WIDTH, DEPTH of sponge JD = X-,X+,Y-,Y+  */
  int    idamp[4];       /* IDAMP(JD): sponge degree, < 0 = no sponge           */
  int    icgtyp;         /* ICGTYP 0 = ILU, otherwise MILU (default 1)         */
  int    icgmax;         /* ICGMAX iteration cap (default 500)                 */
  int    ibsuw0;         /* IBSUW0 0 = linear extrapolation of surface velocity */
  /* Preconditioner decomposition.  The reference run on NPI x NPJ MPI ranks
     (PARALLEL X/Y, vf_cpara.f) factors and sweeps MILU inside each rank's
     x-y block only (vf_mzdcmp.f:53-67 over MYIS..MYIE, MYJS..MYJE), i.e. a
     block-Jacobi MILU.  precond_ti/precond_tj give the interior cells per
     block in x and y; 0 means one block spanning the whole axis (the serial
     NPROCS=1 reference).                                                    */
  int    precond_ti, precond_tj;
  /* 1: after every solve also measure the true residual ||b-Ax||/||b||
     (cadmas_stats.true_relres); costs one extra pass over the system. */
  int    diag_relres;
  /* Pressure solver (no counterpart in the reference, which has only the
     first):
       0  VF_M1BCGS in FP64, converged as the reference does on
          |M^-1 r| <= CGEPSR |M^-1 b| (+ CGEPSA);
       1  mixed precision: FP32 MILU factor and FP32 BiCGSTAB inner solves
          under FP64 iterative refinement, converged on the true residual
          ||b - Ax||_2 <= CGEPSR ||b||_2 computed in FP64.  Falls back to
          solver 0 for a solve whose FP32 factor or inner solve fails.    */
  int    solver;
  /* Initial guess of the pressure solve (no counterpart in the reference,
     which always starts from PT = 0, vf_vpsol.f:52-58):
       0  PT = 0;
       1  the previous step's solution (0 on cells with INDC = -1 now);
       2  the learned guess of cadmas_set_warm_net (below).
     The stopping test is unchanged (|M^-1 r| against |M^-1 b| for
     solver 0), so the result meets the same tolerance.                  */
  int    warm_start;
  /* 0 or 1: one thread block per preconditioner block; 2: two blocks of
     a thread-block cluster, each sweeping precond_tj/2 rows and passing
     its boundary row to the other through distributed shared memory.  The
     preconditioner (and the result) is the same; precond_tj must be even.
     The BiCGSTAB dot products then sum over half-height slabs.           */
  int    precond_split;
  /* IDROP /VF_APHYSI/: 1 = the TimerDoor droplet model VF_FDROPF after the
     flag update of every step (vf_f1cal.f:212-217), the reference's
     default (vf_a2dflt.f:151); 0 = off (DROP OFF).                       */
  int    idrop;
  /* ISCMFF /VF_ACOMPI/: scheme of the F advection in VF_F1CAL
     (vf_f1cal.f:138-146).  0 = donor-acceptor VF_FCONV, the reference's
     default (vf_a2dflt.f:41); 1 = FF-SLOPE VF_FCONVS (input
     'COMP SCHM FF-SLOPE'): a surface cell with a tilted interface moves
     the water under its plane in the swept strip.                      */
  int    iscmff;
  /* LEQK /VF_APHYSI/: 1 = the k-epsilon model: VF_K1CAL between V1CAL and
     F1CAL, then VF_BSSS, VF_CNUT0, VF_CNU00 and VF_BWKE after F1CAL
     (vf_a1main.f:1093-1126), so that ANU = ANU0 + ANUT changes every step;
     0 = off, the reference's default (vf_a2dflt.f:139).  The constants
     are /VF_APHYSR/'s with their defaults (vf_a2dflt.f:61,162,165-176).  */
  int    leqk;
  int    pad0;
  double anu0;                     /* ANU0 molecular viscosity, 1e-6         */
  double scmk;                     /* SCMK upwind weight of k, e convection,
                                      1.0 (donor cell)                       */
  double akmink, akmine;           /* AKMINK, AKMINE cut-offs, 1e-20         */
  double akinik, akinie;           /* AKINIK, AKINIE initial k, e, 1e-20     */
  double akcmu, aksgk, aksge;      /* C_mu 0.09, sigma_k 1.0, sigma_e 1.3    */
  double akc1, akc2, akc3;         /* C1 1.44, C2 1.92, C3 0.0               */
  /* AKK0, AKA0 /VF_APHYSR/: kappa 0.4 and A 5.5 of the log law on
     log-law walls (INDB(3,L) = 6, VF_CLOGLW): the speed over the friction
     velocity is ln(y us / nu) / kappa + A, us the friction velocity; rough
     walls (8) use ln(y / ks) / kappa + A + 3 (VF_CLOGKS)
     (vf_a2dflt.f:175-176, input 'MODEL LOG-LAW', vf_iimdl.f:288-291).      */
  double akk0, aka0;
  /* Inner tolerance of the mixed-precision solver (solver 1; no
     counterpart in the reference).  Each FP32 inner solve is asked for
     the reduction the FP64 residual still needs to reach CGEPSR, times
     0.5, but not below this floor (FP32 sweeps stop gaining near 1e-6).
     0 = the default 1e-5.                                                */
  double mixed_eps_inner;
  /* Time limit in seconds of every device-side wait of the MILU sweeps
     (their bulk-copy mbarriers): a wait that runs out ends the solve
     with CADMAS_ETIMEOUT and leaves the handle usable.  0 = the default
     2 s.                                                                 */
  double wait_limit_s;
  /* Thread blocks of the MILU sweeps per SM (no counterpart in the
     reference): 1 = one block per SM with the deepest bulk-copy ring; 2 =
     two blocks per SM (registers capped, shallower ring), so that the
     wavefronts of two tiles interleave on each SM; it needs blocks of at
     most 256 columns and applies where the ring fits.  0 = the default:
     two blocks for the backward sweeps and the FP32 sweeps when the grid
     has at least two preconditioner blocks per SM, one otherwise; four
     for the FP32 backward sweeps (the mixed solver's) of 16x16 blocks
     (ring depth 4, at most 56 registers) when it has more than two per
     SM.  4 = four blocks for those sweeps at any size, the default for
     the others.  The results do not depend on it.                        */
  int    sweep_occupancy;
  /* Inner products of the mixed solver's FP32 iteration (solver 1; no
     counterpart in the reference): 0 = summed by the backward MILU sweeps
     that produce AP and AE, one partial per preconditioner block, where
     the layout allows (one layout tile per block, at most 512 columns);
     1 = by passes of their own after the sweeps.  The two differ only in
     the order of the double-precision sums of exact products.            */
  int    dot_passes;
} cadmas_params;

/* ---- static fields (set once; host pointers) ---------------------------- */
typedef struct cadmas_static {
  const double *xx, *yy, *zz;      /* XX(6,NUMI), YY(6,NUMJ), ZZ(6,NUMK)      */
  const double *ggv, *ggx, *ggy, *ggz;   /* porosity, face permeabilities     */
  const double *glv, *glx, *gly, *glz;   /* = G + (1-G)*CM (VF_CGLV/CGLXYZ)   */
  const double *cd0;               /* drag coefficient CD0                     */
  const double *anu;               /* ANU molecular (+eddy) viscosity          */
  const int    *indx, *indy, *indz;/* face index (-1 obstacle,0 normal,>0 bnd)*/
  const int    *indb;              /* INDB(4,NUMB)                             */
  /* k-epsilon boundaries, read when leqk != 0 (else may be NULL):
     INDBK(NUMB), INDBE(NUMB) the types of k and e on each boundary face
     (1 fixed, 2 zero gradient, 6/8 log-law and rough wall as set from the
     velocity type; negative, the input's FIX-A/FREE-A: no convective
     flux through the face, vf_iiboun.f:256-330, vf_sconvd.f:86), and
     BCK(NUMB), BCE(NUMB) the input values
     (kept on fixed faces, vf_bwke.f:63-64).                               */
  const int    *indbk, *indbe;
  const double *bck, *bce;
  /* BCVI(NUMB) the roughness ks of rough-wall faces (INDB(3,L) = 8,
     vf_iiboun.f); may be NULL when there are none (read as 0).           */
  const double *bcvi;
} cadmas_static;

/* ---- dynamic state (host pointers; read by set_state, written by get_state)
   NULL pointers are skipped.                                                 */
typedef struct cadmas_state {
  double *uu, *vv, *ww, *pp, *ff;  /* (NUMI,NUMJ,NUMK)                         */
  int    *nf, *indc;               /* NF, INDC                                 */
  double *bcu, *bcv, *bcw, *bcp, *bcf; /* (NUMB) boundary values              */
  double *tbub;                    /* TBUB(NUMK) TimerDoor timers              */
  double tnow;                     /* TNOW                                     */
  int    nnow;                     /* NNOW                                     */
} cadmas_state;

/* ---- per-step record (the list-file line of vf_a1main.f:954-961) -------- */
typedef struct cadmas_stats {
  double fsum, fcut;               /* fluid volume and cut-off volume (FCUT01) */
  double cgbnrm, cgxnrm;           /* |M^-1 b|, |M^-1 r| of the last solve     */
  double divnorm;                  /* |VD| from VF_CDIV00                      */
  double true_relres;              /* ||b-Ax||_2/||b||_2 of the last solve,
                                      INDC != -1 cells; < 0 when not measured  */
  int    icgitr;                   /* ICGITR iterations of the last solve      */
  int    nums;                     /* NUMS surface cells                       */
  int    last_status;              /* status of the last step                  */
  int    fallbacks;                /* solver 1: solves handed to the FP64
                                      solver so far (0 for solver 0)          */
} cadmas_stats;

/* ---- wave-maker boundary, matrix-table form (WAVE-BC ... FUNC MATRIX) ----
   The inflow of a side JD is interpolated from a table in time phase and
   height, as VF_CWMTB1/VF_CWMTB2 do (vf_cwmtb1.f, vf_cwmtb2.f), scaled to
   the current water column and faded in as VF_BWUWN does
   (vf_bwuwn.f:259-470).  Tables are column-major like the Fortran
   DMTBUN(MTBZZ,MTBTT).                                                     */
typedef struct cadmas_wave_table {
  int ntt, nzz;          /* MTBTT, MTBZZ                                     */
  int mtbtyp;            /* MTBTYP: 1 level and velocities (scaled to the
                            column's water level), 2 velocities only,
                            3 level only: the faces act as free faces and
                            the column next to the side takes the level
                            (VF_BWFFSF, vf_bwffsf.f)                      */
  int pad;
  double phase0;         /* DMTBT0: phase at TNOW = 0                        */
  const double *tt;      /* DMTBTT(MTBTT) phase, ascending in [0,1]         */
  const double *hh;      /* DMTBHH(MTBTT) water level above WVLVL            */
  const double *zz;      /* DMTBZZ(MTBZZ) height above WVLVL, ascending      */
  const double *un;      /* DMTBUN(MTBZZ,MTBTT) velocity normal to the side  */
  const double *ut;      /* DMTBUT(MTBZZ,MTBTT) vertical velocity            */
} cadmas_wave_table;

/* ---- wave-maker boundary, wave-theory form (WAVE-BC ... FUNC STREAM N) --
   A steady periodic wave of order N (1..22) by the stream-function
   (Fourier) method with no mean mass transport, the reference's default
   wave theory (vf_cwmak0.f:43-56).  In the frame moving with the wave,
     psi = -ubar (z+d) + sum_j b[j-1] sinh(j k (z+d)) / cosh(j k d) cos(j k X),
   z from the still water level.  cadmas_stream_solve computes it on the
   host (the reference's vf_wsfmb2.f is third-party code; this is
   Fenton's collocation form of the same method), cadmas_set_wave_theory
   drives a side with it: each step the level at the side's phase and the
   face velocities at the heights scaled to the column's water level, as
   VF_BWUWN does with VF_CWMAK1/VF_CWMAK2 (vf_bwuwn.f:259-470), rounded to
   single precision like the reference's REAL*4 wave routines.          */
#define CADMAS_STREAM_NMAX 22
typedef struct cadmas_stream_wave {
  int order;             /* N                                                 */
  int iterations;        /* Newton iterations over all height steps           */
  double depth, period, height, grav;  /* d, T, H, g of the solution         */
  double k;              /* wave number 2 pi / L                              */
  double length;         /* wave length L                                      */
  double celerity;       /* c = L / T                                          */
  double ubar;           /* mean speed of the water past the wave, moving frame */
  double q;              /* volume flux past the wave, moving frame (= c d)    */
  double r;              /* Bernoulli constant                                 */
  double phase0;         /* the phase at TNOW = 0 (BCTYP(6,JD)): where the
                            level crosses zero between the crest (phase 1)
                            and the trough (phase 0.5), found in single
                            precision as VF_CWZERO does (vf_cwzero.f)       */
  double b[CADMAS_STREAM_NMAX];  /* B_1 .. B_N                                 */
} cadmas_stream_wave;
/* Solve for the wave (host only).  CADMAS_EINVAL beyond the reference's
   steepness limits (H/L0 > 0.3 or H/d > 1.5, vf_wsfmb2.f:64-65),
   CADMAS_EWAVE when Newton's method does not converge.                  */
int cadmas_stream_solve(int order, double depth, double period, double height, double grav,
                        cadmas_stream_wave *out);
/* The surface eta at `phase` (theta = 2 pi phase; a crest at 0) and the
   velocities u (direction of travel) and w at height z above the still
   water level, as the wave maker uses them (host only; NULL skips).    */
int cadmas_stream_eval(const cadmas_stream_wave *s, double phase, double z, double *eta, double *u, double *w);

/* ---- wave theories of the wave maker and the wave source ----------------
   FUNC STREAM N | STOKES | CNOIDAL | STK-CND of WAVE-BC and WAVE-SRC
   (IBCTYP(2,JD) / ISCTYP(2), vf_iimdl.f:51-66,133-147).  cadmas_wave_solve
   does at set-up what vf_csetup.f:96-124 (and 270-300 for the source) do:
   the STK-CND choice by the Ursell number, VF_CWMAK0 (the wave and its
   length) and VF_CWZERO (the start phase).  cadmas_wave_eval is
   VF_CWMAK1 (level) and VF_CWMAK2 (velocities).
     type >= 1  the stream-function wave of that order (cadmas_stream_solve);
     type -1    cnoidal, third order (vf_wcnd0.f VF_CND0/1/2);
     type -2    Stokes, fifth order (vf_wstk0.f VF_STK0/1/2);
     type 0     STK-CND: Stokes when GRZ0 H T^2 / D^2 <= 25, else cnoidal.
   The theories use g = 9.8 m/s^2 as the reference's routines do; only the
   Ursell number uses grz0.  Stokes and cnoidal coefficients are kept in the
   units of the reference's routines, centimetres and seconds.            */
#define CADMAS_WAVE_STK_CND 0
#define CADMAS_WAVE_CNOIDAL (-1)
#define CADMAS_WAVE_STOKES (-2)
typedef struct cadmas_stokes_wave {
  double kd;             /* k d                                                */
  double k;              /* wave number, 1/cm                                   */
  double eps;            /* k H / 2, the expansion parameter                    */
  double c0, c;          /* linear and fifth-order celerity, cm/s               */
  double a[5];           /* eta = sum_i a[i-1] cos(i theta), cm                 */
  double b[5];           /* u = b0 + sum_i b[i-1] cosh(i k (z+d)) cos(i theta),
                            w = sum_i b[i-1] sinh(i k (z+d)) sin(i theta), cm/s */
  double b0;             /* cm/s                                                */
  double p0;             /* pressure-head constant, cm                          */
  int iterations, pad;   /* iterations of the dispersion relation              */
} cadmas_stokes_wave;
typedef struct cadmas_cnoidal_wave {
  double ql;             /* pi K'/K of the Jacobi elliptic functions (modulus) */
  double s;              /* the vertical-velocity scale RK of VF_CND0          */
  double d;              /* depth, cm                                           */
  double c0, c;          /* sqrt(g d) and the celerity, cm/s                    */
  double a[4];           /* eta = sum_i a[i-1] cn^(2(i-1)), cm                  */
  double b[12];          /* B(j,i) at (i-1)*3 + j-1: u = sum_i cn^(2(i-1))
                            sum_j B(j,i) Z^(2(j-1)), Z = 1 + z/d, cm/s           */
  double bb[12];         /* BB(j,i): w = Z cn sn dn sum_i cn^(2(i-2))
                            sum_j BB(j,i) Z^(2(j-1)), cm/s                        */
  double p0;             /* pressure-head constant, cm                          */
  int iterations, pad;   /* iterations for the elliptic parameter              */
} cadmas_cnoidal_wave;
typedef struct cadmas_wave_theory {
  int type;              /* after the STK-CND choice: N >= 1, -1 or -2          */
  int pad;
  double depth, period, height;  /* D, T, H (m, s)                             */
  double length;         /* WVLENG (BCTYP(4,JD), SCTYP(4))                      */
  double ursell;         /* GRZ0 H T^2 / D^2 (BCTYP(5,JD), SCTYP(5))           */
  double phase0;         /* VF_CWZERO: the phase in [0.5, 1] where the level
                            crosses zero, found in single precision
                            (BCTYP(6,JD), SCTYP(6))                            */
  cadmas_stream_wave stream;     /* type >= 1                                  */
  cadmas_stokes_wave stokes;     /* type -2                                    */
  cadmas_cnoidal_wave cnoidal;   /* type -1                                    */
} cadmas_wave_theory;
/* Solve for the wave (host only).  CADMAS_EINVAL for an unknown type or
   non-positive D, T, H; CADMAS_EWAVE when the stream-function solution
   does not converge or a theory gives no finite wave.                    */
int cadmas_wave_solve(int type, double depth, double period, double height, double grz0,
                      cadmas_wave_theory *out);
/* The level eta at `phase` (VF_CWMAK1) and the velocities normal to the
   side (u) and vertical (w) at height z above the still water level
   (VF_CWMAK2), in metres and m/s as the wave maker uses them (host only;
   NULL skips).                                                           */
int cadmas_wave_eval(const cadmas_wave_theory *t, double phase, double z, double *eta, double *u, double *w);

typedef struct cadmas_wave_bc {
  int side;              /* JD: 1 X-, 2 X+, 3 Y-, 4 Y+                      */
  int first, last;       /* IBCTYP(3..4,JD): J (X sides) or I (Y sides) of
                            the generated faces, 1-based with ghosts       */
  int pad;
  double depth;          /* BCTYP(1,JD) still-water depth D                  */
  double period;         /* BCTYP(3,JD) period T                             */
  double ramp;           /* BCTYP(8,JD) AMPL: periods of the sine fade-in;
                            0 = none                                        */
} cadmas_wave_bc;

/* ---- wave source (MODEL WAVE-SRC ... FUNC MATRIX) ------------------------
   A line of cells inside the domain that makes waves on both sides by a
   mass source (ISCTYP /VF_APHYSI/, SCTYP /VF_APHYSR/; vf_iimdl.f:115-172).
   Every step the source velocity SRCUV of the line is taken from the
   matrix table at TNOW (VF_CWMSRC, vf_cwmsrc.f:46-143, scaled to the
   column's water level for MTBTYP 1 and faded in over `ramp` periods); it
   enters the momentum sources (VF_VGENE, vf_vgene.f:149-152,225-228,
   304-315), the right-hand side of the pressure equation (VF_VPCOEF,
   vf_vpcoef.f:349-350), the surface cells of the line (VF_BSUWN,
   vf_bsuwn.f:81-118) and F (VF_FGENE, vf_fgene.f:42-70, through
   VF_FEULER's QF).  The table is the one of cadmas_set_wave (MTBTYP 1 or
   2; 3 is 'MTBTYP ERROR.' in the reference, vf_csetup.f:267).  With a
   wave theory (cadmas_set_wave_source_func) the velocities come from
   VF_CWMAK2 at the scaled heights instead, no table needed.              */
typedef struct cadmas_wave_src {
  int line;              /* ISCTYP(1): > 0 the x source at I = line (1-based
                            with ghosts, 2..NUMI-1); < 0 the y source at
                            J = -line (2..NUMJ-1)                           */
  int pad;
  double depth;          /* SCTYP(1) still-water depth D                     */
  double period;         /* SCTYP(3) period T                                */
  double ramp;           /* SCTYP(8) AMPL: periods of the sine fade-in; 0 = none */
} cadmas_wave_src;

typedef struct cadmas_handle cadmas_handle;

/* Defaults of vf_a2dflt.f for every field of cadmas_params. */
void cadmas_default_params(cadmas_params *p);

/* Allocate device state for one grid on the current device.
   Replaces the ALLOCATE block of vf_a1main.f:415-700 for the step arrays. */
int cadmas_create(const cadmas_dims *d, const cadmas_params *p,
                  cadmas_handle **out);
int cadmas_destroy(cadmas_handle *h);

/* Upload metrics, porosity, face indices and the boundary list
   (the fields VF_CGRID/VF_CGLV/VF_CGLXYZ/VF_CINDX/VF_CINDB prepare). */
int cadmas_upload_static(cadmas_handle *h, const cadmas_static *s);

/* Copy host state to the device (NULL members skipped). */
int cadmas_set_state(cadmas_handle *h, const cadmas_state *s);
/* Copy device state to the host (NULL members skipped). */
int cadmas_get_state(cadmas_handle *h, cadmas_state *s);

/* The droplet model's arrays DROPTX, DROPTY, DROPTZ, DROPUU, DROPVV,
   DROPWW, (NUMI,NUMJ,NUMK) column-major host arrays (NULL skipped): the
   arguments of the same names of VF_F1CAL (vf_f1cal.f:3) and of the
   restart file (vf_ir1inp.f:3).  They stay on the device between steps;
   cadmas_create and cadmas_init_state set them to -1e10, 0, 0, 0, 0, 0
   as VF_CINIT does (vf_cinit.f:416-427).                                */
int cadmas_get_drop(cadmas_handle *h, double *droptx, double *dropty, double *droptz, double *dropuu,
                    double *dropvv, double *dropww);
int cadmas_set_drop(cadmas_handle *h, const double *droptx, const double *dropty, const double *droptz,
                    const double *dropuu, const double *dropvv, const double *dropww);

/* The k-epsilon state (params.leqk != 0): AK, AE, ANUT and ANU
   (NUMI,NUMJ,NUMK) column-major, BCK, BCE (NUMB); NULL skipped.  They stay
   on the device between steps.  cadmas_init_state sets them as VF_CINIT
   does (vf_cinit.f:295-315,359-364,397-401).  cadmas_set_turb takes AK,
   AE, BCK, BCE and then forms ANUT (VF_CNUT0) and ANU (VF_CNU00) as the
   restart input does (vf_ir1inp.f:339-340).  CADMAS_EINVAL when leqk is
   0.                                                                    */
int cadmas_get_turb(cadmas_handle *h, double *ak, double *ae, double *anut, double *anu, double *bck,
                    double *bce);
int cadmas_set_turb(cadmas_handle *h, const double *ak, const double *ae, const double *bck,
                    const double *bce);

/* ---- learned warm start: the 3-D U-Net ---------------------------------
   A 3-level U-Net (3x3x3 convolutions, channels 16/32/64, BF16 weights and
   activations, FP32 accumulation on the tensor cores) from 4 input
   channels per voxel to 1 output.  Volumes are nx x ny x nz voxels (each a
   multiple of 4), batch of them; host arrays are C-ordered
   [batch][nz][ny][nx] (x fastest), inputs with 4 channels innermost.
   Parameters: cadmas_unet_param_count() FP32 values.  _grad returns the
   masked mean-square loss against t (mask m, 1 = counted) and its
   parameter gradient; _train_step applies Adam (beta 0.9/0.999, eps 1e-8)
   with learning rate lr.  CADMAS_ETIMEOUT when a tensor-core wait ran
   out of time.                                                         */
typedef struct cadmas_unet cadmas_unet;
size_t cadmas_unet_param_count(void);
int cadmas_unet_create(int nx, int ny, int nz, int batch, cadmas_unet **net);
int cadmas_unet_destroy(cadmas_unet *net);
int cadmas_unet_set_params(cadmas_unet *net, const float *params);
int cadmas_unet_get_params(cadmas_unet *net, float *params);
int cadmas_unet_forward(cadmas_unet *net, const float *x, float *y);
/* Mean device time (CUDA events on the network's stream) of reps forwards
   of the input already on the device (from the last _forward).        */
int cadmas_unet_time_forward(cadmas_unet *net, int reps, float *ms);
int cadmas_unet_grad(cadmas_unet *net, const float *x, const float *t, const float *m, float *loss,
                     float *grad);
int cadmas_unet_train_step(cadmas_unet *net, const float *x, const float *t, const float *m, float lr,
                           float *loss);
/* The loss of the learned guess: w_mse * |m (y - t)|^2 / n + w_res *
   |m (b - c A (m y))|^2 / n, n = sum(m), with b the input's channel 0 and A the
   sample's pressure system a7 ([batch][nz][ny][nx][7] FP32: AD, ALI, ALJ,
   ALK, AUI, AUJ, AUK as VF_MZAX applies them) in the network's volume.
   update != 0: one Adam step; grad (NULL skipped): the gradient.        */
int cadmas_unet_train_sys(cadmas_unet *net, const float *x, const float *t, const float *m, const float *a7,
                          float c, float w_mse, float w_res, float lr, int update, float *loss, float *grad);

/* The learned initial guess of the pressure solve (params.warm_start = 2):
   a network with the given parameters (cadmas_unet_param_count values) is
   run before each solve on (BB / s, F, GGV, INDC != -1), s the RMS of BB
   over computed cells, and PT0 = s * out_scale * output.  PT0 is
   dropped for PT = 0
   (the reference's start, vf_vpsol.f:52-58) unless |BB - A PT0|_2 <
   |BB|_2.  The solve's stopping test is unchanged.  Without a network
   loaded, warm_start 2 starts from PT = 0.  cadmas_warm_stats: guesses
   kept and dropped so far.                                             */
int cadmas_set_warm_net(cadmas_handle *h, const float *params, double out_scale);
int cadmas_warm_stats(cadmas_handle *h, long long *kept, long long *dropped);
/* The right-hand side BB and the solution PT of the last pressure solve
   ((NUMI,NUMJ,NUMK) column-major host arrays, NULL skipped): the training
   pairs of the learned guess.                                          */
int cadmas_get_solve(cadmas_handle *h, double *bb, double *pt);
/* The coefficients AD, ALI, ALJ, ALK, AUI, AUJ, AUK of the last pressure
   system (VF_VPCOEF), valid between cadmas_v1cal and cadmas_f1cal (the
   arrays are the step's work space afterwards).                        */
int cadmas_get_system(cadmas_handle *h, double *ad, double *ali, double *alj, double *alk, double *aui,
                      double *auj, double *auk);

/* ---- restart file (*.rsl / *.res) and list file ----------------------
   The restart file of the reference, byte for byte: a Fortran unformatted
   sequential file (each record framed by its byte count as a 4-byte
   little-endian integer, as gfortran writes one WRITE statement), NPROCS=1.
   cadmas_restart_create writes the header of VF_OR1INI (vf_or1ini.f:38-86):
   version (0,1); NUMI,NUMJ,NUMK,NUMB; the flags LN..L1 of the fields
   present (k-eps, temperature and scalars 0, droplets = IDROP >= 1); GGV.
   cadmas_restart_append writes one output of VF_OR1TRN (vf_or1trn.f:
   104-221) of the present state: NNOW,TNOW,DTNOW; FSUM,FCUT,CGBNRM,CGXNRM,
   ICGITR; NF; UU,BCU; VV,BCV; WW,BCW; PP,BCP; FF,BCF; TBUB; with droplets
   the count of cells with DROPTX >= 0 and one record I,J,K,DROPTX..DROPWW
   each.  When to write (IRSTYP, vf_or1trn.f:87-101) is the caller's call.
   cadmas_restart_load is VF_IR1INP (vf_ir1inp.f:96-336): it checks the
   header against the handle (errors 'INVALID NUMBER OF GRID.', 'INVALID
   NUMBER OF B.C.', 'INVALID EQUATION (...)' as CADMAS_EIO), reads the
   outputs up to the one of step nnow ('INVALID STEP.' if absent) and makes
   it the present state, INDC from NF as VF_CINDC.  Records of 2^31 bytes
   or more (a single 3-D field above 268 M cells) are refused.            */
int cadmas_restart_create(cadmas_handle *h, const char *path);
int cadmas_restart_append(cadmas_handle *h, const char *path);
int cadmas_restart_load(cadmas_handle *h, const char *path, int nnow);
/* VF_CDTCAL (vf_cdtcal.f:46-147), the adaptive time step of IDTTYP = 1
   (the reference's default): the next step's DT from the present state,
   DT = MAX(MIN(dtlim*DTSAFE, 1.2*W), DTMIN) with W = DTNOW of the last step
   (DTINIT before the first), where dtlim is the smallest of DTMAX/DTSAFE
   and every cell's advective limit V/max|face flux| and diffusive limit
   0.5/(1/DX^2+1/DY^2+1/DZ^2)/ANU.  The reference folds the limits into a
   running DT in K,J,I order, whose rounding can differ from the smallest
   limit in the last bits; this function takes the smallest limit itself.
   Reference defaults: DTINIT 1e-6, DTMIN 0, DTMAX 1e20, DTSAFE 0.1
   (vf_a2dflt.f:230-234).                                                  */
int cadmas_cdtcal(cadmas_handle *h, double dtinit, double dtmin, double dtmax, double dtsafe, double *dt);

/* The two lines the time loop writes to the list file after each step
   (vf_a1main.f:954-958, formats 9540 and 9550 of vf_a1main.f:1214-1223):
   STEP, TIME, DT, FSUM, FCUT and !VD! (VF_CDIV00, computed here), then
   !B!, !R! and ITR of the last solve; Fortran 1PE12.5 and I6 fields, each
   line ending in a newline, NUL-terminated in buf (len >= 200 is ample). */
int cadmas_list_step(cadmas_handle *h, char *buf, size_t len);

/* Initial classification and boundary values of VF_CINIT
   (vf_cinit.f:202-207 and the BC calls after :283): FCUT01, BWFF, FNFINI,
   FNFPRV, CINDC; then, if hydrostatic != 0, p = RHO0*GRZ0*(WVLVL - z_c) on
   INDC != -1 cells (vf_cinit.f:283); then BWUWN, BSUWT, BSUWT2, BSUWN3,
   BSPP, BWUWT, BWPP.  F must be set (cadmas_set_state) before the call. */
int cadmas_init_state(cadmas_handle *h, int hydrostatic);

/* One SMAC step of vf_a1main.f:1029-1104 with LOOPS=1: NNOW += 1,
   TNOW += dt, VF_V1CAL, VF_F1CAL. */
int cadmas_step(cadmas_handle *h, double dt);
/* The two halves separately (TNOW/DTNOW already advanced by the caller
   through cadmas_set_time). */
int cadmas_set_time(cadmas_handle *h, double tnow, double dtnow, int nnow);
int cadmas_v1cal(cadmas_handle *h);
int cadmas_f1cal(cadmas_handle *h);

/* VF_CDIV00 (vf_cdiv00.f:38-56) on the current state; also stored in stats. */
int cadmas_divnorm(cadmas_handle *h, double *val);
int cadmas_get_stats(cadmas_handle *h, cadmas_stats *st);

/* Synchronise the handle's stream. */
int cadmas_sync(cadmas_handle *h);

/* ---- ensemble of independent grids (no counterpart in the reference) ----
   One SMAC step of each of the n handles (one host thread per handle, each
   handle on its own stream, so the GPU runs the grids' kernels side by
   side).  dt[i] is handle i's time step; status[i] receives its
   cadmas_step status.  Returns the first non-zero status, or CADMAS_OK. */
int cadmas_step_ensemble(cadmas_handle **h, int n, const double *dt, int *status);

/* ---- batch of grids solved together (no counterpart in the reference) --
   A batch steps n handles of the mixed solver (solver 1, dot_passes 0) on
   one device, all with the same preconditioner block (precond_ti,
   precond_tj; no split).  Each step runs, per grid on its own stream and
   host thread, V1CAL up to the pressure system; then the pressure solves
   of all the grids together on the batch's stream, every solver kernel one
   launch over all the grids' tiles or slabs (a block finds its grid in a
   table of the grids' block ranges); then, per grid again, the rest of
   V1CAL and F1CAL.  The iterations run in lockstep: a grid that has
   converged is marked done and its blocks return at once.  Each grid gets
   the results, iterations and statistics a cadmas_step of its own gives.
   The handles must stay alive and unchanged in their solver parameters
   while the batch exists.  CADMAS_EINVAL for handles that do not match,
   CADMAS_EUNSUPPORTED for blocks too large for the batched sweeps.       */
typedef struct cadmas_batch cadmas_batch;
int cadmas_batch_create(cadmas_handle **h, int n, cadmas_batch **out);
/* One SMAC step of every grid of the batch; dt[i] and status[i] as in
   cadmas_step_ensemble.  Returns the first non-zero status.              */
int cadmas_batch_step(cadmas_batch *b, const double *dt, int *status);
int cadmas_batch_destroy(cadmas_batch *b);

/* Declare side w->side a wave-maker boundary driven by `tab` (copied).  Its
   boundary faces are those of INDB with INDB(3,L) = 5 on that side.  One
   table serves every wave side, as the reference's matrix data does.
   Sides and tables persist until cadmas_destroy. */
int cadmas_set_wave(cadmas_handle *h, const cadmas_wave_bc *w, const cadmas_wave_table *tab);

/* ---- open (radiation) boundary (MODEL OPEN-BC, vf_iimdl.f:176-213) ----
   Side o->side radiates with the phase speed C = L/T of the linear wave of
   period T in still-water depth D (VF_COMAK0, vf_csetup.f:128-143).  Its
   faces are those of INDB with INDB(3,L) = 7 on that side; VF_BWUWN
   blends their values toward the interior each step (vf_bwuwn.f:481-598).
   A side is either a wave maker or open ('DEFINED DOUBLY' otherwise).     */
typedef struct cadmas_open_bc {
  int side;              /* JD: 1 X-, 2 X+, 3 Y-, 4 Y+                      */
  int pad;
  double depth;          /* BCTYP(1,JD) still-water depth D (> 0)            */
  double period;         /* BCTYP(3,JD) period T (> 0)                       */
} cadmas_open_bc;

int cadmas_set_open(cadmas_handle *h, const cadmas_open_bc *o);

/* The phase speed C = BCTYP(6,JD) of an open side: the wave length of
   VF_COMAK0 (Newton on the dispersion relation, vf_comak0.f:31-55) over
   the period.  Host arithmetic only; needs no device. */
int cadmas_open_speed(double depth, double period, double grav, double *c);

/* ---- Fortran-callable step (drop-in for the two CALLs of the time loop) --
   Arguments by reference, as gfortran passes them.  The arrays are the
   caller's host arrays; they are copied in before and out after the step,
   so a Fortran time loop can call it in place of
     CALL VF_V1CAL(...) ; CALL VF_F1CAL(...)
   The handle comes from cadmas_create + cadmas_upload_static.           */
int vf_step_gpu_(cadmas_handle **h, const double *dtnow,
                 double *uu, double *vv, double *ww, double *pp, double *ff,
                 int *nf, int *indc, double *bcu, double *bcv, double *bcw,
                 double *bcp, double *bcf, double *tnow, int *nnow);

/* ---- Fortran-callable V1CAL / F1CAL, one call each -----------------------
   Same arrays as vf_step_gpu_, copied in before and out after the call.
   TNOW, DTNOW and NNOW are taken as the time loop has already advanced
   them (vf_a1main.f:1029-1047) and are not changed, as the COMMON block
   /VF_ATIMER/ is read, not written, by VF_V1CAL and VF_F1CAL.
     vf_v1cal_gpu_  replaces  CALL VF_V1CAL(...)  (vf_a1main.f:1058-1066)
     vf_f1cal_gpu_  replaces  CALL VF_F1CAL(...)  (vf_a1main.f:1104-1115) */
int vf_v1cal_gpu_(cadmas_handle **h, const double *tnow, const double *dtnow, const int *nnow,
                  double *uu, double *vv, double *ww, double *pp, double *ff,
                  int *nf, int *indc, double *bcu, double *bcv, double *bcw,
                  double *bcp, double *bcf);
int vf_f1cal_gpu_(cadmas_handle **h, const double *tnow, const double *dtnow, const int *nnow,
                  double *uu, double *vv, double *ww, double *pp, double *ff,
                  int *nf, int *indc, double *bcu, double *bcv, double *bcw,
                  double *bcp, double *bcf);

/* ---- Poisson solver alone (VF_M1BCGS, vf_m1bcgs.f:1-5) -----------------
   Device pointers, (NUMI,NUMJ,NUMK) each.  x0 is the initial guess on
   entry and the solution on exit when converged (vf_m1bcgs.f:251-261).
   iter receives ICGITR semantics (>icgmax not converged, -1 factorisation
   failed, -2 diverged); bnorm/xnorm receive the square roots of
   |M^-1 b|^2 and |M^-1 r|^2.  Scratch comes from the handle.            */
int cadmas_m1bcgs_dev(cadmas_handle *h,
                      const double *ad, const double *ali, const double *alj,
                      const double *alk, const double *aui, const double *auj,
                      const double *auk, const double *bb, double *x0,
                      const int *indc, int *iter, double *bnorm,
                      double *xnorm);

/* ---- Allocation-free divergence norm (no counterpart in the reference) --
   |VD| of VF_CDIV00 (vf_cdiv00.f:38-56), the value cadmas_divnorm returns
   for a handle's state, computed on arrays the caller holds on the device
   (device pointers, reference layout) without a handle and without
   allocating any memory: the row partials go to a static device array of
   CADMAS_NOALLOC_MAX_ROWS doubles (512 KB).  Runs on `stream`
   (cudaStream_t; NULL = the default stream), waits for it, writes the
   norm to *val (host).
     - NUMJ*NUMK above CADMAS_NOALLOC_MAX_ROWS: CADMAS_ESCRATCH, nothing runs.
     - Nothing in the scratch needs to start at zero (every partial is
       written before it is read).
     - The scratch is one array per device: calls that overlap in time on
       one device (any streams or threads) race; issue them one after
       another.
     - The first call on a device looks the scratch up
       (cudaGetSymbolAddress) and may load the module; make it before any
       phase that must not see such set-up work.
     - `stream` must belong to the current device: the scratch address
       is the current device's.  A stream of another device gets
       CADMAS_EINVAL and nothing runs.
     - A CUDA error that earlier work left pending is reported as
       CADMAS_ECUDA before anything is launched; cadmas_strerror names
       the failing call.                                                  */
#define CADMAS_NOALLOC_MAX_ROWS 65536
int cadmas_divnorm_noalloc(const cadmas_dims *d, const double *xx, const double *yy,
                           const double *zz, const double *ggx, const double *ggy,
                           const double *ggz, const double *uu, const double *vv,
                           const double *ww, const int *indc, void *stream, double *val);

/* Failure injection for tests (no counterpart in the reference): from
   wavefront step `from_step` on (>= 0), the MILU sweeps of this handle
   issue no bulk copies, so their bounded waits run out after
   wait_limit_s and the next solve returns CADMAS_ETIMEOUT; the kernels
   end normally and the handle stays usable.  A negative from_step turns
   the injection off.                                                    */
int cadmas_test_stall_sweeps(cadmas_handle *h, int from_step);

/* Side w->side as a wave maker driven by the wave `s` (WAVE-BC ... FUNC
   STREAM N): depth, period and fade-in from `w`; replaces
   VF_CWMAK0/1/2 calls of VF_BWUWN (vf_bwuwn.f:259-470) for that side.
   The same as cadmas_set_wave_func with a theory of type s->order.      */
int cadmas_set_wave_theory(cadmas_handle *h, const cadmas_wave_bc *w, const cadmas_stream_wave *s);

/* Side w->side as a wave maker driven by the theory `t` (WAVE-BC ... FUNC
   STREAM N | STOKES | CNOIDAL | STK-CND, solved by cadmas_wave_solve with
   the side's depth, height and period): each step the level at the side's
   phase (T0 = t->phase0) and the face velocities at the heights scaled to
   the column's water level (vf_bwuwn.f:259-470).                         */
int cadmas_set_wave_func(cadmas_handle *h, const cadmas_wave_bc *w, const cadmas_wave_theory *t);

/* Oblique incidence of the wave-maker side `side` (WAVE-BC ... ANGLE a X Y,
   BCTYP(9..11,JD)): the wave travels at `angle` degrees from the side's
   inward normal (counter-clockwise), its phase at TNOW = 0 being the
   theory's start phase on the line through (sx, sy) normal to the
   direction of travel.  Each column of the side then has its own phase,
   T0 - (TNOW/T - r/L) with r its distance along the direction of travel
   (vf_bwuwn.f:312-356, 418-430), its own level and its own velocities,
   the normal part times cos and the tangential part times sin of the
   direction.  angle = 0 is normal incidence.  Only wave theories take an
   angle: CADMAS_EINVAL for a matrix-table side ('(WAVE-BC ANGLE) CAN NOT
   USE.', vf_csetup.f:97-99).  Call after the side is set.               */
int cadmas_set_wave_angle(cadmas_handle *h, int side, double angle, double sx, double sy);

/* The wave source of the handle driven by the theory `t` (WAVE-SRC ...
   FUNC STREAM N | STOKES | CNOIDAL | STK-CND), solved with the source's
   depth, height and period: SRCUV of each line from VF_CWMAK2 at the
   heights scaled to the column's level (vf_cwmsrc.f:66-143).             */
int cadmas_set_wave_source_func(cadmas_handle *h, const cadmas_wave_src *s, const cadmas_wave_theory *t);

/* The wave source of the handle (one line, as the reference allows),
   with the matrix table `t` (NULL: the table already given to
   cadmas_set_wave is used).  CADMAS_EINVAL for a line outside the
   interior, MTBTYP 3 or no table.                                         */
int cadmas_set_wave_source(cadmas_handle *h, const cadmas_wave_src *s, const cadmas_wave_table *t);

/* The CUDA stream (cudaStream_t) on which every call of the handle issues
   its work; callers may record CUDA events on it or wait on it. */
int cadmas_get_stream(cadmas_handle *h, void **stream);

/* Number of kernels this library has launched in the process so far. */
long long cadmas_kernel_launches(void);

/* Per-stage GPU time.  While enabled, every launch of a stage is
   bracketed by two CUDA events on the handle's stream; ms[i] and count[i]
   receive the accumulated milliseconds and launches of stage i (see
   CADMAS_STAGE_*), for n <= CADMAS_NSTAGES stages.  enable < 0 only reads;
   enable 0/1 switches timing off/on and clears the totals. */
#define CADMAS_STAGE_FLUX      0  /* VF_VFLXDU/DV/DW                          */
#define CADMAS_STAGE_PREDICT   1  /* VF_VGENE + VF_VEULER                     */
#define CADMAS_STAGE_VPCOEF    2  /* VF_VPCOEF                                */
#define CADMAS_STAGE_DCMP      3  /* VF_MZDCMP                                */
#define CADMAS_STAGE_FWD       4  /* VF_MZAX + VF_MZFRWD (fused)              */
#define CADMAS_STAGE_BWD       5  /* VF_MZBKWD                                */
#define CADMAS_STAGE_DOT       6  /* VF_MZIP dot products and scalar updates  */
#define CADMAS_STAGE_VEC       7  /* BiCGSTAB vector updates                  */
#define CADMAS_STAGE_MODIF     8  /* VF_VMODIF and the V1CAL boundary rules   */
#define CADMAS_STAGE_VOF       9  /* FCONV, FEULER, FMOD1, FCUT01             */
#define CADMAS_STAGE_FLAGS    10  /* FNFINI, FBUBUP, FNFPRV, CINDC            */
#define CADMAS_STAGE_FBC      11  /* F1CAL boundary rules, BSPPFL             */
#define CADMAS_STAGE_TURB     12  /* k-epsilon: VF_K1CAL and the updates after
                                     F1CAL (LEQK != 0)                       */
#define CADMAS_STAGE_WARM     13  /* learned initial guess (warm_start 2)      */
#define CADMAS_NSTAGES        14
int cadmas_stage_timers(cadmas_handle *h, int enable, double *ms, long long *count, int n);

const char *cadmas_strerror(int status);

#ifdef __cplusplus
}
#endif
#endif /* CADMAS_GPU_H */
