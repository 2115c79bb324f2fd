// api.cu -- handle, device memory and the step driver behind the C ABI of
// include/cadmas_gpu.h.
//
// The driver issues the kernels in the call order of VF_V1CAL
// (vf_v1cal.f:118-297) and VF_F1CAL (vf_f1cal.f:121-243) on one stream.
// Host synchronisation happens only where the reference itself takes a
// data-dependent branch on a global value: the BiCGSTAB convergence test
// (batched, see solve()), the NF fixed-point loop of VF_FNFINI, and the
// error flags at the end of a step.
#include <cuda_runtime.h>
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "cadmas_dev.cuh"
#include "kernels.h"

using namespace cadmas;

std::atomic<long long> cadmas::g_kernel_launches{0};

namespace {
thread_local std::string g_last_error;

#define CK(call)                                                              \
  do {                                                                        \
    cudaError_t e_ = (call);                                                  \
    if (e_ != cudaSuccess) {                                                  \
      g_last_error = std::string(#call) + ": " + cudaGetErrorString(e_);      \
      return CADMAS_ECUDA;                                                    \
    }                                                                         \
  } while (0)

template <class T> int dalloc(T **p, size_t n) {
  cudaError_t e = cudaMalloc((void **)p, std::max<size_t>(n, 1) * sizeof(T));
  if (e != cudaSuccess) { g_last_error = cudaGetErrorString(e); *p = nullptr; return CADMAS_ENOMEM; }
  e = cudaMemset(*p, 0, std::max<size_t>(n, 1) * sizeof(T));
  if (e != cudaSuccess) { g_last_error = cudaGetErrorString(e); return CADMAS_ECUDA; }
  return CADMAS_OK;
}
}  // namespace

// Optional per-stage GPU timing with CUDA event pairs on the handle stream.
struct StageTimer {
  bool on = false;
  std::vector<cudaEvent_t> pool;
  struct Pend { int stage; cudaEvent_t a, b; };
  std::vector<Pend> pend;
  cudaEvent_t open_a = nullptr;
  int open_stage = -1;
  double ms[CADMAS_NSTAGES] = {0};
  long long cnt[CADMAS_NSTAGES] = {0};
  cudaEvent_t get() {
    if (pool.empty()) {
      cudaEvent_t e;
      cudaEventCreate(&e);
      return e;
    }
    cudaEvent_t e = pool.back();
    pool.pop_back();
    return e;
  }
  void begin(cudaStream_t s, int stage) {
    if (!on) return;
    open_a = get();
    cudaEventRecord(open_a, s);
    open_stage = stage;
  }
  void end(cudaStream_t s) {
    if (!on || open_stage < 0) return;
    cudaEvent_t b = get();
    cudaEventRecord(b, s);
    pend.push_back({open_stage, open_a, b});
    open_stage = -1;
  }
  void resolve() {
    for (Pend &q : pend) {
      float t = 0.0f;
      cudaEventSynchronize(q.b);
      cudaEventElapsedTime(&t, q.a, q.b);
      ms[q.stage] += t;
      cnt[q.stage] += 1;
      pool.push_back(q.a);
      pool.push_back(q.b);
    }
    pend.clear();
  }
  void clear() {
    resolve();
    for (int i = 0; i < CADMAS_NSTAGES; ++i) { ms[i] = 0.0; cnt[i] = 0; }
  }
  ~StageTimer() {
    resolve();
    for (cudaEvent_t e : pool) cudaEventDestroy(e);
  }
};

struct cadmas_handle {
  int device = 0;
  cudaStream_t s = nullptr;
  cadmas_params P;
  Geo g;
  Prm p;
  Fld f;
  size_t N = 0, NB = 0;
  int TI = 0, TJ = 0;
  bool have_static = false;
  // static
  double *xx = nullptr, *yy = nullptr, *zz = nullptr;
  double *ggv = nullptr, *ggx = nullptr, *ggy = nullptr, *ggz = nullptr;
  double *glv = nullptr, *glx = nullptr, *gly = nullptr, *glz = nullptr, *cd0 = nullptr, *anu = nullptr;
  int *indx = nullptr, *indy = nullptr, *indz = nullptr, *indb = nullptr;
  // state (velocities and pressure double-buffered)
  double *vel[2][3] = {{nullptr, nullptr, nullptr}, {nullptr, nullptr, nullptr}};
  int cur = 0;
  double *pbuf[2] = {nullptr, nullptr};
  int pcur = 0;
  double *ff = nullptr;
  int *nf = nullptr, *indc = nullptr, *nf0 = nullptr, *nlim = nullptr;
  double *bcu = nullptr, *bcv = nullptr, *bcw = nullptr, *bcp = nullptr, *bcf = nullptr;
  // work: 9 flux arrays, reused as the Poisson system (0..7) and PT (8)
  double *wk[9] = {nullptr};
  // solver scratch
  double *xw = nullptr, *y2 = nullptr, *r0 = nullptr, *rr = nullptr, *pv = nullptr,
         *ap = nullptr, *ae = nullptr;
  double *rb0 = nullptr, *rb1 = nullptr, *dres = nullptr;
  double *rb5 = nullptr;  // 5 x nslab sum partials of the regrouped FP32 iteration (solver 1)
  // skewed-layout copies of the system for the MILU kernels, and the
  // forward-sweep result
  SkewGeo q;
  SkewSys S;
  double *bb_sl = nullptr;
  // FP32 system and inner-solve vectors of the mixed solver (solver 1)
  SkewSysF Sf{nullptr, nullptr};
  float *bf = nullptr, *xf = nullptr, *r0f = nullptr, *rrf = nullptr, *pvf = nullptr, *apf = nullptr,
        *aef = nullptr, *y2f = nullptr;
  long long mixed_outer = 0, mixed_fallback = 0;  // refinement passes and FP64 fallbacks so far
  int warm_now = 0;  // the next solve starts from the previous solution (warm_start 1)
  bool have_prev = false;  // xw holds a converged solution of an earlier step
  size_t nsl = 0;        // entries of a skewed vector
  long long nslab = 0;   // slabs of a skewed vector
  long long nrb = 0;     // block partials of a slab sum (slabs / 8, rounded up)
  SolveState *st = nullptr;
  int *dint = nullptr;            // [0] err [1] nch [2] done [3] iter [4] nums
  unsigned char *active = nullptr;
  // pinned host mirrors
  SolveState *h_st = nullptr;
  int *h_int = nullptr;
  double *h_res = nullptr;
  // host-side scalars
  std::vector<double> tbub;
  DropArrays drop{};  // DROPTX..DROPWW (the droplet model's state)
  // k-epsilon (LEQK != 0): AK, AE and their second buffers, ANUT; BCK, BCE,
  // the input values BCK0, BCE0 and the types INDBK, INDBE
  double *ak = nullptr, *ae_k = nullptr, *ak2 = nullptr, *ae2 = nullptr, *anut = nullptr;
  double *bck = nullptr, *bce = nullptr, *bck0 = nullptr, *bce0 = nullptr;
  int *indbk = nullptr, *indbe = nullptr;
  // learned initial guess (warm_start 2): the network, two row buffers,
  // [scale, |r|^2, |b|^2] and [kept, dropped, dropped now]
  cadmas_unet *wnet = nullptr;
  double *ws_rows = nullptr, *ws_scal = nullptr;
  int *ws_cnt = nullptr;
  std::vector<double> zz2;  // ZZ(2,K) on the host, K = 1..NK
  std::vector<unsigned char> h_active;
  double tnow = 0.0, dtnow = 0.0;
  int nnow = 0;
  cadmas_stats stats;
  int last_iter = 8;   // iterations of the previous solve: size of the first batch
  StageTimer tm;
  // wave maker (matrix table): sides JD = 1..4, one table for all of them
  struct WaveSide {
    bool on = false;
    int first = 0, last = 0;
    double d = 0.0, t = 0.0, a = 0.0;
    bool theory = false;     // FUNC STREAM N | STOKES | CNOIDAL: the wave `th`, not the table
    cadmas_wave_theory th{};
    double angle = 0.0, sx = 0.0, sy = 0.0;  // ANGLE: BCTYP(9..11,JD)
    int ncol = 0;                 // oblique incidence: lines first..last, their
    WaveCol *col = nullptr;       // level and phase part (device),
    WaveCol *col_h = nullptr;     // the pinned host copy they are filled in,
    cudaEvent_t col_ev = nullptr; // and the end of its last upload
  } wave[4];
  std::vector<double> xx1, yy1;  // XX(1,I), YY(1,J) on the host, 1-based
  // open (radiation) boundary: sides JD = 1..4 and their phase speed C
  struct OpenSide {
    bool on = false;
    double c = 0.0;
  } open[4];
  long long n_open_faces = 0;  // faces with INDB(3,L) = 7
  long long n_log_faces = 0;   // faces with INDB(3,L) = 6 or 8 (log-law, rough)
  double *bcvi = nullptr;      // BCVI roughness (NUMB)
  int mtbtyp = 0, mtbnow = 0;  // MTBTYP, MTBNOW (persists between calls, vf_a2dflt.f:114)
  double dmtbt0 = 0.0;
  std::vector<double> wtt, whh;  // DMTBTT, DMTBHH (host)
  int nzz = 0;
  double *wzz = nullptr, *wun = nullptr, *wut = nullptr;  // DMTBZZ, DMTBUN, DMTBUT (device)
  double wave_level[4] = {0, 0, 0, 0};  // BCTYP(7,JD) = WVZ*AW of the last call
  // wave source (ISCTYP(1) = line, SCTYP(1,3,8) = d, t, a) and its SRCUV
  struct WaveSrc {
    bool on = false;
    int line = 0;
    double d = 0.0, t = 0.0, a = 0.0;
    bool theory = false;          // a wave theory `th` instead of the table
    cadmas_wave_theory th{};
  } src;
  double *srcuv = nullptr;
  double src_level = 0.0;  // SCTYP(7) = WVZ*AW of the last step
};

#define TB(stage) h->tm.begin(h->s, (stage))
#define TE() h->tm.end(h->s)

static void refresh_fld(cadmas_handle *h) {
  Fld &f = h->f;
  f.ggv = h->ggv; f.ggx = h->ggx; f.ggy = h->ggy; f.ggz = h->ggz;
  f.glv = h->glv; f.glx = h->glx; f.gly = h->gly; f.glz = h->glz;
  f.cd0 = h->cd0; f.anu = h->anu;
  f.indx = h->indx; f.indy = h->indy; f.indz = h->indz; f.indb = h->indb;
  f.uu = h->vel[h->cur][0]; f.vv = h->vel[h->cur][1]; f.ww = h->vel[h->cur][2];
  f.pp = h->pbuf[h->pcur];
  f.ff = h->ff; f.nf = h->nf; f.indc = h->indc; f.nf0 = h->nf0;
  f.bcu = h->bcu; f.bcv = h->bcv; f.bcw = h->bcw; f.bcp = h->bcp; f.bcf = h->bcf;
  f.bcvi = h->bcvi;
  f.srcuv = h->srcuv;
}

static void refresh_prm(cadmas_handle *h) {
  const cadmas_params &P = h->P;
  Prm &p = h->p;
  p.rho0 = P.rho0; p.grz0 = P.grz0; p.vvmax = P.vvmax; p.cgpara = P.cgpara; p.cgepsa = P.cgepsa;
  p.cgepsr = P.cgepsr; p.cgdiv = P.cgdiv; p.flower = P.flower; p.fupper = P.fupper;
  p.plower = P.plower; p.scmvp = P.scmvp; p.wvlvl = P.wvlvl; p.wbub = P.wbub;
  p.glxmin = P.glxmin; p.glxmax = P.glxmax; p.glymin = P.glymin; p.glymax = P.glymax;
  p.dtnow = h->dtnow; p.tnow = h->tnow;
  p.icgtyp = P.icgtyp; p.icgmax = P.icgmax; p.ibsuw0 = P.ibsuw0;
  p.akk0 = P.akk0; p.aka0 = P.aka0; p.anu0 = P.anu0;
  p.loglaw = h->n_log_faces > 0 ? 1 : 0;
  for (int d = 0; d < 4; ++d) p.fixlvl[d] = (h->wave[d].on && !h->wave[d].theory && h->mtbtyp == 3) ? 1 : 0;
  p.iws = (h->src.on && h->src.line > 0) ? h->src.line : 0;
  p.jws = (h->src.on && h->src.line < 0) ? -h->src.line : 0;
  // sponge parameters of vf_veuler.f:77-113
  p.ipa = 0;
  for (int d = 0; d < 4; ++d) {
    p.ip[d] = P.idamp[d];
    p.sw[d] = p.spx[d] = p.spz[d] = 0.0;
    if (p.ip[d] >= 0) {
      p.ipa = p.ipa + 1;
      double D = std::sqrt(P.grz0 / P.damp[d][3]);
      p.sw[d] = P.damp[d][2];
      p.spx[d] = (double)(p.ip[d] + 1) * P.damp[d][0] * D;
      p.spz[d] = (double)(p.ip[d] + 1) * P.damp[d][1] * D;
    }
  }
}

static long long nrows(const cadmas_handle *h) { return (long long)h->g.NJ * h->g.NK; }

// VF_CWMTB1 (vf_cwmtb1.f:26-69): weights of the table rows around phase
// WVT and the interpolated level; the search starts at MTBNOW.
static bool cwmtb1(cadmas_handle *h, double WVT, double &W1, double &W2, double &WVZ) {
  const std::vector<double> &TT = h->wtt;
  const int MTBTT = (int)TT.size();
  int &MTBNOW = h->mtbnow;
  if (MTBNOW <= 0) MTBNOW = MTBTT - 1;
  if (WVT <= TT[0]) {
    MTBNOW = 1; W1 = 1.0; W2 = 0.0;
  } else if (WVT >= TT[MTBTT - 1]) {
    MTBNOW = MTBTT - 1; W1 = 0.0; W2 = 1.0;
  } else {
    int IP = 0;
    W1 = W2 = 0.0;
    for (int I = MTBNOW; I >= 1; --I)
      if (TT[I - 1] <= WVT && WVT <= TT[I]) {
        IP = I; W2 = 1.0 / (TT[I] - TT[I - 1]); W1 = (TT[I] - WVT) * W2; W2 = (WVT - TT[I - 1]) * W2;
        break;
      }
    if (IP == 0)
      for (int I = MTBTT - 1; I >= MTBNOW + 1; --I)
        if (TT[I - 1] <= WVT && WVT <= TT[I]) {
          IP = I; W2 = 1.0 / (TT[I] - TT[I - 1]); W1 = (TT[I] - WVT) * W2; W2 = (WVT - TT[I - 1]) * W2;
          break;
        }
    if (IP == 0) return false;  // 'P.G ERROR.'
    MTBNOW = IP;
  }
  WVZ = (h->mtbtyp != 2) ? W1 * h->whh[MTBNOW - 1] + W2 * h->whh[MTBNOW] : 0.0;
  return true;
}

// Wave-maker part of VF_BWUWN (vf_bwuwn.f:259-470): the time part here
// (phase, fade-in, the table's row weights or the theory's level and phase
// part, per line under oblique incidence), the faces on the device (k_wave).
static int wave_bc(cadmas_handle *h) {
  const double PI = 3.141592653589794, ZERO = 1.0e-20;  // VF_A0PRM.h
  for (int jd = 0; jd < 4; ++jd) {
    cadmas_handle::WaveSide &ws = h->wave[jd];
    if (!ws.on) continue;
    const double T = ws.t, T0 = ws.theory ? ws.th.phase0 : h->dmtbt0;
    float R4TN = (float)(T0 - h->tnow / T);
    R4TN = R4TN - (float)(int)R4TN;
    if (R4TN < 0.0f) R4TN = R4TN + 1.0f;
    double AW = 1.0, A = ws.a;
    if (A >= ZERO) {
      A = h->tnow / T / A;
      if (A < 1.0) AW = 0.5 * std::sin(PI * (A - 0.5)) + 0.5;
    }
    const double WVT = (double)R4TN;
    WaveDev w;
    w.theory = ws.theory ? 1 : 0;
    w.col = nullptr;
    if (ws.theory) {  // VF_CWMAK1: the level at the phase; VF_CWMAK2 per face on the device
      w.wvz = theory_eta(ws.th, WVT);
      theory_phase(ws.th, WVT, w.ph);
      w.wt1 = w.wt2 = 0.0;
    } else {
      if (!cwmtb1(h, WVT, w.wt1, w.wt2, w.wvz)) return CADMAS_EPG;
      std::memset(&w.ph, 0, sizeof(w.ph));
    }
    h->wave_level[jd] = w.wvz * AW;
    w.side = jd + 1; w.first = ws.first; w.last = ws.last;
    w.mtbtyp = ws.theory ? 1 : h->mtbtyp; w.nzz = h->nzz; w.mtbnow = h->mtbnow;
    w.d = ws.d; w.aw = AW; w.wvlvl = h->P.wvlvl;
    w.sa = (jd == 0) ? 1.0 : (jd == 1 ? -1.0 : 0.0);  // normal incidence (vf_bwuwn.f:298-310)
    w.sb = (jd == 2) ? 1.0 : (jd == 3 ? -1.0 : 0.0);
    if (ws.theory && std::fabs(ws.angle) > ZERO) {
      // oblique incidence (vf_bwuwn.f:312-324): the direction of travel,
      // then each line's phase from its distance along it (345-356 on
      // the X sides at the face's x and the cell's middle y, 418-430 on
      // the Y sides the other way round)
      const double off[4] = {0.0, 180.0, 90.0, 270.0};
      double SA = (ws.angle + off[jd]) * PI / 180.0;
      const double SB = std::sin(SA);
      SA = std::cos(SA);
      const double SC = -(SA * ws.sx + SB * ws.sy), DL = ws.th.length;
      if (ws.col_ev) CK(cudaEventSynchronize(ws.col_ev));  // the last upload of col_h is done
      const bool xs = jd <= 1;
      const int NI = h->g.NI, NJ = h->g.NJ;
      for (int n = ws.first; n <= ws.last; ++n) {
        double X0, Y0;
        if (xs) { X0 = h->xx1[jd == 0 ? 2 : NI]; Y0 = (h->yy1[n] + h->yy1[n + 1]) * 0.5; }
        else { Y0 = h->yy1[jd == 2 ? 2 : NJ]; X0 = (h->xx1[n] + h->xx1[n + 1]) * 0.5; }
        const double RR = (SA * X0 + SB * Y0 + SC) / std::sqrt(SA * SA + SB * SB);
        float R4 = (float)(T0 - (h->tnow / T - RR / DL));
        R4 = R4 - (float)(int)R4;
        if (R4 < 0.0f) R4 = R4 + 1.0f;
        WaveCol &c = ws.col_h[n - ws.first];
        c.wvz = theory_eta(ws.th, (double)R4);
        theory_phase(ws.th, (double)R4, c.ph);
      }
      CK(cudaMemcpyAsync(ws.col, ws.col_h, (size_t)ws.ncol * sizeof(WaveCol), cudaMemcpyHostToDevice, h->s));
      CK(cudaEventRecord(ws.col_ev, h->s));
      w.col = ws.col;
      w.sa = SA; w.sb = SB;
    }
    w.zz = h->wzz; w.un = h->wun; w.ut = h->wut;
    // a fixed-water-level table sets no velocities (vf_bwuwn.f:330-331)
    if (ws.theory || h->mtbtyp != 3) launch_wave(h->s, h->g, h->f, w, h->dint);
  }
  return CADMAS_OK;
}

// VF_CWMSRC (vf_cwmsrc.f:46-143): the phase and fade-in at TNOW and
// VF_CWMTB1's row weights or the theory's level and phase part on the
// host, SRCUV of every line of the source on the device (k_srcuv).  The
// reference calls it at TNOW + DT before the step's V1CAL, which is this
// step's TNOW.
static int wave_src(cadmas_handle *h) {
  const double PI = 3.141592653589794, ZERO = 1.0e-20;  // VF_A0PRM.h
  const cadmas_handle::WaveSrc &ws = h->src;
  const double T = ws.t, T0 = ws.theory ? ws.th.phase0 : h->dmtbt0;
  float R4TN = (float)(T0 - h->tnow / T);
  R4TN = R4TN - (float)(int)R4TN;
  if (R4TN < 0.0f) R4TN = R4TN + 1.0f;
  double AW = 1.0, A = ws.a;
  if (A >= ZERO) {
    A = h->tnow / T / A;
    if (A < 1.0) AW = 0.5 * std::sin(PI * (A - 0.5)) + 0.5;
  }
  WaveDev w;
  w.col = nullptr;
  w.theory = ws.theory ? 1 : 0;
  if (ws.theory) {
    w.wvz = theory_eta(ws.th, (double)R4TN);
    theory_phase(ws.th, (double)R4TN, w.ph);
    w.wt1 = w.wt2 = 0.0;
  } else {
    if (!cwmtb1(h, (double)R4TN, w.wt1, w.wt2, w.wvz)) return CADMAS_EPG;
    std::memset(&w.ph, 0, sizeof(w.ph));
  }
  h->src_level = w.wvz * AW;
  w.side = ws.line; w.first = 0; w.last = 0;
  w.mtbtyp = ws.theory ? 1 : h->mtbtyp; w.nzz = h->nzz; w.mtbnow = h->mtbnow;
  w.d = ws.d; w.aw = AW; w.wvlvl = h->P.wvlvl;
  w.sa = 0.0; w.sb = 0.0;
  w.zz = h->wzz; w.un = h->wun; w.ut = h->wut;
  launch_srcuv(h->s, h->g, h->f, w, h->srcuv, h->dint);
  return CADMAS_OK;
}

// VF_BWFFSF (vf_bwffsf.f:43-128): on the sides whose table fixes the water
// level (MTBTYP 3), F of the column next to the side from the level
// WVLVL + the table's level (faded in as VF_BWUWN does) at TNOW.
static int fixed_level_f(cadmas_handle *h) {
  if (h->mtbtyp != 3) return CADMAS_OK;
  const double PI = 3.141592653589794, ZERO = 1.0e-20;
  for (int jd = 0; jd < 4; ++jd) {
    const cadmas_handle::WaveSide &ws = h->wave[jd];
    if (!ws.on || ws.theory) continue;
    const double T = ws.t, T0 = h->dmtbt0;
    float R4TN = (float)(T0 - h->tnow / T);
    R4TN = R4TN - (float)(int)R4TN;
    if (R4TN < 0.0f) R4TN = R4TN + 1.0f;
    double AW = 1.0, A = ws.a;
    if (A >= ZERO) {
      A = h->tnow / T / A;
      if (A < 1.0) AW = 0.5 * std::sin(PI * (A - 0.5)) + 0.5;
    }
    double W1, W2, WVZ;
    if (!cwmtb1(h, (double)R4TN, W1, W2, WVZ)) return CADMAS_EPG;
    h->wave_level[jd] = WVZ * AW;
    launch_bwffsf(h->s, h->g, h->f, jd + 1, ws.first, ws.last, h->P.wvlvl + h->wave_level[jd]);
  }
  return CADMAS_OK;
}

// Open (radiation) part of VF_BWUWN (vf_bwuwn.f:481-598): the phase speed
// of each open side was fixed by cadmas_set_open; the faces are set on the
// device (k_open) from the velocities ub, vb, wb.
static int open_bc(cadmas_handle *h, const double *ub, const double *vb, const double *wb) {
  bool any = false;
  for (int jd = 0; jd < 4; ++jd) {
    if (!h->open[jd].on) continue;
    any = true;
    const OpenDev o{jd + 1, h->nnow, h->open[jd].c, h->dtnow};
    launch_open(h->s, h->g, h->f, o, ub, vb, wb, h->dint);
  }
  if (!any && h->n_open_faces > 0) {
    g_last_error = "faces of type 7 (open boundary) but no side declared open (cadmas_set_open)";
    return CADMAS_EINVAL;
  }
  return CADMAS_OK;
}

// ------------------------------------------------------------ solver
// VF_M1BCGS on the system a with initial guess/result x0.  The BiCGSTAB
// scalars stay on the device; iterations are issued in batches and every
// kernel returns at once after convergence, so results do not depend on
// the batch size.  The host reads the scalars once per batch.
static int solve(cadmas_handle *h, const SysPtr &a, double *x0, const int *indc, int &iter,
                 double &bnorm, double &xnorm) {
  cudaStream_t s = h->s;
  const Geo &g = h->g;
  const size_t vbytes = h->nsl * sizeof(double);
  const double epsa2 = h->P.cgepsa * h->P.cgepsa, epsr2 = h->P.cgepsr * h->P.cgepsr,
               div2 = h->P.cgdiv * h->P.cgdiv;
  const int icgmax = h->P.icgmax;
  const long long nr = h->nrb;
  SolveState *st = h->st;
  const SkewGeo &q = h->q;
  const SkewSys &S = h->S;
  const int *ic = S.indc;  // INDC in the skewed layout (-1 on padding)
  // vf_m1bcgs.f:79-95: XW = X0, work vectors zero
  double *zero_list[] = {h->y2, h->r0, h->rr, h->pv, h->ap, h->ae};
  for (double *z : zero_list) CK(cudaMemsetAsync(z, 0, vbytes, s));
  CK(cudaMemsetAsync(st, 0, SOLVE_CLEAR_BYTES, s));
  const double U = (h->P.icgtyp != 0) ? h->P.cgpara : 0.0;
  TB(CADMAS_STAGE_DCMP);
  launch_to_skew(s, g, q, a, indc, S, x0, h->bb_sl, h->xw, h->warm_now);
  launch_dcmp(s, g, q, U, S, &st->pivot_bad);
  launch_pivot_check(s, st);
  TE();
  // YY = MINV*BB, BNORM = (YY,YY)
  TB(CADMAS_STAGE_FWD); launch_fwd(s, g, q, S, h->bb_sl, nullptr, st, h->y2); TE();
  TB(CADMAS_STAGE_BWD); launch_bwd(s, g, q, S, h->y2, st); TE();
  TB(CADMAS_STAGE_DOT);
  launch_dot(s, q, ic, h->y2, h->y2, nullptr, nullptr, h->rb0, nullptr, st);
  launch_fin(s, FIN_BNORM, h->rb0, nullptr, nr, st, nullptr, epsa2, epsr2, div2, icgmax);
  TE();
  // YY = A*XW; YY = BB - YY; R0 = MINV*YY; S = (R0,R0)
  TB(CADMAS_STAGE_VEC);
  launch_spmv(s, g, q, S, h->xw, h->y2, st);
  launch_bmy(s, q, ic, h->bb_sl, h->y2, st);
  TE();
  TB(CADMAS_STAGE_FWD); launch_fwd(s, g, q, S, h->y2, nullptr, st, h->y2); TE();
  TB(CADMAS_STAGE_BWD); launch_bwd(s, g, q, S, h->r0, st); TE();
  TB(CADMAS_STAGE_DOT);
  launch_dot(s, q, ic, h->r0, h->r0, nullptr, nullptr, h->rb0, nullptr, st);
  launch_fin(s, FIN_START, h->rb0, nullptr, nr, st, nullptr, epsa2, epsr2, div2, icgmax);
  TE();
  TB(CADMAS_STAGE_VEC); launch_copy2(s, q, ic, h->r0, h->rr, h->pv, st); TE();
  // First batch as long as the previous solve; after that batches of 4.
  int batch = std::max(2, std::min(h->last_iter, 64));
  for (int guard = 0; guard < 100000; ++guard) {
    for (int b = 0; b < batch; ++b) {
      // AP = MINV*(A*PP); ALPHA = S/(R0,AP); RR -= ALPHA*AP
      TB(CADMAS_STAGE_FWD); launch_fwd(s, g, q, S, nullptr, h->pv, st, h->y2); TE();
      TB(CADMAS_STAGE_BWD); launch_bwd(s, g, q, S, h->ap, st); TE();
      TB(CADMAS_STAGE_DOT);
      launch_dot(s, q, ic, h->r0, h->ap, nullptr, nullptr, h->rb0, nullptr, st);
      launch_fin(s, FIN_ALPHA, h->rb0, nullptr, nr, st, nullptr, epsa2, epsr2, div2, icgmax);
      TE();
      TB(CADMAS_STAGE_VEC); launch_axpy_rr(s, q, ic, h->ap, h->rr, st); TE();
      // AE = MINV*(A*RR); OMEGA = (RR,AE)/(AE,AE)
      TB(CADMAS_STAGE_FWD); launch_fwd(s, g, q, S, nullptr, h->rr, st, h->y2); TE();
      TB(CADMAS_STAGE_BWD); launch_bwd(s, g, q, S, h->ae, st); TE();
      TB(CADMAS_STAGE_DOT);
      launch_dot(s, q, ic, h->rr, h->ae, h->ae, h->ae, h->rb0, h->rb1, st);
      launch_fin(s, FIN_OMEGA, h->rb0, h->rb1, nr, st, nullptr, epsa2, epsr2, div2, icgmax);
      TE();
      // XW += ALPHA*PP + OMEGA*RR; RR -= OMEGA*AE; convergence; BETA
      TB(CADMAS_STAGE_VEC);
      launch_upd_xr(s, q, ic, h->pv, h->ae, h->r0, h->xw, h->rr, h->rb0, h->rb1, st);
      launch_fin(s, FIN_CONV, h->rb0, h->rb1, nr, st, nullptr, epsa2, epsr2, div2, icgmax);
      launch_upd_p(s, q, ic, h->rr, h->ap, h->pv, st);
      TE();
    }
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(h->h_st, st, sizeof(SolveState), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if (h->h_st->timeout) {
      g_last_error = "a bulk-copy wait of the MILU sweep ran out of time";
      return CADMAS_ETIMEOUT;
    }
    if (h->h_st->done) break;
    batch = 4;
  }
  launch_x0(s, g, q, ic, h->xw, x0, st);
  CK(cudaGetLastError());
  const SolveState &hs = *h->h_st;
  iter = hs.iter;
  if (iter > 0) h->last_iter = iter;
  if (iter == -1) { bnorm = 0.0; xnorm = 0.0; }
  else { bnorm = std::sqrt(hs.bnorm); xnorm = std::sqrt(hs.xnorm); }
  return CADMAS_OK;
}

// ------------------------------------------------ mixed-precision solver
// One FP32 MILU-BiCGSTAB solve of A d = bf from d = 0 (the iteration of
// VF_M1BCGS, vf_m1bcgs.f:76-266, on the FP32 copy of the system), to the
// reference's criterion |M^-1 r| <= eps |M^-1 bf|.  Returns the
// iteration count in `iter` with VF_M1BCGS's meaning (-1 factor failed,
// -2 diverged, > icgmax not converged).
static int solve_inner_f(cadmas_handle *h, double eps, int &iter) {
  cudaStream_t s = h->s;
  const Geo &g = h->g;
  const SkewGeo &q = h->q;
  const SkewSysF &S = h->Sf;
  const int *ic = S.indc;
  const long long nr = h->nrb;
  SolveState *st = h->st;
  const double epsa2 = h->P.cgepsa * h->P.cgepsa, epsr2 = eps * eps, div2 = h->P.cgdiv * h->P.cgdiv;
  const int icgmax = h->P.icgmax;
  const size_t vb = h->nsl * sizeof(float);
  const bool fused_dots = h->P.dot_passes == 0;
  float *zl[] = {h->xf, h->r0f, h->rrf, h->pvf, h->apf, h->aef};
  for (float *z : zl) CK(cudaMemsetAsync(z, 0, vb, s));
  CK(cudaMemsetAsync(st, 0, SOLVE_CLEAR_BYTES, s));
  // YY = MINV*BB, BNORM = (YY,YY); with XW = 0, R0 = YY and S = BNORM
  TB(CADMAS_STAGE_FWD); launch_fwd_f(s, g, q, S, h->bf, nullptr, st, h->y2f); TE();
  TB(CADMAS_STAGE_BWD); launch_bwd_f(s, g, q, S, h->r0f, st); TE();
  TB(CADMAS_STAGE_DOT);
  launch_dot_t<float>(s, q, ic, h->r0f, h->r0f, nullptr, nullptr, h->rb0, nullptr, st);
  launch_fin(s, FIN_BNORM, h->rb0, nullptr, nr, st, nullptr, epsa2, epsr2, div2, icgmax);
  launch_fin(s, FIN_START, h->rb0, nullptr, nr, st, nullptr, epsa2, epsr2, div2, icgmax);
  TE();
  TB(CADMAS_STAGE_VEC); launch_copy2_t<float>(s, q, ic, h->r0f, h->rrf, h->pvf, st); TE();
  int batch = std::max(2, std::min(h->last_iter, 64));
  for (int guard = 0; guard < 100000; ++guard) {
    for (int b = 0; b < batch; ++b) {
      // AP = MINV*(A*PP); ALPHA = S/(R0,AP); RR -= ALPHA*AP.  (R0,AP) is
      // summed by the backward sweep itself where the layout allows
      // (one partial per tile), else by its own pass.
      TB(CADMAS_STAGE_FWD); launch_fwd_f(s, g, q, S, nullptr, h->pvf, st, h->y2f); TE();
      TB(CADMAS_STAGE_BWD);
      const bool d1 = fused_dots && launch_bwd_f_dot1(s, g, q, S, h->r0f, h->apf, h->rb0, st);
      if (!d1) launch_bwd_f(s, g, q, S, h->apf, st);
      TE();
      TB(CADMAS_STAGE_DOT);
      if (!d1) launch_dot2f(s, q, h->r0f, h->apf, h->rb0, st);
      launch_fin(s, FIN_ALPHA, h->rb0, nullptr, d1 ? (long long)q.nb : nr, st, nullptr, epsa2, epsr2, div2, icgmax);
      TE();
      TB(CADMAS_STAGE_VEC); launch_axpyf(s, q, h->apf, h->rrf, st); TE();
      // AE = MINV*(A*RR); the five sums; OMEGA, convergence, BETA; XW,
      // RR and PP in one pass
      TB(CADMAS_STAGE_FWD); launch_fwd_f(s, g, q, S, nullptr, h->rrf, st, h->y2f); TE();
      TB(CADMAS_STAGE_BWD);
      const bool d5 = fused_dots && launch_bwd_f_dot5(s, g, q, S, h->r0f, h->rrf, h->aef, h->rb5, st);
      if (!d5) launch_bwd_f(s, g, q, S, h->aef, st);
      TE();
      TB(CADMAS_STAGE_DOT);
      if (!d5) launch_dot5f(s, q, h->r0f, h->rrf, h->aef, h->rb5, st);
      launch_fin5(s, h->rb5, d5 ? (long long)q.nb : nr, st, epsa2, epsr2, div2, icgmax);
      TE();
      TB(CADMAS_STAGE_VEC);
      launch_upd3f(s, q, h->aef, h->apf, h->xf, h->rrf, h->pvf, st);
      launch_commit(s, st);
      TE();
    }
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(h->h_st, st, sizeof(SolveState), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if (h->h_st->timeout) {
      g_last_error = "a bulk-copy wait of the MILU sweep ran out of time";
      return CADMAS_ETIMEOUT;
    }
    if (h->h_st->done) break;
    batch = 4;
  }
  iter = h->h_st->iter;
  return CADMAS_OK;
}

// Mixed-precision solve of A x = b (solver 1): FP32 MILU factor and FP32
// inner BiCGSTAB solves of A d = r / |r| under FP64 iterative refinement,
// x += |r| d, with r = b - A x and its norm in FP64, until
// |b - A x| <= CGEPSR |b|.  A failed FP32 factor or inner solve hands the
// system to the FP64 solve.  iter = inner iterations of all passes.
static int solve(cadmas_handle *h, const SysPtr &a, double *x0, const int *indc, int &iter,
                 double &bnorm, double &xnorm);
static int solve_mixed(cadmas_handle *h, const SysPtr &a, double *x0, const int *indc, int &iter,
                       double &bnorm, double &xnorm) {
  cudaStream_t s = h->s;
  const Geo &g = h->g;
  const SkewGeo &q = h->q;
  const int *ic = h->S.indc;
  const long long nr = h->nrb;
  SolveState *st = h->st;
  h->Sf.indc = h->S.indc;
  const double U = (h->P.icgtyp != 0) ? h->P.cgpara : 0.0;
  TB(CADMAS_STAGE_DCMP);
  launch_to_skew(s, g, q, a, indc, h->S, x0, h->bb_sl, h->xw, h->warm_now);
  launch_sys_to_f(s, q, h->S.sys, h->Sf.sys);
  CK(cudaMemsetAsync(st, 0, SOLVE_CLEAR_BYTES, s));
  launch_dcmp_f(s, g, q, U, h->Sf, &st->pivot_bad);
  TE();
  CK(cudaMemcpyAsync(h->h_st, st, sizeof(SolveState), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  // FP64 takes over
  auto fallback = [&]() {
    h->mixed_fallback++;
    return solve(h, a, x0, indc, iter, bnorm, xnorm);
  };
  if (h->h_st->pivot_bad) return fallback();
  const double tol2 = h->P.cgepsr * h->P.cgepsr;
  int total = 0;
  bool converged = false;
  double b2 = 0.0, r2 = 0.0;
  for (int outer = 0; outer < 40; ++outer) {
    // r = b - A x and the two norms in FP64
    CK(cudaMemsetAsync(st, 0, SOLVE_CLEAR_BYTES, s));
    TB(CADMAS_STAGE_VEC);
    launch_spmv(s, g, q, h->S, h->xw, h->y2, st);
    launch_bmy(s, q, ic, h->bb_sl, h->y2, st);
    TE();
    TB(CADMAS_STAGE_DOT);
    launch_dot(s, q, ic, h->bb_sl, h->bb_sl, h->y2, h->y2, h->rb0, h->rb1, st);
    launch_fin(s, FIN_STORE, h->rb0, h->rb1, nr, st, h->dres + 6, 0, 0, 0, 0);
    TE();
    CK(cudaMemcpyAsync(h->h_res + 6, h->dres + 6, 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    b2 = h->h_res[6];
    r2 = h->h_res[7];
    h->mixed_outer++;
    if (r2 <= tol2 * b2) { converged = true; break; }
    const double rn = std::sqrt(r2);
    launch_scale_to_f(s, q, ic, h->y2, 1.0 / rn, h->bf);
    // Each pass reduces the residual by about its inner tolerance: ask
    // for half the reduction still needed, no less than the FP32 floor,
    // so the last pass stops near CGEPSR instead of far below it.
    const double need = std::sqrt(tol2 * b2 / r2);
    const double floor_eps = h->P.mixed_eps_inner > 0.0 ? h->P.mixed_eps_inner : 1.0e-5;
    const double eps_in = std::min(0.5, std::max(0.5 * need, floor_eps));
    int it = 0;
    int rc = solve_inner_f(h, eps_in, it);
    if (rc) return rc;
    if (it < 0 || it > h->P.icgmax) return fallback();  // factor, divergence or cap
    total += it;
    launch_add_f(s, q, ic, h->xf, rn, h->xw);
  }
  if (!converged) return fallback();
  // X0 = XW on INDC != -1 (k_x0 requires ITER >= 0: the state is clear)
  CK(cudaMemsetAsync(st, 0, SOLVE_CLEAR_BYTES, s));
  launch_x0(s, g, q, ic, h->xw, x0, st);
  CK(cudaGetLastError());
  iter = total;
  bnorm = std::sqrt(b2);
  xnorm = std::sqrt(r2);
  return CADMAS_OK;
}

static int map_iter(int iter, int icgmax) {
  if (iter > icgmax) return CADMAS_ENOTCONV;
  if (iter == -2) return CADMAS_EDIVERGE;
  if (iter == -1) return CADMAS_EPIVOT;
  return CADMAS_OK;
}

static int read_err(cadmas_handle *h, int &errbits) {
  CK(cudaMemcpyAsync(h->h_int, h->dint, 5 * sizeof(int), cudaMemcpyDeviceToHost, h->s));
  CK(cudaStreamSynchronize(h->s));
  errbits = h->h_int[0];
  return CADMAS_OK;
}
static int map_err(int bits) {
  if (bits & ERR_PG) return CADMAS_EPG;
  if (bits & ERR_UNSUP) return CADMAS_EUNSUPPORTED;
  if (bits & ERR_NOTCONV) return CADMAS_ENOTCONV;
  if (bits & ERR_CAP) return CADMAS_ECAP;
  return CADMAS_OK;
}

// VF_FNFINI: init pass then sweeps until no surface cell changes.
static int fnfini(cadmas_handle *h) {
  cudaStream_t s = h->s;
  launch_fnf_init(s, h->g, h->f, h->p);
  CK(cudaMemsetAsync(h->dint + 1, 0, 3 * sizeof(int), s));  // nch, done, iter
  const int cap = 100000;
  int batch = 2;
  for (int guard = 0; guard < cap; guard += batch) {
    for (int b = 0; b < batch; ++b)
      launch_fnf_sweep(s, h->g, h->nf, h->dint + 1, h->dint + 2, h->dint + 3, cap, h->dint);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(h->h_int, h->dint, 5 * sizeof(int), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if (h->h_int[2]) return CADMAS_OK;
    batch = std::min(batch * 2, 16);
  }
  return CADMAS_ECAP;
}

static int bc_tail_v1(cadmas_handle *h) {
  cudaStream_t s = h->s;
  launch_bsuwt(s, h->g, h->f, h->p);
  launch_bsuwt2(s, h->g, h->f);
  launch_bsuwn(s, h->g, h->f);
  if (h->src.on) launch_bsuwn_src(s, h->g, h->f, h->p);
  launch_bwuwt(s, h->g, h->f, h->p, h->dint);
  launch_bwpp(s, h->g, h->f);
  return CADMAS_OK;
}

// VF_V1CAL in three parts, so that a batch can solve the pressure of
// several grids together: up to the Poisson system and PT's start value
// (vf_v1cal.f:118-271, vf_vpsol.f:52-58), the solve (vf_vpsol.f:59-76),
// and the rest (vf_v1cal.f:272-297).
static SysPtr poisson_sys(const cadmas_handle *h) {
  return SysPtr{h->wk[0], h->wk[1], h->wk[2], h->wk[3], h->wk[4], h->wk[5], h->wk[6], h->wk[7]};
}
static int v1cal_pre(cadmas_handle *h) {
  cudaStream_t s = h->s;
  refresh_prm(h);
  refresh_fld(h);
  CK(cudaMemsetAsync(h->dint, 0, sizeof(int), s));
  // the wave source's velocities of this step (vf_a1main.f:1035-1040)
  if (h->src.on) { const int rs = wave_src(h); if (rs) return rs; }
  // fluxes, sources, provisional velocity (vf_v1cal.f:153-230)
  TB(CADMAS_STAGE_FLUX); launch_flux(s, h->g, h->f, h->p, h->wk); TE();
  const int nxt = h->cur ^ 1;
  TB(CADMAS_STAGE_PREDICT);
  launch_predict(s, h->g, h->f, h->p, h->wk, h->vel[nxt][0], h->vel[nxt][1], h->vel[nxt][2]);
  TE();
  h->cur = nxt;
  refresh_fld(h);
  // normal boundary velocities (vf_v1cal.f:251-254)
  TB(CADMAS_STAGE_MODIF);
  launch_bwuwn(s, h->g, h->f, h->p, h->dint);
  { const int rw = wave_bc(h); if (rw) return rw; }
  // UB, VB, WB: the velocities of the step's start (vf_v1cal.f:125-142)
  { const int ro = open_bc(h, h->vel[nxt ^ 1][0], h->vel[nxt ^ 1][1], h->vel[nxt ^ 1][2]); if (ro) return ro; }
  TE();
  // Poisson system (vf_v1cal.f:259-271)
  const SysPtr a = poisson_sys(h);
  TB(CADMAS_STAGE_VPCOEF); launch_vpcoef(s, h->g, h->f, h->p, a, h->dint); TE();
  // VF_VPSOL: PT = 0, solve (vf_vpsol.f:52-76)
  double *PT = h->wk[8];
  CK(cudaMemsetAsync(PT, 0, h->N * sizeof(double), s));
  if (h->P.warm_start == 2 && h->wnet) {  // the learned PT0 in place of PT = 0
    TB(CADMAS_STAGE_WARM);
    launch_warm_guess(s, h->g, h->f, a, h->wnet, h->ws_rows, h->ws_rows + nrows(h), h->ws_scal, h->ws_cnt, PT);
    TE();
  }
  return CADMAS_OK;
}
static int v1cal_solve(cadmas_handle *h, int &iter, double &bn, double &xn) {
  const SysPtr a = poisson_sys(h);
  double *PT = h->wk[8];
  const bool mixed = (h->P.solver == 1);
  h->warm_now = (h->P.warm_start == 1 && h->have_prev) ? 1 : 0;
  const int rc = mixed ? solve_mixed(h, a, PT, h->indc, iter, bn, xn) : solve(h, a, PT, h->indc, iter, bn, xn);
  h->warm_now = 0;
  return rc;
}
static int v1cal_post(cadmas_handle *h, int rc, int iter, double bn, double xn) {
  cudaStream_t s = h->s;
  double *PT = h->wk[8];
  const bool mixed = (h->P.solver == 1);
  if (rc) return rc;
  h->have_prev = (iter >= 0);
  h->stats.icgitr = iter;
  h->stats.cgbnrm = bn;
  h->stats.cgxnrm = xn;
  rc = mixed ? (iter < 0 ? map_iter(iter, h->P.icgmax) : CADMAS_OK) : map_iter(iter, h->P.icgmax);
  if (rc) return rc;
  if (h->P.diag_relres) {
    launch_relres(s, h->g, h->q, h->S, h->bb_sl, h->xw, h->rb0, h->rb1);
    launch_fin(s, FIN_STORE, h->rb0, h->rb1, h->nrb, h->st, h->dres + 2, 0, 0, 0, 0);
    CK(cudaMemcpyAsync(h->h_res, h->dres, 4 * sizeof(double), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    h->stats.true_relres = h->h_res[3] > 0.0 ? std::sqrt(h->h_res[2]) / std::sqrt(h->h_res[3]) : 0.0;
  }
  // correction and boundary values (vf_v1cal.f:286-297)
  TB(CADMAS_STAGE_MODIF);
  launch_vmodif(s, h->g, h->f, h->p, PT);
  bc_tail_v1(h);
  TE();
  CK(cudaGetLastError());
  return CADMAS_OK;
}
static int do_v1cal(cadmas_handle *h) {
  int rc = v1cal_pre(h);
  if (rc) return rc;
  int iter = 0;
  double bn = 0.0, xn = 0.0;
  rc = v1cal_solve(h, iter, bn, xn);
  return v1cal_post(h, rc, iter, bn, xn);
}

// ------------------------------------------------------------ k-epsilon
static KeConst ke_const(const cadmas_handle *h) {
  const cadmas_params &P = h->P;
  return KeConst{P.anu0, P.scmk, P.akmink, P.akmine, P.akinik, P.akinie, P.akcmu, P.aksgk, P.aksge,
                 P.akc1, P.akc2, P.akc3};
}
static KeArrays ke_arrays(const cadmas_handle *h) {
  return KeArrays{h->ak, h->ae_k, h->anut, h->bck, h->bce, h->indbk, h->indbe};
}

// VF_K1CAL (vf_k1cal.f:84-170): k and e into the second buffers, which
// then become the present ones; surface and gas values; boundary values.
static void do_k1cal(cadmas_handle *h) {
  cudaStream_t s = h->s;
  TB(CADMAS_STAGE_TURB);
  const KeConst kc = ke_const(h);
  launch_kstep(s, h->g, h->f, h->p, kc, ke_arrays(h), h->ak2, h->ae2, h->dint);
  std::swap(h->ak, h->ak2);
  std::swap(h->ae_k, h->ae2);
  launch_kbsss(s, h->g, h->f, kc, h->ak, h->ae_k, h->anut, h->anu, true, false);
  launch_bwke(s, h->g, h->f, ke_arrays(h), h->dint);
  TE();
}

// ANUT and ANU from the present k and e (VF_CNUT0, VF_CNU00)
static void ke_nut(cadmas_handle *h) {
  refresh_fld(h);
  launch_kbsss(h->s, h->g, h->f, ke_const(h), h->ak, h->ae_k, h->anut, h->anu, false, true);
}

// After VF_F1CAL (vf_a1main.f:1119-1127): VF_BSSS with the new NF, ANUT and
// ANU, VF_BWKE, VF_BWUWT.
static void do_kpost(cadmas_handle *h) {
  cudaStream_t s = h->s;
  TB(CADMAS_STAGE_TURB);
  if (h->p.loglaw) launch_bwkelg(s, h->g, h->f, h->p, ke_const(h), h->ak, h->ae_k, h->dint);
  launch_kbsss(s, h->g, h->f, ke_const(h), h->ak, h->ae_k, h->anut, h->anu, true, true);
  launch_bwke(s, h->g, h->f, ke_arrays(h), h->dint);
  launch_bwuwt(s, h->g, h->f, h->p, h->dint);
  TE();
}

void cadmas::set_cuda_error(const char *call, cudaError_t e) {
  g_last_error = std::string(call) + ": " + cudaGetErrorString(e);
}

// ------------------------------------------ kernel shared-memory limits
void cadmas::raise_dynamic_smem(const void *kern, size_t bytes) {
  static std::mutex mu;
  static std::map<std::pair<int, const void *>, size_t> cur;  // (device, kernel) -> limit set
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lk(mu);
  size_t &c = cur[{dev, kern}];
  if (bytes > c) {
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    c = bytes;
  }
}

static int do_f1cal(cadmas_handle *h) {
  cudaStream_t s = h->s;
  refresh_prm(h);
  refresh_fld(h);
  const Geo &g = h->g;
  if (h->P.leqk != 0) do_k1cal(h);  // vf_a1main.f:1093-1100, just before VF_F1CAL
  // fluxes and Euler update (vf_f1cal.f:124-163)
  TB(CADMAS_STAGE_VOF);
  if (h->P.iscmff == 0) launch_fconv(s, g, h->f, h->p, h->wk[0], h->wk[1], h->wk[2]);
  else  // VF_FCONVS: ISTYP in NLIM as in the reference (FMOD1 clears it), SX..SA in wk[3..6]
    launch_fconvs(s, g, h->f, h->p, h->nlim, h->wk[3], h->wk[4], h->wk[5], h->wk[6], h->wk[0], h->wk[1],
                  h->wk[2], h->dint);
  launch_feuler(s, g, h->f, h->p, h->wk[0], h->wk[1], h->wk[2]);
  { const int rl = fixed_level_f(h); if (rl) return rl; }  // vf_f1cal.f:180
  // surface redistribution, cut-off and volume (vf_f1cal.f:185-188)
  launch_fmod1(s, g, h->f, h->nlim);
  launch_fcut(s, g, h->f, h->p, h->rb0, h->rb1);
  launch_fin(s, FIN_STORE, h->rb0, h->rb1, nrows(h), h->st, h->dres, 0, 0, 0, 0);
  TE();
  // boundary values (vf_f1cal.f:192-194)
  TB(CADMAS_STAGE_FBC);
  launch_bwff(s, g, h->f, h->dint);
  launch_bsuwn3(s, g, h->f, h->p);
  launch_bsuwem(s, g, h->f, h->nlim);
  TE();
  // NF before the update (vf_f1cal.f:197-203)
  CK(cudaMemcpyAsync(h->nf0, h->nf, h->N * sizeof(int), cudaMemcpyDeviceToDevice, s));
  // NF and INDC (vf_f1cal.f:207-219)
  TB(CADMAS_STAGE_FLAGS);
  int rc = fnfini(h);
  if (rc) return rc;
  if (h->P.wbub >= 1.0e-20) {
    // VF_FBUBUP level timers (vf_fbubup.f:35-38, 49) on the host
    bool any = false;
    for (int K = h->g.NK - 2; K >= 2; --K) {
      double DTBUB = h->zz2[K] / h->P.wbub;
      h->h_active[K] = 0;
      if (h->tnow - h->tbub[K - 1] > DTBUB) {
        h->h_active[K] = 1;
        any = true;
        h->tbub[K - 1] = h->tbub[K - 1] + DTBUB;
      }
    }
    if (any) {
      CK(cudaMemcpyAsync(h->active, h->h_active.data(), h->h_active.size(), cudaMemcpyHostToDevice, s));
      launch_fbubup(s, g, h->f, h->p, h->active);
    }
    rc = fnfini(h);
    if (rc) return rc;
  }
  if (h->P.idrop >= 1) {  // droplets fall, then the flags again (vf_f1cal.f:212-217)
    launch_fdropf(s, g, h->f, h->p, h->drop);
    rc = fnfini(h);
    if (rc) return rc;
  }
  launch_fnfprv(s, g, h->f, h->dint);
  CK(cudaMemsetAsync(h->dint + 4, 0, sizeof(int), s));
  launch_cindc(s, g, h->f, h->dint + 4);
  TE();
  // gas-to-fluid pressure (vf_f1cal.f:230)
  TB(CADMAS_STAGE_FBC);
  const int pn = h->pcur ^ 1;
  launch_bsppfl(s, g, h->f, h->pbuf[h->pcur], h->pbuf[pn]);
  h->pcur = pn;
  refresh_fld(h);
  // boundary values (vf_f1cal.f:234-239)
  launch_bsuwt(s, g, h->f, h->p);
  launch_bsuwt2(s, g, h->f);
  launch_bsuwn3(s, g, h->f, h->p);
  launch_bspp(s, g, h->f);
  launch_bwuwt(s, g, h->f, h->p, h->dint);
  launch_bwpp(s, g, h->f);
  TE();
  if (h->P.leqk != 0) do_kpost(h);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(h->h_res, h->dres, 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
  int bits;
  rc = read_err(h, bits);
  if (rc) return rc;
  h->tm.resolve();
  h->stats.fsum = h->h_res[0];
  h->stats.fcut = h->h_res[1];
  h->stats.nums = h->h_int[4];
  return map_err(bits);
}

// ====================================================== restart and list I/O
// Fortran unformatted sequential records as gfortran writes them: each
// WRITE is one record, its bytes framed by their count as a 4-byte native
// (little-endian) integer before and after.  Records of 2^31 bytes or more
// would need split markers; they are refused.
struct FRecordFile {
  FILE *f = nullptr;
  ~FRecordFile() { if (f) std::fclose(f); }
  bool put(std::initializer_list<std::pair<const void *, size_t>> parts) {
    size_t n = 0;
    for (auto &p : parts) n += p.second;
    if (n > 0x7fffffffu - 8) return false;
    const int32_t m = (int32_t)n;
    if (std::fwrite(&m, 4, 1, f) != 1) return false;
    for (auto &p : parts)
      if (p.second && std::fwrite(p.first, 1, p.second, f) != p.second) return false;
    return std::fwrite(&m, 4, 1, f) == 1;
  }
  // One record into buf; false at the end of the file or on a bad frame.
  bool get(std::vector<unsigned char> &buf, bool *eof = nullptr) {
    int32_t m = 0, t = 0;
    if (std::fread(&m, 4, 1, f) != 1) { if (eof) *eof = true; return false; }
    if (m < 0) return false;
    buf.resize((size_t)m);
    if (m && std::fread(buf.data(), 1, (size_t)m, f) != (size_t)m) return false;
    return std::fread(&t, 4, 1, f) == 1 && t == m;
  }
};
template <typename T> static T rec_at(const std::vector<unsigned char> &b, size_t off) {
  T v;
  std::memcpy(&v, b.data() + off, sizeof(T));
  return v;
}

// Fortran edit descriptors of the list file: 1PE12.5 and I6.
static std::string f_e12_5(double v) {
  char b[64];
  if (std::isnan(v)) { std::snprintf(b, sizeof b, "%12s", "NaN"); return b; }
  if (std::isinf(v)) { std::snprintf(b, sizeof b, "%12s", v < 0 ? "-Infinity" : "Infinity"); return b; }
  std::snprintf(b, sizeof b, "%.5E", v);  // d.dddddE+xx or d.dddddE+xxx
  std::string t(b);
  const size_t e = t.find('E');
  std::string mant = t.substr(0, e), ex = t.substr(e + 1);  // ex: sign and digits
  const int digits = (int)ex.size() - 1;
  std::string out = digits <= 2 ? mant + "E" + ex : mant + ex;  // E dropped for 3-digit exponents
  if (out.size() < 12) out = std::string(12 - out.size(), ' ') + out;
  return out.size() > 12 ? std::string(12, '*') : out;
}
static std::string f_i6(int v) {
  char b[32];
  std::snprintf(b, sizeof b, "%6d", v);
  std::string t(b);
  return t.size() > 6 ? std::string(6, '*') : t;
}

// ============================================================== C ABI
extern "C" {

const char *cadmas_strerror(int status) {
  switch (status) {
    case CADMAS_OK: return "ok";
    case CADMAS_EINVAL: return "invalid argument";
    case CADMAS_ECUDA: return g_last_error.empty() ? "CUDA error" : g_last_error.c_str();
    case CADMAS_ENOTCONV: return "NOT CONVERGED. (Poisson solve reached ICGMAX)";
    case CADMAS_EDIVERGE: return "INSTABILITY. (Poisson solve diverged)";
    case CADMAS_EPIVOT: return "CAN NOT DECOMPOSITION. (non-positive MILU pivot)";
    case CADMAS_EPG: return "P.G ERROR. (inconsistent cell flags)";
    case CADMAS_ECAP: return "device iteration cap reached";
    case CADMAS_ENOMEM: return "device allocation failed";
    case CADMAS_EUNSUPPORTED: return "option outside the implemented path";
    case CADMAS_ENOSTATIC: return "static fields not uploaded";
    case CADMAS_ETIMEOUT: return "a device-side wait ran out of time";
    case CADMAS_ESCRATCH: return "grid has more than CADMAS_NOALLOC_MAX_ROWS (65536) rows NUMJ*NUMK";
    case CADMAS_EIO: return g_last_error.empty() ? "restart file I/O error" : g_last_error.c_str();
    case CADMAS_EWAVE: return "(VF_SFMB02C) NOT CONVERGED. (the stream-function wave has no solution found)";
    default: return "unknown status";
  }
}

void cadmas_default_params(cadmas_params *p) {
  std::memset(p, 0, sizeof(*p));
  p->rho0 = 1.0e3; p->grz0 = 9.8; p->vvmax = 30.0;
  p->cgpara = 0.95; p->cgepsa = 1.0e-15; p->cgepsr = 1.0e-12; p->cgdiv = 1.0e30;
  p->flower = 1.0e-6; p->fupper = 1.0 - 1.0e-6; p->plower = 1.0e-4; p->scmvp = 1.0;
  p->wvlvl = 0.0; p->wbub = 0.2;
  for (int d = 0; d < 4; ++d) {
    p->idamp[d] = -1;
    p->damp[d][0] = 0.6; p->damp[d][1] = 0.6; p->damp[d][2] = 0.0; p->damp[d][3] = 0.0;
  }
  p->icgtyp = 1; p->icgmax = 500; p->ibsuw0 = 0;
  p->precond_ti = 0; p->precond_tj = 0;
  p->idrop = 1;
  p->iscmff = 0;
  // k-epsilon (vf_a2dflt.f:61,139,162,165-176)
  p->leqk = 0;
  p->anu0 = 1.0e-6; p->scmk = 1.0;
  p->akmink = 1.0e-20; p->akmine = 1.0e-20; p->akinik = 1.0e-20; p->akinie = 1.0e-20;
  p->akcmu = 0.09; p->aksgk = 1.0; p->aksge = 1.3; p->akc1 = 1.44; p->akc2 = 1.92; p->akc3 = 0.0;
  p->akk0 = 0.4; p->aka0 = 5.5;  // vf_a2dflt.f:175-176
  p->mixed_eps_inner = 1.0e-5;
  p->wait_limit_s = 2.0;
}

int cadmas_create(const cadmas_dims *d, const cadmas_params *p, cadmas_handle **out) {
  if (!d || !p || !out) return CADMAS_EINVAL;
  if (d->numi < 5 || d->numj < 3 || d->numk < 5 || d->numb < 0) return CADMAS_EINVAL;
  const long long N = (long long)d->numi * d->numj * d->numk;
  if (N > (1LL << 34)) return CADMAS_EINVAL;
  int TI = p->precond_ti > 0 ? p->precond_ti : d->numi - 2;
  int TJ = p->precond_tj > 0 ? p->precond_tj : d->numj - 2;
  TI = std::min(TI, d->numi - 2);
  TJ = std::min(TJ, d->numj - 2);
  if (TI * TJ > 1024) {
    g_last_error = "preconditioner block of more than 1024 columns; set precond_ti/precond_tj";
    return CADMAS_EUNSUPPORTED;
  }
  cadmas_handle *h = new cadmas_handle();
  h->P = *p;
  h->TI = TI; h->TJ = TJ;
  if (cudaGetDevice(&h->device) != cudaSuccess) { delete h; return CADMAS_ECUDA; }
  if (cudaStreamCreateWithFlags(&h->s, cudaStreamNonBlocking) != cudaSuccess) { delete h; return CADMAS_ECUDA; }
  h->N = (size_t)N;
  h->NB = (size_t)std::max(d->numb, 1);
  h->g.NI = d->numi; h->g.NJ = d->numj; h->g.NK = d->numk; h->g.NB = d->numb; h->g.N = N;
  int rc = CADMAS_OK;
#define AL(ptr, n) if (!rc) rc = dalloc(&(ptr), (n))
  AL(h->xx, 6 * (size_t)d->numi); AL(h->yy, 6 * (size_t)d->numj); AL(h->zz, 6 * (size_t)d->numk);
  AL(h->ggv, h->N); AL(h->ggx, h->N); AL(h->ggy, h->N); AL(h->ggz, h->N);
  AL(h->glv, h->N); AL(h->glx, h->N); AL(h->gly, h->N); AL(h->glz, h->N);
  AL(h->cd0, h->N); AL(h->anu, h->N);
  AL(h->indx, h->N); AL(h->indy, h->N); AL(h->indz, h->N); AL(h->indb, 4 * h->NB);
  for (int b = 0; b < 2; ++b) for (int c = 0; c < 3; ++c) AL(h->vel[b][c], h->N);
  AL(h->pbuf[0], h->N); AL(h->pbuf[1], h->N);
  AL(h->ff, h->N); AL(h->nf, h->N); AL(h->indc, h->N); AL(h->nf0, h->N); AL(h->nlim, h->N);
  AL(h->bcvi, h->NB);
  AL(h->bcu, h->NB); AL(h->bcv, h->NB); AL(h->bcw, h->NB); AL(h->bcp, h->NB); AL(h->bcf, h->NB);
  for (int w = 0; w < 9; ++w) AL(h->wk[w], h->N);
  // layout tiles: TI x TJ, or TI x TJ/2 when each preconditioner block is
  // split over a cluster of two thread blocks
  const int split = (p->precond_split == 2) ? 2 : 1;
  if (p->precond_split < 0 || p->precond_split > 2 || TJ % split != 0) rc = CADMAS_EINVAL;
  const int TJl = TJ / split;
  h->q.split = split;
  h->q.TI = TI; h->q.TJ = TJl; h->q.TIp = (TI + 3) & ~3; h->q.T = h->q.TIp * TJl;
  h->q.W = (d->numk - 2) + (TI - 1) + (TJl - 1);
  h->q.ntx = (d->numi - 2 + TI - 1) / TI;
  h->q.nb = h->q.ntx * ((d->numj - 2 + TJl - 1) / TJl);
  h->q.occ = (p->sweep_occupancy == 1 || p->sweep_occupancy == 2 || p->sweep_occupancy == 4) ? p->sweep_occupancy : 0;
  h->q.nsm = 148;
  {
    int nsm = 0;
    if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, h->device) == cudaSuccess && nsm > 0)
      h->q.nsm = nsm;
  }
  if (!sweep_supported(h->q)) {
    g_last_error = "preconditioner block too large for the MILU sweeps; set precond_ti/precond_tj";
    rc = CADMAS_EUNSUPPORTED;
  }
  h->nsl = (size_t)h->q.nb * h->q.W * h->q.T;
  h->nslab = (long long)h->q.nb * h->q.W;
  h->nrb = (h->nslab + ROWS_PER_BLOCK - 1) / ROWS_PER_BLOCK;
  {
    const size_t nsl = h->nsl;
    AL(h->S.sys, (size_t)SYS_N * nsl);
    AL(h->S.indc, nsl); AL(h->bb_sl, nsl);
    AL(h->xw, nsl); AL(h->y2, nsl); AL(h->r0, nsl); AL(h->rr, nsl);
    AL(h->pv, nsl); AL(h->ap, nsl); AL(h->ae, nsl);
    if (p->solver == 1) {
      if (!sweep_supported_f(h->q)) {
        g_last_error = "preconditioner block too large for the FP32 sweeps; set precond_ti/precond_tj";
        rc = rc ? rc : CADMAS_EUNSUPPORTED;
      }
      AL(h->Sf.sys, (size_t)SYS_N * nsl);
      AL(h->bf, nsl); AL(h->xf, nsl); AL(h->r0f, nsl); AL(h->rrf, nsl); AL(h->pvf, nsl);
      AL(h->apf, nsl); AL(h->aef, nsl); AL(h->y2f, nsl);
      AL(h->rb5, 5 * (size_t)h->nrb);
    } else if (p->solver != 0) {
      rc = rc ? rc : CADMAS_EINVAL;
    }
  }
  AL(h->rb0, (size_t)std::max<long long>(nrows(h), h->nslab)); AL(h->rb1, (size_t)std::max<long long>(nrows(h), h->nslab)); AL(h->dres, 10);
  AL(h->st, 1); AL(h->dint, 8); AL(h->active, (size_t)d->numk + 1);
  AL(h->drop.tx, h->N); AL(h->drop.ty, h->N); AL(h->drop.tz, h->N);
  AL(h->drop.uu, h->N); AL(h->drop.vv, h->N); AL(h->drop.ww, h->N);
  if (p->leqk != 0) {
    AL(h->ak, h->N); AL(h->ae_k, h->N); AL(h->ak2, h->N); AL(h->ae2, h->N); AL(h->anut, h->N);
    AL(h->bck, h->NB); AL(h->bce, h->NB); AL(h->bck0, h->NB); AL(h->bce0, h->NB);
    AL(h->indbk, h->NB); AL(h->indbe, h->NB);
  }
  if (p->idrop >= 1 && !drop_supported(h->g)) {
    g_last_error = "x lines too long for the droplet model's shared-memory walk";
    rc = rc ? rc : CADMAS_EUNSUPPORTED;
  }
#undef AL
  if (!rc && cudaMallocHost((void **)&h->h_st, sizeof(SolveState)) != cudaSuccess) rc = CADMAS_ENOMEM;
  if (!rc && cudaMallocHost((void **)&h->h_int, 8 * sizeof(int)) != cudaSuccess) rc = CADMAS_ENOMEM;
  if (!rc && cudaMallocHost((void **)&h->h_res, 10 * sizeof(double)) != cudaSuccess) rc = CADMAS_ENOMEM;
  if (!rc) {  // the sweeps' wait limit and (no) stall, kept across solves
    const double lim = p->wait_limit_s > 0.0 ? std::min(p->wait_limit_s, 60.0) : 2.0;
    std::memset(h->h_st, 0, sizeof(SolveState));
    h->h_st->wait_ns = (long long)(lim * 1.0e9);
    h->h_st->stall_from = 1 << 30;
    if (cudaMemcpy(h->st, h->h_st, sizeof(SolveState), cudaMemcpyHostToDevice) != cudaSuccess) rc = CADMAS_ECUDA;
  }
  if (rc) { cadmas_destroy(h); return rc; }
  // NF starts as all obstacle until set_state; INDC as non-computed.
  cudaMemset(h->nf, 0xff, h->N * sizeof(int));
  cudaMemset(h->indc, 0xff, h->N * sizeof(int));
  launch_drop_reset(h->s, (long long)h->N, h->drop);
  h->tbub.assign(d->numk, 0.0);
  h->h_active.assign(d->numk + 1, 0);
  std::memset(&h->stats, 0, sizeof(h->stats));
  h->stats.true_relres = -1.0;
  h->g.XX = h->xx; h->g.YY = h->yy; h->g.ZZ = h->zz;
  refresh_prm(h);
  refresh_fld(h);
  *out = h;
  return CADMAS_OK;
}

int cadmas_destroy(cadmas_handle *h) {
  if (!h) return CADMAS_OK;
  cudaStreamSynchronize(h->s);
  double *dl[] = {h->xx, h->yy, h->zz, h->ggv, h->ggx, h->ggy, h->ggz, h->glv, h->glx, h->gly, h->glz,
                  h->cd0, h->anu, h->pbuf[0], h->pbuf[1], h->ff, h->bcvi, h->bcu, h->bcv, h->bcw, h->bcp, h->bcf,
                  h->xw, h->y2, h->r0, h->rr, h->pv, h->ap, h->ae, h->rb0, h->rb1, h->dres,
                  h->S.sys, h->bb_sl, h->rb5};
  for (double *q : dl) if (q) cudaFree(q);
  for (int b = 0; b < 2; ++b) for (int c = 0; c < 3; ++c) if (h->vel[b][c]) cudaFree(h->vel[b][c]);
  for (double *q : h->wk) if (q) cudaFree(q);
  int *il[] = {h->indx, h->indy, h->indz, h->indb, h->nf, h->indc, h->nf0, h->nlim, h->dint, h->S.indc};
  for (int *q : il) if (q) cudaFree(q);
  if (h->st) cudaFree(h->st);
  if (h->active) cudaFree(h->active);
  if (h->h_st) cudaFreeHost(h->h_st);
  if (h->h_int) cudaFreeHost(h->h_int);
  if (h->h_res) cudaFreeHost(h->h_res);
  for (double *q : {h->wzz, h->wun, h->wut, h->srcuv}) if (q) cudaFree(q);
  for (auto &ws : h->wave) {
    if (ws.col) cudaFree(ws.col);
    if (ws.col_h) cudaFreeHost(ws.col_h);
    if (ws.col_ev) cudaEventDestroy(ws.col_ev);
  }
  for (double *q : {h->drop.tx, h->drop.ty, h->drop.tz, h->drop.uu, h->drop.vv, h->drop.ww}) if (q) cudaFree(q);
  for (double *q : {h->ak, h->ae_k, h->ak2, h->ae2, h->anut, h->bck, h->bce, h->bck0, h->bce0}) if (q) cudaFree(q);
  if (h->wnet) cadmas_unet_destroy(h->wnet);
  for (double *q : {h->ws_rows, h->ws_scal}) if (q) cudaFree(q);
  if (h->ws_cnt) cudaFree(h->ws_cnt);
  for (int *q : {h->indbk, h->indbe}) if (q) cudaFree(q);
  for (float *q : {h->Sf.sys, h->bf, h->xf, h->r0f, h->rrf, h->pvf, h->apf, h->aef, h->y2f})
    if (q) cudaFree(q);
  if (h->s) cudaStreamDestroy(h->s);
  delete h;
  return CADMAS_OK;
}

// The matrix table (/VF_AFILEI/ DMTB*), one for the wave sides and the
// wave source as in the reference.
static int set_table(cadmas_handle *h, const cadmas_wave_table *t) {
  if (!t->tt || !t->hh || !t->zz || !t->un || !t->ut) return CADMAS_EINVAL;
  if (t->ntt < 2 || t->nzz < 2 || t->mtbtyp < 1 || t->mtbtyp > 3) return CADMAS_EINVAL;
  for (int i = 1; i < t->ntt; ++i) if (!(t->tt[i] >= t->tt[i - 1])) return CADMAS_EINVAL;
  for (int k = 1; k < t->nzz; ++k) if (!(t->zz[k] > t->zz[k - 1])) return CADMAS_EINVAL;
  const size_t nzt = (size_t)t->nzz * t->ntt;
  if (h->nzz != 0 && (h->nzz != t->nzz || (int)h->wtt.size() != t->ntt)) return CADMAS_EINVAL;
  if (!h->wzz) {
    int rc = CADMAS_OK;
    if (!rc) rc = dalloc(&h->wzz, (size_t)t->nzz);
    if (!rc) rc = dalloc(&h->wun, nzt);
    if (!rc) rc = dalloc(&h->wut, nzt);
    if (rc) return rc;
  }
  CK(cudaMemcpy(h->wzz, t->zz, (size_t)t->nzz * sizeof(double), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(h->wun, t->un, nzt * sizeof(double), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(h->wut, t->ut, nzt * sizeof(double), cudaMemcpyHostToDevice));
  h->wtt.assign(t->tt, t->tt + t->ntt);
  h->whh.assign(t->hh, t->hh + t->ntt);
  h->nzz = t->nzz;
  h->mtbtyp = t->mtbtyp;
  h->dmtbt0 = t->phase0;
  return CADMAS_OK;
}

// The side's oblique-incidence buffers: one WaveCol per line, on the
// device and pinned on the host, (re)made for the side's line range.
static int wave_cols(cadmas_handle::WaveSide &ws, bool need) {
  const int n = need ? ws.last - ws.first + 1 : 0;
  if (n == ws.ncol) return CADMAS_OK;
  if (ws.col_ev) cudaEventSynchronize(ws.col_ev);
  if (ws.col) cudaFree(ws.col);
  if (ws.col_h) cudaFreeHost(ws.col_h);
  ws.col = nullptr; ws.col_h = nullptr; ws.ncol = 0;
  if (n == 0) return CADMAS_OK;
  CK(cudaMalloc(&ws.col, (size_t)n * sizeof(WaveCol)));
  CK(cudaMallocHost(&ws.col_h, (size_t)n * sizeof(WaveCol)));
  if (!ws.col_ev) CK(cudaEventCreateWithFlags(&ws.col_ev, cudaEventDisableTiming));
  ws.ncol = n;
  return CADMAS_OK;
}

// The checks of a wave-maker side common to the table and the theories.
static int wave_side_ok(cadmas_handle *h, const cadmas_wave_bc *w) {
  if (w->side < 1 || w->side > 4) return CADMAS_EINVAL;
  if (h->open[w->side - 1].on) {  // vf_iimdl.f: 'DEFINED DOUBLY.'
    g_last_error = "side already declared open";
    return CADMAS_EINVAL;
  }
  const int lim = (w->side <= 2) ? h->g.NJ - 1 : h->g.NI - 1;  // vf_iimdl.f:101-106
  if (w->first < 2 || w->last > lim || w->first > w->last) return CADMAS_EINVAL;
  return CADMAS_OK;
}

int cadmas_set_wave(cadmas_handle *h, const cadmas_wave_bc *w, const cadmas_wave_table *t) {
  if (!h || !w || !t) return CADMAS_EINVAL;
  { const int rs = wave_side_ok(h, w); if (rs) return rs; }
  if (t->mtbtyp < 1 || t->mtbtyp > 3) return CADMAS_EINVAL;
  if (!(w->period > 0.0) || (t->mtbtyp == 1 && !(w->depth > 0.0))) return CADMAS_EINVAL;
  cadmas_handle::WaveSide &ws = h->wave[w->side - 1];
  if (std::fabs(ws.angle) > 1.0e-20) {  // vf_csetup.f:97-99
    g_last_error = "(WAVE-BC ANGLE) CAN NOT USE.";
    return CADMAS_EINVAL;
  }
  { const int rt = set_table(h, t); if (rt) return rt; }
  ws.on = true; ws.first = w->first; ws.last = w->last;
  ws.d = w->depth; ws.t = w->period; ws.a = w->ramp;
  ws.theory = false;
  refresh_prm(h);
  return CADMAS_OK;
}

// A side driven by a solved wave theory.
static int set_wave_side(cadmas_handle *h, const cadmas_wave_bc *w, const cadmas_wave_theory &th) {
  { const int rs = wave_side_ok(h, w); if (rs) return rs; }
  if (!(w->period > 0.0) || !(w->depth > 0.0)) return CADMAS_EINVAL;
  cadmas_handle::WaveSide &ws = h->wave[w->side - 1];
  ws.on = true; ws.first = w->first; ws.last = w->last;
  ws.d = w->depth; ws.t = w->period; ws.a = w->ramp;
  ws.theory = true; ws.th = th;
  { const int rc = wave_cols(ws, std::fabs(ws.angle) > 1.0e-20); if (rc) return rc; }
  refresh_prm(h);
  return CADMAS_OK;
}

static bool theory_ok(const cadmas_wave_theory *t) {
  if (!t || t->type == 0 || t->type < CADMAS_WAVE_STOKES || t->type > CADMAS_STREAM_NMAX) return false;
  if (t->type >= 1) return t->stream.order == t->type && t->stream.k > 0.0;
  if (t->type == CADMAS_WAVE_STOKES) return t->stokes.k > 0.0 && t->length > 0.0;
  return t->cnoidal.ql > 0.0 && t->cnoidal.d > 0.0 && t->length > 0.0;
}

int cadmas_set_wave_theory(cadmas_handle *h, const cadmas_wave_bc *w, const cadmas_stream_wave *sw) {
  if (!h || !w || !sw) return CADMAS_EINVAL;
  if (sw->order < 1 || sw->order > CADMAS_STREAM_NMAX || !(sw->k > 0.0)) return CADMAS_EINVAL;
  cadmas_wave_theory th;
  theory_from_stream(*sw, th);
  return set_wave_side(h, w, th);
}

int cadmas_set_wave_func(cadmas_handle *h, const cadmas_wave_bc *w, const cadmas_wave_theory *t) {
  if (!h || !w || !theory_ok(t)) return CADMAS_EINVAL;
  return set_wave_side(h, w, *t);
}

int cadmas_set_wave_angle(cadmas_handle *h, int side, double angle, double sx, double sy) {
  if (!h || side < 1 || side > 4 || !std::isfinite(angle) || !std::isfinite(sx) || !std::isfinite(sy))
    return CADMAS_EINVAL;
  cadmas_handle::WaveSide &ws = h->wave[side - 1];
  if (!ws.on || !ws.theory) {  // vf_csetup.f:97-99 (and vf_bwuwn.f:351-356)
    g_last_error = "(WAVE-BC ANGLE) CAN NOT USE.";
    return CADMAS_EINVAL;
  }
  ws.angle = angle; ws.sx = sx; ws.sy = sy;
  return wave_cols(ws, std::fabs(angle) > 1.0e-20);
}

// The line and the SRCUV array of the wave source.
static int set_source_line(cadmas_handle *h, const cadmas_wave_src *src) {
  const size_t n = (size_t)(src->line > 0 ? h->g.NJ : h->g.NI) * h->g.NK;
  if (h->srcuv) { cudaFree(h->srcuv); h->srcuv = nullptr; }
  { const int ra = dalloc(&h->srcuv, n); if (ra) return ra; }  // SRCUV = 0 (vf_a1main.f:690)
  h->src.on = true; h->src.line = src->line;
  h->src.d = src->depth; h->src.t = src->period; h->src.a = src->ramp;
  refresh_fld(h);
  refresh_prm(h);
  return CADMAS_OK;
}

static bool source_line_ok(const cadmas_handle *h, int L) {  // vf_iimdl.f:119-133
  return !(L == 0 || (L > 0 && (L < 2 || L > h->g.NI - 1)) || (L < 0 && (-L < 2 || -L > h->g.NJ - 1)));
}

int cadmas_set_wave_source(cadmas_handle *h, const cadmas_wave_src *src, const cadmas_wave_table *t) {
  if (!h || !src) return CADMAS_EINVAL;
  if (!source_line_ok(h, src->line)) return CADMAS_EINVAL;
  if (t) { const int rt = set_table(h, t); if (rt) return rt; }
  if (h->nzz == 0) { g_last_error = "the wave source needs a matrix table"; return CADMAS_EINVAL; }
  if (h->mtbtyp == 3) { g_last_error = "(WAVE-SRC) MTBTYP ERROR."; return CADMAS_EINVAL; }  // vf_csetup.f:267
  if (!(src->period > 0.0) || (h->mtbtyp == 1 && !(src->depth > 0.0))) return CADMAS_EINVAL;
  h->src.theory = false;
  return set_source_line(h, src);
}

int cadmas_set_wave_source_func(cadmas_handle *h, const cadmas_wave_src *src, const cadmas_wave_theory *t) {
  if (!h || !src || !theory_ok(t)) return CADMAS_EINVAL;
  if (!source_line_ok(h, src->line)) return CADMAS_EINVAL;
  if (!(src->period > 0.0) || !(src->depth > 0.0)) return CADMAS_EINVAL;
  h->src.theory = true;
  h->src.th = *t;
  return set_source_line(h, src);
}

int cadmas_open_speed(double depth, double period, double grav, double *c) {
  if (!c || !(depth > 0.0) || !(period > 0.0) || !(grav > 0.0)) return CADMAS_EINVAL;
  // VF_COMAK0 (vf_comak0.f:24-55): x = k D from x = d coth(x),
  // d = 4 pi^2 D / (g T^2), Newton from d (deep) or sqrt(d) (shallow)
  const double PI = 3.141592653589794;  // VF_A0PRM.h
  const int MI = 10;
  const double EPS = 1.0e-10;
  const double D = 4.0 * PI * PI * depth / grav / period / period;
  double X = (D >= 1.0) ? D : std::sqrt(D);
  for (int it = 1; it <= MI; ++it) {
    const double EXPX = std::exp(X);
    const double EXPXI = 1.0 / EXPX;
    const double COTHX = (EXPX + EXPXI) / (EXPX - EXPXI);
    const double DX = (X - D * COTHX) / (1.0 + D * (COTHX * COTHX - 1.0));
    X = X - DX;
    if (std::fabs(DX / X) <= EPS) break;
  }
  const double WLN = 2.0 * PI * depth / X;
  *c = WLN / period;  // BCTYP(6,JD) = WLN/T (vf_csetup.f:143)
  return std::isfinite(*c) ? CADMAS_OK : CADMAS_EINVAL;
}

int cadmas_set_open(cadmas_handle *h, const cadmas_open_bc *o) {
  if (!h || !o || o->side < 1 || o->side > 4) return CADMAS_EINVAL;
  if (h->wave[o->side - 1].on) {  // vf_iimdl.f: 'DEFINED DOUBLY.'
    g_last_error = "side already declared a wave maker";
    return CADMAS_EINVAL;
  }
  double c;
  const int rc = cadmas_open_speed(o->depth, o->period, h->P.grz0, &c);
  if (rc) return rc;
  h->open[o->side - 1].on = true;
  h->open[o->side - 1].c = c;
  return CADMAS_OK;
}

int cadmas_upload_static(cadmas_handle *h, const cadmas_static *st) {
  if (!h || !st) return CADMAS_EINVAL;
  const double *req[] = {st->xx, st->yy, st->zz, st->ggv, st->ggx, st->ggy, st->ggz, st->glv,
                         st->glx, st->gly, st->glz, st->cd0, st->anu};
  for (const double *q : req) if (!q) return CADMAS_EINVAL;
  if (!st->indx || !st->indy || !st->indz || (h->g.NB > 0 && !st->indb)) return CADMAS_EINVAL;
  cudaStream_t s = h->s;
  const size_t b8 = h->N * sizeof(double), b4 = h->N * sizeof(int);
  CK(cudaMemcpyAsync(h->xx, st->xx, 6 * h->g.NI * sizeof(double), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(h->yy, st->yy, 6 * h->g.NJ * sizeof(double), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(h->zz, st->zz, 6 * h->g.NK * sizeof(double), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(h->ggv, st->ggv, b8, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(h->ggx, st->ggx, b8, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(h->ggy, st->ggy, b8, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(h->ggz, st->ggz, b8, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(h->glv, st->glv, b8, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(h->glx, st->glx, b8, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(h->gly, st->gly, b8, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(h->glz, st->glz, b8, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(h->cd0, st->cd0, b8, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(h->anu, st->anu, b8, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(h->indx, st->indx, b4, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(h->indy, st->indy, b4, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(h->indz, st->indz, b4, cudaMemcpyHostToDevice, s));
  if (h->g.NB > 0) CK(cudaMemcpyAsync(h->indb, st->indb, 4 * h->g.NB * sizeof(int), cudaMemcpyHostToDevice, s));
  h->n_open_faces = 0;
  h->n_log_faces = 0;
  for (long long L = 0; L < h->g.NB; ++L) {
    const int ib = st->indb[4 * L + 2];
    h->n_open_faces += (ib == 7);
    h->n_log_faces += (ib == 6 || ib == 8);
  }
  if (h->g.NB > 0) {
    if (st->bcvi) CK(cudaMemcpyAsync(h->bcvi, st->bcvi, h->g.NB * sizeof(double), cudaMemcpyHostToDevice, s));
    else CK(cudaMemsetAsync(h->bcvi, 0, h->g.NB * sizeof(double), s));
  }
  refresh_prm(h);
  if (h->P.leqk != 0 && h->g.NB > 0) {  // k-epsilon boundaries (vf_iiboun.f:250-330)
    if (!st->indbk || !st->indbe || !st->bck || !st->bce) return CADMAS_EINVAL;
    const size_t nb = (size_t)h->g.NB;
    CK(cudaMemcpyAsync(h->indbk, st->indbk, nb * sizeof(int), cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(h->indbe, st->indbe, nb * sizeof(int), cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(h->bck0, st->bck, nb * sizeof(double), cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(h->bce0, st->bce, nb * sizeof(double), cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(h->bck, st->bck, nb * sizeof(double), cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(h->bce, st->bce, nb * sizeof(double), cudaMemcpyHostToDevice, s));
  }
  // host copies of XX(1,I), YY(1,J) (oblique wave makers)
  h->xx1.assign(h->g.NI + 2, 0.0);
  h->yy1.assign(h->g.NJ + 2, 0.0);
  for (int i = 1; i <= h->g.NI; ++i) h->xx1[i] = st->xx[6 * (i - 1)];
  for (int j = 1; j <= h->g.NJ; ++j) h->yy1[j] = st->yy[6 * (j - 1)];
  // host copy of ZZ(2,K) for the bubble timers
  h->zz2.assign(h->g.NK + 1, 0.0);
  std::vector<double> zz(6 * h->g.NK);
  std::memcpy(zz.data(), st->zz, zz.size() * sizeof(double));
  for (int k = 1; k <= h->g.NK; ++k) h->zz2[k] = zz[1 + 6 * (k - 1)];
  CK(cudaStreamSynchronize(s));
  h->have_static = true;
  return CADMAS_OK;
}

int cadmas_set_state(cadmas_handle *h, const cadmas_state *st) {
  if (!h || !st) return CADMAS_EINVAL;
  cudaStream_t s = h->s;
  const size_t b8 = h->N * sizeof(double), b4 = h->N * sizeof(int), bb = (size_t)h->g.NB * sizeof(double);
  refresh_fld(h);
  if (st->uu) CK(cudaMemcpyAsync(h->f.uu, st->uu, b8, cudaMemcpyHostToDevice, s));
  if (st->vv) CK(cudaMemcpyAsync(h->f.vv, st->vv, b8, cudaMemcpyHostToDevice, s));
  if (st->ww) CK(cudaMemcpyAsync(h->f.ww, st->ww, b8, cudaMemcpyHostToDevice, s));
  if (st->pp) CK(cudaMemcpyAsync(h->f.pp, st->pp, b8, cudaMemcpyHostToDevice, s));
  if (st->ff) CK(cudaMemcpyAsync(h->ff, st->ff, b8, cudaMemcpyHostToDevice, s));
  if (st->nf) CK(cudaMemcpyAsync(h->nf, st->nf, b4, cudaMemcpyHostToDevice, s));
  if (st->indc) CK(cudaMemcpyAsync(h->indc, st->indc, b4, cudaMemcpyHostToDevice, s));
  if (bb) {
    if (st->bcu) CK(cudaMemcpyAsync(h->bcu, st->bcu, bb, cudaMemcpyHostToDevice, s));
    if (st->bcv) CK(cudaMemcpyAsync(h->bcv, st->bcv, bb, cudaMemcpyHostToDevice, s));
    if (st->bcw) CK(cudaMemcpyAsync(h->bcw, st->bcw, bb, cudaMemcpyHostToDevice, s));
    if (st->bcp) CK(cudaMemcpyAsync(h->bcp, st->bcp, bb, cudaMemcpyHostToDevice, s));
    if (st->bcf) CK(cudaMemcpyAsync(h->bcf, st->bcf, bb, cudaMemcpyHostToDevice, s));
  }
  if (st->tbub) std::memcpy(h->tbub.data(), st->tbub, h->g.NK * sizeof(double));
  h->tnow = st->tnow;
  h->nnow = st->nnow;
  CK(cudaStreamSynchronize(s));
  return CADMAS_OK;
}

int cadmas_get_state(cadmas_handle *h, cadmas_state *st) {
  if (!h || !st) return CADMAS_EINVAL;
  cudaStream_t s = h->s;
  const size_t b8 = h->N * sizeof(double), b4 = h->N * sizeof(int), bb = (size_t)h->g.NB * sizeof(double);
  refresh_fld(h);
  if (st->uu) CK(cudaMemcpyAsync(st->uu, h->f.uu, b8, cudaMemcpyDeviceToHost, s));
  if (st->vv) CK(cudaMemcpyAsync(st->vv, h->f.vv, b8, cudaMemcpyDeviceToHost, s));
  if (st->ww) CK(cudaMemcpyAsync(st->ww, h->f.ww, b8, cudaMemcpyDeviceToHost, s));
  if (st->pp) CK(cudaMemcpyAsync(st->pp, h->f.pp, b8, cudaMemcpyDeviceToHost, s));
  if (st->ff) CK(cudaMemcpyAsync(st->ff, h->ff, b8, cudaMemcpyDeviceToHost, s));
  if (st->nf) CK(cudaMemcpyAsync(st->nf, h->nf, b4, cudaMemcpyDeviceToHost, s));
  if (st->indc) CK(cudaMemcpyAsync(st->indc, h->indc, b4, cudaMemcpyDeviceToHost, s));
  if (bb) {
    if (st->bcu) CK(cudaMemcpyAsync(st->bcu, h->bcu, bb, cudaMemcpyDeviceToHost, s));
    if (st->bcv) CK(cudaMemcpyAsync(st->bcv, h->bcv, bb, cudaMemcpyDeviceToHost, s));
    if (st->bcw) CK(cudaMemcpyAsync(st->bcw, h->bcw, bb, cudaMemcpyDeviceToHost, s));
    if (st->bcp) CK(cudaMemcpyAsync(st->bcp, h->bcp, bb, cudaMemcpyDeviceToHost, s));
    if (st->bcf) CK(cudaMemcpyAsync(st->bcf, h->bcf, bb, cudaMemcpyDeviceToHost, s));
  }
  if (st->tbub) std::memcpy(st->tbub, h->tbub.data(), h->g.NK * sizeof(double));
  st->tnow = h->tnow;
  st->nnow = h->nnow;
  CK(cudaStreamSynchronize(s));
  return CADMAS_OK;
}

int cadmas_get_drop(cadmas_handle *h, double *tx, double *ty, double *tz, double *uu, double *vv, double *ww) {
  if (!h) return CADMAS_EINVAL;
  const size_t b8 = h->N * sizeof(double);
  double *dst[6] = {tx, ty, tz, uu, vv, ww};
  const double *src[6] = {h->drop.tx, h->drop.ty, h->drop.tz, h->drop.uu, h->drop.vv, h->drop.ww};
  for (int a = 0; a < 6; ++a)
    if (dst[a]) CK(cudaMemcpyAsync(dst[a], src[a], b8, cudaMemcpyDeviceToHost, h->s));
  CK(cudaStreamSynchronize(h->s));
  return CADMAS_OK;
}

int cadmas_set_drop(cadmas_handle *h, const double *tx, const double *ty, const double *tz, const double *uu,
                    const double *vv, const double *ww) {
  if (!h) return CADMAS_EINVAL;
  const size_t b8 = h->N * sizeof(double);
  const double *src[6] = {tx, ty, tz, uu, vv, ww};
  double *dst[6] = {h->drop.tx, h->drop.ty, h->drop.tz, h->drop.uu, h->drop.vv, h->drop.ww};
  for (int a = 0; a < 6; ++a)
    if (src[a]) CK(cudaMemcpyAsync(dst[a], src[a], b8, cudaMemcpyHostToDevice, h->s));
  CK(cudaStreamSynchronize(h->s));
  return CADMAS_OK;
}

// VF_OR1INI (vf_or1ini.f:38-86) for NPROCS = 1: version, sizes, the
// flags of the fields that follow every output, GGV.
int cadmas_restart_create(cadmas_handle *h, const char *path) {
  if (!h || !path) return CADMAS_EINVAL;
  if (!h->have_static) return CADMAS_ENOSTATIC;
  FRecordFile r;
  r.f = std::fopen(path, "wb");
  if (!r.f) { g_last_error = "CAN NOT OPEN (*****.rsl)."; return CADMAS_EIO; }
  const int32_t ver[2] = {0, 1};  // IVR001, IVR002 (VF_A0PRM.h)
  const int32_t dims[4] = {h->g.NI, h->g.NJ, h->g.NK, h->g.NB};
  // LN, LV, LP, LF, LK, LT, LS, LG, LD, L1: k-eps when LEQK != 0, no
  // temperature, scalars or time-dependent porosity here; droplets when
  // IDROP >= 1
  const int32_t flags[10] = {1, 1, 1, 1, h->P.leqk != 0 ? 1 : 0, 0, 0, 0, h->P.idrop >= 1 ? 1 : 0, 0};
  std::vector<double> ggv(h->N);
  CK(cudaMemcpy(ggv.data(), h->ggv, h->N * sizeof(double), cudaMemcpyDeviceToHost));
  if (!r.put({{ver, sizeof ver}}) || !r.put({{dims, sizeof dims}}) || !r.put({{flags, sizeof flags}}) ||
      !r.put({{ggv.data(), h->N * sizeof(double)}})) {
    g_last_error = "WRITE ERROR (*****.rsl).";
    return CADMAS_EIO;
  }
  return CADMAS_OK;
}

// VF_OR1TRN (vf_or1trn.f:104-221): one output of the present state
// appended to a file made by cadmas_restart_create.
int cadmas_restart_append(cadmas_handle *h, const char *path) {
  if (!h || !path) return CADMAS_EINVAL;
  const size_t N = h->N, NB = (size_t)h->g.NB;
  std::vector<double> a[5];
  std::vector<double> bc[5];
  std::vector<int32_t> nf(N);
  cadmas_state st;
  std::memset(&st, 0, sizeof st);
  for (int k = 0; k < 5; ++k) { a[k].resize(N); bc[k].resize(NB); }
  st.uu = a[0].data(); st.vv = a[1].data(); st.ww = a[2].data(); st.pp = a[3].data(); st.ff = a[4].data();
  st.nf = nf.data();
  if (NB) { st.bcu = bc[0].data(); st.bcv = bc[1].data(); st.bcw = bc[2].data(); st.bcp = bc[3].data(); st.bcf = bc[4].data(); }
  int rc = cadmas_get_state(h, &st);
  if (rc) return rc;
  std::vector<double> dr[6];
  for (auto &v : dr) v.resize(N);
  if (h->P.idrop >= 1) {
    rc = cadmas_get_drop(h, dr[0].data(), dr[1].data(), dr[2].data(), dr[3].data(), dr[4].data(), dr[5].data());
    if (rc) return rc;
  }
  std::vector<double> ke[4];  // AK, BCK, AE, BCE
  if (h->P.leqk != 0) {
    ke[0].resize(N); ke[2].resize(N); ke[1].resize(NB); ke[3].resize(NB);
    rc = cadmas_get_turb(h, ke[0].data(), ke[2].data(), nullptr, nullptr, NB ? ke[1].data() : nullptr,
                         NB ? ke[3].data() : nullptr);
    if (rc) return rc;
  }
  FRecordFile r;
  r.f = std::fopen(path, "ab");
  if (!r.f) { g_last_error = "CAN NOT OPEN (*****.rsl)."; return CADMAS_EIO; }
  const int32_t nnow = h->nnow, icgitr = h->stats.icgitr;
  const double tn = h->tnow, dtn = h->dtnow;
  const double sums[4] = {h->stats.fsum, h->stats.fcut, h->stats.cgbnrm, h->stats.cgxnrm};
  const size_t b8 = N * sizeof(double), bb = NB * sizeof(double);
  bool ok = r.put({{&nnow, 4}, {&tn, 8}, {&dtn, 8}}) && r.put({{sums, sizeof sums}, {&icgitr, 4}}) &&
            r.put({{nf.data(), N * 4}});
  for (int k = 0; k < 5 && ok; ++k) ok = r.put({{a[k].data(), b8}}) && r.put({{bc[k].data(), bb}});
  if (h->P.leqk != 0)  // vf_or1trn.f:134-146
    for (int k = 0; k < 4 && ok; ++k) ok = r.put({{ke[k].data(), (k % 2 ? bb : b8)}});
  ok = ok && r.put({{h->tbub.data(), (size_t)h->g.NK * sizeof(double)}});
  if (ok && h->P.idrop >= 1) {
    // the droplet cells (DROPTX >= 0), K, J, I order
    const int NI = h->g.NI, NJ = h->g.NJ, NK = h->g.NK;
    std::vector<size_t> cells;
    for (int K = 2; K <= NK - 1; ++K)
      for (int J = 2; J <= NJ - 1; ++J)
        for (int I = 2; I <= NI - 1; ++I) {
          const size_t c = (size_t)(I - 1) + (size_t)NI * ((size_t)(J - 1) + (size_t)NJ * (K - 1));
          if (dr[0][c] >= 0.0) cells.push_back(c);
        }
    const int32_t nd = (int32_t)cells.size();
    ok = r.put({{&nd, 4}});
    for (size_t c : cells) {
      if (!ok) break;
      const int32_t ijk[3] = {(int32_t)(c % NI) + 1, (int32_t)((c / NI) % NJ) + 1, (int32_t)(c / ((size_t)NI * NJ)) + 1};
      const double v[6] = {dr[0][c], dr[1][c], dr[2][c], dr[3][c], dr[4][c], dr[5][c]};
      ok = r.put({{ijk, sizeof ijk}, {v, sizeof v}});
    }
  }
  if (!ok) { g_last_error = "WRITE ERROR (*****.rsl)."; return CADMAS_EIO; }
  return CADMAS_OK;
}

// VF_IR1INP (vf_ir1inp.f:96-336) for NPROCS = 1: read the outputs of a
// restart file up to the one of step nnow and make it the present state
// (time, step, sums, flags, fields, boundary values, TBUB, droplets), with
// INDC from NF (VF_CINDC).
int cadmas_restart_load(cadmas_handle *h, const char *path, int nnow) {
  if (!h || !path) return CADMAS_EINVAL;
  if (!h->have_static) return CADMAS_ENOSTATIC;
  FRecordFile r;
  r.f = std::fopen(path, "rb");
  if (!r.f) { g_last_error = "CAN NOT OPEN (*****.res)."; return CADMAS_EIO; }
  const size_t N = h->N, NB = (size_t)h->g.NB, NK = (size_t)h->g.NK;
  auto bad = [&](const char *m) { g_last_error = m; return CADMAS_EIO; };
  std::vector<unsigned char> b;
  if (!r.get(b) || b.size() != 8) return bad("READ ERROR (*****.res).");
  if (!r.get(b) || b.size() != 16) return bad("READ ERROR (*****.res).");
  if (rec_at<int32_t>(b, 0) != h->g.NI || rec_at<int32_t>(b, 4) != h->g.NJ || rec_at<int32_t>(b, 8) != h->g.NK)
    return bad("INVALID NUMBER OF GRID.");
  if (rec_at<int32_t>(b, 12) != h->g.NB) return bad("INVALID NUMBER OF B.C.");
  if (!r.get(b) || b.size() != 40) return bad("READ ERROR (*****.res).");
  int32_t L[10];
  std::memcpy(L, b.data(), sizeof L);
  if (L[4] != (h->P.leqk != 0 ? 1 : 0)) return bad("INVALID EQUATION (K-EPS).");
  if (L[5] != 0) return bad("INVALID EQUATION (TEMP).");
  if (L[6] != 0) return bad("INVALID EQUATION (CONC).");
  const int LG = L[7], LD = L[8];
  if (LG == 0 && (!r.get(b) || b.size() != N * 8)) return bad("READ ERROR (*****.res).");  // GGV, unused
  std::vector<unsigned char> rec[14], kr[4];  // kr: AK, BCK, AE, BCE
  for (;;) {
    bool eof = false;
    if (!r.get(rec[0], &eof)) return bad(eof ? "INVALID STEP." : "READ ERROR (*****.res).");
    if (rec[0].size() != 20) return bad("READ ERROR (*****.res).");
    // rec[1] sums, [2] NF, [3] UU, [4] BCU, [5] VV, [6] BCV, [7] WW, [8] BCW,
    // [9] PP, [10] BCP, [11] FF, [12] BCF, (GGV when LG != 0), [13] TBUB
    const size_t want[12] = {36, N * 4, N * 8, NB * 8, N * 8, NB * 8, N * 8, NB * 8, N * 8, NB * 8, N * 8, NB * 8};
    for (int k = 1; k <= 12; ++k)
      if (!r.get(rec[k]) || rec[k].size() != want[k - 1]) return bad("READ ERROR (*****.res).");
    if (L[4] != 0) {  // vf_ir1inp.f:213-225
      const size_t kw[4] = {N * 8, NB * 8, N * 8, NB * 8};
      for (int k = 0; k < 4; ++k)
        if (!r.get(kr[k]) || kr[k].size() != kw[k]) return bad("READ ERROR (*****.res).");
    }
    if (LG != 0 && !r.get(b)) return bad("READ ERROR (*****.res).");  // GGV of IPRNT > 1, unused
    if (!r.get(rec[13]) || rec[13].size() != NK * 8) return bad("READ ERROR (*****.res).");
    const int32_t step = rec_at<int32_t>(rec[0], 0);
    std::vector<double> dr[6];
    if (LD >= 1) {
      if (!r.get(b) || b.size() != 4) return bad("READ ERROR (*****.res).");
      const int32_t nd = rec_at<int32_t>(b, 0);
      const bool use = h->P.idrop >= 1 && step == nnow;
      if (use) {
        for (auto &v : dr) v.assign(N, 0.0);
        std::fill(dr[0].begin(), dr[0].end(), -1.0e10);
      }
      for (int32_t n = 0; n < nd; ++n) {
        if (!r.get(b) || b.size() != 60) return bad("READ ERROR (*****.res).");
        if (!use) continue;
        const int I = rec_at<int32_t>(b, 0), J = rec_at<int32_t>(b, 4), K = rec_at<int32_t>(b, 8);
        if (I < 1 || I > h->g.NI || J < 1 || J > h->g.NJ || K < 1 || K > h->g.NK) return bad("READ ERROR (*****.res).");
        const size_t c = (size_t)(I - 1) + (size_t)h->g.NI * ((size_t)(J - 1) + (size_t)h->g.NJ * (K - 1));
        for (int a = 0; a < 6; ++a) dr[a][c] = rec_at<double>(b, 12 + 8 * a);
      }
    }
    if (step != nnow) continue;
    // the output of step nnow: make it the state
    cadmas_state st;
    std::memset(&st, 0, sizeof st);
    st.nf = reinterpret_cast<int *>(rec[2].data());
    st.uu = reinterpret_cast<double *>(rec[3].data()); st.vv = reinterpret_cast<double *>(rec[5].data());
    st.ww = reinterpret_cast<double *>(rec[7].data()); st.pp = reinterpret_cast<double *>(rec[9].data());
    st.ff = reinterpret_cast<double *>(rec[11].data());
    if (NB) {
      st.bcu = reinterpret_cast<double *>(rec[4].data()); st.bcv = reinterpret_cast<double *>(rec[6].data());
      st.bcw = reinterpret_cast<double *>(rec[8].data()); st.bcp = reinterpret_cast<double *>(rec[10].data());
      st.bcf = reinterpret_cast<double *>(rec[12].data());
    }
    st.tbub = reinterpret_cast<double *>(rec[13].data());
    st.tnow = rec_at<double>(rec[0], 4);
    st.nnow = step;
    int rc = cadmas_set_state(h, &st);
    if (rc) return rc;
    h->dtnow = rec_at<double>(rec[0], 12);
    h->stats.fsum = rec_at<double>(rec[1], 0); h->stats.fcut = rec_at<double>(rec[1], 8);
    h->stats.cgbnrm = rec_at<double>(rec[1], 16); h->stats.cgxnrm = rec_at<double>(rec[1], 24);
    h->stats.icgitr = rec_at<int32_t>(rec[1], 32);
    if (h->P.leqk != 0) {  // k, e, their boundary values, then ANUT, ANU (vf_ir1inp.f:339-340)
      rc = cadmas_set_turb(h, reinterpret_cast<double *>(kr[0].data()), reinterpret_cast<double *>(kr[2].data()),
                           reinterpret_cast<double *>(kr[1].data()), reinterpret_cast<double *>(kr[3].data()));
      if (rc) return rc;
    }
    if (h->P.idrop >= 1) {
      if (LD >= 1) rc = cadmas_set_drop(h, dr[0].data(), dr[1].data(), dr[2].data(), dr[3].data(), dr[4].data(), dr[5].data());
      else launch_drop_reset(h->s, (long long)N, h->drop);  // vf_ir1inp.f:96-108
      if (rc) return rc;
    }
    // INDC from NF (vf_ir1inp.f:316-322)
    refresh_fld(h);
    CK(cudaMemsetAsync(h->indc, 0xff, N * sizeof(int), h->s));
    CK(cudaMemsetAsync(h->dint + 4, 0, sizeof(int), h->s));
    launch_cindc(h->s, h->g, h->f, h->dint + 4);
    int bits;
    rc = read_err(h, bits);
    if (rc) return rc;
    h->stats.nums = h->h_int[4];
    return CADMAS_OK;
  }
}

// The two lines the time loop writes to the list file after a step
// (vf_a1main.f:954-958, formats 9540 and 9550), with !VD! from VF_CDIV00.
int cadmas_list_step(cadmas_handle *h, char *buf, size_t len) {
  if (!h || !buf || len == 0) return CADMAS_EINVAL;
  double dv;
  int rc = cadmas_divnorm(h, &dv);
  if (rc) return rc;
  const cadmas_stats &S = h->stats;
  std::string t = " STEP=" + f_i6(h->nnow) + " : TIME= " + f_e12_5(h->tnow) + " : DT  = " + f_e12_5(h->dtnow) +
                  " : FSUM= " + f_e12_5(S.fsum) + " : FCUT= " + f_e12_5(S.fcut) + " : !VD!= " + f_e12_5(dv) + "\n" +
                  " " + std::string(11, ' ') + " : !B! = " + f_e12_5(S.cgbnrm) + " : !R! = " + f_e12_5(S.cgxnrm) +
                  " : ITR = " + f_i6(S.icgitr) + "\n";
  if (t.size() + 1 > len) return CADMAS_EINVAL;
  std::memcpy(buf, t.c_str(), t.size() + 1);
  return CADMAS_OK;
}

int cadmas_init_state(cadmas_handle *h, int hydrostatic) {
  if (!h) return CADMAS_EINVAL;
  if (!h->have_static) return CADMAS_ENOSTATIC;
  cudaStream_t s = h->s;
  refresh_prm(h);
  refresh_fld(h);
  CK(cudaMemsetAsync(h->dint, 0, 8 * sizeof(int), s));
  { const int rl = fixed_level_f(h); if (rl) return rl; }  // vf_cinit.f:177
  // vf_cinit.f:202-207
  launch_fcut(s, h->g, h->f, h->p, h->rb0, h->rb1);
  launch_fin(s, FIN_STORE, h->rb0, h->rb1, nrows(h), h->st, h->dres, 0, 0, 0, 0);
  launch_bwff(s, h->g, h->f, h->dint);
  int rc = fnfini(h);
  if (rc) return rc;
  launch_fnfprv(s, h->g, h->f, h->dint);
  CK(cudaMemsetAsync(h->indc, 0xff, h->N * sizeof(int), s));
  CK(cudaMemsetAsync(h->dint + 4, 0, sizeof(int), s));
  launch_cindc(s, h->g, h->f, h->dint + 4);
  if (hydrostatic) {
    // p = RHO0*GRZ0*(WVLVL - z_c) on INDC != -1 (vf_cinit.f:273-285)
    std::vector<double> pp(h->N, 0.0);
    std::vector<int> indc(h->N);
    std::vector<double> zz(6 * h->g.NK);
    CK(cudaMemcpyAsync(indc.data(), h->indc, h->N * sizeof(int), cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(zz.data(), h->zz, zz.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    const int NI = h->g.NI, NJ = h->g.NJ, NK = h->g.NK;
    for (int K = 2; K <= NK - 1; ++K) {
      double VAL = h->P.rho0 * h->P.grz0 * (h->P.wvlvl - (zz[6 * (K - 1)] + zz[6 * K]) * 0.5);
      for (int J = 2; J <= NJ - 1; ++J)
        for (int I = 2; I <= NI - 1; ++I) {
          size_t c = (size_t)(I - 1) + (size_t)NI * ((size_t)(J - 1) + (size_t)NJ * (K - 1));
          if (indc[c] != -1) pp[c] = VAL;
        }
    }
    CK(cudaMemcpyAsync(h->f.pp, pp.data(), h->N * sizeof(double), cudaMemcpyHostToDevice, s));
    CK(cudaStreamSynchronize(s));
  }
  // vf_cinit.f:376-394: the open boundary reads a copy of the present
  // velocities as those of the previous step
  const bool any_open = h->open[0].on || h->open[1].on || h->open[2].on || h->open[3].on;
  if (any_open)
    for (int c = 0; c < 3; ++c)
      CK(cudaMemcpyAsync(h->wk[c], h->vel[h->cur][c], h->N * sizeof(double), cudaMemcpyDeviceToDevice, s));
  launch_bwuwn(s, h->g, h->f, h->p, h->dint);
  { const int rw = wave_bc(h); if (rw) return rw; }
  { const int ro = open_bc(h, h->wk[0], h->wk[1], h->wk[2]); if (ro) return ro; }
  // vf_cinit.f:295-315 and 359-364: k, e, ANUT and ANU before the wall
  // functions of VF_BWUWT read ANU
  if (h->P.leqk != 0) launch_kinit(s, h->g, h->f, ke_const(h), h->ak, h->ae_k, h->anut, h->anu);
  launch_bsuwt(s, h->g, h->f, h->p);
  launch_bsuwt2(s, h->g, h->f);
  launch_bsuwn3(s, h->g, h->f, h->p);
  launch_bspp(s, h->g, h->f);
  launch_bwuwt(s, h->g, h->f, h->p, h->dint);
  launch_bwpp(s, h->g, h->f);
  if (h->P.leqk != 0) {
    // vf_cinit.f:397-401
    const KeConst kc = ke_const(h);
    if (h->g.NB > 0) {
      CK(cudaMemcpyAsync(h->bck, h->bck0, (size_t)h->g.NB * sizeof(double), cudaMemcpyDeviceToDevice, s));
      CK(cudaMemcpyAsync(h->bce, h->bce0, (size_t)h->g.NB * sizeof(double), cudaMemcpyDeviceToDevice, s));
    }
    launch_kbsss(s, h->g, h->f, kc, h->ak, h->ae_k, h->anut, h->anu, true, false);
    launch_bwke(s, h->g, h->f, ke_arrays(h), h->dint);
  }
  std::fill(h->tbub.begin(), h->tbub.end(), 0.0);
  launch_drop_reset(s, (long long)h->N, h->drop);  // vf_cinit.f:416-427
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(h->h_res, h->dres, 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
  int bits;
  rc = read_err(h, bits);
  if (rc) return rc;
  h->stats.fsum = h->h_res[0];
  h->stats.fcut = h->h_res[1];
  h->stats.nums = h->h_int[4];
  return map_err(bits);
}

int cadmas_get_turb(cadmas_handle *h, double *ak, double *ae, double *anut, double *anu, double *bck,
                    double *bce) {
  if (!h || h->P.leqk == 0) return CADMAS_EINVAL;
  cudaStream_t s = h->s;
  const size_t b8 = h->N * sizeof(double), bb = (size_t)h->g.NB * sizeof(double);
  if (ak) CK(cudaMemcpyAsync(ak, h->ak, b8, cudaMemcpyDeviceToHost, s));
  if (ae) CK(cudaMemcpyAsync(ae, h->ae_k, b8, cudaMemcpyDeviceToHost, s));
  if (anut) CK(cudaMemcpyAsync(anut, h->anut, b8, cudaMemcpyDeviceToHost, s));
  if (anu) CK(cudaMemcpyAsync(anu, h->anu, b8, cudaMemcpyDeviceToHost, s));
  if (bck && bb) CK(cudaMemcpyAsync(bck, h->bck, bb, cudaMemcpyDeviceToHost, s));
  if (bce && bb) CK(cudaMemcpyAsync(bce, h->bce, bb, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  return CADMAS_OK;
}

int cadmas_set_turb(cadmas_handle *h, const double *ak, const double *ae, const double *bck, const double *bce) {
  if (!h || h->P.leqk == 0 || !ak || !ae || (h->g.NB > 0 && (!bck || !bce))) return CADMAS_EINVAL;
  if (!h->have_static) return CADMAS_ENOSTATIC;
  cudaStream_t s = h->s;
  const size_t b8 = h->N * sizeof(double), bb = (size_t)h->g.NB * sizeof(double);
  CK(cudaMemcpyAsync(h->ak, ak, b8, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(h->ae_k, ae, b8, cudaMemcpyHostToDevice, s));
  if (bb) {
    CK(cudaMemcpyAsync(h->bck, bck, bb, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(h->bce, bce, bb, cudaMemcpyHostToDevice, s));
  }
  ke_nut(h);  // vf_ir1inp.f:339-340
  CK(cudaStreamSynchronize(s));
  return CADMAS_OK;
}

int cadmas_set_warm_net(cadmas_handle *h, const float *params, double out_scale) {
  if (!h || !params || !(out_scale > 0.0)) return CADMAS_EINVAL;
  if (!h->wnet) {
    const int X = (h->g.NI + 3) & ~3, Y = (h->g.NJ + 3) & ~3, Z = (h->g.NK + 3) & ~3;
    int rc = unet_new(X, Y, Z, 1, h->s, &h->wnet);
    if (rc) return rc;
    if (dalloc(&h->ws_rows, 2 * (size_t)nrows(h)) || dalloc(&h->ws_scal, 4) || dalloc(&h->ws_cnt, 4))
      return CADMAS_ENOMEM;
    CK(cudaMemsetAsync(h->ws_cnt, 0, 4 * sizeof(int), h->s));
  }
  // scal = [s, |r|^2, |b|^2, output scale]
  CK(cudaMemcpyAsync(h->ws_scal + 3, &out_scale, sizeof(double), cudaMemcpyHostToDevice, h->s));
  return cadmas_unet_set_params(h->wnet, params);
}

int cadmas_warm_stats(cadmas_handle *h, long long *kept, long long *dropped) {
  if (!h) return CADMAS_EINVAL;
  int c[2] = {0, 0};
  if (h->ws_cnt) {
    CK(cudaMemcpyAsync(c, h->ws_cnt, 2 * sizeof(int), cudaMemcpyDeviceToHost, h->s));
    CK(cudaStreamSynchronize(h->s));
    const int e = unet_error_host(h->wnet);
    if (e) return e;
  }
  if (kept) *kept = c[0];
  if (dropped) *dropped = c[1];
  return CADMAS_OK;
}

int cadmas_get_system(cadmas_handle *h, double *ad, double *ali, double *alj, double *alk, double *aui,
                      double *auj, double *auk) {
  if (!h) return CADMAS_EINVAL;
  double *out[7] = {ad, ali, alj, alk, aui, auj, auk};
  for (int k = 0; k < 7; ++k)
    if (out[k]) CK(cudaMemcpyAsync(out[k], h->wk[k], h->N * sizeof(double), cudaMemcpyDeviceToHost, h->s));
  CK(cudaStreamSynchronize(h->s));
  return CADMAS_OK;
}

int cadmas_get_solve(cadmas_handle *h, double *bb, double *pt) {
  if (!h) return CADMAS_EINVAL;
  const size_t b8 = h->N * sizeof(double);
  if (bb) CK(cudaMemcpyAsync(bb, h->wk[7], b8, cudaMemcpyDeviceToHost, h->s));
  if (pt) CK(cudaMemcpyAsync(pt, h->wk[8], b8, cudaMemcpyDeviceToHost, h->s));
  CK(cudaStreamSynchronize(h->s));
  return CADMAS_OK;
}

int cadmas_set_time(cadmas_handle *h, double tnow, double dtnow, int nnow) {
  if (!h) return CADMAS_EINVAL;
  h->tnow = tnow; h->dtnow = dtnow; h->nnow = nnow;
  return CADMAS_OK;
}

int cadmas_v1cal(cadmas_handle *h) {
  if (!h) return CADMAS_EINVAL;
  if (!h->have_static) return CADMAS_ENOSTATIC;
  int rc = do_v1cal(h);
  if (rc == CADMAS_OK) {
    int bits;
    rc = read_err(h, bits);
    if (rc == CADMAS_OK) rc = map_err(bits);
  }
  h->stats.last_status = rc;
  return rc;
}

int cadmas_f1cal(cadmas_handle *h) {
  if (!h) return CADMAS_EINVAL;
  if (!h->have_static) return CADMAS_ENOSTATIC;
  int rc = do_f1cal(h);
  h->stats.last_status = rc;
  return rc;
}

int cadmas_step(cadmas_handle *h, double dt) {
  if (!h) return CADMAS_EINVAL;
  if (!h->have_static) return CADMAS_ENOSTATIC;
  if (!(dt > 0.0)) return CADMAS_EINVAL;
  // vf_a1main.f:1029-1047 with LOOPS = 1
  h->dtnow = dt;
  h->nnow = h->nnow + 1;
  h->tnow = h->tnow + h->dtnow;
  int rc = cadmas_v1cal(h);
  if (rc == CADMAS_OK) rc = cadmas_f1cal(h);
  h->stats.last_status = rc;
  return rc;
}

int cadmas_step_ensemble(cadmas_handle **hs, int n, const double *dt, int *status) {
  if (!hs || !dt || !status || n < 0) return CADMAS_EINVAL;
  for (int i = 0; i < n; ++i)
    if (!hs[i]) return CADMAS_EINVAL;
  if (n == 1) return status[0] = cadmas_step(hs[0], dt[0]);
  std::vector<std::thread> pool;
  pool.reserve((size_t)n);
  for (int i = 0; i < n; ++i)
    pool.emplace_back([=]() {
      cudaSetDevice(hs[i]->device);
      status[i] = cadmas_step(hs[i], dt[i]);
    });
  for (std::thread &t : pool) t.join();
  for (int i = 0; i < n; ++i)
    if (status[i]) return status[i];
  return CADMAS_OK;
}

// ------------------------------------------------------------ batches
// Grids stepped together with one launch of each solver kernel for all of
// them (the mixed solver's FP32 iteration, its FP64 residuals, the layout
// conversions and the factorisation).  The parts of a step around the
// solve run per grid on the grid's own stream and host thread.
struct cadmas_batch {
  std::vector<cadmas_handle *> h;
  int device = 0, nsm = 148, occ = 0;
  cudaStream_t s = nullptr;
  BatchMember *d_m = nullptr, *h_m = nullptr;  // member table (device, pinned host)
  int *d_pre = nullptr;                          // block prefixes (BR_N x (n+1))
  double *d_g = nullptr, *h_g = nullptr;         // gathered per member
  cudaEvent_t ev = nullptr;
  std::vector<cudaEvent_t> ev_m;
  long long launches_solve = 0;
};

namespace {
// A member's part of the batched solve from its handle.
BatchMember batch_member_of(cadmas_handle *h) {
  BatchMember m;
  std::memset(&m, 0, sizeof(m));
  h->Sf.indc = h->S.indc;
  m.g = h->g; m.q = h->q; m.S = h->S; m.Sf = h->Sf; m.a = poisson_sys(h);
  m.indc = h->indc; m.pt = h->wk[8];
  float *vf[BF_N] = {h->bf, h->xf, h->r0f, h->rrf, h->pvf, h->apf, h->aef, h->y2f};
  for (int i = 0; i < BF_N; ++i) m.vf[i] = vf[i];
  m.vd[BD_B] = h->bb_sl; m.vd[BD_X] = h->xw; m.vd[BD_Y2] = h->y2;
  m.rb0 = h->rb0; m.rb1 = h->rb1; m.rb5 = h->rb5; m.dres = h->dres;
  m.st = h->st; m.pivot_bad = &h->st->pivot_bad;
  m.nrb = h->nrb;
  m.epsa2 = h->P.cgepsa * h->P.cgepsa; m.div2 = h->P.cgdiv * h->P.cgdiv; m.tol2 = h->P.cgepsr * h->P.cgepsr;
  m.U = (h->P.icgtyp != 0) ? h->P.cgpara : 0.0;
  m.icgmax = h->P.icgmax;
  m.warm = (h->P.warm_start == 1 && h->have_prev) ? 1 : 0;
  m.active = 1;
  return m;
}
}  // namespace

// The mixed solve (solve_mixed, solve_inner_f) of the members `idx` of a
// batch in lockstep: every refinement pass and every FP32 iteration is one
// launch per kernel over all members still refining; a member that has
// converged is marked done and its blocks return at once.  A member whose
// FP32 factor or inner solve fails is solved alone by the FP64 solver, as
// solve_mixed does.  Results, iterations and status per member.
static void solve_mixed_batch(cadmas_batch *b, const std::vector<int> &idx, std::vector<int> &iter,
                              std::vector<double> &bn, std::vector<double> &xn, std::vector<int> &rc) {
  cudaStream_t s = b->s;
  const int nm = (int)idx.size();
  std::vector<cadmas_handle *> hs(nm);
  for (int j = 0; j < nm; ++j) hs[j] = b->h[idx[j]];
  iter.assign(nm, 0); bn.assign(nm, 0.0); xn.assign(nm, 0.0); rc.assign(nm, CADMAS_OK);
  if (nm == 0) return;
  auto fail = [&](int code) { for (int j = 0; j < nm; ++j) if (!rc[j]) rc[j] = code; };
  // member table and block prefixes
  std::vector<int> pre((size_t)BR_N * (nm + 1), 0);
  long long ntiles = 0, nslab = 0, nelem = 0;
  for (int j = 0; j < nm; ++j) {
    b->h_m[j] = batch_member_of(hs[j]);
    const SkewGeo &q = hs[j]->q;
    const long long n = (long long)q.nb * q.W * q.T;
    pre[BR_TILE * (nm + 1) + j] = (int)ntiles;
    pre[BR_SLAB * (nm + 1) + j] = (int)nslab;
    pre[BR_ELEM * (nm + 1) + j] = (int)nelem;
    ntiles += q.nb;
    nslab += hs[j]->nrb;
    nelem += (n + BATCH_ELEM - 1) / BATCH_ELEM;
  }
  pre[BR_TILE * (nm + 1) + nm] = (int)ntiles;
  pre[BR_SLAB * (nm + 1) + nm] = (int)nslab;
  pre[BR_ELEM * (nm + 1) + nm] = (int)nelem;
  const SkewGeo qref = hs[0]->q;
  const BatchMember *bm = b->d_m;
  const int *dp = b->d_pre;
  const int nsm = b->nsm, occ = b->occ;
  auto upload = [&]() -> bool {
    return cudaMemcpyAsync(b->d_m, b->h_m, (size_t)nm * sizeof(BatchMember), cudaMemcpyHostToDevice, s) ==
           cudaSuccess;
  };
  auto gather = [&]() -> bool {
    launch_b_gather(s, bm, nm, b->d_g);
    return cudaMemcpyAsync(b->h_g, b->d_g, (size_t)nm * BATCH_GATHER * sizeof(double), cudaMemcpyDeviceToHost,
                           s) == cudaSuccess &&
           cudaStreamSynchronize(s) == cudaSuccess;
  };
  auto G = [&](int j, int c) { return b->h_g[(size_t)j * BATCH_GATHER + c]; };
  if (cudaMemcpyAsync(b->d_pre, pre.data(), pre.size() * sizeof(int), cudaMemcpyHostToDevice, s) != cudaSuccess ||
      !upload()) { set_cuda_error("batch upload", cudaGetLastError()); fail(CADMAS_ECUDA); return; }
  // the FP64 system, INDC, B and the initial guess in the skewed layout;
  // the FP32 system and its factor
  launch_b_to_skew(s, bm, dp, nm, nelem);
  launch_b_sys_to_f(s, bm, dp, nm, nelem);
  launch_b_clear(s, bm, nm);
  if (!launch_b_dcmp_f(s, bm, dp, nm, ntiles, qref.T) || !gather()) { fail(CADMAS_ECUDA); return; }
  std::vector<char> fallback(nm, 0), conv(nm, 0);
  std::vector<double> b2(nm, 0.0), r2(nm, 0.0);
  std::vector<int> total(nm, 0);
  for (int j = 0; j < nm; ++j)
    if (G(j, 3) != 0.0) { fallback[j] = 1; b->h_m[j].active = 0; }
  bool error = false;
  for (int outer = 0; outer < 40 && !error; ++outer) {
    // r = b - A x and the two norms in FP64 for every member still refining
    if (!upload()) { error = true; break; }
    launch_b_clear(s, bm, nm);
    launch_b_residual(s, bm, dp, nm, nslab);
    launch_b_fin(s, FIN_STORE, bm, nm, false);
    if (!gather()) { error = true; break; }
    int nact = 0;
    for (int j = 0; j < nm; ++j) {
      BatchMember &M = b->h_m[j];
      if (!M.active) continue;
      cadmas_handle *h = hs[j];
      b2[j] = G(j, 4);
      r2[j] = G(j, 5);
      h->mixed_outer++;
      if (r2[j] <= M.tol2 * b2[j]) { conv[j] = 1; M.active = 0; continue; }
      const double rn = std::sqrt(r2[j]);
      const double need = std::sqrt(M.tol2 * b2[j] / r2[j]);
      const double floor_eps = h->P.mixed_eps_inner > 0.0 ? h->P.mixed_eps_inner : 1.0e-5;
      const double eps_in = std::min(0.5, std::max(0.5 * need, floor_eps));
      M.rn = rn; M.scale = 1.0 / rn; M.eps2 = eps_in * eps_in;
      ++nact;
    }
    if (nact == 0) break;
    if (!upload()) { error = true; break; }
    // the inner FP32 solve of every member refining (solve_inner_f)
    launch_b_start_f(s, bm, dp, nm, nslab);
    launch_b_clear(s, bm, nm);
    bool ok = launch_b_sweep(s, SWEEP_FWD, bm, dp, nm, ntiles, qref, BF_B, -1, -1, false, nsm, occ) &&
              launch_b_sweep(s, SWEEP_BWD, bm, dp, nm, ntiles, qref, -1, BF_R0, -1, false, nsm, occ);
    launch_b_dot_r0f(s, bm, dp, nm, nslab);
    launch_b_fin(s, FIN_BNORM, bm, nm, false);
    launch_b_fin(s, FIN_START, bm, nm, false);
    launch_b_copy2_f(s, bm, dp, nm, nslab);
    int last = 8;
    for (int j = 0; j < nm; ++j) last = std::max(last, hs[j]->last_iter);
    int batch = std::max(2, std::min(last, 64));
    for (int guard = 0; guard < 100000 && ok; ++guard) {
      for (int k = 0; k < batch && ok; ++k) {
        ok = launch_b_sweep(s, SWEEP_FWD_AX, bm, dp, nm, ntiles, qref, BF_PV, -1, -1, false, nsm, occ) &&
             launch_b_sweep(s, SWEEP_BWD1, bm, dp, nm, ntiles, qref, BF_R0, BF_AP, -1, false, nsm, occ);
        launch_b_fin(s, FIN_ALPHA, bm, nm, true);
        launch_b_axpyf(s, bm, dp, nm, nslab);
        ok = ok && launch_b_sweep(s, SWEEP_FWD_AX, bm, dp, nm, ntiles, qref, BF_RR, -1, -1, false, nsm, occ) &&
             launch_b_sweep(s, SWEEP_BWD5, bm, dp, nm, ntiles, qref, BF_R0, BF_AE, BF_RR, true, nsm, occ);
        launch_b_fin5(s, bm, nm);
        launch_b_upd3f(s, bm, dp, nm, nslab);
        launch_b_commit(s, bm, nm);
      }
      if (!ok || !gather()) { ok = false; break; }
      bool all = true;
      for (int j = 0; j < nm; ++j) {
        if (!b->h_m[j].active) continue;
        if (G(j, 1) != 0.0) {  // a bounded wait ran out: this member's step fails
          g_last_error = "a bulk-copy wait of the MILU sweep ran out of time";
          rc[j] = CADMAS_ETIMEOUT;
        }
        if (G(j, 0) == 0.0) all = false;
      }
      if (all) break;
      batch = 4;
    }
    if (!ok) { error = true; break; }
    for (int j = 0; j < nm; ++j) {
      BatchMember &M = b->h_m[j];
      if (!M.active) continue;
      if (rc[j]) { M.active = 0; continue; }
      const int it = (int)G(j, 2);
      if (it < 0 || it > M.icgmax) { fallback[j] = 1; M.active = 0; continue; }  // FP64 takes over
      total[j] += it;
    }
    launch_b_add_f(s, bm, dp, nm, nslab);  // XW += |r| D where the inner solve ended in ICGMAX
  }
  if (error) { set_cuda_error("batched solve", cudaGetLastError()); fail(CADMAS_ECUDA); return; }
  for (int j = 0; j < nm; ++j)
    if (b->h_m[j].active && !rc[j]) { fallback[j] = 1; b->h_m[j].active = 0; }  // not converged in 40 passes
  // X0 = XW of the converged members (k_x0 needs ITER >= 0: the state cleared)
  for (int j = 0; j < nm; ++j) b->h_m[j].active = (conv[j] && !rc[j]) ? 1 : 0;
  if (!upload()) { fail(CADMAS_ECUDA); return; }
  launch_b_clear(s, bm, nm);
  launch_b_x0(s, bm, dp, nm, nslab);
  if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(s) != cudaSuccess) { fail(CADMAS_ECUDA); return; }
  for (int j = 0; j < nm; ++j) {
    if (rc[j]) continue;
    cadmas_handle *h = hs[j];
    if (fallback[j]) {  // the FP64 solver alone, from the guess of this step (solve_mixed's fallback)
      h->mixed_fallback++;
      h->warm_now = b->h_m[j].warm;
      rc[j] = solve(h, poisson_sys(h), h->wk[8], h->indc, iter[j], bn[j], xn[j]);
      h->warm_now = 0;
      if (cudaStreamSynchronize(h->s) != cudaSuccess) rc[j] = CADMAS_ECUDA;
      continue;
    }
    iter[j] = total[j];
    bn[j] = std::sqrt(b2[j]);
    xn[j] = std::sqrt(r2[j]);
  }
}

int cadmas_batch_create(cadmas_handle **hs, int n, cadmas_batch **out) {
  if (!hs || !out || n < 1) return CADMAS_EINVAL;
  *out = nullptr;
  long long ntiles = 0;
  for (int i = 0; i < n; ++i) {
    cadmas_handle *h = hs[i];
    if (!h) return CADMAS_EINVAL;
    if (h->P.solver != 1 || h->P.dot_passes != 0) {
      g_last_error = "a batch takes handles of the mixed solver (solver 1, dot_passes 0)";
      return CADMAS_EINVAL;
    }
    if (h->device != hs[0]->device || h->q.split != 1 || h->q.TI != hs[0]->q.TI || h->q.TJ != hs[0]->q.TJ ||
        h->q.TIp != hs[0]->q.TIp) {
      g_last_error = "a batch takes handles of one device with the same preconditioner block, unsplit";
      return CADMAS_EINVAL;
    }
    for (int j = 0; j < i; ++j)
      if (hs[j] == h) { g_last_error = "a handle twice in a batch"; return CADMAS_EINVAL; }
    ntiles += h->q.nb;
  }
  cadmas_batch *b = new cadmas_batch();
  b->h.assign(hs, hs + n);
  b->device = hs[0]->device;
  b->nsm = hs[0]->q.nsm;
  b->occ = hs[0]->q.occ;
  if (!b_sweeps_supported(hs[0]->q, b->nsm, b->occ, ntiles)) {
    delete b;
    g_last_error = "preconditioner block too large for the batched FP32 sweeps";
    return CADMAS_EUNSUPPORTED;
  }
  int rc = CADMAS_OK;
  if (cudaStreamCreateWithFlags(&b->s, cudaStreamNonBlocking) != cudaSuccess) rc = CADMAS_ECUDA;
  if (!rc && cudaMalloc(&b->d_m, (size_t)n * sizeof(BatchMember)) != cudaSuccess) rc = CADMAS_ENOMEM;
  if (!rc && cudaMallocHost(&b->h_m, (size_t)n * sizeof(BatchMember)) != cudaSuccess) rc = CADMAS_ENOMEM;
  if (!rc && cudaMalloc(&b->d_pre, (size_t)BR_N * (n + 1) * sizeof(int)) != cudaSuccess) rc = CADMAS_ENOMEM;
  if (!rc && cudaMalloc(&b->d_g, (size_t)n * BATCH_GATHER * sizeof(double)) != cudaSuccess) rc = CADMAS_ENOMEM;
  if (!rc && cudaMallocHost(&b->h_g, (size_t)n * BATCH_GATHER * sizeof(double)) != cudaSuccess) rc = CADMAS_ENOMEM;
  if (!rc && cudaEventCreateWithFlags(&b->ev, cudaEventDisableTiming) != cudaSuccess) rc = CADMAS_ECUDA;
  b->ev_m.assign(n, nullptr);
  for (int i = 0; i < n && !rc; ++i)
    if (cudaEventCreateWithFlags(&b->ev_m[i], cudaEventDisableTiming) != cudaSuccess) rc = CADMAS_ECUDA;
  if (rc) { cadmas_batch_destroy(b); return rc; }
  *out = b;
  return CADMAS_OK;
}

int cadmas_batch_destroy(cadmas_batch *b) {
  if (!b) return CADMAS_OK;
  if (b->s) cudaStreamSynchronize(b->s);
  if (b->d_m) cudaFree(b->d_m);
  if (b->h_m) cudaFreeHost(b->h_m);
  if (b->d_pre) cudaFree(b->d_pre);
  if (b->d_g) cudaFree(b->d_g);
  if (b->h_g) cudaFreeHost(b->h_g);
  if (b->ev) cudaEventDestroy(b->ev);
  for (cudaEvent_t e : b->ev_m) if (e) cudaEventDestroy(e);
  if (b->s) cudaStreamDestroy(b->s);
  delete b;
  return CADMAS_OK;
}

int cadmas_batch_step(cadmas_batch *b, const double *dt, int *status) {
  if (!b || !dt || !status) return CADMAS_EINVAL;
  const int n = (int)b->h.size();
  std::vector<int> rc1(n, CADMAS_OK);
  auto par = [&](auto fn) {  // fn(i) on one host thread per member
    std::vector<std::thread> pool;
    pool.reserve((size_t)n);
    for (int i = 0; i < n; ++i)
      pool.emplace_back([&, i]() { cudaSetDevice(b->device); fn(i); });
    for (std::thread &t : pool) t.join();
  };
  // V1CAL up to the pressure system (vf_a1main.f:1029-1058)
  par([&](int i) {
    cadmas_handle *h = b->h[i];
    if (!h->have_static) { rc1[i] = CADMAS_ENOSTATIC; return; }
    if (!(dt[i] > 0.0)) { rc1[i] = CADMAS_EINVAL; return; }
    h->dtnow = dt[i];
    h->nnow = h->nnow + 1;
    h->tnow = h->tnow + h->dtnow;
    rc1[i] = v1cal_pre(h);
    if (!rc1[i] && cudaEventRecord(b->ev_m[i], h->s) != cudaSuccess) rc1[i] = CADMAS_ECUDA;
  });
  cudaSetDevice(b->device);
  std::vector<int> idx;
  for (int i = 0; i < n; ++i)
    if (!rc1[i]) {
      idx.push_back(i);
      cudaStreamWaitEvent(b->s, b->ev_m[i], 0);
    }
  // the pressure solves together
  std::vector<int> iter, rc2;
  std::vector<double> bn, xn;
  solve_mixed_batch(b, idx, iter, bn, xn, rc2);
  cudaEventRecord(b->ev, b->s);
  std::vector<int> slot(n, -1);
  for (int j = 0; j < (int)idx.size(); ++j) slot[idx[j]] = j;
  // the rest of V1CAL and F1CAL (vf_a1main.f:1058-1115)
  par([&](int i) {
    cadmas_handle *h = b->h[i];
    int rc = rc1[i];
    if (!rc) {
      const int j = slot[i];
      cudaStreamWaitEvent(h->s, b->ev, 0);
      rc = v1cal_post(h, rc2[j], iter[j], bn[j], xn[j]);
      if (rc == CADMAS_OK) {
        int bits;
        rc = read_err(h, bits);
        if (rc == CADMAS_OK) rc = map_err(bits);
      }
      if (rc == CADMAS_OK) rc = do_f1cal(h);
    }
    h->stats.last_status = rc;
    status[i] = rc;
  });
  for (int i = 0; i < n; ++i)
    if (status[i]) return status[i];
  return CADMAS_OK;
}

// VF_CDTCAL (vf_cdtcal.f:46-147): the time step for the next step from
// the present state; the caller's DTINIT, DTMIN, DTMAX and DTSAFE.
int cadmas_cdtcal(cadmas_handle *h, double dtinit, double dtmin, double dtmax, double dtsafe, double *dt) {
  if (!h || !dt || !(dtsafe > 0.0)) return CADMAS_EINVAL;
  if (!h->have_static) return CADMAS_ENOSTATIC;
  refresh_fld(h);
  const double w = (h->nnow == 0) ? dtinit : h->dtnow;
  launch_cdtcal(h->s, h->g, h->f, h->rb0, dtmax / dtsafe, dtsafe, w, dtmin, h->dres + 8);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(h->h_res + 8, h->dres + 8, sizeof(double), cudaMemcpyDeviceToHost, h->s));
  CK(cudaStreamSynchronize(h->s));
  *dt = h->h_res[8];
  return CADMAS_OK;
}

int cadmas_divnorm(cadmas_handle *h, double *val) {
  if (!h || !val) return CADMAS_EINVAL;
  refresh_fld(h);
  launch_cdiv(h->s, h->g, h->f, h->rb0);
  launch_fin(h->s, FIN_STORE, h->rb0, h->rb0, nrows(h), h->st, h->dres + 4, 0, 0, 0, 0);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(h->h_res, h->dres, 6 * sizeof(double), cudaMemcpyDeviceToHost, h->s));
  CK(cudaStreamSynchronize(h->s));
  *val = std::sqrt(h->h_res[4]);
  h->stats.divnorm = *val;
  return CADMAS_OK;
}

int cadmas_get_stats(cadmas_handle *h, cadmas_stats *st) {
  if (!h || !st) return CADMAS_EINVAL;
  h->stats.fallbacks = (int)h->mixed_fallback;
  *st = h->stats;
  return CADMAS_OK;
}

int cadmas_test_stall_sweeps(cadmas_handle *h, int from_step) {
  if (!h) return CADMAS_EINVAL;
  const int v = from_step >= 0 ? from_step : (1 << 30);
  CK(cudaMemcpyAsync(&h->st->stall_from, &v, sizeof(int), cudaMemcpyHostToDevice, h->s));
  CK(cudaStreamSynchronize(h->s));
  return CADMAS_OK;
}

int cadmas_get_stream(cadmas_handle *h, void **stream) {
  if (!h || !stream) return CADMAS_EINVAL;
  *stream = (void *)h->s;
  return CADMAS_OK;
}

long long cadmas_kernel_launches(void) { return g_kernel_launches.load(); }

int cadmas_stage_timers(cadmas_handle *h, int enable, double *ms, long long *count, int n) {
  if (!h || n < 0 || n > CADMAS_NSTAGES) return CADMAS_EINVAL;
  CK(cudaStreamSynchronize(h->s));
  h->tm.resolve();
  for (int i = 0; i < n; ++i) {
    if (ms) ms[i] = h->tm.ms[i];
    if (count) count[i] = h->tm.cnt[i];
  }
  if (enable >= 0) {
    h->tm.clear();
    h->tm.on = (enable != 0);
  }
  return CADMAS_OK;
}

int cadmas_sync(cadmas_handle *h) {
  if (!h) return CADMAS_EINVAL;
  CK(cudaStreamSynchronize(h->s));
  return CADMAS_OK;
}

int vf_step_gpu_(cadmas_handle **hp, const double *dtnow, double *uu, double *vv, double *ww,
                 double *pp, double *ff, int *nf, int *indc, double *bcu, double *bcv, double *bcw,
                 double *bcp, double *bcf, double *tnow, int *nnow) {
  if (!hp || !*hp || !dtnow || !tnow || !nnow) return CADMAS_EINVAL;
  cadmas_handle *h = *hp;
  cadmas_state s{uu, vv, ww, pp, ff, nf, indc, bcu, bcv, bcw, bcp, bcf, nullptr, *tnow, *nnow};
  int rc = cadmas_set_state(h, &s);
  if (rc) return rc;
  rc = cadmas_step(h, *dtnow);
  int rc2 = cadmas_get_state(h, &s);
  *tnow = s.tnow;
  *nnow = s.nnow;
  return rc ? rc : rc2;
}

// One of V1CAL/F1CAL through host arrays: state in, call, state out.
static int fortran_call(cadmas_handle **hp, const double *tnow, const double *dtnow, const int *nnow,
                        double *uu, double *vv, double *ww, double *pp, double *ff, int *nf, int *indc,
                        double *bcu, double *bcv, double *bcw, double *bcp, double *bcf,
                        int (*call)(cadmas_handle *)) {
  if (!hp || !*hp || !tnow || !dtnow || !nnow) return CADMAS_EINVAL;
  if (!(*dtnow > 0.0)) return CADMAS_EINVAL;
  cadmas_handle *h = *hp;
  cadmas_state s{uu, vv, ww, pp, ff, nf, indc, bcu, bcv, bcw, bcp, bcf, nullptr, *tnow, *nnow};
  int rc = cadmas_set_state(h, &s);
  if (rc) return rc;
  rc = cadmas_set_time(h, *tnow, *dtnow, *nnow);
  if (rc) return rc;
  rc = call(h);
  const int rc2 = cadmas_get_state(h, &s);
  return rc ? rc : rc2;
}

int vf_v1cal_gpu_(cadmas_handle **h, const double *tnow, const double *dtnow, const int *nnow, double *uu,
                  double *vv, double *ww, double *pp, double *ff, int *nf, int *indc, double *bcu, double *bcv,
                  double *bcw, double *bcp, double *bcf) {
  return fortran_call(h, tnow, dtnow, nnow, uu, vv, ww, pp, ff, nf, indc, bcu, bcv, bcw, bcp, bcf, cadmas_v1cal);
}

int vf_f1cal_gpu_(cadmas_handle **h, const double *tnow, const double *dtnow, const int *nnow, double *uu,
                  double *vv, double *ww, double *pp, double *ff, int *nf, int *indc, double *bcu, double *bcv,
                  double *bcw, double *bcp, double *bcf) {
  return fortran_call(h, tnow, dtnow, nnow, uu, vv, ww, pp, ff, nf, indc, bcu, bcv, bcw, bcp, bcf, cadmas_f1cal);
}

int cadmas_m1bcgs_dev(cadmas_handle *h, const double *ad, const double *ali, const double *alj,
                      const double *alk, const double *aui, const double *auj, const double *auk,
                      const double *bb, double *x0, const int *indc, int *iter, double *bnorm,
                      double *xnorm) {
  if (!h || !ad || !ali || !alj || !alk || !aui || !auj || !auk || !bb || !x0 || !indc || !iter ||
      !bnorm || !xnorm)
    return CADMAS_EINVAL;
  SysPtr a{const_cast<double *>(ad), const_cast<double *>(ali), const_cast<double *>(alj),
           const_cast<double *>(alk), const_cast<double *>(aui), const_cast<double *>(auj),
           const_cast<double *>(auk), const_cast<double *>(bb)};
  int it;
  double bn, xn;
  int rc = solve(h, a, x0, indc, it, bn, xn);
  if (rc) return rc;
  CK(cudaStreamSynchronize(h->s));
  *iter = it; *bnorm = bn; *xnorm = xn;
  return CADMAS_OK;
}

}  // extern "C"
