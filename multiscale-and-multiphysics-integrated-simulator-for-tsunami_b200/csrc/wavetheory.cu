// wavetheory.cu -- steady periodic water waves by the Fourier
// (stream-function) method, for the wave maker's FUNC STREAM N
// (IWVTYP >= 1; vf_cwmak0.f:43-56, vf_cwmak1.f, vf_cwmak2.f).
//
// The reference solves the same steady-wave problem with a third-party
// least-squares routine (vf_wsfmb2.f, "stream function method B" with the
// mean mass transport as the current definition).  This file solves it
// with Fenton's collocation form of the method (J. D. Fenton, "The
// numerical solution of steady water wave problems", Computers &
// Geosciences 14(3), 1988): in the frame moving with the wave,
//   psi(X, z) = -UB (z + d) + sum_{j=1..N} B_j sinh(j k (z+d)) / cosh(j k d) cos(j k X),
// which satisfies the field equation and the bed condition; at the N+1
// points k X_m = m pi / N of half a wave the surface eta_m must satisfy
//   psi(X_m, eta_m) = -Q                       (kinematic)
//   (U_m^2 + W_m^2) / 2 + g eta_m = R          (dynamic, Bernoulli)
// together with a zero mean level (trapezoidal rule over the N+1
// points), the wave height eta_0 - eta_N = H, and the current definition
// of the reference: no mean mass transport in the fixed frame, c = Q / d,
// with c = 2 pi / (k T).  2N+5 equations in k, UB, Q, R, B_1..B_N,
// eta_0..eta_N, solved by Newton's method (central-difference Jacobian,
// Gaussian elimination with partial pivoting) in units of d and sqrt(g d),
// the height raised to H in steps from the linear wave.
//
// Everything here runs on the host, once per wave maker; the per-step
// evaluation is wavetheory.cuh.
#include <cmath>
#include <cstring>
#include <vector>

#include "wavetheory.cuh"
#include "../../include/cadmas_gpu.h"

namespace cadmas {
double stream_eta(const cadmas_stream_wave &s, double wvt);
double stream_zero_phase(const cadmas_stream_wave &s);
}  // namespace cadmas

namespace {

const double PI = 3.141592653589793;

// residuals of the 2N+5 equations at x (nondimensional)
void stream_residual(int N, double Tn, double Hn, const double *x, double *f) {
  const double K = x[0], U = x[1], Q = x[2], R = x[3];
  const double *B = x + 4, *E = x + 4 + N;
  for (int m = 0; m <= N; ++m) {
    const double th = PI * m / N;
    double psi = -U * (E[m] + 1.0) + Q, um = -U, wm = 0.0;
    for (int j = 1; j <= N; ++j) {
      const double a = j * K * (E[m] + 1.0), cd = std::cosh(j * K);
      const double s = std::sinh(a) / cd, ch = std::cosh(a) / cd;
      const double cs = std::cos(j * th), sn = std::sin(j * th);
      psi += B[j - 1] * s * cs;
      um += j * K * B[j - 1] * ch * cs;
      wm += j * K * B[j - 1] * s * sn;
    }
    f[m] = psi;
    f[N + 1 + m] = 0.5 * (um * um + wm * wm) + E[m] - R;
  }
  double mean = 0.5 * (E[0] + E[N]);
  for (int m = 1; m < N; ++m) mean += E[m];
  f[2 * N + 2] = mean / N;
  f[2 * N + 3] = E[0] - E[N] - Hn;
  f[2 * N + 4] = 2.0 * PI / (K * Tn) - Q;
}

// A x = b in place (partial pivoting); false when singular
bool gauss(int n, std::vector<double> &A, std::vector<double> &b) {
  for (int c = 0; c < n; ++c) {
    int p = c;
    for (int r = c + 1; r < n; ++r)
      if (std::fabs(A[r * n + c]) > std::fabs(A[p * n + c])) p = r;
    if (!(std::fabs(A[p * n + c]) > 0.0)) return false;
    if (p != c) {
      for (int k = 0; k < n; ++k) std::swap(A[c * n + k], A[p * n + k]);
      std::swap(b[c], b[p]);
    }
    for (int r = c + 1; r < n; ++r) {
      const double f = A[r * n + c] / A[c * n + c];
      if (f == 0.0) continue;
      for (int k = c; k < n; ++k) A[r * n + k] -= f * A[c * n + k];
      b[r] -= f * b[c];
    }
  }
  for (int c = n - 1; c >= 0; --c) {
    double s = b[c];
    for (int k = c + 1; k < n; ++k) s -= A[c * n + k] * b[k];
    b[c] = s / A[c * n + c];
  }
  return true;
}

// linear dispersion: w^2 d / g = K tanh(K), K = k d
double linear_kd(double w2) {
  double K = w2 > 1.0 ? w2 : std::sqrt(w2);
  for (int i = 0; i < 100; ++i) {
    const double th = std::tanh(K);
    const double f = K * th - w2, df = th + K * (1.0 - th * th);
    const double dK = f / df;
    K -= dK;
    if (std::fabs(dK) < 1e-15 * K) break;
  }
  return K;
}

}  // namespace

extern "C" int cadmas_stream_solve(int order, double depth, double period, double height, double grav,
                                   cadmas_stream_wave *out) {
  if (!out || order < 1 || order > CADMAS_STREAM_NMAX || !(depth > 0.0) || !(period > 0.0) || !(height > 0.0) ||
      !(grav > 0.0))
    return CADMAS_EINVAL;
  const int N = order, n = 2 * N + 5;
  const double sgd = std::sqrt(grav * depth);
  const double Tn = period * std::sqrt(grav / depth), Hn = height / depth;
  const double w = 2.0 * PI / Tn;  // nondimensional angular frequency
  const double K0 = linear_kd(w * w);
  // the reference's limits on the steepness (vf_wsfmb2.f:64-65)
  const double L0 = grav * period * period / (2.0 * PI);
  if (height / L0 > 0.3 || height / depth > 1.5) return CADMAS_EINVAL;
  // height steps from the linear wave
  const double Llin = 2.0 * PI * depth / K0;
  const int steps = std::max(2, (int)std::ceil(40.0 * height / Llin));
  std::vector<double> x(n, 0.0), f(n), f1(n), f2(n), J((size_t)n * n), dx(n);
  int iters = 0;
  for (int st = 1; st <= steps; ++st) {
    const double Hs = Hn * st / steps;
    if (st == 1) {  // the linear wave of height Hs
      const double U = std::sqrt(std::tanh(K0) / K0);
      x[0] = K0; x[1] = U; x[2] = 2.0 * PI / (K0 * Tn); x[3] = 0.5 * U * U;
      x[4] = U * 0.5 * Hs / std::tanh(K0);
      for (int m = 0; m <= N; ++m) x[4 + N + m] = 0.5 * Hs * std::cos(PI * m / N);
    } else {  // the previous height's wave, its B and eta scaled up
      const double s = (double)st / (st - 1);
      for (int j = 0; j < N; ++j) x[4 + j] *= s;
      for (int m = 0; m <= N; ++m) x[4 + N + m] *= s;
    }
    bool conv = false;
    for (int it = 0; it < 100 && !conv; ++it) {
      stream_residual(N, Tn, Hs, x.data(), f.data());
      double fm = 0.0;
      for (int r = 0; r < n; ++r) fm = std::max(fm, std::fabs(f[r]));
      if (fm < 1e-14) { conv = true; break; }  // every equation holds to 1e-14 (units of d, sqrt(g d))
      for (int c = 0; c < n; ++c) {
        const double h = 1e-7 * std::max(std::fabs(x[c]), 1e-3);
        const double x0 = x[c];
        x[c] = x0 + h; stream_residual(N, Tn, Hs, x.data(), f1.data());
        x[c] = x0 - h; stream_residual(N, Tn, Hs, x.data(), f2.data());
        x[c] = x0;
        for (int r = 0; r < n; ++r) J[(size_t)r * n + c] = (f1[r] - f2[r]) / (2.0 * h);
      }
      for (int r = 0; r < n; ++r) dx[r] = -f[r];
      if (!gauss(n, J, dx)) return CADMAS_EWAVE;
      double mx = 0.0;
      for (int r = 0; r < n; ++r) {
        x[r] += dx[r];
        mx = std::max(mx, std::fabs(dx[r]));
      }
      ++iters;
      if (!(mx == mx) || !(x[0] > 0.0)) return CADMAS_EWAVE;
      if (mx < 1e-15) conv = true;  // no further change at working precision
    }
    if (!conv) return CADMAS_EWAVE;
  }
  std::memset(out, 0, sizeof(*out));
  out->order = N;
  out->iterations = iters;
  out->depth = depth; out->period = period; out->height = height; out->grav = grav;
  out->k = x[0] / depth;
  out->length = 2.0 * PI / out->k;
  out->celerity = out->length / period;
  out->ubar = x[1] * sgd;
  out->q = x[2] * depth * sgd;
  out->r = x[3] * grav * depth;
  for (int j = 0; j < N; ++j) out->b[j] = x[4 + j] * depth * sgd;
  out->phase0 = cadmas::stream_zero_phase(*out);
  return CADMAS_OK;
}

namespace cadmas {

// The series coefficients at phase `wvt` (theta = 2 pi wvt).
void stream_phase(const cadmas_stream_wave &s, double wvt, WavePhase &ph) {
  const double th = 2.0 * PI * wvt;
  ph.n = s.order; ph.k = s.k; ph.d = s.depth; ph.ub = s.celerity - s.ubar;
  for (int j = 1; j <= s.order; ++j) {
    double ch, sh;
    wt_coshsinh((double)j * s.k * s.depth, ch, sh);
    const double a = (double)j * s.k * s.b[j - 1] / ch;
    ph.cj[j - 1] = a * std::cos((double)j * th);
    ph.sj[j - 1] = a * std::sin((double)j * th);
  }
}

// The surface eta at phase `wvt`: psi(theta, eta) + Q = 0 by Newton's
// method from eta = 0 (VF_SFMB1 starts there too), rounded to single
// precision.
double stream_eta(const cadmas_stream_wave &s, double wvt) {
  const double th = 2.0 * PI * wvt, d = s.depth, k = s.k;
  double e = 0.0;
  for (int it = 0; it < 60; ++it) {
    double f = -s.ubar * (e + d) + s.q, df = -s.ubar;
    for (int j = 1; j <= s.order; ++j) {
      double chd, shd, ch, sh;
      wt_coshsinh((double)j * k * d, chd, shd);
      wt_coshsinh((double)j * k * (e + d), ch, sh);
      const double cs = std::cos((double)j * th);
      f = f + s.b[j - 1] * sh / chd * cs;
      df = df + (double)j * k * s.b[j - 1] * ch / chd * cs;
    }
    const double de = f / df;
    e = e - de;
    if (std::fabs(de) < 1e-14 * d) break;
  }
  return (double)(float)e;
}

// VF_CWZERO (vf_cwzero.f): the phase in [0.5, 1] where the level
// crosses zero, in single precision: 100 steps down from phase 1 to
// bracket it, then at most 20 bisections, |eta| < 1e-6 accepted as zero;
// 0.5 when no crossing is bracketed.
double stream_zero_phase(const cadmas_stream_wave &s) {
  const int NB = 100, NI = 20;
  const float EPS = 1.0e-6f;
  double WVZERO = 0.5;
  float T1 = 1.0f, Z1 = (float)stream_eta(s, (double)T1), T2 = T1, Z2 = Z1;
  if (std::fabs(Z1) < EPS) return (double)T1;
  for (int L = 1; L <= NB; ++L) {
    T2 = 1.0f - 0.5f * (float)L / (float)NB;
    Z2 = (float)stream_eta(s, (double)T2);
    if (Z1 * Z2 <= 0.0f) break;
    T1 = T2;
    Z1 = Z2;
  }
  if (std::fabs(Z2) < EPS) return (double)T2;
  if (T1 == T2) return WVZERO;
  for (int L = 1; L <= NI; ++L) {
    const float T = (T1 + T2) * 0.5f;
    WVZERO = (double)T;
    const float Z = (float)stream_eta(s, WVZERO);
    if (std::fabs(Z) < EPS) break;
    if (Z1 * Z >= 0.0f) { T1 = T; Z1 = Z; }
    else { T2 = T; Z2 = Z; }
  }
  return WVZERO;
}

}  // namespace cadmas

extern "C" int cadmas_stream_eval(const cadmas_stream_wave *s, double phase, double z, double *eta, double *u,
                                  double *w) {
  if (!s || s->order < 1 || s->order > CADMAS_STREAM_NMAX) return CADMAS_EINVAL;
  if (eta) *eta = cadmas::stream_eta(*s, phase);
  if (u || w) {
    cadmas::WavePhase ph;
    cadmas::stream_phase(*s, phase, ph);
    double uu, ww;
    cadmas::wt_velocity(ph, z, uu, ww);
    if (u) *u = uu;
    if (w) *w = ww;
  }
  return CADMAS_OK;
}
