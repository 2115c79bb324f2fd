// wavetheory.cu -- the wave theories of the wave maker and the wave
// source (VF_CWMAK0/1/2 and VF_CWZERO: FUNC STREAM N, STOKES, CNOIDAL,
// STK-CND; vf_cwmak0.f, vf_cwmak1.f, vf_cwmak2.f, vf_cwzero.f), on the
// host: each wave is solved once, and each step its level at the phase and
// the phase's part of the velocity series are formed here; the per-face
// evaluation is wavetheory.cuh.
//
// Stream function (IWVTYP >= 1).  The reference solves the steady-wave
// problem with a third-party least-squares routine (vf_wsfmb2.f, "stream
// function method B" with the mean mass transport as the current
// definition).  This file solves it with Fenton's collocation form of the
// method (J. D. Fenton, "The numerical solution of steady water wave
// problems", Computers & Geosciences 14(3), 1988): in the frame moving
// with the wave,
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
// Stokes, fifth order (IWVTYP -2), and cnoidal, third order (IWVTYP -1).
// The reference carries the perturbation solutions of Isobe's programs
// (vf_wstk0.f, vf_wcnd0.f): the fifth-order Stokes wave in the expansion
// parameter kH/2 with the celerity of zero mean mass transport, and the
// third-order cnoidal wave in H/d (Isobe and Kraus's form) with Jacobi's
// elliptic functions.  Their coefficient polynomials are the theories
// themselves; they are written here as tables of the same numbers, the
// accumulation order of the reference kept, and evaluated in double
// precision in the reference's units (cm, s, g = 980 cm/s^2).  The
// iterations (the dispersion relation, the elliptic parameter) take the
// reference's start values, updates and stopping tests.  Jacobi's sn, cn,
// dn come from the arithmetic-geometric mean (the descending Landen
// transformation, Abramowitz and Stegun 16.4) with the modulus from the
// theta series of the smaller of the two nomes; the reference sums
// truncated theta series instead.  Results leave the routines in single
// precision, as the reference's REAL*4 routines return them.
#include <cmath>
#include <cstring>
#include <initializer_list>
#include <vector>

#include "wavetheory.cuh"
#include "../../include/cadmas_gpu.h"

namespace cadmas {
double stream_eta(const cadmas_stream_wave &s, double wvt);
double stream_zero_phase(const cadmas_stream_wave &s);
void stream_phase(const cadmas_stream_wave &s, double wvt, WavePhase &ph);
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
  std::memset(&ph, 0, sizeof(ph));
  ph.n = s.order; ph.kind = WT_SERIES; ph.clamp = 1; ph.zs = 1.0; ph.us = 1.0;
  ph.k = s.k; ph.d = s.depth; ph.ub = s.celerity - s.ubar;
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

// ------------------------------------------------ Stokes, fifth order
namespace {

// c[0] + R (c[1] + R (c[2] + ...)): the nested polynomials of the theories
double horner(double R, const double *c, int n) {
  double p = c[n - 1];
  for (int i = n - 2; i >= 0; --i) p = c[i] + p * R;
  return p;
}
#define HR(R, ...) ([&] { static const double c_[] = {__VA_ARGS__}; return horner((R), c_, (int)(sizeof(c_) / sizeof(double))); }())

// VF_HK (vf_wstk0.f): k d of the linear wave from w^2 d / g, Newton's
// method from sqrt(WW) to a relative step of 1e-6 (10 steps at most);
// WW itself in deep water (WW > 15).
double linear_hk(double WW) {
  if (WW > 15.0) return WW;
  double hk = std::sqrt(WW);
  for (int n = 1; n <= 10; ++n) {
    const double t = std::tanh(hk);
    const double d = (hk * t - WW) / (t + hk * (1.0 - t * t));
    hk = hk - d;
    if (std::fabs(d / hk) < 1.0e-6) break;
  }
  return hk;
}

// The fifth-order celerity factor C1 (c = C1 c0) at k d = dk for the
// half-height ratio hd = H / (2 d), with tanh, coth and coth^2 there.
double stokes_c1(double dk, double hd, double &th, double &ct, double &R) {
  th = std::tanh(dk);
  ct = 1.0 / th;
  R = ct * ct;
  const double f = (hd * dk) * (hd * dk);
  double c1 = HR(R, 39., 351., -2194., 2454., -117., -405.) / 1024. - HR(R, 3., -7., -3., -9.) * ct / (64. * dk);
  c1 = c1 * f + HR(R, 9., -10., 9.) / 16. - ct / (2. * dk);
  c1 = c1 * f + 1.;
  return c1;
}

// VF_STK0 with N = 5 (vf_wstk0.f): the dispersion relation
// sqrt(kd tanh kd) C1(kd) = w sqrt(d/g) by the reference's secant steps
// (a forward difference of relative size 1e-5, stop at a relative change
// below 1e-5, 20 steps), then the coefficients of the level and the
// velocities.  Lengths in cm.
int stokes_solve(double depth, double period, double height, cadmas_stokes_wave &o, double &RL) {
  const double G = 980.0, EPS = 1.0e-5;
  const double D = depth * 100.0, T = period, H = height * 100.0;
  const double SGM = 2.0 * PI / T, WW = SGM * SGM * D / G, W = std::sqrt(WW), HD = H / (2.0 * D);
  double DK = linear_hk(WW), DDDK = 0.0, th, ct, R, c1;
  auto resid = [&](double dk) {
    c1 = stokes_c1(dk, HD, th, ct, R);
    return std::sqrt(dk * th) * c1 - W;
  };
  bool conv = false;
  int it = 0;
  while (it < 20) {
    ++it;
    const double DDK = (DDDK >= 0.0) ? std::fabs(DK * EPS) : -std::fabs(DK * EPS);
    const double R2 = resid(DK + DDK);
    const double R1 = resid(DK);
    DDDK = -R1 * DDK / (R2 - R1);
    DK = DK + DDDK;
    if (!(std::fabs(DDDK / DK) >= EPS)) { conv = true; break; }
  }
  if (conv) resid(DK);   // tanh, coth, C1 at the result
  else DK = DK - DDDK;   // the last point evaluated
  if (!(DK > 0.0) || !std::isfinite(c1)) return CADMAS_EWAVE;
  const double RK = DK / D;
  RL = 2.0 * PI / RK;
  const double E = DK * HD;
  const double C0 = std::sqrt(G * th / RK);
  std::memset(&o, 0, sizeof(o));
  o.kd = DK; o.k = RK; o.eps = E; o.c0 = C0; o.c = c1 * C0; o.iterations = it;
  const double E2 = E * E, E3 = E2 * E, E4 = E3 * E, E5 = E4 * E;
  const double q1 = 1. + 5. * R, q3 = 3. + 5. * R;
  double *A = o.a, *B = o.b, B0, P0;
  // fifth order
  A[0] = E5 * HR(R, -225., 2370., 14622., -6070., 53932., -340410., -764046., 203310., 188325.) / (12288. * q1 * q3);
  A[2] = E5 * HR(R, -180., -1008., 900., -5328., 46980., -7776., -14580.) * R / (4096. * q1);
  A[4] = E5 * HR(R, 45., -150., -570., 2618., -3896., -498., 25866., 8910., 6075.) * 5. / (12288. * q1 * q3);
  B[0] = E5 * HR(R, 861., 12262., 30114., -75986., -131460., -91438., -199602., 89370., 62775.) / (4096. * q1 * q3);
  B[2] = E5 * HR(R, 173., 1413., 1665., -6591., -7569., 10935., 4131., -3645.) / (1024. * q1);
  B[4] = E5 * HR(R, 1083., 15230., 39970., -78730., -89928., 157690., -16290., -39150., 10125.) / (4096. * q1 * q3);
  // fourth order
  A[1] = E4 * HR(R, 12., -352., 792., 0., -324.) * ct / 384.;
  A[3] = E4 * HR(R, 21., 1., -262., 522., 81., 405.) * ct / (384. * q1);
  B[1] = E4 * HR(R, -103., 19., 261., 81., -162.) * ct / 192.;
  B[3] = E4 * HR(R, -197., -747., 1466., 342., -1269., 405.) * ct / (384. * q1);
  B0 = E4 * HR(R, -3., 7., 3., 9.) * ct / (64. * DK);
  P0 = E4 * ((-1. + R) * HR(R, 21., 13., -57., -9.) / 128. - 3. * ct * (-1. + R) * HR(R, 7., -2., 3.) / (64. * DK) -
             R / (8. * DK * DK));
  // third order
  A[0] = A[0] + E3 * HR(R, 1., -3., 3., -9.) * 3. / 64.;
  A[2] = A[2] + E3 * HR(R, -1., 3., -3., 9.) * 3. / 64.;
  B[0] = B[0] + E3 * HR(R, 39., -41., -3., -27.) / 64.;
  B[2] = B[2] + E3 * HR(R, 13., 17., -57., 27.) / 64.;
  // second order
  A[1] = A[1] + E2 * (-1. + 3. * R) * ct / 4.;
  B[1] = B[1] + E2 * (-1. + R) * ct * 3. / 4.;
  B0 = B0 + E2 * (-ct / (2. * DK));
  P0 = P0 + E2 * ((-1. + R) / 4. + ct / (2. * DK));
  // first order
  A[0] = A[0] + E;
  B[0] = B[0] + E;
  for (int i = 1; i <= 5; ++i) {
    A[i - 1] = A[i - 1] / RK;
    B[i - 1] = B[i - 1] * C0 * (double)i / std::sinh((double)i * DK);
  }
  o.b0 = B0 * C0;
  o.p0 = P0 * C0 * C0 / G;
  return CADMAS_OK;
}

// ------------------------------------------------ cnoidal, third order

// VF_CND0 with N = 3 (vf_wcnd0.f): the elliptic parameter from the Ursell
// number (held at 10 or more, as the reference's branch does) by the
// reference's fixed-point iteration on QQL = pi K/K' (start sqrt(3 Ur/4),
// stop at a relative change below 1e-5, 20 steps), the coefficients of
// the level and the velocities from the parameters R and O of the last
// step.  Lengths in cm.
int cnoidal_solve(double depth, double period, double height, cadmas_cnoidal_wave &o, double &RL) {
  const double G = 980.0, EPS = 1.0e-5;
  const double D = depth * 100.0, T = period, H = height * 100.0;
  const double C0 = std::sqrt(G * D);
  const double E = H / D, E2 = E * E, E3 = E2 * E;
  double UR = G * H * T * T / (D * D);
  if (UR < 10.0) UR = 10.0;
  const double UR34 = UR * 0.75;
  double QQL = std::sqrt(UR34);
  double C00 = E2 * 0.2, C01 = E2 * (-0.25), C10 = E2 * 0.825, C11 = E2 * (-0.5), C20 = E2 * 0.825;
  C00 = C00 + E * (-0.25);
  C10 = C10 + E * (-0.5);
  C00 = C00 + 1.;
  auto p4 = [](double x) { const double x2 = x * x; return x2 * x2; };
  double R = 0.0, O = 0.0, T3 = 1.0;
  int it = 0;
  while (it < 20) {
    ++it;
    const double QQ = std::exp(-QQL), Q2 = QQ * QQ, Q4 = Q2 * Q2;
    const double T2 = p4(1. + 2. * (-QQ + Q4));
    T3 = p4(1. + 2. * (QQ + Q4));
    const double T4 = p4(1. + Q2 * (1. + Q4));
    const double S = 1. + 8. * Q2 * (1. - Q2);
    R = 16. * QQ * T4 / T2;
    O = (2. / QQL + T3 - S) / T2;
    const double QQLL = QQL;
    QQL = std::sqrt(UR34 * (C00 + R * (C10 + R * C20) + O * (C01 + R * C11)) / T2);
    if (std::fabs((QQLL - QQL) / QQL) < EPS) break;
  }
  if (!(QQL > 0.0) || !std::isfinite(QQL)) return CADMAS_EWAVE;
  // monomials 1, R, O, RR, RO, OO, RRR, RRO, ROO, OOO
  const double RR = R * R, RO = R * O, OO = O * O;
  const double m[10] = {1., R, O, RR, RO, OO, RR * R, RR * O, RO * O, OO * O};
  auto sum = [&](std::initializer_list<double> c) {
    double s = 0.0;
    int i = 0;
    for (double ci : c) s = s + ci * m[i++];
    return s;
  };
  double A[4], B[3][4], P0, C;  // B[j-1][i-1] = B(j,i)
  // third order
  A[0] = E3 * sum({0., 133., -16., 399., -466., 100., 266., -466., 200.}) / 400.;
  A[1] = E3 * sum({50., -1., -60.}) / 80.;
  A[2] = E3 * sum({-151., 1., 60.}) / 80.;
  A[3] = E3 * 101. / 80.;
  B[0][0] = E3 * sum({0., -71., 47., -23., 97., -50., 153., -153., -25., 25.}) / 200.;
  B[1][0] = E3 * sum({0., 6., 0., 24., -21.}) / 8.;
  B[2][0] = E3 * sum({0., 3., 0., -3.}) / 16.;
  B[0][1] = E3 * sum({-19., -27., 10., 101., -100., 15.}) / 40.;
  B[1][1] = E3 * sum({6., 36., -21., -24., 21.}) / 4.;
  B[2][1] = E3 * sum({6., -39., 0., 6.}) / 16.;
  B[0][2] = E3 * sum({-2., 32., -15.}) / 10.;
  B[1][2] = E3 * sum({30., -120., 63.}) / 8.;
  B[2][2] = E3 * sum({-45., 45.}) / 16.;
  B[0][3] = E3 * 6. / 5.;
  B[1][3] = E3 * (-15.) / 2.;
  B[2][3] = E3 * 45. / 16.;
  P0 = E3 * sum({0., 3., -6., 9., -26., 5., 6., -26., 10., 10.}) / 20.;
  C = E3 * sum({150., 1079., -203., 2337., -2653., 350., 1558., -2653., 700., 175.}) / 2800.;
  // second order
  A[0] = A[0] + E2 * sum({0., -2., 1., -2., 2.}) / 4.;
  A[1] = A[1] + E2 * (-0.75);
  A[2] = A[2] + E2 * (0.75);
  B[0][0] = B[0][0] + E2 * sum({0., 1., -1., -2., 0., 2.}) / 4.;
  B[1][0] = B[1][0] + E2 * (-0.75 * R);
  B[0][1] = B[0][1] + E2 * sum({1., -6., 2.}) / 4.;
  B[1][1] = B[1][1] + E2 * sum({-3., 3.}) / 2.;
  B[0][2] = B[0][2] + E2 * (-1.);
  B[1][2] = B[1][2] + E2 * 2.25;
  P0 = P0 + E2 * sum({0., -1., 2., -1., 4., -3.}) / 2.;
  C = C + E2 * sum({-6., -16., 5., -16., 10., 15.}) / 40.;
  // first order
  A[0] = A[0] + E * (R - O);
  A[1] = A[1] + E;
  B[0][0] = B[0][0] + E * (R - O);
  B[0][1] = B[0][1] + E;
  C = C + E * (1. + 2. * R - 3. * O) / 2. + 1.;
  const double CC = C * C0;
  RL = T * CC;
  const double DL = D / RL;
  const double S = 2. * std::sqrt(T3) * QQL * DL;
  std::memset(&o, 0, sizeof(o));
  for (int i = 1; i <= 4; ++i) {
    o.a[i - 1] = A[i - 1] * D;
    for (int j = 1; j <= 3; ++j) {
      const double b = B[j - 1][i - 1] * C0;
      o.b[(i - 1) * 3 + (j - 1)] = b;
      o.bb[(i - 1) * 3 + (j - 1)] = b * S * (double)(i - 1) / (double)(2 * j - 1);
    }
  }
  o.p0 = P0 * C0 * C0 / G;
  o.ql = PI * PI / QQL;
  o.s = S;
  o.d = D;
  o.c0 = C0;
  o.c = CC;
  o.iterations = it;
  if (!std::isfinite(RL) || !(RL > 0.0)) return CADMAS_EWAVE;
  return CADMAS_OK;
}

}  // namespace

namespace cadmas {

// Jacobi's elliptic functions cn, sn, dn at u = 4 K x (x in periods of
// cn) for the modulus whose quarter-period ratio is ql = pi K'/K.  The
// moduli k, k' from the theta series of the nome exp(-ql) when ql >= pi,
// else of the complementary nome exp(-pi^2/ql) (both below exp(-pi), six
// terms), x reduced to [-1/4, 1/4] (cn and sn change sign over half a
// period), then the arithmetic-geometric mean of 1 and k' and the
// descending recursion phi_{n-1} = (phi_n + asin(c_n/a_n sin phi_n)) / 2
// from phi_N = 2^N a_N u = 2^N 2 pi x (Abramowitz and Stegun 16.4.2-3).
void jacobi_cn(double ql, double x, double &cn, double &sn, double &dn) {
  auto thetas = [](double q, double &t2, double &t3, double &t4) {
    double s2 = 0.0, s3 = 0.0, s4 = 0.0;
    for (int n = 6; n >= 1; --n) {
      s3 = s3 + std::pow(q, (double)(n * n));
      s4 = s4 + ((n & 1) ? -1.0 : 1.0) * std::pow(q, (double)(n * n));
    }
    for (int n = 6; n >= 0; --n) s2 = s2 + std::pow(q, (double)(n * (n + 1)));
    t2 = 2.0 * std::pow(q, 0.25) * s2;
    t3 = 1.0 + 2.0 * s3;
    t4 = 1.0 + 2.0 * s4;
  };
  double k, kp, t2, t3, t4;
  if (ql >= PI) {
    thetas(std::exp(-ql), t2, t3, t4);
    k = (t2 / t3) * (t2 / t3);
    kp = (t4 / t3) * (t4 / t3);
  } else {
    thetas(std::exp(-PI * PI / ql), t2, t3, t4);
    kp = (t2 / t3) * (t2 / t3);
    k = (t4 / t3) * (t4 / t3);
  }
  double x1 = x - std::floor(x + 0.5), sig = 1.0;
  if (x1 > 0.25) { x1 = x1 - 0.5; sig = -1.0; }
  else if (x1 < -0.25) { x1 = x1 + 0.5; sig = -1.0; }
  double a[48], c[48], b = kp;
  a[0] = 1.0; c[0] = k;
  int n = 0;
  while (n < 46 && std::fabs(c[n]) > 1e-15 * a[n]) {
    a[n + 1] = 0.5 * (a[n] + b);
    c[n + 1] = 0.5 * (a[n] - b);
    b = std::sqrt(a[n] * b);
    ++n;
  }
  double phi = std::ldexp(2.0 * PI * x1, n), phi1 = phi;
  for (int m = n; m >= 1; --m) {
    phi1 = phi;
    phi = 0.5 * (phi + std::asin(c[m] / a[m] * std::sin(phi)));
  }
  sn = sig * std::sin(phi);
  cn = sig * std::cos(phi);
  dn = (n == 0) ? 1.0 : std::cos(phi) / std::cos(phi1 - phi);
}

// VF_CWMAK1 (vf_cwmak1.f): the level at phase `wvt`, in metres, from the
// single-precision result of the theory's routine.
double theory_eta(const cadmas_wave_theory &t, double wvt) {
  if (t.type >= 1) return stream_eta(t.stream, wvt);
  double zs = 0.0;
  if (t.type == CADMAS_WAVE_STOKES) {  // VF_STK1
    const double th = 2.0 * PI * wvt;
    for (int i = 1; i <= 5; ++i) zs = zs + t.stokes.a[i - 1] * std::cos((double)i * th);
  } else {  // VF_CND1
    double cn, sn, dn;
    jacobi_cn(t.cnoidal.ql, wvt / 2.0, cn, sn, dn);
    const double cn2 = cn * cn;
    for (int L = 4; L >= 1; --L) zs = zs * cn2 + t.cnoidal.a[L - 1];
  }
  return (double)(float)zs * 0.01;
}

// The phase's part of VF_CWMAK2 (vf_cwmak2.f) for wt_velocity.
void theory_phase(const cadmas_wave_theory &t, double wvt, WavePhase &ph) {
  if (t.type >= 1) { stream_phase(t.stream, wvt, ph); return; }
  std::memset(&ph, 0, sizeof(ph));
  ph.zs = 100.0;
  ph.us = 0.01;
  if (t.type == CADMAS_WAVE_STOKES) {  // VF_STK2
    const double th = 2.0 * PI * wvt;
    ph.kind = WT_SERIES; ph.n = 5; ph.clamp = 0;
    ph.k = t.stokes.k; ph.d = t.depth * 100.0; ph.ub = t.stokes.b0;
    for (int i = 1; i <= 5; ++i) {
      ph.cj[i - 1] = t.stokes.b[i - 1] * std::cos((double)i * th);
      ph.sj[i - 1] = t.stokes.b[i - 1] * std::sin((double)i * th);
    }
  } else {  // VF_CND2
    double cn, sn, dn;
    jacobi_cn(t.cnoidal.ql, wvt / 2.0, cn, sn, dn);
    ph.kind = WT_CNOIDAL; ph.n = 12;
    ph.d = t.cnoidal.d;
    ph.cn2 = cn * cn;
    ph.csd = cn * sn * dn;
    for (int i = 0; i < 12; ++i) { ph.cj[i] = t.cnoidal.b[i]; ph.sj[i] = t.cnoidal.bb[i]; }
  }
}

// VF_CWZERO (vf_cwzero.f) for any theory: |eta| below 1e-6 m (stream
// function) or 1e-8 m (Stokes, cnoidal) counts as zero.
double theory_zero_phase(const cadmas_wave_theory &t) {
  const int NB = 100, NI = 20;
  const float EPS = (t.type >= 1) ? 1.0e-6f : 1.0e-8f;
  double WVZERO = 0.5;
  float T1 = 1.0f, Z1 = (float)theory_eta(t, (double)T1), T2 = T1, Z2 = Z1;
  if (std::fabs(Z1) < EPS) return (double)T1;
  for (int L = 1; L <= NB; ++L) {
    T2 = 1.0f - 0.5f * (float)L / (float)NB;
    Z2 = (float)theory_eta(t, (double)T2);
    if (Z1 * Z2 <= 0.0f) break;
    T1 = T2;
    Z1 = Z2;
  }
  if (std::fabs(Z2) < EPS) return (double)T2;
  if (T1 == T2) return WVZERO;
  for (int L = 1; L <= NI; ++L) {
    const float Tm = (T1 + T2) * 0.5f;
    WVZERO = (double)Tm;
    const float Z = (float)theory_eta(t, WVZERO);
    if (std::fabs(Z) < EPS) break;
    if (Z1 * Z >= 0.0f) { T1 = Tm; Z1 = Z; }
    else { T2 = Tm; Z2 = Z; }
  }
  return WVZERO;
}

// A theory of type `order` from a solved stream-function wave.
void theory_from_stream(const cadmas_stream_wave &s, cadmas_wave_theory &t) {
  std::memset(&t, 0, sizeof(t));
  t.type = s.order;
  t.depth = s.depth; t.period = s.period; t.height = s.height;
  t.length = (double)(float)s.length;
  t.stream = s;
  t.phase0 = s.phase0;
}

}  // namespace cadmas

extern "C" int cadmas_wave_solve(int type, double depth, double period, double height, double grz0,
                                 cadmas_wave_theory *out) {
  if (!out || type > CADMAS_STREAM_NMAX || type < CADMAS_WAVE_STOKES || !(depth > 0.0) || !(period > 0.0) ||
      !(height > 0.0) || !(grz0 > 0.0))
    return CADMAS_EINVAL;
  std::memset(out, 0, sizeof(*out));
  // the Ursell number and the STK-CND choice (vf_csetup.f:100-109)
  const double WUS = grz0 * height * period * period / depth / depth;
  if (type == CADMAS_WAVE_STK_CND) type = (WUS <= 25.0) ? CADMAS_WAVE_STOKES : CADMAS_WAVE_CNOIDAL;
  out->type = type;
  out->depth = depth; out->period = period; out->height = height;
  out->ursell = WUS;
  // WVLENG: the single-precision length of the theory's routine, in m
  // (vf_cwmak0.f:36-51)
  double RL = 0.0;
  int rc;
  if (type >= 1) {  // the reference's stream routine works with g = 9.8 (vf_wsfmb2.f:247)
    rc = cadmas_stream_solve(type, depth, period, height, 9.8, &out->stream);
    if (!rc) out->length = (double)(float)out->stream.length;
  } else if (type == CADMAS_WAVE_STOKES) {
    rc = stokes_solve(depth, period, height, out->stokes, RL);
    out->length = (double)(float)RL * 0.01;
  } else {
    rc = cnoidal_solve(depth, period, height, out->cnoidal, RL);
    out->length = (double)(float)RL * 0.01;
  }
  if (rc) { std::memset(out, 0, sizeof(*out)); return rc; }
  out->phase0 = cadmas::theory_zero_phase(*out);
  return CADMAS_OK;
}

extern "C" int cadmas_wave_eval(const cadmas_wave_theory *t, double phase, double z, double *eta, double *u,
                                double *w) {
  if (!t || t->type > CADMAS_STREAM_NMAX || t->type < CADMAS_WAVE_STOKES || t->type == 0) return CADMAS_EINVAL;
  if (eta) *eta = cadmas::theory_eta(*t, phase);
  if (u || w) {
    cadmas::WavePhase ph;
    cadmas::theory_phase(*t, phase, ph);
    double uu, ww;
    cadmas::wt_velocity(ph, z, uu, ww);
    if (u) *u = uu;
    if (w) *w = ww;
  }
  return CADMAS_OK;
}
