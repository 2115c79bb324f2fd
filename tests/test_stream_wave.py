"""The stream-function wave of the wave maker (WAVE-BC ... FUNC STREAM N,
cadmas_stream_solve / cadmas_stream_eval, host code of the library).

The reference's own solver (vf_wsfmb2.f) cannot be run here (no Fortran
compiler), so the solution is checked against what any exact steady-wave
solution must satisfy:
  * order 1 and a vanishing height: the linear dispersion relation
    w^2 = g k tanh(k d), to 1e-9 relative in L;
  * the orders converge: L, crest and trough of N = 12 and N = 20 agree to
    1e-9 m (the config-1 wave, H = 0.08 m, T = 1.5 s, d = 0.5 m);
  * the height eta(0) - eta(1/2) is H, the mean level over a period is 0
    (to the single precision the wave routines return: 1e-6 m);
  * Bernoulli's equation holds between the collocation points, to 1e-5 g H;
  * no mean mass transport in the fixed frame (the reference's current
    definition): the period-mean flux under the surface is 0 to 1e-5 c d;
  * second-order Stokes theory: the crest height a + k a^2 cosh(kd)
    (2 + cosh 2kd) / (4 sinh^3 kd) within 5 % of its second-order part;
  * the start phase: eta(phase0) = 0 with phase0 in [0.5, 1].
"""
import math

import numpy as np
import pytest

D, T, H, G = 0.5, 1.5, 0.08, 9.8


def _linear_k(T, d, g=G):
    w2 = (2 * math.pi / T) ** 2 * d / g
    K = max(w2, math.sqrt(w2))
    for _ in range(100):
        th = math.tanh(K)
        K -= (K * th - w2) / (th + K * (1 - th * th))
    return K / d


def test_linear_limit(pkg):
    k = _linear_k(T, D)
    sw = pkg.stream_solve(1, D, T, 1e-5)
    assert abs(sw.length - 2 * math.pi / k) <= 1e-9 * sw.length
    assert abs(sw.celerity - sw.length / T) <= 1e-12


def test_orders_converge_and_shape(pkg):
    a, b = pkg.stream_solve(12, D, T, H), pkg.stream_solve(20, D, T, H)
    assert abs(a.length - b.length) <= 1e-9
    for ph in (0.0, 0.5, 0.25):
        assert abs(pkg.stream_eval(a, ph)[0] - pkg.stream_eval(b, ph)[0]) <= 1e-6  # float results
    crest, trough = pkg.stream_eval(b, 0.0)[0], pkg.stream_eval(b, 0.5)[0]
    assert abs(crest - trough - H) <= 1e-6
    phases = np.linspace(0.0, 1.0, 200, endpoint=False)
    eta = np.array([pkg.stream_eval(b, p)[0] for p in phases])
    assert abs(eta.mean()) <= 1e-6
    assert crest > H / 2 > -trough  # crest higher than the trough is deep


def test_bernoulli_between_collocation_points(pkg):
    sw = pkg.stream_solve(16, D, T, H)
    c = sw.celerity
    rng = np.random.default_rng(3)
    worst = 0.0
    for ph in rng.uniform(0, 1, 40):
        eta, u, w = pkg.stream_eval(sw, ph, 0.0)
        _, u, w = pkg.stream_eval(sw, ph, eta)
        worst = max(worst, abs(0.5 * ((u - c) ** 2 + w * w) + G * eta - sw.r))
    assert worst <= 1e-5 * G * H


def test_no_mean_mass_transport(pkg):
    sw = pkg.stream_solve(16, D, T, H)
    phases = np.linspace(0.0, 1.0, 100, endpoint=False)
    flux = []
    for ph in phases:
        eta = pkg.stream_eval(sw, ph)[0]
        z = np.linspace(-D, eta, 201)
        u = np.array([pkg.stream_eval(sw, ph, zz)[1] for zz in z])
        flux.append(np.trapezoid(u, z))
    assert abs(np.mean(flux)) <= 1e-5 * sw.celerity * D


def test_second_order_crest(pkg):
    sw = pkg.stream_solve(16, D, T, H)
    k, a = sw.k, H / 2
    kd = k * D
    second = k * a * a * math.cosh(kd) * (2 + math.cosh(2 * kd)) / (4 * math.sinh(kd) ** 3)
    crest = pkg.stream_eval(sw, 0.0)[0]
    assert abs(crest - (a + second)) <= 0.05 * second


def test_start_phase_is_a_zero_crossing(pkg):
    for n in (1, 5):
        sw = pkg.stream_solve(n, D, T, H)
        assert 0.5 <= sw.phase0 <= 1.0
        assert abs(pkg.stream_eval(sw, sw.phase0)[0]) <= 1e-4 * H


def test_steepness_limits(pkg):
    with pytest.raises(pkg.CadmasError):
        pkg.stream_solve(5, D, T, 1.0)  # H/d > 1.5 is refused (vf_wsfmb2.f:64-65)
