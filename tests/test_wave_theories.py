"""The Stokes and cnoidal wave theories of the wave maker and the wave
source (FUNC STOKES | CNOIDAL | STK-CND; cadmas_wave_solve and
cadmas_wave_eval, host code of the library).

The reference's routines (vf_wstk0.f, vf_wcnd0.f) cannot be run here (no
Fortran compiler), so the solutions are checked against what the theories
must satisfy:
  * a vanishing height: Stokes reduces to the linear wave (dispersion
    relation w^2 = g k tanh(k d) to 1e-6 in L, amplitude H/2);
  * Stokes is fifth order: against the stream-function wave of order 22
    (an exact steady wave to working precision, the same zero-mass-
    transport current) the level and the velocities differ by O(eps^6),
    so halving H divides the differences by about 64 (at least 45 is
    asserted; an error in a fourth- or fifth-order coefficient would give
    16 or 32), with the differences themselves below 1e-4 H;
  * the Stokes surface is a streamline at zero pressure: the pressure
    head p0 + (c u - (u^2 + w^2)/2)/g equals eta on the surface to 1e-4 H;
  * cnoidal is third order in H/d: against the stream-function wave in
    shallow water the differences are O(eps^4) (halving H at fixed period
    divides the level's by at least 12) and below 5e-5 H at H/d = 1/15;
  * Jacobi's elliptic functions of the cnoidal level against
    scipy.special.ellipj at the modulus of the solved parameter pi K'/K;
  * STK-CND picks Stokes up to an Ursell number of 25, cnoidal above
    (vf_csetup.f:100-109); the start phase is a zero of the level in
    [0.5, 1] (VF_CWZERO);
  * the oracle's restatement of the per-phase evaluation (VF_CWMAK1/2)
    gives the library's results bit for bit.
"""
import math

import numpy as np
import pytest


def _linear_k(T, d, g=9.8):
    w2 = (2 * math.pi / T) ** 2 * d / g
    K = max(w2, math.sqrt(w2))
    for _ in range(100):
        th = math.tanh(K)
        K -= (K * th - w2) / (th + K * (1 - th * th))
    return K / d


def _diffs(pkg, a, b, d, n=61):
    ph = np.linspace(0.0, 1.0, n)
    zs = (-0.9 * d, -0.5 * d, -0.1 * d)
    de = max(abs(pkg.wave_eval(a, p)[0] - pkg.wave_eval(b, p)[0]) for p in ph)
    du = max(abs(pkg.wave_eval(a, p, z)[1] - pkg.wave_eval(b, p, z)[1]) for p in ph for z in zs)
    dw = max(abs(pkg.wave_eval(a, p, z)[2] - pkg.wave_eval(b, p, z)[2]) for p in ph for z in zs)
    return de, du, dw


def test_stokes_small_height_is_linear(pkg):
    d, T, H = 0.5, 1.5, 1e-4
    s = pkg.wave_solve("stokes", d, T, H)
    assert s.type == pkg.WAVE_STOKES
    L = 2 * math.pi / _linear_k(T, d)
    assert abs(s.length - L) <= 1e-6 * L
    crest, trough = pkg.wave_eval(s, 0.0)[0], pkg.wave_eval(s, 0.5)[0]
    assert abs(crest - H / 2) <= 1e-3 * H and abs(trough + H / 2) <= 1e-3 * H


@pytest.mark.parametrize("d,T,H", [(1.0, 1.2, 0.1), (0.5, 1.5, 0.08), (0.3, 2.0, 0.02)])
def test_stokes_is_fifth_order_against_the_stream_function(pkg, d, T, H):
    hi = _diffs(pkg, pkg.wave_solve("stokes", d, T, H), pkg.wave_solve(22, d, T, H), d)
    lo = _diffs(pkg, pkg.wave_solve("stokes", d, T, H / 2), pkg.wave_solve(22, d, T, H / 2), d)
    assert hi[0] <= 1e-4 * H
    for a, b in zip(hi, lo):
        assert a / b >= 45.0, (hi, lo)


def test_stokes_surface_is_at_zero_pressure(pkg):
    d, T, H = 0.5, 1.5, 0.08
    s = pkg.wave_solve("stokes", d, T, H)
    c, g = s.stokes.c, 980.0  # cm/s, cm/s^2, as the theory's routine
    for p in np.linspace(0.0, 1.0, 41):
        e = pkg.wave_eval(s, p)[0]
        _, u, w = pkg.wave_eval(s, p, e)
        U, W = u * 100.0, w * 100.0
        head = s.stokes.p0 + (c * U - (U * U + W * W) / 2.0) / g
        assert abs(head - e * 100.0) <= 1e-4 * H * 100.0


@pytest.mark.parametrize("d,T,H", [(0.3, 4.0, 0.04), (0.5, 5.0, 0.1)])
def test_cnoidal_is_third_order_against_the_stream_function(pkg, d, T, H):
    hi = _diffs(pkg, pkg.wave_solve("cnoidal", d, T, H), pkg.wave_solve(22, d, T, H), d, n=81)
    lo = _diffs(pkg, pkg.wave_solve("cnoidal", d, T, H / 2), pkg.wave_solve(22, d, T, H / 2), d, n=81)
    assert lo[0] <= 1.2e-4 * (H / 2)
    assert hi[0] / lo[0] >= 12.0 and hi[1] / lo[1] >= 12.0, (hi, lo)


def test_cnoidal_shallow_agreement(pkg):
    d, T, H = 0.3, 4.0, 0.02
    c, f = pkg.wave_solve("cnoidal", d, T, H), pkg.wave_solve(22, d, T, H)
    assert c.ursell > 25.0
    assert abs(c.length - f.length) <= 1e-4 * f.length
    de, du, _ = _diffs(pkg, c, f, d, n=81)
    assert de <= 5e-5 * H and du <= 5e-4 * 0.073


def test_cnoidal_elliptic_functions_match_scipy(pkg):
    sp = pytest.importorskip("scipy.special")
    opt = pytest.importorskip("scipy.optimize")
    d, T, H = 0.3, 4.0, 0.04
    c = pkg.wave_solve("cnoidal", d, T, H)
    ql = c.cnoidal.ql  # pi K'/K
    m1 = opt.brentq(lambda m1: math.pi * sp.ellipk(m1) / sp.ellipk(1.0 - m1) - ql, 1e-300, 1.0 - 1e-16,
                    xtol=1e-300, rtol=1e-15)
    m = 1.0 - m1
    K = sp.ellipk(m)
    a = np.array(c.cnoidal.a[:4])
    for p in np.linspace(0.0, 1.0, 33):
        sn, cn, dn, _ = sp.ellipj(2.0 * K * p, m)
        eta = sum(a[i] * cn ** (2 * i) for i in range(4)) * 0.01
        assert abs(pkg.wave_eval(c, p)[0] - eta) <= 2e-7 * H


def test_stk_cnd_choice_and_start_phase(pkg):
    s = pkg.wave_solve("stk-cnd", 0.5, 1.5, 0.08)
    c = pkg.wave_solve("stk-cnd", 0.3, 4.0, 0.04)
    assert s.ursell <= 25.0 and s.type == pkg.WAVE_STOKES
    assert c.ursell > 25.0 and c.type == pkg.WAVE_CNOIDAL
    assert abs(c.ursell - 9.8 * 0.04 * 16.0 / 0.09) <= 1e-12 * c.ursell
    for th in (s, c):
        assert 0.5 <= th.phase0 <= 1.0
        assert abs(pkg.wave_eval(th, th.phase0)[0]) <= 2e-5 * th.height  # a zero in single precision
        assert pkg.wave_eval(th, 1.0)[0] > 0.0 > pkg.wave_eval(th, 0.5)[0]


def test_invalid_theories(pkg):
    for args in ((23, 0.5, 1.5, 0.08), (-3, 0.5, 1.5, 0.08), ("stokes", 0.5, 1.5, 0.0), ("stokes", -1.0, 1.5, 0.1)):
        with pytest.raises(pkg.CadmasError):
            pkg.wave_solve(*args)
    th = pkg.WaveTheory()  # type 0: not resolved
    with pytest.raises(pkg.CadmasError):
        pkg.wave_eval(th, 0.0)


def test_oracle_restatement_is_bitwise(pkg, orc):
    for th in (pkg.wave_solve("stokes", 0.5, 1.5, 0.08), pkg.wave_solve("cnoidal", 0.3, 4.0, 0.04),
               pkg.wave_solve(5, 0.5, 1.5, 0.08)):
        for p in np.linspace(0.0, 1.0, 37):
            for z in (-0.29, -0.1, 0.0, 0.02):
                assert pkg.wave_eval(th, p, z) == orc.wave_eval(th, p, z)
