"""FF-SLOPE advection (ISCMFF = 1, VF_FCONVS) in the oracle.

The reference ships no test of it, so the pieces are checked against what
they compute: the elementary functions of VF_CROOT3 against libm, VF_CROOT3
against numpy's polynomial roots, VF_FSLP2A/3A against VF_FSLP2F/3F (the
plane found for a water fraction must hold that fraction) and against a
closed form, and whole steps for conservation of water and for the slope
branches they exercise.
"""
import math

import numpy as np
import pytest

ULP = 2.0 ** -52


def test_cube_root_within_one_ulp(orc):
    rng = np.random.default_rng(0)
    xs = np.concatenate([np.logspace(-300, 300, 601), rng.uniform(1e-6, 10.0, 4000), [1.0, 8.0, 27.0, 0.125]])
    for x in xs:
        got, want = orc.slope_fn(0, x), np.cbrt(x)
        assert abs(got - want) <= ULP * want, x
    assert orc.slope_fn(0, 0.0) == 0.0


def test_arctangent_within_two_ulps(orc):
    ys = np.concatenate([np.linspace(-40.0, 40.0, 8001), [1e-300, -1e-300, 1e300, 1.0, -1.0, 0.0]])
    for y in ys:
        got, want = orc.slope_fn(1, y), math.atan(y)
        assert abs(got - want) <= 2 * ULP * abs(want) + 1e-320, y


def test_cosine_on_the_cardano_range(orc):
    # VF_CROOT3 takes cos of T/3, (PI-T)/3, (PI+T)/3 with T in (-pi/2, 3pi/2]
    for x in np.linspace(-math.pi / 6, 5 * math.pi / 6, 4001):
        assert abs(orc.slope_fn(2, x) - math.cos(x)) <= 4 * ULP, x


@pytest.mark.parametrize("coef", [
    (1.0, -6.0, 11.0, -6.0),      # (x-1)(x-2)(x-3): three real roots
    (2.0, 0.0, 3.0, -5.0),        # one real root
    (1.0, -3.0, 3.0, -1.0 + 1e-9),  # near-triple root
    (0.0, 1.0, -3.0, 2.0),        # quadratic through VF_CROOT2
    (-1.0, 0.3, 0.02, -0.0004),
])
def test_croot3_against_numpy(orc, coef):
    roots, n = orc.croot3(*coef)
    want = np.roots(coef)
    real = sorted(r.real for r in want if abs(r.imag) < 1e-6)
    assert n == len(real) or (n == 1 and len(real) == 3 and coef[2] == 3.0)  # near-triple: one root
    scale = max(1.0, max(abs(r) for r in real))
    for r in roots:
        assert min(abs(r - w) for w in real) < 1e-5 * scale, (roots, real)


def test_plane_round_trip(orc):
    """VF_FSLP2F/3F of the plane VF_FSLP2A/3A finds gives back the water
    fraction it was given."""
    rng = np.random.default_rng(1)
    for t in range(4000):
        dim = 2 if t % 2 else 3
        s = rng.normal(size=dim)
        s /= np.linalg.norm(s)
        s[np.abs(s) < 1e-4] = 1e-4
        d = rng.uniform(0.005, 0.05, size=dim)
        f = rng.uniform(1e-6, 1 - 1e-6)
        aa, fb = orc.fslp(list(s), list(d), f)
        assert abs(fb - f) < 1e-10, (s, d, f)


def test_plane_closed_form_2d(orc):
    # 45 degrees in a unit square: F = 1/2 puts the plane on the diagonal,
    # F = 1/8 cuts the corner triangle of legs 1/2
    s = [math.sqrt(0.5)] * 2
    aa, _ = orc.fslp(s, [1.0, 1.0], 0.5)
    assert abs(aa - math.sqrt(0.5)) < 1e-15
    aa, _ = orc.fslp(s, [1.0, 1.0], 0.125)
    assert abs(aa - 0.5 * math.sqrt(0.5)) < 1e-15
    # 3-D: the corner tetrahedron x+y+z <= a of the unit cube holds a^3/6
    s3 = [1.0 / math.sqrt(3.0)] * 3
    aa, _ = orc.fslp(s3, [1.0, 1.0, 1.0], 1.0 / 48.0)
    assert abs(aa - 0.5 / math.sqrt(3.0)) < 1e-14


@pytest.mark.parametrize("builder,kw,steps,sloped", [("random_tank", dict(seed=1), 20, True),
                                                     ("droplet_tank", dict(seed=1), 20, False),
                                                     ("dam_break", dict(nx=32, ny=4, nz=16, dt=2e-4), 20, True)])
def test_ffslope_conserves_water(pkg, orc, builder, kw, steps, sloped):
    """The slope fluxes move water between cells and nowhere else: FSUM +
    the cut-off volume stays constant, as with donor-acceptor."""
    c = getattr(pkg.cases, builder)(**kw)
    o = orc.Oracle(c, iscmff=1)
    o.init_state(c.hydrostatic)
    if getattr(c, "drop_state", None) is not None:
        o.set_drop(c.drop_state)
    v0 = o.stats()["fsum"]
    cut = 0.0
    for _ in range(steps):
        o.step(c.dt)
        cut += o.stats()["fcut"]
    s = o.stats()
    assert abs(s["fsum"] + cut - v0) <= 1e-12 * v0
    if sloped:  # (the droplet tank's level surface has no slope)
        assert sum(o.slope_counts()[3:]) > 0
    assert not np.isnan(o.get_state()["ff"]).any()


def test_ffslope_exercises_every_type_and_changes_f(pkg, orc):
    c = pkg.cases.random_tank(0)
    ff = {}
    for sch in (0, 1):
        o = orc.Oracle(c, iscmff=sch)
        o.init_state(c.hydrostatic)
        for _ in range(20):
            o.step(c.dt)
        ff[sch] = o.get_state()["ff"]
        if sch:
            counts = o.slope_counts()
    assert all(counts[k] > 0 for k in (3, 5, 6, 7)), counts
    assert counts[1] == counts[2] == counts[4] == 0  # one component is never a slope
    assert (ff[0] != ff[1]).sum() > 10
