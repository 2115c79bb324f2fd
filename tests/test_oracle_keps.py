"""The k-epsilon model (LEQK = 1: VF_K1CAL, VF_CNUT0, VF_CNU00, VF_BSSS,
VF_BWKE) in the oracle.

The reference ships no test of it.  Its known answer is decaying
homogeneous turbulence: in still water with uniform k and e, production is
zero (no velocity gradient), zero-gradient walls carry no flux and the
upwind fluxes vanish, so every fluid cell follows the explicit Euler steps
of dk/dt = -e, de/dt = -C2 e^2/k that VF_KGENE and VF_SEULER form.  Around
it: the eddy viscosity C_mu k^2/e and ANU = ANU0 + ANUT after each step,
the boundary rules of VF_BWKE, water conservation and a moving case with
random boundary types.
"""
import numpy as np
import pytest


def fluid(st):
    return st["nf"].reshape(-1, order="F") == 0


def still_tank(pkg, k0, e0, **kw):
    c = pkg.cases.random_tank(0, nobst=0, nporous=0, nbox=0, **kw)
    return pkg.cases.turbulence(c, k0, e0)


def test_decaying_homogeneous_turbulence(pkg, orc):
    k0, e0 = 1.0e-3, 2.0e-4
    c = still_tank(pkg, k0, e0)
    o = orc.Oracle(c)
    o.init_state(True)
    C2, dt = 1.92, c.dt
    k, e = k0, e0
    for n in range(50):
        o.step(dt)
        # VF_KGENE: QK = -e, QE = -C2 (e/k) e; VF_SEULER with GGV cancelling
        k, e = k - dt * e, e - dt * (C2 * (e / k) * e)
    t = o.get_turb()
    m = fluid(o.get_state())
    assert m.sum() > 100
    np.testing.assert_allclose(t["ak"][m], k, rtol=1e-9)
    np.testing.assert_allclose(t["ae"][m], e, rtol=1e-9)
    # and the continuous law k(t) = k0 (1 + (C2-1) e0 t / k0)^(-1/(C2-1))
    T = 50 * dt
    k_exact = k0 * (1.0 + (C2 - 1.0) * e0 * T / k0) ** (-1.0 / (C2 - 1.0))
    assert abs(t["ak"][m].mean() - k_exact) < 2e-3 * k_exact


def test_eddy_viscosity_and_anu(pkg, orc):
    c = pkg.cases.turbulent_tank(1)
    o = orc.Oracle(c)
    o.init_state(True)
    for _ in range(5):
        o.step(c.dt)
    t = o.get_turb()
    st = o.get_state()
    nf = st["nf"].reshape(-1, order="F")
    inner = np.zeros((c.ni, c.nj, c.nk), bool)
    inner[1:-1, 1:-1, 1:-1] = True
    inner = inner.reshape(-1, order="F")
    live = inner & (nf != -1)
    want = 0.09 * t["ak"][live] * t["ak"][live] / np.maximum(t["ae"][live], 1e-20)
    assert np.array_equal(t["anut"][live], want)
    assert np.array_equal(t["anu"][live], 1.0e-6 + t["anut"][live])
    assert not t["anu"][inner & (nf == -1)].any()
    # gas cells carry no turbulence, surface cells the mean of fluid ones
    assert not t["ak"][inner & (nf == 8)].any()


def test_boundary_rules(pkg, orc):
    """VF_BWKE: fixed faces keep the input value, zero-gradient faces take
    the value of the cell inside."""
    c = pkg.cases.turbulent_tank(2)
    o = orc.Oracle(c)
    o.init_state(True)
    for _ in range(3):
        o.step(c.dt)
    t = o.get_turb()
    fixed = np.abs(c.indbk) == 1
    assert fixed.any() and (~fixed).any()
    np.testing.assert_array_equal(t["bck"][fixed], c.bck[fixed])
    ak = t["ak"]
    for L in np.nonzero(~fixed)[0][:50]:
        ijk, ns = int(c.indb[0, L]) - 1, int(c.indb[1, L])
        off = {1: 0, 2: -1, 3: 0, 4: -c.ni, 5: 0, 6: -c.ni * c.nj}[ns]
        assert t["bck"][L] == ak[ijk + off]


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_turbulent_tank_conserves_water_and_stays_finite(pkg, orc, seed):
    c = pkg.cases.turbulent_tank(seed)
    o = orc.Oracle(c)
    o.init_state(True)
    v0 = o.stats()["fsum"]
    cut = 0.0
    for _ in range(20):
        o.step(c.dt)
        cut += o.stats()["fcut"]
    assert abs(o.stats()["fsum"] + cut - v0) <= 1e-12 * v0
    t = o.get_turb()
    for n in ("ak", "ae", "anut", "anu", "bck", "bce"):
        assert np.isfinite(t[n]).all(), n
    m = fluid(o.get_state())
    assert (t["ak"][m] >= 1e-20).all() and (t["ae"][m] >= 1e-20).all()


def test_turbulence_changes_the_flow(pkg, orc):
    """The eddy viscosity reaches the momentum step (ANU of VF_V1CAL)."""
    base = pkg.cases.dam_break(nx=32, ny=4, nz=16, dt=2e-4)
    turb = pkg.cases.turbulence(pkg.cases.dam_break(nx=32, ny=4, nz=16, dt=2e-4), 1e-2, 1e-3)
    uu = []
    for c in (base, turb):
        o = orc.Oracle(c)
        o.init_state(True)
        for _ in range(10):
            o.step(c.dt)
        uu.append(o.get_state()["uu"])
    assert np.abs(uu[0] - uu[1]).max() > 1e-8
