"""Log-law (INDB(3,L) = 6) and fully rough (8) walls in the oracle.

- The logarithm the oracle and the kernels share (frexp reduction and the
  atanh series) is within 1 ulp of libm's over 600 decades.
- VF_CLOGLW's friction velocity satisfies the log law
  VA = u*/kappa ln(DL u*/nu) + A u* to rounding; VF_CLOGKS is
  VA / (ln(DL/ks)/kappa + A + 3).
- After VF_CINIT the tangential values of every log-law and rough face are
  VF_BWUWT's, computed here in numpy from the state: the adjacent cell's
  averages V reduced to V (1 - DL u*^2 / (ANU |V|)).
- k and e of the cells next to such walls are VF_BWKELG's.
"""
import numpy as np
import pytest


def test_ln_is_within_one_ulp_of_libm(orc):
    rng = np.random.default_rng(5)
    xs = np.concatenate([rng.uniform(1e-3, 1e3, 3000), 10.0 ** rng.uniform(-300, 300, 3000),
                         [0.5, 2.0, np.sqrt(0.5), np.sqrt(2.0), 1.0 + 2.0 ** -52, 1e-310, 1.7e308]])
    for x in xs:
        y = orc.ln(x)
        assert abs(y - np.log(x)) <= np.spacing(abs(np.log(x))), x
    assert orc.ln(1.0) == 0.0
    assert orc.ln(0.0) == -np.inf
    assert np.isnan(orc.ln(-1.0))


def test_ln_ulp_bound_on_the_wall_function_range(orc):
    """The largest difference from libm's log over the arguments the wall
    functions take: DL u*/nu (log law) and DL/ks (rough walls) from 1e-2 to
    1e7.  At most 1 ulp of the result from 10 up (where the log law holds),
    2 ulps below 10, where |ln x| is small and its ulp finer than the
    series' absolute error of about 1e-16."""
    rng = np.random.default_rng(7)
    for lo, hi, bound in ((1.0, 7.0, 1.0), (-2.0, 1.0, 2.0)):
        xs = 10.0 ** rng.uniform(lo, hi, 4000)
        ulps = np.array([abs(orc.ln(x) - np.log(x)) / np.spacing(abs(np.log(x))) for x in xs])
        assert ulps.max() <= bound, (lo, hi, ulps.max())


@pytest.mark.parametrize("dl,va", [(0.005, 0.05), (0.005, 1e-6), (0.01, 2.0), (5e-4, 1e-3), (0.1, 10.0)])
def test_friction_velocity_satisfies_the_log_law(orc, dl, va):
    vt = orc.cloglw(dl, va)
    res = vt / 0.4 * np.log(dl * vt / 1e-6) + 5.5 * vt - va
    assert abs(res) <= 1e-12 * va
    ks = 1e-3
    assert orc.clogks(dl, va, ks) == va / (np.log(dl / ks) / 0.4 + 5.5 + 3.0) or \
        abs(orc.clogks(dl, va, ks) - va / (np.log(dl / ks) / 0.4 + 8.5)) <= 1e-15 * va
    assert orc.cloglw(dl, 1e-21) == 0.0 and orc.clogks(dl, 1e-21, ks) == 0.0


def _cell_avgs(s, I, J, K, NS):
    at = lambda a, i, j, k: s[a][i - 1, j - 1, k - 1]
    if NS in (1, 2):
        i = I if NS == 1 else I - 1
        return (at("vv", i, J, K) + at("vv", i, J + 1, K)) * 0.5, (at("ww", i, J, K) + at("ww", i, J, K + 1)) * 0.5, \
            ("x", i, J, K)
    if NS in (3, 4):
        j = J if NS == 3 else J - 1
        return (at("uu", I, j, K) + at("uu", I + 1, j, K)) * 0.5, (at("ww", I, j, K) + at("ww", I, j, K + 1)) * 0.5, \
            ("y", I, j, K)
    k = K if NS == 5 else K - 1
    return (at("uu", I, J, k) + at("uu", I + 1, J, k)) * 0.5, (at("vv", I, J, k) + at("vv", I, J + 1, k)) * 0.5, \
        ("z", I, J, k)


def test_init_sets_wall_function_values(orc, pkg):
    c = pkg.cases.loglaw_tank(0)
    o = orc.Oracle(c)
    o.init_state(True)
    s = o.get_state()
    n6 = n8 = 0
    for L in range(c.indb.shape[1]):
        ib = int(c.indb[2, L])
        if ib not in (6, 8):
            continue
        ijk, NS = int(c.indb[0, L]), int(c.indb[1, L])
        I = (ijk - 1) % c.ni + 1
        J = ((ijk - 1) // c.ni) % c.nj + 1
        K = (ijk - 1) // (c.ni * c.nj) + 1
        V1, V2, (ax, i, j, k) = _cell_avgs(s, I, J, K, NS)
        DL = {"x": c.xx[1, i - 1], "y": c.yy[1, j - 1], "z": c.zz[1, k - 1]}[ax] * 0.5
        AN = c.anu[i - 1, j - 1, k - 1]
        VA = np.sqrt(V1 * V1 + V2 * V2)
        if VA < 1e-20 or AN < 1e-20:
            V1 = V2 = 0.0
        else:
            VT = orc.cloglw(DL, VA) if ib == 6 else orc.clogks(DL, VA, c.bcvi[L])
            R = DL / AN * VT * VT / VA
            V1, V2 = V1 - R * V1, V2 - R * V2
            n6 += ib == 6
            n8 += ib == 8
        got = {1: ("bcv", "bcw"), 2: ("bcv", "bcw"), 3: ("bcu", "bcw"), 4: ("bcu", "bcw")}.get(NS, ("bcu", "bcv"))
        assert s[got[0]][L] == V1 and s[got[1]][L] == V2, (L, NS, ib)
    assert n6 > 20 and n8 > 20


def test_bwkelg_sets_k_and_e_next_to_walls(orc, pkg):
    c = pkg.cases.loglaw_tank(2, turb=True)
    o = orc.Oracle(c)
    o.init_state(True)
    for _ in range(3):
        o.step(c.dt)
    ak = o.get_turb()["ak"].reshape((c.ni, c.nj, c.nk), order="F")
    s = o.get_state()
    # one fluid cell whose only wall face is a single log-law z- face
    at = lambda a, i, j, k: a[i - 1, j - 1, k - 1]
    found = 0
    for K in range(2, c.nk):
        for J in range(2, c.nj):
            for I in range(2, c.ni):
                if at(s["nf"], I, J, K) != 0:
                    continue
                Ls = [int(at(c.indx, I, J, K)), int(at(c.indx, I + 1, J, K)), int(at(c.indy, I, J, K)),
                      int(at(c.indy, I, J + 1, K)), int(at(c.indz, I, J, K)), int(at(c.indz, I, J, K + 1))]
                types = [int(c.indb[2, L - 1]) if L >= 1 else 0 for L in Ls]
                if types[4] != 6 or any(tp in (6, 8) for q, tp in enumerate(types) if q != 4):
                    continue
                UC = (at(s["uu"], I, J, K) + at(s["uu"], I + 1, J, K)) * 0.5
                VC = (at(s["vv"], I, J, K) + at(s["vv"], I, J + 1, K)) * 0.5
                DZ = c.zz[1, K - 1] * 0.5
                WT = orc.cloglw(DZ, np.sqrt(UC * UC + VC * VC))
                # k after the step's cut-off and BSSS: the wall value unless cut off
                k = at(ak, I, J, K)
                assert k == pytest.approx(WT * WT / np.sqrt(0.09), rel=1e-12, abs=1e-20), (I, J, K)
                found += 1
    assert found > 0
