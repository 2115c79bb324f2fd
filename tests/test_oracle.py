"""The CPU oracle against its pins and the invariants the reference's own
logic implies (the reference ships no tests or golden outputs)."""
import json
import pathlib
import sys

import numpy as np
import pytest

HERE = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(HERE / "golden"))
import make_golden  # noqa: E402


@pytest.mark.parametrize("name", sorted(make_golden.CASES))
def test_oracle_pins(name, orc):
    pins = json.loads((HERE / "golden" / "oracle_pins.json").read_text())
    got = make_golden.run(name, make_golden.CASES[name])
    assert got["digest"] == pins[name]["digest"]
    for k, v in pins[name]["stats"].items():
        assert got["stats"][k] == v, k


def test_dam_break_volume_balance(pkg, orc):
    """FSUM + cumulative FCUT is conserved in a closed box (vf_fcut01.f)."""
    c = pkg.cases.dam_break()
    o = orc.Oracle(c)
    o.init_state(True)
    v0 = o.stats()["fsum"]
    cut = 0.0
    for _ in range(40):
        o.step(c.dt)
        s = o.stats()
        cut += s["fcut"]
    assert abs(s["fsum"] + cut - v0) / v0 < 1e-10


def test_still_water_stays_at_rest(pkg, orc):
    """Hydrostatic still water in a closed box (p = rho g (WVLVL - z),
    vf_cinit.f:283) stays at rest."""
    c = pkg.cases.new_case("still", np.arange(13) * 0.01, np.arange(5) * 0.01, np.arange(11) * 0.01)
    c.params.update(wvlvl=0.045, wbub=-1.0)
    pkg.cases.init_f_still_water(c, 0.045)
    pkg.cases.finish(c)
    o = orc.Oracle(c)
    o.init_state(True)
    for _ in range(20):
        o.step(1e-3)
    st = o.get_state()
    assert max(np.abs(st[n]).max() for n in ("uu", "vv", "ww")) < 1e-9
    assert abs(o.stats()["fsum"] - 0.12 * 0.04 * 0.045) < 1e-13


def test_ilu_equals_milu_at_zero_parameter(pkg, orc):
    """MILU with CGPARA=0 is plain ILU (vf_mzdcmp.f:48-49)."""
    c = pkg.cases.random_tank(2)
    a = orc.Oracle(c, icgtyp=0)
    b = orc.Oracle(c, icgtyp=1, cgpara=0.0)
    for o in (a, b):
        o.init_state(True)
        for _ in range(3):
            o.step(c.dt)
    sa, sb = a.get_state(), b.get_state()
    for n in ("uu", "vv", "ww", "pp", "ff"):
        np.testing.assert_array_equal(sa[n], sb[n])


def _dense(sys7, indc, ni, nj):
    ad, ali, alj, alk, aui, auj, auk = sys7
    idx = np.nonzero(indc.reshape(-1, order="F") != -1)[0]
    pos = {c: r for r, c in enumerate(idx)}
    A = np.zeros((idx.size, idx.size))
    offs = [(ad, 0), (ali, -1), (alj, -ni), (alk, -ni * nj), (aui, 1), (auj, ni), (auk, ni * nj)]
    for r, c in enumerate(idx):
        for arr, o in offs:
            v = arr.reshape(-1, order="F")[c]
            if v != 0.0:
                A[r, pos[c + o]] += v
    return A, idx


def test_bicgstab_matches_dense_solve(pkg, orc):
    """VF_M1BCGS on the pressure system of a real step against LAPACK."""
    c = pkg.cases.random_tank(4)
    o = orc.Oracle(c, cgepsr=1e-14)
    o.init_state(True)
    o.step(c.dt)
    indc = o.get_state()["indc"]      # flags the next system is assembled with
    o.step(c.dt)
    sysa = [o.poisson(w) for w in range(8)]
    x, it, bn, xn = o.m1bcgs(*sysa, np.zeros_like(sysa[0]), indc)
    assert 0 < it < 500
    A, idx = _dense(sysa[:7], indc, c.ni, c.nj)
    b = sysa[7].reshape(-1, order="F")[idx]
    xd = np.linalg.solve(A, b)
    xs = x.reshape(-1, order="F")[idx]
    assert np.abs(xs - xd).max() <= 1e-9 * max(np.abs(xd).max(), 1e-30)


def test_block_jacobi_and_serial_agree_to_tolerance(pkg, orc):
    """The emulated NPI x NPJ decomposition (block-Jacobi MILU, as the
    reference runs on several ranks) and the serial MILU solve the same
    system to the solver tolerance."""
    c = pkg.cases.random_tank(6, nx=16, ny=8)
    a = orc.Oracle(c, cgepsr=1e-13)
    b = orc.Oracle(c, cgepsr=1e-13, precond_ti=4, precond_tj=4)
    for o in (a, b):
        o.init_state(True)
        o.step(c.dt)
    sa, sb = a.get_state(), b.get_state()
    np.testing.assert_array_equal(sa["nf"], sb["nf"])
    scale = np.abs(sa["pp"]).max()
    assert np.abs(sa["pp"] - sb["pp"]).max() < 1e-8 * scale


def test_ref_and_tree_order_close(pkg, orc):
    """The GPU summation order changes only the last bits."""
    c = pkg.cases.dam_break()
    a = orc.Oracle(c, sum_mode=orc.SUM_REF)
    b = orc.Oracle(c, sum_mode=orc.SUM_GPU)
    for o in (a, b):
        o.init_state(True)
        for _ in range(5):
            o.step(c.dt)
    sa, sb = a.get_state(), b.get_state()
    np.testing.assert_array_equal(sa["nf"], sb["nf"])
    for n in ("uu", "ww", "pp", "ff"):
        d = np.abs(sa[n] - sb[n]).max()
        assert d <= 1e-9 * max(np.abs(sa[n]).max(), 1e-12), n


def test_error_status_not_converged(pkg, orc):
    """ICGITR > ICGMAX maps to 'NOT CONVERGED.' (vf_vpsol.f:71-72)."""
    c = pkg.cases.dam_break()
    o = orc.Oracle(c, icgmax=1)
    o.init_state(True)
    with pytest.raises(pkg.CadmasError) as e:
        o.step(c.dt)
    assert e.value.status == pkg.ENOTCONV


def test_wave_maker_injects_the_table_wave(pkg, orc):
    """Matrix-table wave maker on the X- side: the boundary faces carry the
    table's velocity profile scaled by the fade-in, the inflow-side water
    level rises during the crest phase, and the solver still converges."""
    c = pkg.cases.porous_flume(nx=48, ny=2, nz=64, block=(0.6, 0.7, 0.6), sponge_width=0.2)
    pkg.cases.wave_maker(c, 0.08, 1.5, 0.5)          # no fade-in: full amplitude at once
    o = orc.Oracle(c, sum_mode=orc.SUM_REF)
    o.init_state(True)
    v0 = o.stats()["fsum"]
    o.step(c.dt)
    st = o.get_state()
    wave = c.indb[2] == 5
    assert wave.sum() == (c.nj - 2) * (c.nk - 2)
    bcu = st["bcu"][wave]
    # crest at the boundary at t = dt: inflow everywhere below the surface,
    # growing towards the surface (cosh profile)
    tab = c.wave["table"]
    assert np.all(bcu > 0.0)
    assert bcu.max() <= tab["un"].max() * 1.2
    col = st["uu"][1, 1, 1:-1]
    wet = st["ff"][1, 1, 1:-1] > 0
    assert np.all(np.diff(col[wet][: int(wet.sum()) - 1]) >= 0.0)
    for _ in range(40):
        o.step(c.dt)
    assert o.stats()["fsum"] > v0
    assert o.stats()["icgitr"] < 500


def test_droplets_move_water_and_conserve_it(pkg, orc):
    """VF_FDROPF: with IDROP=1 the droplet water moves (cells' F change and
    droplets split); the total volume FSUM + cut-off stays within rounding
    plus the cut-off of tiny leftovers; with IDROP=0 the droplet cells keep
    their water (gas cells carry no flux)."""
    c = pkg.cases.droplet_tank(0)
    runs = {}
    for idrop in (0, 1):
        o = orc.Oracle(c, idrop=idrop)
        o.init_state(True)
        o.set_drop(c.drop_state)
        v0 = o.stats()["fsum"]
        f0 = o.get_state()["ff"].copy()
        cut = 0.0
        for _ in range(20):
            o.step(c.dt)
            cut += o.stats()["fcut"]
        st = o.get_state()
        runs[idrop] = (f0, st["ff"], o.get_drop(), o.stats()["fsum"], v0, cut)
    f0, f1, d1, v1, v0, cut = runs[1]
    drop0 = c.drop_state["droptx"] > -1e9
    assert np.abs(f1 - f0).max() > 0.1                       # droplet water moved
    assert int((d1["droptx"] > -1e9).sum()) > int(drop0.sum())  # and split over more cells
    assert abs(v1 + cut - v0) <= 1e-9 * v0
    f0n, f1n = runs[0][0], runs[0][1]
    np.testing.assert_array_equal(f1n.reshape(-1, order="F")[drop0], f0n.reshape(-1, order="F")[drop0])


def test_droplet_free_fall_time(pkg, orc):
    """A droplet at rest in the air leaves its cell after the free-fall time
    of one cell, sqrt(2 dz / g) (vf_fdropf.f:548-556), and not before."""
    c = pkg.cases.droplet_tank(1, ndrop=1)
    o = orc.Oracle(c)
    o.init_state(True)
    ds = {k: v.copy() for k, v in c.drop_state.items()}
    cell = int(np.argmax(ds["droptx"] > -1e9))
    for k in ("dropuu", "dropvv", "dropww"):
        ds[k][cell] = 0.0
    o.set_drop(ds)
    f0 = o.get_state()["ff"].reshape(-1, order="F")[cell]
    ni, nj = c.ni, c.nj
    kc = cell // (ni * nj)
    dz = c.zz[1, kc]
    t_fall = np.sqrt(2.0 * dz / 9.8)
    left = None
    for n in range(1, int(2 * t_fall / c.dt) + 3):
        o.step(c.dt)
        if o.get_state()["ff"].reshape(-1, order="F")[cell] < f0 and left is None:
            left = n * c.dt
    assert left is not None and t_fall < left <= t_fall + 2 * c.dt
