"""The k-epsilon model (LEQK = 1: k_kstep, k_kbsss, k_bwke, k_kinit) on
the GPU against the oracle, through the C ABI.

Bit-identical like the rest of the step: every field, NF/INDC, the step
statistics and the turbulence arrays AK, AE, ANUT, ANU, BCK, BCE after
every checked step.  The restart file carries AK, BCK, AE, BCE after BCF
(vf_or1trn.f:134-146) and a restart continues bit for bit.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FIELDS = ("uu", "vv", "ww", "pp", "ff", "nf", "indc", "bcu", "bcv", "bcw", "bcp", "bcf")
TURB = ("ak", "ae", "anut", "anu", "bck", "bce")


def assert_same(ga, oa, names, where):
    for n in names:
        a, b = ga[n], oa[n]
        if a.tobytes() != b.tobytes():
            bad = np.argwhere(a != b)
            d = np.abs(a.astype(np.float64) - b.astype(np.float64)).max()
            raise AssertionError(f"{where}: {n} differs at {bad.shape[0]} places, first {bad[:3].tolist()}, max |d| {d}")


def run_pair(pkg, orc, c, steps, check_every=5, **over):
    t = pkg.Tank(c, **over)
    o = orc.Oracle(c, sum_mode=orc.SUM_GPU, **over)
    t.init_state(c.hydrostatic)
    o.init_state(c.hydrostatic)
    if getattr(c, "drop_state", None) is not None:
        t.set_drop(c.drop_state)
        o.set_drop(c.drop_state)
    assert_same(t.get_turb(), o.get_turb(), TURB, "init")
    for n in range(1, steps + 1):
        t.step(c.dt)
        o.step(c.dt)
        if n % check_every == 0 or n == steps:
            assert_same(t.get_state(), o.get_state(), FIELDS, f"step {n}")
            assert_same(t.get_turb(), o.get_turb(), TURB, f"step {n}")
            sg, so = t.stats(), o.stats()
            for k in ("fsum", "fcut", "cgbnrm", "cgxnrm", "icgitr", "nums"):
                assert sg[k] == so[k], (n, k, sg[k], so[k])
    return t, o


@pytest.mark.parametrize("seed", [0, 1, 2, 3])
def test_turbulent_tanks_bitwise(gpu_lib, pkg, orc, seed):
    c = pkg.cases.turbulent_tank(seed)
    run_pair(pkg, orc, c, 20)


def test_turbulent_dam_break_bitwise(gpu_lib, pkg, orc):
    c = pkg.cases.turbulence(pkg.cases.dam_break(), 1e-2, 1e-3)
    t, o = run_pair(pkg, orc, c, 20)
    assert t.get_turb()["anut"].max() > 1e-5  # the eddy viscosity is live


def test_turbulence_with_droplets_and_ffslope_bitwise(gpu_lib, pkg, orc):
    c = pkg.cases.turbulence(pkg.cases.random_tank(0), 1e-3, 1e-4, seed=5)
    run_pair(pkg, orc, c, 15, iscmff=1)
    d = pkg.cases.turbulence(pkg.cases.droplet_tank(1), 1e-3, 1e-4, seed=6)
    run_pair(pkg, orc, d, 15)


def test_set_turb_forms_the_eddy_viscosity(gpu_lib, pkg, orc):
    """cadmas_set_turb: AK, AE, BCK, BCE in, ANUT and ANU as VF_CNUT0 and
    VF_CNU00 form them (the restart input's rule)."""
    c = pkg.cases.turbulent_tank(1)
    t = pkg.Tank(c)
    o = orc.Oracle(c, sum_mode=orc.SUM_GPU)
    t.init_state(True)
    o.init_state(True)
    rng = np.random.default_rng(3)
    n = c.ni * c.nj * c.nk
    arrs = dict(ak=rng.uniform(1e-5, 1e-3, n), ae=rng.uniform(1e-6, 1e-4, n),
                bck=rng.uniform(0, 1e-3, c.numb), bce=rng.uniform(0, 1e-4, c.numb))
    t.set_turb(arrs)
    o.set_turb(arrs)
    assert_same(t.get_turb(), o.get_turb(), TURB, "set_turb")
    for _ in range(3):
        t.step(c.dt)
        o.step(c.dt)
    assert_same(t.get_turb(), o.get_turb(), TURB, "after set_turb")


def test_restart_with_turbulence(gpu_lib, pkg, tmp_path):
    from test_gpu_restart import records
    c = pkg.cases.turbulent_tank(2)
    path = tmp_path / "keps.rsl"
    t = pkg.Tank(c)
    t.init_state(True)
    t.restart_create(path)
    for _ in range(4):
        t.step(c.dt)
    t.restart_append(path)
    kept = t.get_turb()
    R = records(path)
    assert np.frombuffer(R[2], "<i4").tolist() == [1, 1, 1, 1, 1, 0, 0, 0, 1, 0]
    # output: header, sums, NF, 5 x (field, BC), then AK, BCK, AE, BCE,
    # TBUB, the droplet count and the droplets
    base = 4 + 3 + 10
    for k, n in enumerate(("ak", "bck", "ae", "bce")):
        assert R[base + k] == kept[n].tobytes(), n
    assert len(R[base + 4]) == 8 * c.nk
    nd = int(np.frombuffer(R[base + 5], "<i4")[0])
    assert len(R) == base + 6 + nd
    # a restart continues bit for bit
    u = pkg.Tank(c)
    u.init_state(True)
    u.restart_load(path, 4)
    for _ in range(3):
        t.step(c.dt)
        u.step(c.dt)
    assert_same(u.get_turb(), t.get_turb(), TURB, "restart")
    assert_same(u.get_state(), t.get_state(), FIELDS, "restart")
    # a file without k-epsilon is refused by a k-epsilon run
    plain = pkg.Tank(pkg.cases.random_tank(2))
    plain.init_state(True)
    p2 = tmp_path / "plain.rsl"
    plain.restart_create(p2)
    plain.restart_append(p2)
    with pytest.raises(pkg.CadmasError, match="K-EPS"):
        u.restart_load(p2, 0)
