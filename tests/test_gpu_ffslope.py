"""FF-SLOPE advection of F (ISCMFF = 1: k_fslope + k_fconvs, restating
VF_FCONVS) on the GPU against the oracle, through the C ABI.

Same bar as the donor-acceptor path: with --fmad=false, the Fortran
operand order and the cube root, arctangent and cosine of VF_CROOT3 built
from the same basic operations on both sides, every field after every
checked step is bit-identical to the oracle's.  The oracle's counts of
slope types show that the 2-D (types 5, 6) and 3-D (type 7) plane
branches ran.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FIELDS = ("uu", "vv", "ww", "pp", "ff", "nf", "indc", "bcu", "bcv", "bcw", "bcp", "bcf")


def assert_same(ga, oa, where):
    for n in FIELDS:
        a, b = ga[n], oa[n]
        if a.tobytes() != b.tobytes():
            bad = np.argwhere(a != b)
            d = np.abs(a.astype(np.float64) - b.astype(np.float64)).max()
            raise AssertionError(f"{where}: {n} differs at {bad.shape[0]} places, first {bad[:3].tolist()}, max |d| {d}")


def run_pair(pkg, orc, c, steps, check_every=5, **over):
    t = pkg.Tank(c, iscmff=1, **over)
    o = orc.Oracle(c, sum_mode=orc.SUM_GPU, iscmff=1, **over)
    t.init_state(c.hydrostatic)
    o.init_state(c.hydrostatic)
    if getattr(c, "drop_state", None) is not None:
        t.set_drop(c.drop_state)
        o.set_drop(c.drop_state)
    for n in range(1, steps + 1):
        t.step(c.dt)
        o.step(c.dt)
        if n % check_every == 0 or n == steps:
            assert_same(t.get_state(), o.get_state(), f"step {n}")
            sg, so = t.stats(), o.stats()
            for k in ("fsum", "fcut", "cgbnrm", "cgxnrm", "icgitr", "nums"):
                assert sg[k] == so[k], (n, k, sg[k], so[k])
    return t, o


@pytest.mark.parametrize("seed", [0, 2, 3, 6])
def test_ffslope_random_tanks_bitwise(gpu_lib, pkg, orc, seed):
    c = pkg.cases.random_tank(seed)
    t, o = run_pair(pkg, orc, c, 20)
    counts = o.slope_counts()
    assert sum(counts[3:]) > 0, counts


def test_ffslope_dam_break_bitwise(gpu_lib, pkg, orc):
    c = pkg.cases.dam_break()
    t, o = run_pair(pkg, orc, c, 20)
    assert o.slope_counts()[5] > 0
    assert t.divnorm() == o.divnorm()


def test_ffslope_droplets_bitwise(gpu_lib, pkg, orc):
    """Droplets over a level pool (no slope cells: the donor-acceptor faces
    of VF_FCONVS and the droplet model under ISCMFF = 1)."""
    c = pkg.cases.droplet_tank(1)
    t, o = run_pair(pkg, orc, c, 20)
    dg, do = t.get_drop(), o.get_drop()
    for k in pkg.DROP_ARRAYS:
        assert dg[k].tobytes() == do[k].tobytes(), k


def test_ffslope_every_type_and_scheme_matters(gpu_lib, pkg, orc):
    """Seed 0 has surface cells of types 3, 5, 6 and 7; the GPU's F differs
    between the two schemes (the switch reaches the kernels)."""
    c = pkg.cases.random_tank(0)
    t, o = run_pair(pkg, orc, c, 20, check_every=20)
    counts = o.slope_counts()
    assert all(counts[k] > 0 for k in (3, 5, 6, 7)), counts
    d = pkg.Tank(c)
    d.init_state(c.hydrostatic)
    for _ in range(20):
        d.step(c.dt)
    assert (d.get_state()["ff"] != t.get_state()["ff"]).sum() > 10
