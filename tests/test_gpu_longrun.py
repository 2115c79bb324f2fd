"""Long runs at the benchmark sizes, GPU against the oracle.

* Config 0, the 64x8x32 dam break, for its full 2000 steps (dt = 1e-4 s,
  R-ERROR 1e-10, the time loop of vf_a1main.f:919-1145):
  - the GPU equals the oracle in the GPU summation order bit for bit
    (every field, NF, INDC, the solver statistics), checked every 250
    steps;
  - the GPU against the oracle in the reference's own summation order
    (sequential K,J,I sums, as the Fortran loops add): the fields differ
    only by the rounding of the global sums, within
        |u|, |v|, |w|  max-abs 1e-12 m/s   (|u| up to 2.4 m/s)
        p              max-abs 1e-8 Pa     (p up to 1.3e3 Pa)
        F              max-abs 1e-12
        NF             no cell differs
        FSUM           relative difference 1e-12,
    about 100 times the differences seen over the 2000 steps (velocity
    1.2e-14, p 7.3e-11, F 3.6e-14, FSUM 2.5e-14 relative).
* Config 1, the full 512x32x96 porous flume with its wave maker (the
  first-order stream-function wave, FUNC STREAM 1), 20 steps with 16x16
  preconditioner blocks: bit for bit against the oracle in the GPU order
  every 5 steps.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FIELDS = ("uu", "vv", "ww", "pp", "ff", "nf", "indc", "bcu", "bcv", "bcw", "bcp", "bcf")
STATS = ("fsum", "fcut", "cgbnrm", "cgxnrm", "icgitr", "nums")
TOL_REF_ORDER = {"uu": 1e-12, "vv": 1e-12, "ww": 1e-12, "pp": 1e-8, "ff": 1e-12}


def _bitwise(a, b, where):
    for n in FIELDS:
        if a[n].tobytes() != b[n].tobytes():
            d = np.abs(a[n].astype(np.float64) - b[n].astype(np.float64)).max()
            raise AssertionError(f"{where}: {n} differs (max |d| {d})")


def test_dam_break_2000_steps(gpu_lib, pkg, orc):
    c = pkg.cases.dam_break()
    assert (c.ni - 2, c.nj - 2, c.nk - 2) == (64, 8, 32) and c.dt == 1.0e-4
    t = pkg.Tank(c)
    og = orc.Oracle(c, sum_mode=orc.SUM_GPU)
    orf = orc.Oracle(c, sum_mode=orc.SUM_REF)
    for x in (t, og, orf):
        x.init_state(True)
    fsum0 = t.stats()["fsum"]
    worst = {n: 0.0 for n in TOL_REF_ORDER}
    for n in range(1, 2001):
        for x in (t, og, orf):
            x.step(c.dt)
        if n % 250 == 0:
            sg, so, sr = t.get_state(), og.get_state(), orf.get_state()
            _bitwise(sg, so, f"step {n}")
            a, b = t.stats(), og.stats()
            for k in STATS:
                assert a[k] == b[k], (n, k, a[k], b[k])
            for f, tol in TOL_REF_ORDER.items():
                d = float(np.abs(sg[f] - sr[f]).max())
                worst[f] = max(worst[f], d)
                assert d <= tol, f"step {n}: {f} differs from the reference order by {d} > {tol}"
            assert int((sg["nf"] != sr["nf"]).sum()) == 0, f"step {n}: NF differs from the reference order"
            fr = orf.stats()["fsum"]
            assert abs(a["fsum"] - fr) <= 1e-12 * abs(fr), (n, a["fsum"], fr)
    # the water column has collapsed and run along the floor
    st = t.get_state()
    assert np.abs(st["uu"]).max() > 1.0
    assert abs(t.stats()["fsum"] - fsum0) <= 1e-3 * fsum0
    t.close()


def test_flume_full_size_20_steps_bitwise(gpu_lib, pkg, orc):
    c = pkg.cases.porous_flume()
    pkg.cases.wave_maker(c, 0.08, 1.5, 0.5, stream=1)  # WAVE-BC X- FUNC STREAM 1
    pkg.cases.linear_wave_initial(c, 0.08, 1.5, 0.5, phase0=c.wave["stream"].phase0)
    assert (c.ni - 2, c.nj - 2, c.nk - 2) == (512, 32, 96)
    over = dict(precond_ti=16, precond_tj=16)
    t = pkg.Tank(c, **over)
    o = orc.Oracle(c, sum_mode=orc.SUM_GPU, **over)
    t.init_state(True)
    o.init_state(True)
    _bitwise(t.get_state(), o.get_state(), "init")
    for n in range(1, 21):
        t.step(c.dt)
        o.step(c.dt)
        if n % 5 == 0:
            _bitwise(t.get_state(), o.get_state(), f"step {n}")
            a, b = t.stats(), o.stats()
            for k in STATS:
                assert a[k] == b[k], (n, k, a[k], b[k])
    assert t.stats()["icgitr"] > 0
    t.close()
