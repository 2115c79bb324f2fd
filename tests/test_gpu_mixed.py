"""Mixed-precision pressure solver (solver 1: FP32 MILU-BiCGSTAB inner
solves under FP64 iterative refinement) against the FP64 solver (solver 0)
and the FP64 oracle on the same inputs.

Solver 1 converges on the true residual |b - Ax| <= CGEPSR |b| instead of
the reference's preconditioned criterion, so its fields are not bit-equal
to the reference's; the tolerances below state how far they may be:
  pressure        max |dp| <= 1e-8 * max |p|
  velocities      max |du| <= 1e-9 m/s
  F               max |dF| <= 1e-8
  fluid volume    |FSUM_1 - FSUM_0| <= 1e-10 * FSUM_0
  true residual   ||b - Ax|| / ||b|| <= CGEPSR (measured, diag_relres)
after 16 steps of the porous wave flume with its wave maker.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = dict(pp_rel=1e-8, vel=1e-9, ff=1e-8, vol=1e-10)


def _flume(pkg):
    c = pkg.cases.porous_flume(nx=96, ny=4, nz=64, block=(1.2, 1.4, 0.6), sponge_width=0.4)
    pkg.cases.linear_wave_initial(c, 0.08, 1.5, 0.5)
    pkg.cases.wave_maker(c, 0.08, 1.5, 0.5)
    return c


def _run(pkg, c, steps, **over):
    t = pkg.Tank(c, diag_relres=1, cgepsr=1e-10, **over)
    t.init_state(True)
    rel = []
    for _ in range(steps):
        t.step(c.dt)
        rel.append(t.stats()["true_relres"])
    return t, rel


def _errors(a, b):
    return dict(pp_rel=np.abs(a["pp"] - b["pp"]).max() / np.abs(b["pp"]).max(),
                vel=max(np.abs(a[n] - b[n]).max() for n in ("uu", "vv", "ww")),
                ff=np.abs(a["ff"] - b["ff"]).max())


def test_mixed_solver_against_fp64(gpu_lib, pkg):
    c = _flume(pkg)
    t0, rel0 = _run(pkg, c, 16, solver=0)
    t1, rel1 = _run(pkg, c, 16, solver=1)
    s0, s1 = t0.get_state(), t1.get_state()
    err = _errors(s1, s0)
    vol = abs(t1.stats()["fsum"] - t0.stats()["fsum"]) / t0.stats()["fsum"]
    print("mixed vs FP64:", err, "volume", vol, "relres", max(rel1), "fallbacks", t1.stats()["fallbacks"])
    assert max(rel1) <= 1e-10
    assert t1.stats()["fallbacks"] == 0
    for k, v in err.items():
        assert v <= TOL[k], (k, v)
    assert vol <= TOL["vol"]
    assert np.array_equal(s1["nf"], s0["nf"])


def test_mixed_solver_against_oracle(gpu_lib, pkg, orc):
    c = _flume(pkg)
    t1, rel1 = _run(pkg, c, 8, solver=1)
    o = orc.Oracle(c, sum_mode=orc.SUM_REF, cgepsr=1e-10)
    o.init_state(True)
    for _ in range(8):
        o.step(c.dt)
    err = _errors(t1.get_state(), o.get_state())
    print("mixed vs oracle:", err)
    for k, v in err.items():
        assert v <= TOL[k], (k, v)


@pytest.mark.parametrize("over", [dict(precond_ti=16, precond_tj=4), dict(precond_ti=16, precond_tj=4,
                                                                           sweep_occupancy=2), {}])
def test_inner_products_in_the_sweeps(gpu_lib, pkg, over):
    """The FP32 iteration's inner products summed by the backward sweeps
    (dot_passes 0: (R0,AP) and the five sums after AE, one partial per
    preconditioner block) against separate passes (dot_passes 1).  The
    products are exact in double and only the order of the sums differs;
    the FP32 iteration's path reacts to last-bit differences (single solves
    take a few iterations more or fewer either way), so the iterations of
    12 steps agree within 6 % in total and the fields within the solver's
    tolerance; six blocks with one or two sweep blocks per SM, and one
    block."""
    c = _flume(pkg)
    res = []
    for dp in (0, 1):
        t = pkg.Tank(c, diag_relres=1, cgepsr=1e-10, solver=1, dot_passes=dp, **over)
        t.init_state(True)
        its, rel = [], []
        for _ in range(12):
            t.step(c.dt)
            its.append(t.stats()["icgitr"])
            rel.append(t.stats()["true_relres"])
        assert max(rel) <= 1e-10 and t.stats()["fallbacks"] == 0
        res.append((sum(its), t.get_state()))
    assert abs(res[0][0] - res[1][0]) <= 0.06 * res[1][0], (res[0][0], res[1][0])
    err = _errors(res[0][1], res[1][1])
    for k, v in err.items():
        assert v <= TOL[k], (k, v)


def test_batch_matches_each_grid_alone(gpu_lib, pkg):
    """A batch of grids of different sizes whose mixed pressure solves run
    together (cadmas_batch_step: one launch per solver kernel over all the
    grids, iterations in lockstep, converged grids skipped) gives each grid
    bit for bit what it gives stepped alone, with the same iterations;
    with the previous-step guess, over 8 steps."""
    mk = lambda: [pkg.cases.porous_flume(nx=96 + 48 * i, ny=16 + 8 * (i % 2), nz=48 + 8 * i, depth=0.3,
                                         block=(1.0, 1.3, 0.4), sponge_width=0.4) for i in range(4)]
    kw = dict(solver=1, warm_start=1, precond_ti=16, precond_tj=8)
    together = [pkg.Tank(c, **kw) for c in mk()]
    alone = [pkg.Tank(c, **kw) for c in mk()]
    for t in together + alone:
        t.init_state(True)
    batch = pkg.Batch(together)
    for _ in range(8):
        assert batch.step() == [0] * len(together)
        for t in alone:
            t.step()
        for a, b in zip(together, alone):
            assert a.stats()["icgitr"] == b.stats()["icgitr"]
    batch.close()
    for a, b in zip(together, alone):
        sa, sb = a.get_state(), b.get_state()
        for k in ("uu", "vv", "ww", "pp", "ff", "nf"):
            assert sa[k].tobytes() == sb[k].tobytes(), k
        assert a.stats()["fallbacks"] == b.stats()["fallbacks"] == 0


def test_batch_rejects_mismatched_handles(gpu_lib, pkg):
    c = pkg.cases.porous_flume(nx=64, ny=16, nz=40, depth=0.3, block=(0.6, 0.8, 0.4), sponge_width=0.3)
    a = pkg.Tank(c, solver=1, precond_ti=16, precond_tj=8)
    b = pkg.Tank(c, solver=1, precond_ti=8, precond_tj=8)
    p = pkg.Tank(c, solver=0, precond_ti=16, precond_tj=8)
    for bad in ([a, b], [a, p], [a, a]):
        with pytest.raises(pkg.CadmasError):
            pkg.Batch(bad)
