"""Bounded device-side waits of the MILU sweeps, made to run out.

Every mbarrier wait of the sweeps gives up after the handle's
wait_limit_s; the sweep then lets its issued bulk copies land, flags the
solve as timed out and ends, and the host returns CADMAS_ETIMEOUT.  The
failure is injected on the host side of the kernel's contract: with
cadmas_test_stall_sweeps the producer warp issues no copies from a given
wavefront step on, so the waits for those steps have nothing to wait for
(no fault, no endless loop: every wait is bounded).  After the injection
is switched off the same handle must step exactly like a handle that never
timed out.
"""
import numpy as np
import pytest


def _copy_state(src, dst):
    st = src.get_state()
    dst.set_state(st)
    dst.set_time(st["tnow"], src.case.dt, st["nnow"])


@pytest.mark.gpu
@pytest.mark.parametrize("solver", [0, 1])
def test_sweep_wait_runs_out_then_handle_recovers(gpu_lib, pkg, solver):
    c = pkg.cases.dam_break(nx=32, ny=4, nz=16, column=(8, 8), dt=1.0e-4)
    t = pkg.Tank(c, wait_limit_s=0.05, solver=solver)
    ref = pkg.Tank(c, solver=solver)
    for x in (t, ref):
        x.init_state(True)
        x.step(c.dt)
    t.test_stall_sweeps(5)
    with pytest.raises(pkg.CadmasError) as e:
        t.step(c.dt)
    assert e.value.status == pkg.ETIMEOUT
    assert b"time" in t.lib.cadmas_strerror(pkg.ETIMEOUT)
    # the context and the handle stay usable
    t.test_stall_sweeps(-1)
    _copy_state(ref, t)
    for step in range(3):
        t.step(c.dt)
        ref.step(c.dt)
        a, b = t.get_state(), ref.get_state()
        for n in ("uu", "vv", "ww", "pp", "ff", "nf", "indc"):
            assert np.array_equal(a[n], b[n]), f"step {step}: {n} differs after recovery"
        assert t.stats()["icgitr"] == ref.stats()["icgitr"]
    t.close()
    ref.close()


@pytest.mark.gpu
def test_default_wait_limit_is_not_reached(gpu_lib, pkg):
    """A normal solve with a short limit (10 ms) never comes near it."""
    c = pkg.cases.dam_break(nx=32, ny=4, nz=16, column=(8, 8), dt=1.0e-4)
    t = pkg.Tank(c, wait_limit_s=0.01)
    t.init_state(True)
    for _ in range(3):
        t.step(c.dt)
    assert t.stats()["icgitr"] > 0
    t.close()
