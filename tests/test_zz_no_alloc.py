"""cadmas_divnorm_noalloc: the divergence norm of VF_CDIV00 on device arrays,
without a handle and without allocating (static device scratch).

It runs the same kernels in the same summation order as the handle's
cadmas_divnorm, so the test tolerance is 0: both must return the same
double.  The file name sorts last so the test also runs after every other
GPU test in the same process; it passes alone as well.
"""
import ctypes

import numpy as np
import pytest


def test_noalloc_rejects_grid_beyond_scratch(pkg):
    """NUMJ*NUMK above the static scratch: CADMAS_ESCRATCH before any CUDA call."""
    lib = pkg.load_library()
    d = pkg.Dims(10, 300, 300, 0)  # 90,000 rows > 65,536
    fake = [ctypes.c_void_p(256)] * 10  # never dereferenced: rejected first
    v = ctypes.c_double(-1.0)
    rc = lib.cadmas_divnorm_noalloc(ctypes.byref(d), *fake, ctypes.c_void_p(0), ctypes.byref(v))
    assert rc == pkg.ESCRATCH
    assert v.value == -1.0
    assert b"65536" in lib.cadmas_strerror(rc)


def _check_against_handle(pkg, c, steps, **over):
    """cadmas_divnorm_noalloc on copies of a tank's arrays equals the
    handle's cadmas_divnorm, bit for bit, twice in a row after each step."""
    import torch

    t = pkg.Tank(c, **over)
    t.init_state(True)
    dims = (c.ni, c.nj, c.nk)

    def dev(a):
        return torch.from_numpy(np.ascontiguousarray(np.asarray(a).ravel(order="F"))).cuda()

    static = {n: dev(getattr(c, n)) for n in ("xx", "yy", "zz", "ggx", "ggy", "ggz")}
    for step in range(steps):
        t.step(c.dt)
        ref = t.divnorm()
        st = t.get_state()
        fld = {n: dev(st[n]) for n in ("uu", "vv", "ww", "indc")}
        torch.cuda.synchronize()
        ptr = lambda n: (static[n] if n in static else fld[n]).data_ptr()
        for call in range(2):  # two calls in a row on the same state
            v = pkg.divnorm_noalloc(dims, *(ptr(n) for n in ("xx", "yy", "zz", "ggx", "ggy", "ggz",
                                                              "uu", "vv", "ww", "indc")))
            assert v == ref, f"{c.name} step {step} call {call}: {v!r} != {ref!r}"
        assert ref > 0.0
    t.close()


@pytest.mark.gpu
def test_noalloc_matches_handle_divnorm(gpu_lib, pkg):
    _check_against_handle(pkg, pkg.cases.random_tank(2), steps=2)


@pytest.mark.gpu
def test_noalloc_full_scratch_then_small_grid(gpu_lib, pkg):
    """NUMJ*NUMK exactly CADMAS_NOALLOC_MAX_ROWS (4x254x254 interior, so
    NUMJ = NUMK = 256): every row slot of the scratch is used next to the
    result slot.  A small grid right after it must read none of the large
    grid's stale row partials."""
    big = pkg.cases.random_tank(5, nx=4, ny=254, nz=254, nobst=6, nporous=6, nbox=6)
    assert big.nj * big.nk == 65536
    _check_against_handle(pkg, big, steps=1, precond_ti=4, precond_tj=16)
    _check_against_handle(pkg, pkg.cases.random_tank(3), steps=1)
