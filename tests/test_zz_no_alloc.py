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


@pytest.mark.gpu
def test_noalloc_matches_handle_divnorm(gpu_lib, pkg):
    import torch

    c = pkg.cases.random_tank(2)
    t = pkg.Tank(c)
    t.init_state(True)
    dims = (c.ni, c.nj, c.nk)

    def dev(a):
        return torch.from_numpy(np.ascontiguousarray(np.asarray(a).ravel(order="F"))).cuda()

    static = {n: dev(getattr(c, n)) for n in ("xx", "yy", "zz", "ggx", "ggy", "ggz")}
    for step in range(2):
        t.step(c.dt)
        ref = t.divnorm()
        st = t.get_state()
        fld = {n: dev(st[n]) for n in ("uu", "vv", "ww", "indc")}
        torch.cuda.synchronize()
        ptr = lambda n: (static[n] if n in static else fld[n]).data_ptr()
        for call in range(2):  # two calls in a row on the same state
            v = pkg.divnorm_noalloc(dims, *(ptr(n) for n in ("xx", "yy", "zz", "ggx", "ggy", "ggz",
                                                              "uu", "vv", "ww", "indc")))
            assert v == ref, f"step {step} call {call}: {v!r} != {ref!r}"
        assert ref > 0.0
    t.close()
