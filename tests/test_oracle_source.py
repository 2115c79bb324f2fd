"""The wave source (MODEL WAVE-SRC ... FUNC MATRIX) in the oracle.

A source line in the middle of still water between two damping zones,
driven by a first-order wave table (H = 0.03 m, T = 1.2 s, depth 0.25 m)
and faded in over half a period:
  * the waves it makes are mirror images on its two sides (VF_CWMSRC's
    SRCUV enters VF_VGENE on the faces on both sides of the line,
    VF_VPCOEF, VF_BSUWN and VF_FGENE symmetrically): the column water
    levels left and right of the line agree to 1e-6 m;
  * the y source on the transposed grid makes the same levels as the x
    source, to 1e-8 m (only the summation order of the global sums
    differs);
  * the wave it makes has about the table's amplitude H/2: between 0.5
    and 1.5 times H/2 within 300 steps (0.6 s).
"""
import numpy as np


def _levels(orc, pkg, axis, steps):
    c = pkg.cases.source_flume(axis=axis)
    o = orc.Oracle(c, sum_mode=orc.SUM_REF)
    o.init_state(True)
    for _ in range(steps):
        o.step(c.dt)
    ff = o.get_state()["ff"]
    dz = c.zz[1, 1:-1]
    lvl = (ff[1:-1, 2, 1:-1] * dz).sum(axis=1) if axis == "x" else (ff[2, 1:-1, 1:-1] * dz).sum(axis=1)
    return lvl, c


def test_source_waves_are_symmetric_and_sized(orc, pkg):
    lx, c = _levels(orc, pkg, "x", 300)
    mid = len(lx) // 2  # the source column I = nx/2 + 2 is interior index nx/2
    left, right = lx[:mid][::-1], lx[mid + 1:]
    n = min(len(left), len(right))
    assert np.abs(left[:n] - right[:n]).max() <= 1e-6
    amp = np.abs(lx - 0.25).max()
    assert 0.5 * 0.015 <= amp <= 1.5 * 0.015, amp
    ly, _ = _levels(orc, pkg, "y", 300)
    assert np.abs(lx - ly).max() <= 1e-8
