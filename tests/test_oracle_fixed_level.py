"""Fixed-water-level wave boundary (WAVE-BC ... FUNC MATRIX with MTBTYP 3)
in the oracle.

- VF_BWFFSF (vf_bwffsf.f:43-128): after every step the F of the column next
  to the side is the level WVLVL + the table's level at TNOW, cell by cell,
  computed here from the table in numpy.
- VF_BWUWN's fixed-level faces (vf_bwuwn.f:161-216) copy the face inside,
  as free faces do.
"""
import numpy as np


def _level(c, tnow):
    w = c.wave
    t = w["table"]
    p = np.float32(0.0 - tnow / w["period"])
    p = p - np.float32(int(p))
    if p < 0:
        p = p + np.float32(1.0)
    return c.params["wvlvl"] + float(np.interp(float(p), t["tt"], t["hh"]))


def test_boundary_column_follows_the_level_table(orc, pkg):
    c = pkg.cases.fixed_level_flume(nx=48, nz=40, amp=0.04, T=2.0)
    o = orc.Oracle(c)
    o.init_state(True)
    zz = c.zz[0]
    for n in range(1, 31):
        o.step(c.dt)
        if n % 10:
            continue
        s = o.get_state()
        wl = _level(c, n * c.dt)
        for K in range(2, c.nk):
            z0, z1 = zz[K - 1], zz[K]
            exp = 0.0 if z0 > wl else 1.0 if z1 < wl else (wl - z0) / (z1 - z0)
            for J in range(2, c.nj):
                got = s["ff"][1, J - 1, K - 1]
                assert abs(got - exp) <= 1e-12, (n, J, K, got, exp)


def test_fixed_level_faces_copy_the_face_inside(orc, pkg):
    c = pkg.cases.fixed_level_flume(nx=48, nz=40, amp=0.04, T=2.0)
    o = orc.Oracle(c)
    o.init_state(True)
    for _ in range(30):
        o.step(c.dt)
    s = o.get_state()
    assert np.abs(s["uu"][2, 2:-2, 2:20]).max() > 1e-5  # inflow under way
    for L in range(c.indb.shape[1]):
        if c.indb[2, L] != 5:
            continue
        ijk = int(c.indb[0, L])
        I = (ijk - 1) % c.ni + 1
        J = ((ijk - 1) // c.ni) % c.nj + 1
        K = (ijk - 1) // (c.ni * c.nj) + 1
        assert I == 2 and s["bcu"][L] == s["uu"][I - 1, J - 1, K - 1]
