"""Case builder (host-side set-up) checks on CPU."""
import numpy as np


def test_grid_metrics_uniform(pkg):
    x = pkg.cases.grid_metrics(np.arange(5) * 0.5)
    assert x.shape == (6, 6)
    np.testing.assert_allclose(x[1], 0.5)
    np.testing.assert_allclose(x[3], 2.0)
    assert x[2, 0] == 0 and x[4, 0] == 0 and x[5, 0] == 0
    np.testing.assert_allclose(x[2, 1:], 0.5)
    np.testing.assert_allclose(x[5, 1:], 1.0)
    assert x[0, 0] == -0.5


def test_dam_break_layout(pkg):
    c = pkg.cases.dam_break()
    assert (c.ni, c.nj, c.nk) == (66, 10, 34)
    # closed box: every wall face of the interior is a boundary face
    nwall = 2 * (8 * 32) + 2 * (64 * 32) + 2 * (64 * 8)
    assert c.numb == nwall
    assert (c.indb[2] == pkg.cases.VP_SLIP).all() and (c.indb[3] == pkg.cases.F_FREE).all()
    assert set(np.unique(c.indb[1])) == {1, 2, 3, 4, 5, 6}
    # water only where x < 0.16 and z < 0.16
    vol = (c.ff[1:-1, 1:-1, 1:-1] * 1e-6).sum()
    assert abs(vol - 0.16 * 0.08 * 0.16) < 1e-12


def test_boundary_numbering_order(pkg):
    c = pkg.cases.random_tank(5)
    flat = lambda a: a.reshape(-1, order="F")
    nums = np.concatenate([flat(c.indx)[flat(c.indx) > 0], flat(c.indy)[flat(c.indy) > 0],
                           flat(c.indz)[flat(c.indz) > 0]])
    np.testing.assert_array_equal(nums, np.arange(1, c.numb + 1))
    # INDB(1) decodes back to the face position
    for L in range(1, c.numb + 1, 7):
        ijk = c.indb[0, L - 1]
        k = (ijk - 1) // (c.ni * c.nj) + 1
        r = ijk - c.ni * c.nj * (k - 1)
        j = (r - 1) // c.ni + 1
        i = r - c.ni * (j - 1)
        ns = c.indb[1, L - 1]
        ind = (c.indx, c.indx, c.indy, c.indy, c.indz, c.indz)[ns - 1]
        assert ind[i - 1, j - 1, k - 1] == L


def test_inertia_fast_matches_loop(pkg):
    c1 = pkg.cases.random_tank(11)
    g = (c1.glx.copy(), c1.gly.copy(), c1.glz.copy(), c1.glv.copy())
    pkg.cases.build_inertia_fast(c1)
    for a, b in zip(g, (c1.glx, c1.gly, c1.glz, c1.glv)):
        np.testing.assert_array_equal(a, b)
