"""Open (radiation) boundary, MODEL OPEN-BC (vf_bwuwn.f:481-598), in the
oracle and in the library's host set-up.

- The phase speed C = L/T (VF_COMAK0, vf_comak0.f:31-55) solves the linear
  dispersion relation w^2 = g k tanh(k D) in shallow, intermediate and deep
  water, and the library's host function gives the oracle's bits.
- One oracle step moves every X+ open face as VF_BWUWN's blend says,
  computed here in numpy from the state before the step: the normal value
  toward the face one cell inside with ALN = min(C dt / dx, 1), the
  tangential ones toward the cell-centre averages with ALT = min(2 ALN, 1),
  zero next to non-fluid cells, and surface cells' faces copied from the
  face below or above.
- A side cannot be both a wave maker and open.
"""
import numpy as np
import pytest


@pytest.mark.parametrize("depth,T", [(0.05, 8.0), (0.4, 1.2), (3.0, 2.0), (20.0, 1.0)])
def test_phase_speed_solves_the_dispersion_relation(orc, pkg, depth, T):
    c = orc.open_speed(depth, T)
    k, w = 2.0 * np.pi / (c * T), 2.0 * np.pi / T
    assert abs(w * w - 9.8 * k * np.tanh(k * depth)) <= 1e-12 * w * w
    assert pkg.open_speed(depth, T) == c  # same bits from the library's host code
    assert c <= np.sqrt(9.8 * depth) * (1.0 + 1e-12)  # below the shallow-water speed


@pytest.mark.parametrize("bad", [(0.0, 1.0), (-1.0, 1.0), (1.0, 0.0), (1.0, -2.0)])
def test_phase_speed_rejects_bad_input(orc, pkg, bad):
    assert orc.open_speed(*bad) is None
    with pytest.raises(pkg.CadmasError):
        pkg.open_speed(*bad)


def _faces_x(c, I):
    """(J, K, L) of the boundary faces INDX(I, J, K) = L >= 1 of type 7."""
    out = []
    for K in range(2, c.nk):
        for J in range(2, c.nj):
            L = int(c.indx[I - 1, J - 1, K - 1])
            if L >= 1 and c.indb[2, L - 1] == 7:
                out.append((J, K, L))
    return out


def test_one_step_moves_open_faces_as_the_reference_blend(orc, pkg):
    c = pkg.cases.open_flume(nx=64, ny=4, nz=48, seed=2)
    o = orc.Oracle(c)
    o.init_state(True)
    for _ in range(6):
        o.step(c.dt)
    s0 = o.get_state()
    o.step(c.dt)
    s1 = o.get_state()
    C = orc.open_speed(c.open[0]["depth"], c.open[0]["period"])
    NI = c.ni
    I, IC, I2 = NI, NI - 1, NI - 1
    aln = min(C * c.dt / c.xx[1, IC - 1], 1.0)
    alt = min(aln * 2.0, 1.0)
    assert 0.0 < aln < 1.0
    faces = _faces_x(c, I)
    assert len(faces) == (c.nj - 2) * (c.nk - 2)
    at = lambda a, i, j, k: a[i - 1, j - 1, k - 1]
    nf0 = s0["nf"]
    exp_u, exp_v, exp_w = {}, {}, {}
    for J, K, L in faces:
        if at(nf0, IC, J, K) == 0:
            vc = (at(s0["vv"], IC, J, K) + at(s0["vv"], IC, J + 1, K)) * 0.5
            wc = (at(s0["ww"], IC, J, K) + at(s0["ww"], IC, J, K + 1)) * 0.5
            exp_u[L] = (1.0 - aln) * s0["bcu"][L - 1] + aln * at(s0["uu"], I2, J, K)
            exp_v[L] = (1.0 - alt) * s0["bcv"][L - 1] + alt * vc
            exp_w[L] = (1.0 - alt) * s0["bcw"][L - 1] + alt * wc
        else:
            exp_u[L] = exp_v[L] = exp_w[L] = 0.0
    ncopy = 0
    for J, K, L in faces:  # surface cells: the face below (NF 5) or above (NF 6)
        n = at(nf0, IC, J, K)
        if n in (5, 6):
            L2 = int(at(c.indx, I, J, K - 1 if n == 5 else K + 1))
            exp_u[L], exp_v[L], exp_w[L] = exp_u[L2], exp_v[L2], exp_w[L2]
            ncopy += 1
    assert ncopy > 0
    nfluid = sum(at(nf0, IC, J, K) == 0 for J, K, _ in faces)
    assert nfluid > 0
    for J, K, L in faces:
        assert s1["bcu"][L - 1] == exp_u[L], (J, K)
        assert s1["bcv"][L - 1] == exp_v[L], (J, K)
        assert s1["bcw"][L - 1] == exp_w[L], (J, K)


def test_wave_and_open_on_one_side_are_refused(orc, pkg):
    c = pkg.cases.open_flume(nx=32, ny=4, nz=32, depth=0.2, H=0.02)
    c.open = [dict(side=1, depth=0.2, period=1.2)]  # side 1 is the wave maker
    with pytest.raises(pkg.CadmasError):
        orc.Oracle(c)


def test_open_faces_without_an_open_side_are_refused(orc, pkg):
    c = pkg.cases.open_flume(nx=32, ny=4, nz=32, depth=0.2, H=0.02)
    c.open = None
    o = orc.Oracle(c)
    with pytest.raises(pkg.CadmasError):
        o.init_state(True)
