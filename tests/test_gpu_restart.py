"""Restart file and list-file lines (cadmas_restart_*, cadmas_list_step).

The reference cannot run here (no Fortran compiler), so no .rsl file of
its own exists to compare with.  The layout is restated below from
vf_or1ini.f:38-86, vf_or1trn.f:104-221 and vf_ir1inp.f:96-336 as a plain
reader of Fortran unformatted sequential records (4-byte little-endian
byte counts around each record, as gfortran writes them), independent of
the library's writer, and every record is checked against the state the
library reports.  A restart from the file must continue bit for bit like
the run that wrote it.
"""
import re

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def records(path):
    """The records of a Fortran unformatted sequential file."""
    data = open(path, "rb").read()
    out, pos = [], 0
    while pos < len(data):
        n = int.from_bytes(data[pos:pos + 4], "little", signed=True)
        rec = data[pos + 4:pos + 4 + n]
        tail = int.from_bytes(data[pos + 4 + n:pos + 8 + n], "little", signed=True)
        assert tail == n and len(rec) == n
        out.append(rec)
        pos += 8 + n
    return out


def parse(path, ni, nj, nk, nb, idrop):
    """Header and outputs of a restart file, NPROCS = 1 (vf_or1ini.f,
    vf_or1trn.f)."""
    R = records(path)
    n = ni * nj * nk
    ver = np.frombuffer(R[0], "<i4")
    dims = np.frombuffer(R[1], "<i4")
    flags = np.frombuffer(R[2], "<i4")
    ggv = np.frombuffer(R[3], "<f8")
    assert ver.tolist() == [0, 1]
    assert dims.tolist() == [ni, nj, nk, nb]
    assert flags.tolist() == [1, 1, 1, 1, 0, 0, 0, 0, 1 if idrop else 0, 0]
    assert ggv.size == n
    outs, i = [], 4
    while i < len(R):
        o = {}
        o["nnow"] = int(np.frombuffer(R[i][:4], "<i4")[0])
        o["tnow"], o["dtnow"] = np.frombuffer(R[i][4:20], "<f8").tolist()
        sums = R[i + 1]
        o["fsum"], o["fcut"], o["cgbnrm"], o["cgxnrm"] = np.frombuffer(sums[:32], "<f8").tolist()
        o["icgitr"] = int(np.frombuffer(sums[32:36], "<i4")[0])
        o["nf"] = np.frombuffer(R[i + 2], "<i4")
        names = ["uu", "bcu", "vv", "bcv", "ww", "bcw", "pp", "bcp", "ff", "bcf"]
        for k, nm in enumerate(names):
            o[nm] = np.frombuffer(R[i + 3 + k], "<f8")
        o["tbub"] = np.frombuffer(R[i + 13], "<f8")
        i += 14
        if idrop:
            nd = int(np.frombuffer(R[i], "<i4")[0])
            i += 1
            o["drops"] = []
            for _ in range(nd):
                ijk = np.frombuffer(R[i][:12], "<i4").tolist()
                vals = np.frombuffer(R[i][12:60], "<f8").tolist()
                o["drops"].append((ijk, vals))
                i += 1
        outs.append(o)
    return ggv, outs


def e12_5(v):
    """Fortran 1PE12.5."""
    t = f"{v:.5E}"
    m, e = t.split("E")
    t = m + ("E" + e if len(e) <= 3 else e)
    return t.rjust(12)


def test_restart_file_layout_and_continuation(gpu_lib, pkg, tmp_path):
    c = pkg.cases.droplet_tank(2)
    path = tmp_path / "droplets.rsl"
    t = pkg.Tank(c)
    t.init_state(True)
    t.set_drop(c.drop_state)
    t.restart_create(path)
    kept = {}
    for n in range(1, 7):
        t.step(c.dt)
        if n in (3, 6):
            t.restart_append(path)
            kept[n] = (t.get_state(), t.get_drop(), t.stats())
    ggv, outs = parse(path, c.ni, c.nj, c.nk, c.numb, 1)
    np.testing.assert_array_equal(ggv, c.ggv.reshape(-1, order="F"))
    assert [o["nnow"] for o in outs] == [3, 6]
    for o in outs:
        st, dr, stats = kept[o["nnow"]]
        assert o["tnow"] == st["tnow"] and o["dtnow"] == c.dt
        for k in ("fsum", "fcut", "cgbnrm", "cgxnrm", "icgitr"):
            assert o[k] == stats[k], k
        for k in ("nf", "uu", "vv", "ww", "pp", "ff", "bcu", "bcv", "bcw", "bcp", "bcf", "tbub"):
            assert o[k].tobytes() == np.ascontiguousarray(st[k]).reshape(-1, order="F").tobytes(), k
        cells = np.nonzero(dr["droptx"] >= 0.0)[0]
        # interior cells in K, J, I order (column-major order of the arrays)
        cells = [q for q in cells if 0 < q % c.ni < c.ni - 1 and 0 < (q // c.ni) % c.nj < c.nj - 1
                 and 0 < q // (c.ni * c.nj) < c.nk - 1]
        assert len(o["drops"]) == len(cells) > 0
        for (ijk, vals), q in zip(o["drops"], cells):
            assert ijk == [q % c.ni + 1, (q // c.ni) % c.nj + 1, q // (c.ni * c.nj) + 1]
            assert vals == [dr[k][q] for k in pkg.DROP_ARRAYS]
    # restart from step 3 and run to step 6: the same state bit for bit
    u = pkg.Tank(c)
    u.init_state(True)
    u.restart_load(path, 3)
    su = u.get_state()
    assert su["nnow"] == 3 and su["tnow"] == kept[3][0]["tnow"]
    for n in range(3):
        u.step(c.dt)
    s6, d6, _ = kept[6]
    got = u.get_state()
    for k in ("nf", "indc", "uu", "vv", "ww", "pp", "ff", "bcu", "bcv", "bcw", "bcp", "bcf"):
        assert got[k].tobytes() == s6[k].tobytes(), k
    gd = u.get_drop()
    for k in pkg.DROP_ARRAYS:
        assert gd[k].tobytes() == d6[k].tobytes(), k


def test_restart_errors(gpu_lib, pkg, tmp_path):
    c = pkg.cases.droplet_tank(0)
    path = tmp_path / "a.rsl"
    t = pkg.Tank(c)
    t.init_state(True)
    t.restart_create(path)
    t.step(c.dt)
    t.restart_append(path)
    with pytest.raises(pkg.CadmasError, match="INVALID STEP"):
        t.restart_load(path, 7)
    other = pkg.cases.droplet_tank(0, nx=20)
    u = pkg.Tank(other)
    u.init_state(True)
    with pytest.raises(pkg.CadmasError, match="INVALID NUMBER OF GRID"):
        u.restart_load(path, 1)
    with pytest.raises(pkg.CadmasError, match="CAN NOT OPEN"):
        t.restart_load(tmp_path / "missing.res", 1)


def test_list_step_lines(gpu_lib, pkg):
    c = pkg.cases.random_tank(3)
    t = pkg.Tank(c)
    t.init_state(True)
    for _ in range(3):
        t.step(c.dt)
    text = t.list_step()
    st, s = t.get_state(), t.stats()
    dv = t.divnorm()
    want = (f" STEP={st['nnow']:6d} : TIME= {e12_5(st['tnow'])} : DT  = {e12_5(c.dt)}"
            f" : FSUM= {e12_5(s['fsum'])} : FCUT= {e12_5(s['fcut'])} : !VD!= {e12_5(dv)}\n"
            f" {' ' * 11} : !B! = {e12_5(s['cgbnrm'])} : !R! = {e12_5(s['cgxnrm'])} : ITR = {s['icgitr']:6d}\n")
    assert text == want
    assert re.fullmatch(r" STEP= {0,5}\d+ : TIME= .{12} : DT  = .{12} : FSUM= .{12} : FCUT= .{12} : !VD!= .{12}",
                        text.splitlines()[0])


@pytest.mark.parametrize("builder", ["open_flume", "fixed_level_flume"])
def test_restart_continues_wave_and_open_boundaries(gpu_lib, pkg, tmp_path, builder):
    """The open boundary blends from the stored BCU/BCV/BCW and the fixed
    level follows TNOW, both of which the restart records carry
    (vf_or1trn.f:102-118): a run restarted at step 4 reaches step 10 bit
    for bit."""
    c = getattr(pkg.cases, builder)(nx=64, ny=4, nz=40) if builder == "open_flume" else \
        pkg.cases.fixed_level_flume(nx=48, nz=40, amp=0.04, T=2.0)
    path = tmp_path / "b.rsl"
    t = pkg.Tank(c)
    t.init_state(True)
    t.restart_create(path)
    for n in range(1, 11):
        t.step(c.dt)
        if n == 4:
            t.restart_append(path)
    ref = t.get_state()
    u = pkg.Tank(c)
    u.init_state(True)
    u.restart_load(path, 4)
    for n in range(6):
        u.step(c.dt)
    got = u.get_state()
    for k in ("nf", "indc", "uu", "vv", "ww", "pp", "ff", "bcu", "bcv", "bcw", "bcp", "bcf"):
        assert got[k].tobytes() == ref[k].tobytes(), k
