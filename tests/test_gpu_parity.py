"""GPU library against the oracle, through the C ABI.

The oracle runs in the GPU's summation order (the only order-dependent
values are global sums), the library is compiled with --fmad=false, and
every per-cell expression keeps the Fortran operand order, so the state
after every step must be bit-identical: tolerance 0 on every field, on
NF/INDC and on the step statistics.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FIELDS = ("uu", "vv", "ww", "pp", "ff", "nf", "indc", "bcu", "bcv", "bcw", "bcp", "bcf")


def assert_same(ga, oa, where):
    for n in FIELDS:
        a, b = ga[n], oa[n]
        if a.tobytes() != b.tobytes():
            bad = np.argwhere(a != b)
            d = np.abs(a.astype(np.float64) - b.astype(np.float64)).max()
            raise AssertionError(f"{where}: {n} differs at {bad.shape[0]} places, first {bad[:3].tolist()}, max |d| {d}")


def run_pair(pkg, orc, case, steps, check_every=1, **over):
    t = pkg.Tank(case, **over)
    o = orc.Oracle(case, sum_mode=orc.SUM_GPU, **over)
    t.init_state(case.hydrostatic)
    o.init_state(case.hydrostatic)
    assert_same(t.get_state(), o.get_state(), "init")
    for n in range(1, steps + 1):
        t.step(case.dt)
        o.step(case.dt)
        if n % check_every == 0 or n == steps:
            assert_same(t.get_state(), o.get_state(), f"step {n}")
            sg, so = t.stats(), o.stats()
            for k in ("fsum", "fcut", "cgbnrm", "cgxnrm", "icgitr", "nums"):
                assert sg[k] == so[k], (n, k, sg[k], so[k])
    return t, o


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_droplets_bitwise(gpu_lib, pkg, orc, seed):
    """The TimerDoor droplet model (VF_FDROPF, k_drop.cu) with droplets
    already in flight: every field, flag and droplet array equals the
    oracle's bit for bit."""
    c = pkg.cases.droplet_tank(seed)
    t = pkg.Tank(c)
    o = orc.Oracle(c, sum_mode=orc.SUM_GPU)
    t.init_state(True)
    o.init_state(True)
    t.set_drop(c.drop_state)
    o.set_drop(c.drop_state)
    moved = 0
    for n in range(1, 31):
        t.step(c.dt)
        o.step(c.dt)
        if n % 5 == 0:
            assert_same(t.get_state(), o.get_state(), f"step {n}")
            dg, do = t.get_drop(), o.get_drop()
            for k in pkg.DROP_ARRAYS:
                assert dg[k].tobytes() == do[k].tobytes(), (n, k, np.abs(dg[k] - do[k]).max())
            moved = max(moved, int((dg["droptx"] > -1e9).sum()))
            assert t.stats()["fsum"] == o.stats()["fsum"]
    assert moved >= 7  # droplets were present throughout


def test_dam_break_bitwise(gpu_lib, pkg, orc):
    c = pkg.cases.dam_break()
    t, o = run_pair(pkg, orc, c, 30, check_every=5)
    assert t.divnorm() == o.divnorm()


@pytest.mark.parametrize("seed", [0, 1, 2, 3, 5, 8])
def test_random_tanks_bitwise(gpu_lib, pkg, orc, seed):
    c = pkg.cases.random_tank(seed)
    run_pair(pkg, orc, c, 8)


def test_block_jacobi_preconditioner_bitwise(gpu_lib, pkg, orc):
    c = pkg.cases.dam_break()
    run_pair(pkg, orc, c, 10, check_every=5, precond_ti=16, precond_tj=4)


@pytest.mark.parametrize("solver,occ", [(0, 2), (1, 2), (1, 4)])
def test_two_sweep_blocks_per_sm_bitwise(gpu_lib, pkg, orc, solver, occ):
    """Two thread blocks of the MILU sweeps per SM (sweep_occupancy 2, a
    shallower ring under a register cap), or four for the FP32 backward
    sweeps (sweep_occupancy 4), change the schedule only: the FP64 run
    equals the oracle bit for bit, and the mixed solver's run equals the
    same run with one block per SM bit for bit."""
    c = pkg.cases.porous_flume(nx=96, ny=32, nz=30, dx=0.05, dz=0.025, depth=0.4,
                               block=(1.2, 1.8, 0.5), sponge_width=0.6, dt=2e-3)
    over = dict(precond_ti=16, precond_tj=16, cgepsr=1e-10)
    if solver == 0:
        run_pair(pkg, orc, c, 6, check_every=3, sweep_occupancy=2, **over)
        return
    a = pkg.Tank(c, solver=1, sweep_occupancy=occ, **over)
    b = pkg.Tank(c, solver=1, sweep_occupancy=1, **over)
    for t in (a, b):
        t.init_state(True)
    for n in range(4):
        a.step(c.dt)
        b.step(c.dt)
        assert_same(a.get_state(), b.get_state(), f"mixed step {n}")


def test_porous_flume_with_sponge_bitwise(gpu_lib, pkg, orc):
    c = pkg.cases.porous_flume(nx=64, ny=6, nz=30, dx=0.05, dz=0.025, depth=0.4,
                               block=(1.2, 1.8, 0.5), sponge_width=0.6, dt=2e-3)
    run_pair(pkg, orc, c, 10, check_every=5)


def test_bubble_rise_bitwise(gpu_lib, pkg, orc):
    c = pkg.cases.random_tank(9)
    run_pair(pkg, orc, c, 6, wbub=0.2)


def test_ilu_bitwise(gpu_lib, pkg, orc):
    c = pkg.cases.random_tank(4)
    run_pair(pkg, orc, c, 4, icgtyp=0)


def test_solver_alone_through_c_abi(gpu_lib, pkg, orc):
    """cadmas_m1bcgs_dev on device buffers equals VF_M1BCGS of the oracle."""
    import torch
    c = pkg.cases.random_tank(4)
    o = orc.Oracle(c, sum_mode=orc.SUM_GPU)
    o.init_state(True)
    o.step(c.dt)
    indc = o.get_state()["indc"]      # flags the next system is assembled with
    o.step(c.dt)
    sysa = [o.poisson(w) for w in range(8)]
    xo, ito, bno, xno = o.m1bcgs(*sysa, np.zeros_like(sysa[0]), indc)
    t = pkg.Tank(c)
    dev = [torch.from_numpy(a.reshape(-1, order="F").copy()).cuda() for a in sysa]
    x = torch.zeros_like(dev[0])
    ic = torch.from_numpy(indc.reshape(-1, order="F").copy()).cuda()
    it, bn, xn = pkg.m1bcgs_dev(t, *[d.data_ptr() for d in dev], x.data_ptr(), ic.data_ptr())
    assert (it, bn, xn) == (ito, bno, xno)
    assert np.array_equal(x.cpu().numpy(), xo.reshape(-1, order="F"))


def test_not_converged_status(gpu_lib, pkg):
    c = pkg.cases.dam_break()
    t = pkg.Tank(c, icgmax=1)
    t.init_state(True)
    with pytest.raises(pkg.CadmasError) as e:
        t.step(c.dt)
    assert e.value.status == pkg.ENOTCONV


def test_pivot_failure_status(gpu_lib, pkg):
    """A non-positive MILU pivot gives ITER=-1 ('CAN NOT DECOMPOSITION.')."""
    import torch
    c = pkg.cases.random_tank(1)
    t = pkg.Tank(c)
    t.init_state(True)
    n = c.ni * c.nj * c.nk
    indc = torch.from_numpy(t.get_state()["indc"].reshape(-1, order="F").copy()).cuda()
    ad = torch.full((n,), -1.0, dtype=torch.float64, device="cuda")
    z = [torch.zeros(n, dtype=torch.float64, device="cuda") for _ in range(7)]
    x = torch.zeros(n, dtype=torch.float64, device="cuda")
    it, bn, xn = pkg.m1bcgs_dev(t, ad.data_ptr(), *[q.data_ptr() for q in z[:6]], z[6].data_ptr(),
                                x.data_ptr(), indc.data_ptr())
    assert it == -1 and bn == 0.0 and xn == 0.0


def test_wave_maker_flume_bitwise(gpu_lib, pkg, orc):
    """Wave-maker inflow (matrix table, X- side, fade-in over one period)
    into the porous flume: VF_BWUWN's wave part on the GPU, bit for bit."""
    c = pkg.cases.porous_flume(nx=96, ny=4, nz=64, block=(1.2, 1.4, 0.6), sponge_width=0.4)
    pkg.cases.wave_maker(c, 0.08, 1.5, 0.5, ramp=1.0)
    run_pair(pkg, orc, c, 24, check_every=8)


def test_open_flume_bitwise(gpu_lib, pkg, orc):
    """Wave maker at X- and a radiation outlet at X+ (MODEL OPEN-BC,
    VF_BWUWN vf_bwuwn.f:481-598 in k_open) with a wave train and seeded
    velocity noise in the flume: bit for bit."""
    c = pkg.cases.open_flume()
    run_pair(pkg, orc, c, 24, check_every=8)


def test_open_flume_two_open_sides_tiles_bitwise(gpu_lib, pkg, orc):
    """Open X+ and Y+ sides (the Y form of the blend), 16x8 blocks."""
    c = pkg.cases.open_flume(nx=96, ny=16, nz=48, depth=0.3, H=0.05, seed=1, y_open=True)
    run_pair(pkg, orc, c, 16, check_every=8, precond_ti=16, precond_tj=8)


@pytest.mark.parametrize("seed", [0, 1, 3])
def test_loglaw_walls_bitwise(gpu_lib, pkg, orc, seed):
    """Log-law (6) and rough (8) walls (VF_BWUWT's wall functions with the
    series logarithm, vf_bwuwt.f:116-176) in a random tank with a seeded
    flow: bit for bit."""
    c = pkg.cases.loglaw_tank(seed)
    run_pair(pkg, orc, c, 20, check_every=5)


@pytest.mark.parametrize("seed", [2, 4])
def test_loglaw_walls_with_turbulence_bitwise(gpu_lib, pkg, orc, seed):
    """The same with k-epsilon: VF_BWKELG fused into the k-e step and after
    F1CAL; k, e, ANUT, ANU and their boundary values bit for bit too."""
    c = pkg.cases.loglaw_tank(seed, turb=True)
    t, o = run_pair(pkg, orc, c, 16, check_every=4)
    tg, to = t.get_turb(), o.get_turb()
    for k in ("ak", "ae", "anut", "anu", "bck", "bce"):
        assert tg[k].tobytes() == to[k].tobytes(), k


def test_loglaw_walls_larger_tank_tiles_bitwise(gpu_lib, pkg, orc):
    c = pkg.cases.loglaw_tank(5, turb=True, nx=40, ny=20, nz=24)
    run_pair(pkg, orc, c, 10, check_every=5, precond_ti=16, precond_tj=8)


def test_fixed_level_flume_bitwise(gpu_lib, pkg, orc):
    """Fixed water level at X- (MTBTYP 3: free faces in VF_BWUWN, VF_VPCOEF,
    VF_VMODIF and VF_BWUWT, F from the level in VF_BWFFSF) and an open X+
    side: bit for bit."""
    c = pkg.cases.fixed_level_flume()
    run_pair(pkg, orc, c, 40, check_every=10)


def test_fixed_level_flume_fade_in_tiles_bitwise(gpu_lib, pkg, orc):
    c = pkg.cases.fixed_level_flume(nx=128, ny=16, nz=40, amp=0.08, T=1.5, ramp=0.5, open_end=False)
    run_pair(pkg, orc, c, 24, check_every=8, precond_ti=16, precond_tj=8)


@pytest.mark.parametrize("side", [3, 4])
def test_fixed_level_on_a_y_side_bitwise(gpu_lib, pkg, orc, side):
    """The Y forms of the fixed-level rules (VF_VPCOEF's y faces,
    VF_VMODIF's y loop, VF_BWUWT's NS 3/4, VF_BWFFSF's y column)."""
    c = pkg.cases.fixed_level_flume(nx=48, ny=24, nz=40, amp=0.05, T=1.5, side=side)
    run_pair(pkg, orc, c, 24, check_every=8, precond_ti=16, precond_tj=8)


def test_open_y_minus_side_bitwise(gpu_lib, pkg, orc):
    """An open Y- side (J = 2, the blend toward J = 3) beside the X+ one."""
    c = pkg.cases.open_flume(nx=64, ny=12, nz=40, depth=0.25, H=0.04, seed=4)
    pkg.cases.open_boundary(c, 0.25, 1.2, side=3)
    run_pair(pkg, orc, c, 20, check_every=5)


def test_all_boundary_models_together_bitwise(gpu_lib, pkg, orc):
    """Wave maker, open outlet, log-law and rough walls, k-epsilon and
    FF-SLOPE in one flume: every field, k, e and the eddy viscosity bit for
    bit."""
    c = pkg.cases.open_flume(nx=96, ny=8, nz=48, depth=0.3, H=0.05, seed=3)
    pkg.cases.turbulence(c)
    pkg.cases.loglaw_walls(c, seed=3)
    t, o = run_pair(pkg, orc, c, 20, check_every=5, iscmff=1, precond_ti=16, precond_tj=8)
    tg, to = t.get_turb(), o.get_turb()
    for k in ("ak", "ae", "anut", "anu", "bck", "bce"):
        assert tg[k].tobytes() == to[k].tobytes(), k


def test_open_faces_need_an_open_side(gpu_lib, pkg):
    c = pkg.cases.open_flume(nx=32, ny=4, nz=32, depth=0.2, H=0.02)
    c.open = None
    t = pkg.Tank(c)
    with pytest.raises(pkg.CadmasError):
        t.init_state(True)
    c.open = [dict(side=1, depth=0.2, period=1.2)]  # side 1 is the wave maker
    with pytest.raises(pkg.CadmasError):
        pkg.Tank(c)


def test_wave_maker_flume_tiles_bitwise(gpu_lib, pkg, orc):
    """The same with a wave train already in the flume, no fade-in and
    16x2 preconditioner blocks."""
    c = pkg.cases.porous_flume(nx=96, ny=4, nz=64, block=(1.2, 1.4, 0.6), sponge_width=0.4)
    pkg.cases.linear_wave_initial(c, 0.08, 1.5, 0.5)
    pkg.cases.wave_maker(c, 0.08, 1.5, 0.5)
    run_pair(pkg, orc, c, 16, check_every=8, precond_ti=16, precond_tj=2)


@pytest.mark.parametrize("case,over", [
    ("flume", dict(precond_ti=16, precond_tj=4, precond_split=2)),
    ("flume10", dict(precond_ti=24, precond_tj=8, precond_split=2)),
    ("dam", dict(precond_split=2)),
    ("tank", dict(precond_ti=6, precond_tj=4, precond_split=2)),
])
def test_split_preconditioner_blocks_bitwise(gpu_lib, pkg, orc, case, over):
    """Each preconditioner block swept by a cluster of two thread blocks
    that pass their boundary row through distributed shared memory: the
    same MILU as one block per preconditioner block, bit for bit (the dot
    products sum over the half-height slabs, as the oracle does).
    flume10: 10 rows in y with 8-row blocks, so the top block has one
    4-row-or-less layout tile and its cluster partner has no tile."""
    if case == "flume":
        c = pkg.cases.porous_flume(nx=96, ny=4, nz=64, block=(1.2, 1.4, 0.6), sponge_width=0.4)
        pkg.cases.linear_wave_initial(c, 0.08, 1.5, 0.5)
        pkg.cases.wave_maker(c, 0.08, 1.5, 0.5)
        steps = 12
    elif case == "flume10":
        c = pkg.cases.porous_flume(nx=72, ny=10, nz=64, block=(0.8, 1.0, 0.6), sponge_width=0.3)
        pkg.cases.linear_wave_initial(c, 0.08, 1.5, 0.5)
        steps = 8
    elif case == "dam":
        c = pkg.cases.dam_break()
        steps = 10
    else:
        c = pkg.cases.random_tank(4, ny=10)
        steps = 10
    run_pair(pkg, orc, c, steps, check_every=steps // 2, **over)


def test_fortran_entry_point(gpu_lib, pkg, orc):
    """vf_step_gpu_ (host arrays in, host arrays out) equals cadmas_step."""
    c = pkg.cases.random_tank(3)
    t = pkg.Tank(c)
    t.init_state(True)
    st = t.get_state()
    t2 = pkg.Tank(c)
    t2.set_state(st)
    t2.step(c.dt)
    ref = t2.get_state()
    lib = gpu_lib
    hp = ctypes.c_void_p(t.h.value)
    dt = ctypes.c_double(c.dt)
    tnow = ctypes.c_double(st["tnow"])
    nnow = ctypes.c_int(st["nnow"])
    dp = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    ip = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))
    rc = lib.vf_step_gpu_(ctypes.byref(hp), ctypes.byref(dt), dp(st["uu"]), dp(st["vv"]), dp(st["ww"]),
                          dp(st["pp"]), dp(st["ff"]), ip(st["nf"]), ip(st["indc"]), dp(st["bcu"]),
                          dp(st["bcv"]), dp(st["bcw"]), dp(st["bcp"]), dp(st["bcf"]), ctypes.byref(tnow),
                          ctypes.byref(nnow))
    assert rc == 0
    assert nnow.value == ref["nnow"] and tnow.value == ref["tnow"]
    assert_same(st, ref, "vf_step_gpu_")


def test_fortran_v1cal_f1cal_entry_points(gpu_lib, pkg):
    """vf_v1cal_gpu_ then vf_f1cal_gpu_, with the time advanced by the
    caller as the reference loop does, equal cadmas_step."""
    c = pkg.cases.random_tank(5)
    t = pkg.Tank(c)
    t.init_state(True)
    st = t.get_state()
    t2 = pkg.Tank(c)
    t2.set_state(st)
    t2.step(c.dt)
    ref = t2.get_state()
    lib = gpu_lib
    hp = ctypes.c_void_p(t.h.value)
    dt = ctypes.c_double(c.dt)
    tnow = ctypes.c_double(st["tnow"] + c.dt)
    nnow = ctypes.c_int(st["nnow"] + 1)
    dp = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    ip = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))
    for fn in (lib.vf_v1cal_gpu_, lib.vf_f1cal_gpu_):
        rc = fn(ctypes.byref(hp), ctypes.byref(tnow), ctypes.byref(dt), ctypes.byref(nnow), dp(st["uu"]),
                dp(st["vv"]), dp(st["ww"]), dp(st["pp"]), dp(st["ff"]), ip(st["nf"]), ip(st["indc"]),
                dp(st["bcu"]), dp(st["bcv"]), dp(st["bcw"]), dp(st["bcp"]), dp(st["bcf"]))
        assert rc == 0
    assert nnow.value == ref["nnow"] and tnow.value == ref["tnow"]
    assert_same(st, ref, "vf_v1cal_gpu_/vf_f1cal_gpu_")


def test_flume_full_size_properties(gpu_lib, pkg):
    """512x32x96 porous flume (block-Jacobi tiles): a few steps keep the
    fluid volume (closed box) and a divergence-free correction."""
    c = pkg.cases.porous_flume()
    pkg.cases.linear_wave_initial(c, 0.08, 1.5, 0.5)
    t = pkg.Tank(c, precond_ti=32, precond_tj=8, diag_relres=1, cgepsr=1e-10)
    t.init_state(True)
    v0 = t.stats()["fsum"]
    cut = 0.0
    for _ in range(3):
        t.step(c.dt)
        s = t.stats()
        cut += s["fcut"]
        assert s["true_relres"] < 1e-8
    assert abs(s["fsum"] + cut - v0) / v0 < 1e-10
    assert np.isfinite(t.divnorm())


@pytest.mark.parametrize("builder,kw,active", [("random_tank", dict(seed=5), False),
                                               ("droplet_tank", dict(seed=1), False), ("dam_break", {}, True)])
def test_adaptive_time_step_bitwise(gpu_lib, pkg, orc, builder, kw, active):
    """VF_CDTCAL: the next step's DT from the GPU equals the oracle's
    (smallest-limit order) bit for bit, and within 1e-13 of the reference's
    running minimum; ten steps each taken with that DT stay bitwise equal."""
    c = getattr(pkg.cases, builder)(**kw)
    t = pkg.Tank(c)
    o = orc.Oracle(c, sum_mode=orc.SUM_GPU)
    r = orc.Oracle(c, sum_mode=orc.SUM_REF)
    for x in (t, o, r):
        x.init_state(c.hydrostatic)
    dt0 = t.cdtcal()
    assert dt0 == o.cdtcal() and abs(dt0 - 1.2e-6) <= 1e-20  # NNOW = 0: 1.2 DTINIT caps it
    dt = c.dt
    # DTSAFE 1e-3: the cells' limits, not the 1.2*DTNOW cap, decide DT
    kw = dict(dtmax=c.dt / 0.1, dtsafe=1.0e-3)
    limited = 0
    for n in range(1, 11):
        t.step(dt)
        o.step(dt)
        dg, do = t.cdtcal(**kw), o.cdtcal(**kw)
        st = o.get_state()
        r.set_state(st)
        r.set_time(st["tnow"], dt, st["nnow"])
        dr = r.cdtcal(**kw)
        assert dg == do, (n, dg, do)
        assert abs(dg - dr) <= 1e-13 * dr
        assert dg <= 1.2 * dt
        limited += dg < 1.2 * dt
        dt = dg
    assert limited > 0 or not active  # the collapsing dam's velocities limit DT
    assert_same(t.get_state(), o.get_state(), "after 10 adaptive steps")


def test_solitary_beach_small_bitwise(gpu_lib, pkg, orc):
    """Config 2's shape at small size: staircase beach, porous boxes and an
    injected solitary wave (set as the initial state), 16x8 blocks."""
    c = pkg.cases.solitary_beach(nx=128, ny=32, nz=48, x_toe=1.0, x0=0.6, amp=0.08, depth=0.3, nbox=6, seed=3,
                                 dt=1.0e-3)
    t = pkg.Tank(c, precond_ti=16, precond_tj=8)
    o = orc.Oracle(c, sum_mode=orc.SUM_GPU, precond_ti=16, precond_tj=8)
    init = pkg.initial_state(c)
    t.set_state(init)
    o.set_state(init)
    t.init_state(c.hydrostatic)
    o.init_state(c.hydrostatic)
    for n in range(1, 13):
        t.step(c.dt)
        o.step(c.dt)
        if n % 4 == 0:
            assert_same(t.get_state(), o.get_state(), f"step {n}")


def test_wave_maker_flume_with_turbulence_bitwise(gpu_lib, pkg, orc):
    """k-epsilon in the porous flume driven by the wave maker."""
    c = pkg.cases.porous_flume(nx=96, ny=4, nz=64, block=(1.2, 1.4, 0.6), sponge_width=0.4)
    pkg.cases.wave_maker(c, 0.08, 1.5, 0.5, ramp=1.0)
    pkg.cases.turbulence(c, 1e-4, 1e-5)
    t, o = run_pair(pkg, orc, c, 16, check_every=8)
    gt, ot = t.get_turb(), o.get_turb()
    for k in ("ak", "ae", "anut", "anu", "bck", "bce"):
        assert gt[k].tobytes() == ot[k].tobytes(), k


def test_ensemble_of_mixed_tile_shapes(gpu_lib, pkg):
    """Handles of different grids and preconditioner block shapes stepped
    together (cadmas_step_ensemble, one host thread each) give exactly what
    each gives stepped alone."""
    shapes = [(16, 16), (8, 8), (16, 8), (32, 8)]
    mk = lambda: [pkg.cases.porous_flume(nx=96 + 32 * i, ny=16, nz=48, depth=0.3, block=(1.0, 1.3, 0.4),
                                         sponge_width=0.4)
                  for i in range(len(shapes))]
    together = [pkg.Tank(c, precond_ti=ti, precond_tj=tj) for c, (ti, tj) in zip(mk(), shapes)]
    alone = [pkg.Tank(c, precond_ti=ti, precond_tj=tj) for c, (ti, tj) in zip(mk(), shapes)]
    for t in together + alone:
        t.init_state(True)
    for _ in range(6):
        pkg.step_ensemble(together)
        for t in alone:
            t.step()
    for a, b in zip(together, alone):
        sa, sb = a.get_state(), b.get_state()
        for k in ("uu", "pp", "ff", "nf"):
            assert sa[k].tobytes() == sb[k].tobytes(), k


@pytest.mark.parametrize("axis", ["x", "y"])
def test_wave_source_bitwise(gpu_lib, pkg, orc, axis):
    """A wave source line (MODEL WAVE-SRC ... FUNC MATRIX: k_srcuv for
    VF_CWMSRC, the source terms of VF_VGENE, VF_VPCOEF, VF_BSUWN and
    VF_FGENE) along x and along y: bit for bit with the oracle, through the
    fade-in and beyond."""
    c = pkg.cases.source_flume(nx=64, nz=32, axis=axis, ramp=0.2)
    t, o = run_pair(pkg, orc, c, 60, check_every=10)
    st = t.get_state()
    assert np.abs(st["ww"]).max() > 1e-3  # the source moves the water


@pytest.mark.parametrize("order", [1, 5])
def test_stream_function_wave_maker_bitwise(gpu_lib, pkg, orc, order):
    """The wave maker driven by the stream-function wave (WAVE-BC ... FUNC
    STREAM N): the level at the phase on the host, the face velocities at
    the scaled heights in k_wave from the wave's series; bit for bit with
    the oracle's own evaluation of the same wave."""
    c = pkg.cases.porous_flume(nx=96, ny=4, nz=64, block=(1.2, 1.4, 0.6), sponge_width=0.4)
    pkg.cases.wave_maker(c, 0.08, 1.5, 0.5, ramp=0.5, stream=order)
    t, o = run_pair(pkg, orc, c, 30, check_every=10)
    assert np.abs(t.get_state()["uu"][1, :, :]).max() > 2e-4  # the wave maker drives the inflow (faded in)


@pytest.mark.parametrize("func,H,T,ramp", [("stokes", 0.08, 1.5, 0.5), ("cnoidal", 0.05, 4.0, 0.05),
                                            ("stk-cnd", 0.05, 4.0, 0.05)])
def test_stokes_cnoidal_wave_maker_bitwise(gpu_lib, pkg, orc, func, H, T, ramp):
    """The wave maker driven by the fifth-order Stokes or the third-order
    cnoidal wave (WAVE-BC ... FUNC STOKES | CNOIDAL | STK-CND, the last
    choosing cnoidal at an Ursell number of 31): the level at the phase and
    the phase's part of the series on the host, the face velocities in
    k_wave; bit for bit with the oracle's evaluation of the same wave."""
    c = pkg.cases.porous_flume(nx=96, ny=4, nz=64, block=(1.2, 1.4, 0.6), sponge_width=0.4)
    pkg.cases.wave_maker(c, H, T, 0.5, ramp=ramp, func=func)
    assert c.wave["theory"].type == (pkg.WAVE_STOKES if func == "stokes" else pkg.WAVE_CNOIDAL)
    t, o = run_pair(pkg, orc, c, 30, check_every=10)
    assert np.abs(t.get_state()["uu"][1, :, :]).max() > 2e-4  # the wave maker drives the inflow (faded in)


@pytest.mark.parametrize("func,side,angle", [(5, 1, (25.0, 0.3, 0.2)), ("stokes", 3, (-30.0, 0.1, 0.4)),
                                             ("cnoidal", 2, (15.0, 0.0, 0.0))])
def test_oblique_wave_maker_bitwise(gpu_lib, pkg, orc, func, side, angle):
    """Oblique incidence (WAVE-BC ... ANGLE a X Y) on an X side and a Y
    side: each line's phase from its distance along the direction of
    travel, its own level and velocities (the table of lines uploaded each
    step), the normal and tangential parts of the face velocity; bit for
    bit with the oracle."""
    c = pkg.cases.porous_flume(nx=48, ny=24, nz=64, block=(0.6, 0.7, 0.3), sponge_width=0.3)
    kw = dict(stream=func) if isinstance(func, int) else dict(func=func)
    H, T, ramp = (0.05, 4.0, 0.02) if func == "cnoidal" else (0.06, 1.5, 0.2)
    pkg.cases.wave_maker(c, H, T, 0.5, side=side, ramp=ramp, angle=angle, **kw)
    t, o = run_pair(pkg, orc, c, 20, check_every=10, precond_ti=16, precond_tj=8)
    st = t.get_state()
    if side <= 2:
        I = 1 if side == 1 else c.ni - 1
        face = st["uu"][I, 1:-1, 10]  # below the still water level, along the side
    else:
        face = st["vv"][1:-1, 1, 10]
    assert np.ptp(face) > 1e-5  # the phase varies along the side


@pytest.mark.parametrize("func", [3, "stokes"])
def test_wave_source_with_a_theory_bitwise(gpu_lib, pkg, orc, func):
    """A wave source line driven by a wave theory (WAVE-SRC ... FUNC STREAM
    N | STOKES): SRCUV from VF_CWMAK2 at the heights scaled to each
    column's level in k_srcuv; bit for bit with the oracle."""
    c = pkg.cases.source_flume(nx=64, nz=32, ramp=0.2, func=func)
    t, o = run_pair(pkg, orc, c, 40, check_every=10)
    assert np.abs(t.get_state()["ww"]).max() > 1e-3  # the source moves the water
