"""Generate tests/golden/oracle_pins.json: SHA-256 pins of the oracle's
state after a few steps of small cases, in the reference summation order.

The reference ships no tests, golden outputs or example cases and cannot be
compiled here (no Fortran compiler), so these pins do not come from the
reference itself: they freeze the CPU restatement so that any change to it
shows up, and the GPU parity tests compare against the same restatement.
Run from the repository root:  python tests/golden/make_golden.py
"""
import hashlib
import json
import pathlib
import sys

ROOT = pathlib.Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT / "tests"))
from conftest import load_oracle, load_pkg  # noqa: E402

CASES = {
    "dam_break_10": dict(builder="dam_break", kw={}, steps=10, sum_mode=0, over={}),
    "dam_break_10_gpuorder": dict(builder="dam_break", kw={}, steps=10, sum_mode=1, over={}),
    "random_tank_3_8": dict(builder="random_tank", kw=dict(seed=3), steps=8, sum_mode=0, over={}),
    "random_tank_7_8_tiles": dict(builder="random_tank", kw=dict(seed=7), steps=8, sum_mode=0,
                                  over=dict(precond_ti=4, precond_tj=3)),
    "porous_flume_small_5": dict(builder="porous_flume",
                                 kw=dict(nx=40, ny=4, nz=24, dx=0.05, dz=0.025, depth=0.3,
                                         block=(0.8, 1.2, 0.35), sponge_width=0.5, dt=2e-3),
                                 steps=5, sum_mode=0, over={}),
    "bubble_tank_6": dict(builder="random_tank", kw=dict(seed=9), steps=6, sum_mode=0,
                          over=dict(wbub=0.2)),
    "droplet_tank_0_20": dict(builder="droplet_tank", kw=dict(seed=0), steps=20, sum_mode=0, over={}),
    # FF-SLOPE advection of F (ISCMFF = 1, VF_FCONVS)
    "ffslope_tank_1_20": dict(builder="random_tank", kw=dict(seed=1), steps=20, sum_mode=0,
                              over=dict(iscmff=1)),
    "ffslope_dam_break_10": dict(builder="dam_break", kw={}, steps=10, sum_mode=0, over=dict(iscmff=1)),
    # k-epsilon (LEQK = 1) with random k, e boundary types
    "turbulent_tank_0_10": dict(builder="turbulent_tank", kw=dict(seed=0), steps=10, sum_mode=0, over={}),
    # log-law (6) and rough (8) walls, without and with k-epsilon (VF_BWKELG)
    "loglaw_tank_1_20": dict(builder="loglaw_tank", kw=dict(seed=1), steps=20, sum_mode=0, over={}),
    "loglaw_turb_tank_2_10": dict(builder="loglaw_tank", kw=dict(seed=2, turb=True), steps=10, sum_mode=0,
                                  over={}),
    # fixed water level at X- (MTBTYP 3), open X+
    "fixed_level_flume_20": dict(builder="fixed_level_flume", kw=dict(nx=48, nz=40, amp=0.04, T=2.0), steps=20,
                                 sum_mode=0, over={}),
    # wave maker at X-, open (radiation) boundaries at X+ and Y+
    "open_flume_0_10": dict(builder="open_flume", kw=dict(nx=64, ny=4, nz=48, y_open=True), steps=10,
                            sum_mode=0, over={}),
    # wave source line (MODEL WAVE-SRC ... FUNC MATRIX) along x
    "source_flume_x_40": dict(builder="source_flume", kw=dict(nx=64, nz=32, ramp=0.2), steps=40, sum_mode=0,
                              over={}),
}
DROP = ("droptx", "dropty", "droptz", "dropuu", "dropvv", "dropww")
TURB = ("ak", "ae", "anut", "anu", "bck", "bce")
FIELDS = ("uu", "vv", "ww", "pp", "ff", "nf", "indc", "bcu", "bcv", "bcw", "bcp", "bcf")


def digest(arrs):
    return {n: hashlib.sha256(arrs[n].tobytes(order="F")).hexdigest()[:32] for n in FIELDS}


def run(name, spec):
    P = load_pkg()
    O = load_oracle()
    c = getattr(P.cases, spec["builder"])(**spec["kw"])
    o = O.Oracle(c, sum_mode=spec["sum_mode"], **spec["over"])
    o.init_state(c.hydrostatic)
    drops = getattr(c, "drop_state", None)
    if drops is not None:  # droplets already in flight (cases.droplet_tank)
        o.set_drop(drops)
    for _ in range(spec["steps"]):
        o.step(c.dt)
    st = o.stats()
    dig = digest(o.get_state())
    if drops is not None:
        d = o.get_drop()
        dig.update({n: hashlib.sha256(d[n].tobytes()).hexdigest()[:32] for n in DROP})
    if c.params.get("leqk", 0):
        t = o.get_turb()
        dig.update({n: hashlib.sha256(t[n].tobytes()).hexdigest()[:32] for n in TURB})
    return dict(digest=dig, stats={k: st[k] for k in ("fsum", "fcut", "cgbnrm", "cgxnrm", "icgitr", "nums")})


if __name__ == "__main__":
    out = {name: run(name, spec) for name, spec in CASES.items()}
    p = pathlib.Path(__file__).with_name("oracle_pins.json")
    p.write_text(json.dumps(out, indent=1, sort_keys=True) + "\n")
    print(p)
