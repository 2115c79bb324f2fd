"""Python host side of libcadmas_gpu.so, the B200 SMAC step of CADMAS-SURF/3D.

This mirrors the per-step driver interface of the reference
(VF_V1CAL, Simulators/CADMAS-SURF-3D/Source code/vf_v1cal.f:1-9, and
VF_F1CAL, vf_f1cal.f:1-20, called once per step from the time loop at
vf_a1main.f:1058 and :1104) over the C ABI declared in
include/cadmas_gpu.h.  Arrays are numpy arrays of shape (NUMI,NUMJ,NUMK) in
Fortran order, exactly the Fortran arrays.  The reference aborts through
VF_A2ERR on an error; here every call raises CadmasError carrying the status
code and the reference's message.

The CUDA library is required: importing this package does not need a GPU,
but creating a Tank without libcadmas_gpu.so, or without a CUDA device,
raises.  There is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import pathlib

import numpy as np

from . import cases  # noqa: F401  (re-exported)

HERE = pathlib.Path(__file__).resolve().parent
LIB_PATH = HERE / "libcadmas_gpu.so"

(OK, EINVAL, ECUDA, ENOTCONV, EDIVERGE, EPIVOT, EPG, ECAP, ENOMEM, EUNSUPPORTED, ENOSTATIC, ETIMEOUT, ESCRATCH,
 EIO, EWAVE) = range(15)

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


class Dims(C.Structure):
    _fields_ = [("numi", C.c_int), ("numj", C.c_int), ("numk", C.c_int), ("numb", C.c_int)]


class WaveTable(C.Structure):
    _fields_ = [("ntt", C.c_int), ("nzz", C.c_int), ("mtbtyp", C.c_int), ("pad", C.c_int),
                ("phase0", C.c_double), ("tt", _dp), ("hh", _dp), ("zz", _dp), ("un", _dp), ("ut", _dp)]


class WaveBC(C.Structure):
    _fields_ = [("side", C.c_int), ("first", C.c_int), ("last", C.c_int), ("pad", C.c_int),
                ("depth", C.c_double), ("period", C.c_double), ("ramp", C.c_double)]


STREAM_NMAX = 22


class StreamWave(C.Structure):
    _fields_ = [("order", C.c_int), ("iterations", C.c_int)] + [
        (n, C.c_double) for n in ("depth", "period", "height", "grav", "k", "length", "celerity", "ubar", "q",
                                  "r", "phase0")] + [("b", C.c_double * STREAM_NMAX)]


def stream_solve(order, depth, period, height, grav=9.8, lib=None) -> StreamWave:
    """The stream-function wave of order N (cadmas_stream_solve, host only)."""
    lib = lib or load_library()
    out = StreamWave()
    lib.cadmas_stream_solve.argtypes = [C.c_int] + [C.c_double] * 4 + [C.POINTER(StreamWave)]
    _check(lib, lib.cadmas_stream_solve(int(order), float(depth), float(period), float(height), float(grav),
                                        C.byref(out)))
    return out


def stream_eval(sw: StreamWave, phase, z=0.0, lib=None):
    """(eta, u, w) of a stream-function wave at `phase` and height z above
    the still water level, as the wave maker uses them (cadmas_stream_eval)."""
    lib = lib or load_library()
    e, u, w = C.c_double(), C.c_double(), C.c_double()
    lib.cadmas_stream_eval.argtypes = [C.POINTER(StreamWave), C.c_double, C.c_double, _dp, _dp, _dp]
    _check(lib, lib.cadmas_stream_eval(C.byref(sw), float(phase), float(z), C.byref(e), C.byref(u), C.byref(w)))
    return e.value, u.value, w.value


WAVE_STK_CND, WAVE_CNOIDAL, WAVE_STOKES = 0, -1, -2
_WAVE_FUNCS = {"stk-cnd": WAVE_STK_CND, "cnoidal": WAVE_CNOIDAL, "stokes": WAVE_STOKES}


class StokesWave(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("kd", "k", "eps", "c0", "c")] + [
        ("a", C.c_double * 5), ("b", C.c_double * 5), ("b0", C.c_double), ("p0", C.c_double),
        ("iterations", C.c_int), ("pad", C.c_int)]


class CnoidalWave(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("ql", "s", "d", "c0", "c")] + [
        ("a", C.c_double * 4), ("b", C.c_double * 12), ("bb", C.c_double * 12), ("p0", C.c_double),
        ("iterations", C.c_int), ("pad", C.c_int)]


class WaveTheory(C.Structure):
    _fields_ = [("type", C.c_int), ("pad", C.c_int)] + [
        (n, C.c_double) for n in ("depth", "period", "height", "length", "ursell", "phase0")] + [
        ("stream", StreamWave), ("stokes", StokesWave), ("cnoidal", CnoidalWave)]


def wave_type(func) -> int:
    """IWVTYP of a wave-theory name ("stokes", "cnoidal", "stk-cnd") or a
    stream-function order N >= 1."""
    if isinstance(func, str):
        return _WAVE_FUNCS[func.lower()]
    return int(func)


def wave_solve(func, depth, period, height, grz0=9.8, lib=None) -> WaveTheory:
    """A wave theory of the wave maker or the wave source (cadmas_wave_solve,
    host only): `func` a stream-function order N or "stokes", "cnoidal",
    "stk-cnd" (the choice by the Ursell number)."""
    lib = lib or load_library()
    out = WaveTheory()
    lib.cadmas_wave_solve.argtypes = [C.c_int] + [C.c_double] * 4 + [C.POINTER(WaveTheory)]
    _check(lib, lib.cadmas_wave_solve(wave_type(func), float(depth), float(period), float(height), float(grz0),
                                      C.byref(out)))
    return out


def wave_eval(th: WaveTheory, phase, z=0.0, lib=None):
    """(eta, u, w) of a wave theory at `phase` and height z above the still
    water level, as the wave maker uses them (cadmas_wave_eval)."""
    lib = lib or load_library()
    e, u, w = C.c_double(), C.c_double(), C.c_double()
    lib.cadmas_wave_eval.argtypes = [C.POINTER(WaveTheory), C.c_double, C.c_double, _dp, _dp, _dp]
    _check(lib, lib.cadmas_wave_eval(C.byref(th), float(phase), float(z), C.byref(e), C.byref(u), C.byref(w)))
    return e.value, u.value, w.value


class WaveSrc(C.Structure):
    _fields_ = [("line", C.c_int), ("pad", C.c_int), ("depth", C.c_double), ("period", C.c_double),
                ("ramp", C.c_double)]


def source_structs(src):
    """(WaveSrc, WaveTable or None, keep-alive arrays) of a case's wave
    source dict (cases.wave_source)."""
    tab, arrs = None, {}
    if src.get("table") is not None:
        _, tab, arrs = wave_structs(dict(side=1, first=2, last=2, depth=src["depth"], period=src["period"],
                                         table=src["table"]))
    ws = WaveSrc(int(src["line"]), 0, float(src["depth"]), float(src["period"]), float(src.get("ramp", 0.0)))
    return ws, tab, arrs


class OpenBC(C.Structure):
    _fields_ = [("side", C.c_int), ("pad", C.c_int), ("depth", C.c_double), ("period", C.c_double)]


def wave_structs(wave):
    """(WaveBC, WaveTable, keep-alive arrays) of a case's wave-maker dict
    (cases.wave_maker)."""
    t = wave["table"]
    arrs = {n: np.ascontiguousarray(t[n], dtype=np.float64) for n in ("tt", "hh", "zz")}
    for n in ("un", "ut"):
        arrs[n] = np.asfortranarray(t[n], dtype=np.float64)  # (MTBZZ, MTBTT)
    tab = WaveTable(len(arrs["tt"]), len(arrs["zz"]), int(t.get("mtbtyp", 1)), 0, float(t.get("phase0", 0.0)),
                    *(arrs[n].ctypes.data_as(_dp) for n in ("tt", "hh", "zz", "un", "ut")))
    bc = WaveBC(int(wave["side"]), int(wave["first"]), int(wave["last"]), 0, float(wave["depth"]),
                float(wave["period"]), float(wave.get("ramp", 0.0)))
    return bc, tab, arrs


class Params(C.Structure):
    _fields_ = [(n, C.c_double) for n in (
        "rho0", "grz0", "vvmax", "cgpara", "cgepsa", "cgepsr", "cgdiv", "flower", "fupper",
        "plower", "scmvp", "wvlvl", "wbub", "glxmin", "glxmax", "glymin", "glymax")] + [
        ("damp", (C.c_double * 4) * 4),
        ("idamp", C.c_int * 4),
        ("icgtyp", C.c_int), ("icgmax", C.c_int), ("ibsuw0", C.c_int),
        ("precond_ti", C.c_int), ("precond_tj", C.c_int),
        ("diag_relres", C.c_int), ("solver", C.c_int), ("warm_start", C.c_int), ("precond_split", C.c_int),
        ("idrop", C.c_int), ("iscmff", C.c_int), ("leqk", C.c_int), ("pad0", C.c_int)] + [
        (n, C.c_double) for n in ("anu0", "scmk", "akmink", "akmine", "akinik", "akinie", "akcmu", "aksgk",
                                  "aksge", "akc1", "akc2", "akc3", "akk0", "aka0",
                                  "mixed_eps_inner", "wait_limit_s")] + [
        ("sweep_occupancy", C.c_int), ("dot_passes", C.c_int)]


class Static(C.Structure):
    _fields_ = [(n, _dp) for n in ("xx", "yy", "zz", "ggv", "ggx", "ggy", "ggz", "glv", "glx",
                                   "gly", "glz", "cd0", "anu")] + [
        (n, _ip) for n in ("indx", "indy", "indz", "indb", "indbk", "indbe")] + [
        (n, _dp) for n in ("bck", "bce", "bcvi")]


class State(C.Structure):
    _fields_ = [(n, _dp) for n in ("uu", "vv", "ww", "pp", "ff")] + [
        ("nf", _ip), ("indc", _ip)] + [(n, _dp) for n in ("bcu", "bcv", "bcw", "bcp", "bcf", "tbub")] + [
        ("tnow", C.c_double), ("nnow", C.c_int)]


class Stats(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("fsum", "fcut", "cgbnrm", "cgxnrm", "divnorm", "true_relres")] + [
        (n, C.c_int) for n in ("icgitr", "nums", "last_status", "fallbacks")]


EXPORTED = ["cadmas_default_params", "cadmas_create", "cadmas_destroy", "cadmas_upload_static",
            "cadmas_set_state", "cadmas_get_state", "cadmas_init_state", "cadmas_step",
            "cadmas_set_time", "cadmas_v1cal", "cadmas_f1cal", "cadmas_divnorm", "cadmas_get_stats",
            "cadmas_sync", "vf_step_gpu_", "vf_v1cal_gpu_", "vf_f1cal_gpu_", "cadmas_m1bcgs_dev",
            "cadmas_strerror", "cadmas_divnorm_noalloc", "cadmas_set_wave", "cadmas_set_open", "cadmas_open_speed", "cadmas_step_ensemble",
            "cadmas_get_stream", "cadmas_kernel_launches", "cadmas_stage_timers", "cadmas_get_drop",
            "cadmas_set_drop", "cadmas_restart_create", "cadmas_restart_append", "cadmas_restart_load",
            "cadmas_list_step", "cadmas_cdtcal", "cadmas_get_turb", "cadmas_set_turb",
            "cadmas_unet_param_count", "cadmas_unet_create", "cadmas_unet_destroy", "cadmas_unet_set_params",
            "cadmas_unet_get_params", "cadmas_unet_forward", "cadmas_unet_grad", "cadmas_unet_train_step",
            "cadmas_set_warm_net", "cadmas_warm_stats", "cadmas_get_solve", "cadmas_get_system",
            "cadmas_unet_train_sys", "cadmas_unet_time_forward", "cadmas_test_stall_sweeps",
            "cadmas_set_wave_source", "cadmas_stream_solve", "cadmas_stream_eval", "cadmas_set_wave_theory",
            "cadmas_wave_solve", "cadmas_wave_eval", "cadmas_set_wave_func", "cadmas_set_wave_angle",
            "cadmas_set_wave_source_func", "cadmas_batch_create", "cadmas_batch_step", "cadmas_batch_destroy"]

DROP_ARRAYS = ("droptx", "dropty", "droptz", "dropuu", "dropvv", "dropww")
TURB_CELLS = ("ak", "ae", "anut", "anu")   # (NUMI,NUMJ,NUMK)
TURB_FACES = ("bck", "bce")                # (NUMB)

STAGES = ["flux", "predict", "vpcoef", "dcmp", "fwd", "bwd", "dot", "vec", "modif", "vof", "flags", "fbc", "turb",
          "warm"]


class CadmasError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"{msg} (status {status})")
        self.status = status


_lib = None


def build_library(force: bool = False, verbose: bool = False) -> pathlib.Path:
    """Compile libcadmas_gpu.so for sm_100a if its sources changed (nvcc)."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("cadmas_b200_build", pathlib.Path(__file__).parent / "build.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod.build(force=force, verbose=verbose)


def load_library(path: pathlib.Path | None = None):
    """Load libcadmas_gpu.so (no GPU needed to load it)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = pathlib.Path(path) if path else LIB_PATH
    if not p.exists():
        raise CadmasError(EINVAL, f"{p} not built: run build.py (nvcc, sm_100a)")
    lib = C.CDLL(str(p))
    lib.cadmas_default_params.argtypes = [C.POINTER(Params)]
    lib.cadmas_default_params.restype = None
    lib.cadmas_create.argtypes = [C.POINTER(Dims), C.POINTER(Params), C.POINTER(C.c_void_p)]
    lib.cadmas_destroy.argtypes = [C.c_void_p]
    lib.cadmas_upload_static.argtypes = [C.c_void_p, C.POINTER(Static)]
    lib.cadmas_set_state.argtypes = [C.c_void_p, C.POINTER(State)]
    lib.cadmas_get_state.argtypes = [C.c_void_p, C.POINTER(State)]
    lib.cadmas_get_drop.argtypes = [C.c_void_p] + [_dp] * 6
    lib.cadmas_restart_create.argtypes = [C.c_void_p, C.c_char_p]
    lib.cadmas_restart_append.argtypes = [C.c_void_p, C.c_char_p]
    lib.cadmas_restart_load.argtypes = [C.c_void_p, C.c_char_p, C.c_int]
    lib.cadmas_list_step.argtypes = [C.c_void_p, C.c_char_p, C.c_size_t]
    lib.cadmas_cdtcal.argtypes = [C.c_void_p] + [C.c_double] * 4 + [C.POINTER(C.c_double)]
    lib.cadmas_set_drop.argtypes = [C.c_void_p] + [_dp] * 6
    lib.cadmas_get_turb.argtypes = [C.c_void_p] + [_dp] * 6
    _fp = C.POINTER(C.c_float)
    lib.cadmas_unet_param_count.restype = C.c_size_t
    lib.cadmas_unet_param_count.argtypes = []
    lib.cadmas_unet_create.argtypes = [C.c_int] * 4 + [C.POINTER(C.c_void_p)]
    lib.cadmas_unet_destroy.argtypes = [C.c_void_p]
    lib.cadmas_unet_set_params.argtypes = [C.c_void_p, _fp]
    lib.cadmas_unet_get_params.argtypes = [C.c_void_p, _fp]
    lib.cadmas_unet_forward.argtypes = [C.c_void_p, _fp, _fp]
    lib.cadmas_unet_time_forward.argtypes = [C.c_void_p, C.c_int, _fp]
    lib.cadmas_unet_grad.argtypes = [C.c_void_p, _fp, _fp, _fp, _fp, _fp]
    lib.cadmas_unet_train_step.argtypes = [C.c_void_p, _fp, _fp, _fp, C.c_float, _fp]
    lib.cadmas_set_warm_net.argtypes = [C.c_void_p, _fp, C.c_double]
    lib.cadmas_get_system.argtypes = [C.c_void_p] + [_dp] * 7
    lib.cadmas_unet_train_sys.argtypes = [C.c_void_p, _fp, _fp, _fp, _fp, C.c_float, C.c_float, C.c_float,
                                          C.c_float, C.c_int, _fp, _fp]
    lib.cadmas_warm_stats.argtypes = [C.c_void_p, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)]
    lib.cadmas_get_solve.argtypes = [C.c_void_p, _dp, _dp]
    lib.cadmas_v1cal.argtypes = [C.c_void_p]
    lib.cadmas_f1cal.argtypes = [C.c_void_p]
    lib.cadmas_set_turb.argtypes = [C.c_void_p] + [_dp] * 4
    lib.cadmas_init_state.argtypes = [C.c_void_p, C.c_int]
    lib.cadmas_step.argtypes = [C.c_void_p, C.c_double]
    lib.cadmas_set_time.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_int]
    lib.cadmas_v1cal.argtypes = [C.c_void_p]
    lib.cadmas_f1cal.argtypes = [C.c_void_p]
    lib.cadmas_divnorm.argtypes = [C.c_void_p, _dp]
    lib.cadmas_get_stats.argtypes = [C.c_void_p, C.POINTER(Stats)]
    lib.cadmas_sync.argtypes = [C.c_void_p]
    lib.cadmas_m1bcgs_dev.argtypes = [C.c_void_p] + [C.c_void_p] * 10 + [_ip, _dp, _dp]
    lib.cadmas_get_stream.argtypes = [C.c_void_p, C.POINTER(C.c_void_p)]
    lib.cadmas_kernel_launches.argtypes = []
    lib.cadmas_kernel_launches.restype = C.c_longlong
    lib.cadmas_stage_timers.argtypes = [C.c_void_p, C.c_int, _dp, C.POINTER(C.c_longlong), C.c_int]
    lib.cadmas_strerror.argtypes = [C.c_int]
    lib.cadmas_strerror.restype = C.c_char_p
    vf = lib.vf_step_gpu_
    vf.argtypes = [C.POINTER(C.c_void_p), _dp] + [_dp] * 5 + [_ip, _ip] + [_dp] * 5 + [_dp, _ip]
    lib.cadmas_divnorm_noalloc.argtypes = [C.POINTER(Dims)] + [C.c_void_p] * 11 + [_dp]
    lib.cadmas_set_wave.argtypes = [C.c_void_p, C.POINTER(WaveBC), C.POINTER(WaveTable)]
    lib.cadmas_set_open.argtypes = [C.c_void_p, C.POINTER(OpenBC)]
    lib.cadmas_open_speed.argtypes = [C.c_double, C.c_double, C.c_double, _dp]
    lib.cadmas_step_ensemble.argtypes = [C.POINTER(C.c_void_p), C.c_int, _dp, _ip]
    if path is None:
        _lib = lib
    return lib


def _check(lib, rc):
    if rc != OK:
        raise CadmasError(rc, lib.cadmas_strerror(rc).decode())


def _dptr(a):
    return a.ctypes.data_as(_dp) if a is not None else None


def _iptr(a):
    return a.ctypes.data_as(_ip) if a is not None else None


def default_params(lib=None) -> Params:
    lib = lib or load_library()
    p = Params()
    lib.cadmas_default_params(C.byref(p))
    return p


def make_params(case, base: Params | None = None, **over) -> Params:
    """cadmas_params for a case: library defaults (vf_a2dflt.f), then the
    case's settings, then keyword overrides."""
    p = base if base is not None else default_params()
    d = dict(case.params)
    d.update(over)
    for k, v in d.items():
        if k in ("idamp",):
            for i in range(4):
                p.idamp[i] = int(v[i])
        elif k.startswith("damp_"):
            jd = {"damp_xm": 0, "damp_xp": 1, "damp_ym": 2, "damp_yp": 3}[k]
            for m in range(4):
                p.damp[jd][m] = float(v[m])
        elif hasattr(p, k):
            setattr(p, k, type(getattr(p, k))(v))
        else:
            raise KeyError(f"unknown parameter {k}")
    return p


def static_of(case) -> Static:
    s = Static()
    for n in ("xx", "yy", "zz", "ggv", "ggx", "ggy", "ggz", "glv", "glx", "gly", "glz", "cd0", "anu"):
        a = getattr(case, n)
        assert a.dtype == np.float64 and (a.flags.f_contiguous or a.ndim == 1)
        setattr(s, n, _dptr(a))
    for n in ("indx", "indy", "indz", "indb"):
        a = getattr(case, n)
        assert a.dtype == np.int32 and a.flags.f_contiguous
        setattr(s, n, _iptr(a))
    # k-epsilon boundaries (read only when leqk != 0)
    for n in ("indbk", "indbe"):
        a = getattr(case, n, None)
        if a is not None:
            assert a.dtype == np.int32 and a.ndim == 1
            setattr(s, n, _iptr(a))
    for n in ("bck", "bce", "bcvi"):
        a = getattr(case, n, None)
        if a is not None:
            assert a.dtype == np.float64 and a.ndim == 1
            setattr(s, n, _dptr(a))
    return s


def new_state_arrays(ni, nj, nk, nb):
    f3 = lambda dt: np.zeros((ni, nj, nk), dtype=dt, order="F")
    nbx = max(nb, 1)
    return dict(uu=f3(np.float64), vv=f3(np.float64), ww=f3(np.float64), pp=f3(np.float64),
                ff=f3(np.float64), nf=f3(np.int32), indc=f3(np.int32),
                bcu=np.zeros(nbx), bcv=np.zeros(nbx), bcw=np.zeros(nbx), bcp=np.zeros(nbx),
                bcf=np.zeros(nbx), tbub=np.zeros(nk), tnow=0.0, nnow=0)


def state_struct(arrs) -> State:
    s = State()
    for n in ("uu", "vv", "ww", "pp", "ff", "bcu", "bcv", "bcw", "bcp", "bcf", "tbub"):
        setattr(s, n, _dptr(arrs.get(n)))
    s.nf = _iptr(arrs.get("nf"))
    s.indc = _iptr(arrs.get("indc"))
    s.tnow = float(arrs.get("tnow", 0.0))
    s.nnow = int(arrs.get("nnow", 0))
    return s


def initial_state(case):
    """Host arrays of the initial state of a case (F, velocities; NF from
    the obstacle map, INDC unset) for cadmas_set_state."""
    st = new_state_arrays(case.ni, case.nj, case.nk, case.numb)
    st["uu"][...] = case.uu
    st["vv"][...] = case.vv
    st["ww"][...] = case.ww
    st["pp"][...] = case.pp
    st["ff"][...] = case.ff
    st["nf"][...] = case.nf
    st["indc"][...] = -1
    for n in ("bcu", "bcv", "bcw", "bcp", "bcf"):
        st[n][...] = getattr(case, n)
    return st


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _fptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_float)) if a is not None else None


class UNet:
    """The learned warm start's 3-D U-Net on the GPU (cadmas_unet_*):
    volumes (batch, nz, ny, nx) of 4 input channels and one output."""

    def __init__(self, nx, ny, nz, batch=1, lib=None):
        self.lib = lib or load_library()
        self.shape = (batch, nz, ny, nx)
        self.h = C.c_void_p()
        _check(self.lib, self.lib.cadmas_unet_create(nx, ny, nz, batch, C.byref(self.h)))
        self.nparam = int(self.lib.cadmas_unet_param_count())

    def set_params(self, p):
        p = _f32(p)
        assert p.size == self.nparam
        _check(self.lib, self.lib.cadmas_unet_set_params(self.h, _fptr(p)))

    def get_params(self):
        p = np.zeros(self.nparam, np.float32)
        _check(self.lib, self.lib.cadmas_unet_get_params(self.h, _fptr(p)))
        return p

    def forward(self, x):
        x = _f32(x)
        assert x.shape == self.shape + (4,)
        y = np.zeros(self.shape, np.float32)
        _check(self.lib, self.lib.cadmas_unet_forward(self.h, _fptr(x), _fptr(y)))
        return y

    def time_forward(self, reps=5):
        """Mean device milliseconds of a forward of the resident input."""
        ms = C.c_float()
        _check(self.lib, self.lib.cadmas_unet_time_forward(self.h, int(reps), C.byref(ms)))
        return ms.value

    def grad(self, x, t, m):
        """(loss, gradient over the parameters) of the masked MSE."""
        x, t, m = _f32(x), _f32(t), _f32(m)
        loss = C.c_float()
        g = np.zeros(self.nparam, np.float32)
        _check(self.lib, self.lib.cadmas_unet_grad(self.h, _fptr(x), _fptr(t), _fptr(m), C.byref(loss), _fptr(g)))
        return loss.value, g

    def train_sys(self, x, t, m, a7, c=1.0, w_mse=1.0, w_res=1.0, lr=1.0e-3, update=True, want_grad=False):
        """MSE plus residual loss against the samples' systems a7; (loss,
        gradient or None)."""
        x, t, m, a7 = _f32(x), _f32(t), _f32(m), _f32(a7)
        loss = C.c_float()
        g = np.zeros(self.nparam, np.float32) if want_grad else None
        _check(self.lib, self.lib.cadmas_unet_train_sys(self.h, _fptr(x), _fptr(t), _fptr(m), _fptr(a7), float(c),
                                                        float(w_mse), float(w_res), float(lr), int(update),
                                                        C.byref(loss), _fptr(g)))
        return loss.value, g

    def train_step(self, x, t, m, lr=1.0e-3):
        x, t, m = _f32(x), _f32(t), _f32(m)
        loss = C.c_float()
        _check(self.lib, self.lib.cadmas_unet_train_step(self.h, _fptr(x), _fptr(t), _fptr(m), float(lr),
                                                         C.byref(loss)))
        return loss.value

    def close(self):
        if getattr(self, "h", None) and self.h.value:
            self.lib.cadmas_unet_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Tank:
    """One grid on the GPU: the state of the time loop between two steps."""

    def __init__(self, case, lib=None, **over):
        self.lib = lib or load_library()
        self.case = case
        self.params = make_params(case, default_params(self.lib), **over)
        d = Dims(case.ni, case.nj, case.nk, case.numb)
        h = C.c_void_p()
        _check(self.lib, self.lib.cadmas_create(C.byref(d), C.byref(self.params), C.byref(h)))
        self.h = h
        self._static = static_of(case)   # keep the pointers' owners alive
        _check(self.lib, self.lib.cadmas_upload_static(self.h, C.byref(self._static)))
        if getattr(case, "wave", None):
            self.set_wave(case.wave)
        for op in getattr(case, "open", None) or []:
            self.set_open(op)
        if getattr(case, "source", None):
            self.set_wave_source(case.source)
        self.set_state(initial_state(case))

    def set_wave_source(self, src):
        """Wave source line from a dict made by cases.wave_source
        (cadmas_set_wave_source with a table, cadmas_set_wave_source_func
        with a wave theory)."""
        ws, tab, keep = source_structs(src)
        if src.get("theory") is not None:
            self.lib.cadmas_set_wave_source_func.argtypes = [C.c_void_p, C.POINTER(WaveSrc), C.POINTER(WaveTheory)]
            _check(self.lib, self.lib.cadmas_set_wave_source_func(self.h, C.byref(ws), C.byref(src["theory"])))
            return
        self.lib.cadmas_set_wave_source.argtypes = [C.c_void_p, C.POINTER(WaveSrc), C.POINTER(WaveTable)]
        _check(self.lib, self.lib.cadmas_set_wave_source(self.h, C.byref(ws), C.byref(tab) if tab else None))

    def set_open(self, op):
        """Open (radiation) side from a dict made by cases.open_boundary
        (cadmas_set_open)."""
        o = OpenBC(int(op["side"]), 0, float(op["depth"]), float(op["period"]))
        _check(self.lib, self.lib.cadmas_set_open(self.h, C.byref(o)))

    def set_wave(self, wave):
        """Wave-maker side from a dict made by cases.wave_maker
        (cadmas_set_wave with a table, cadmas_set_wave_theory with a
        stream-function wave, cadmas_set_wave_func with a wave theory, then
        cadmas_set_wave_angle for oblique incidence)."""
        bc = WaveBC(int(wave["side"]), int(wave["first"]), int(wave["last"]), 0, float(wave["depth"]),
                    float(wave["period"]), float(wave.get("ramp", 0.0)))
        if wave.get("theory") is not None:
            self.lib.cadmas_set_wave_func.argtypes = [C.c_void_p, C.POINTER(WaveBC), C.POINTER(WaveTheory)]
            _check(self.lib, self.lib.cadmas_set_wave_func(self.h, C.byref(bc), C.byref(wave["theory"])))
        elif wave.get("stream") is not None:
            self.lib.cadmas_set_wave_theory.argtypes = [C.c_void_p, C.POINTER(WaveBC), C.POINTER(StreamWave)]
            _check(self.lib, self.lib.cadmas_set_wave_theory(self.h, C.byref(bc), C.byref(wave["stream"])))
        else:
            bc, tab, keep = wave_structs(wave)
            _check(self.lib, self.lib.cadmas_set_wave(self.h, C.byref(bc), C.byref(tab)))
        if wave.get("angle") is not None:
            a, sx, sy = (float(v) for v in wave["angle"])
            self.lib.cadmas_set_wave_angle.argtypes = [C.c_void_p, C.c_int] + [C.c_double] * 3
            _check(self.lib, self.lib.cadmas_set_wave_angle(self.h, int(wave["side"]), a, sx, sy))

    # ------------------------------------------------------------ state
    def set_state(self, arrs):
        s = state_struct(arrs)
        _check(self.lib, self.lib.cadmas_set_state(self.h, C.byref(s)))

    def get_state(self):
        arrs = new_state_arrays(self.case.ni, self.case.nj, self.case.nk, self.case.numb)
        s = state_struct(arrs)
        _check(self.lib, self.lib.cadmas_get_state(self.h, C.byref(s)))
        arrs["tnow"], arrs["nnow"] = s.tnow, s.nnow
        return arrs

    def init_state(self, hydrostatic=True):
        _check(self.lib, self.lib.cadmas_init_state(self.h, int(bool(hydrostatic))))

    def get_drop(self):
        """The droplet model's arrays {droptx, dropty, droptz, dropuu, dropvv, dropww}."""
        arrs = {n: np.zeros(self.case.ni * self.case.nj * self.case.nk) for n in DROP_ARRAYS}
        _check(self.lib, self.lib.cadmas_get_drop(self.h, *(_dptr(arrs[n]) for n in DROP_ARRAYS)))
        return arrs

    def restart_create(self, path):
        """Header of a restart file (VF_OR1INI)."""
        _check(self.lib, self.lib.cadmas_restart_create(self.h, str(path).encode()))

    def restart_append(self, path):
        """One output of the present state (VF_OR1TRN)."""
        _check(self.lib, self.lib.cadmas_restart_append(self.h, str(path).encode()))

    def restart_load(self, path, nnow):
        """The state of step nnow from a restart file (VF_IR1INP)."""
        _check(self.lib, self.lib.cadmas_restart_load(self.h, str(path).encode(), int(nnow)))

    def cdtcal(self, dtinit=1.0e-6, dtmin=0.0, dtmax=1.0e20, dtsafe=0.1):
        """The next step's DT of VF_CDTCAL (defaults of vf_a2dflt.f:230-234)."""
        dt = C.c_double()
        _check(self.lib, self.lib.cadmas_cdtcal(self.h, dtinit, dtmin, dtmax, dtsafe, C.byref(dt)))
        return dt.value

    def list_step(self):
        """The list-file lines of the last step (formats 9540 and 9550)."""
        buf = C.create_string_buffer(512)
        _check(self.lib, self.lib.cadmas_list_step(self.h, buf, 512))
        return buf.value.decode()

    def set_drop(self, arrs):
        keep = {n: np.ascontiguousarray(arrs[n], dtype=np.float64) for n in DROP_ARRAYS}
        _check(self.lib, self.lib.cadmas_set_drop(self.h, *(_dptr(keep[n]) for n in DROP_ARRAYS)))

    def set_warm_net(self, params, out_scale=1.0):
        """Load the learned guess's network (used with warm_start=2)."""
        p = _f32(params)
        _check(self.lib, self.lib.cadmas_set_warm_net(self.h, _fptr(p), float(out_scale)))

    def get_system(self):
        """The last pressure system {ad, ali, alj, alk, aui, auj, auk}; call
        between v1cal() and f1cal()."""
        c = self.case
        names = ("ad", "ali", "alj", "alk", "aui", "auj", "auk")
        arrs = {n: np.zeros((c.ni, c.nj, c.nk), order="F") for n in names}
        _check(self.lib, self.lib.cadmas_get_system(self.h, *(_dptr(arrs[n]) for n in names)))
        return arrs

    def warm_stats(self):
        """(kept, dropped) learned guesses so far."""
        k, d = C.c_longlong(), C.c_longlong()
        _check(self.lib, self.lib.cadmas_warm_stats(self.h, C.byref(k), C.byref(d)))
        return k.value, d.value

    def get_solve(self):
        """(BB, PT) of the last pressure solve, (ni, nj, nk) Fortran order."""
        c = self.case
        bb = np.zeros((c.ni, c.nj, c.nk), order="F")
        pt = np.zeros((c.ni, c.nj, c.nk), order="F")
        _check(self.lib, self.lib.cadmas_get_solve(self.h, _dptr(bb), _dptr(pt)))
        return bb, pt

    def v1cal(self):
        _check(self.lib, self.lib.cadmas_v1cal(self.h))

    def f1cal(self):
        _check(self.lib, self.lib.cadmas_f1cal(self.h))

    def get_turb(self):
        """The k-epsilon state {ak, ae, anut, anu} (flat, cells) and {bck, bce}."""
        c = self.case
        arrs = {n: np.zeros(c.ni * c.nj * c.nk) for n in TURB_CELLS}
        arrs.update({n: np.zeros(max(c.numb, 1)) for n in TURB_FACES})
        _check(self.lib, self.lib.cadmas_get_turb(self.h, *(_dptr(arrs[n]) for n in TURB_CELLS + TURB_FACES)))
        return arrs

    def set_turb(self, arrs):
        """AK, AE, BCK, BCE; ANUT and ANU follow (VF_CNUT0, VF_CNU00)."""
        keep = {n: np.ascontiguousarray(arrs[n], dtype=np.float64).reshape(-1, order="F")
                for n in ("ak", "ae", "bck", "bce")}
        _check(self.lib, self.lib.cadmas_set_turb(self.h, *(_dptr(keep[n]) for n in ("ak", "ae", "bck", "bce"))))

    # ------------------------------------------------------------ step
    def step(self, dt=None):
        _check(self.lib, self.lib.cadmas_step(self.h, float(dt if dt is not None else self.case.dt)))

    def set_time(self, tnow, dtnow, nnow):
        _check(self.lib, self.lib.cadmas_set_time(self.h, float(tnow), float(dtnow), int(nnow)))

    def test_stall_sweeps(self, from_step):
        """Failure injection: the MILU sweeps issue no bulk copies from
        wavefront step `from_step` on (negative: off), so their bounded
        waits run out (cadmas_test_stall_sweeps)."""
        _check(self.lib, self.lib.cadmas_test_stall_sweeps(self.h, int(from_step)))

    def divnorm(self):
        v = C.c_double()
        _check(self.lib, self.lib.cadmas_divnorm(self.h, C.byref(v)))
        return v.value

    def stats(self):
        st = Stats()
        _check(self.lib, self.lib.cadmas_get_stats(self.h, C.byref(st)))
        return {n: getattr(st, n) for n, _ in Stats._fields_}

    def sync(self):
        _check(self.lib, self.lib.cadmas_sync(self.h))

    def stream(self) -> int:
        """Address of the cudaStream_t all work of this tank runs on."""
        p = C.c_void_p()
        _check(self.lib, self.lib.cadmas_get_stream(self.h, C.byref(p)))
        return p.value or 0

    def stage_timers(self, enable=-1):
        """Per-stage GPU milliseconds and launch counts; enable 1/0 also
        switches timing on/off and clears the totals."""
        n = len(STAGES)
        ms = (C.c_double * n)()
        cnt = (C.c_longlong * n)()
        _check(self.lib, self.lib.cadmas_stage_timers(self.h, int(enable), ms, cnt, n))
        return {STAGES[i]: (ms[i], cnt[i]) for i in range(n)}

    def close(self):
        if getattr(self, "h", None):
            self.lib.cadmas_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def kernel_launches(lib=None) -> int:
    """Kernels launched by libcadmas_gpu.so in this process so far."""
    return int((lib or load_library()).cadmas_kernel_launches())


def m1bcgs_dev(tank: Tank, ad, ali, alj, alk, aui, auj, auk, bb, x0, indc):
    """VF_M1BCGS on device buffers (integer device addresses, e.g. from
    torch.Tensor.data_ptr()).  Returns (iter, bnorm, xnorm); x0 is updated
    in place on convergence."""
    it, bn, xn = C.c_int(), C.c_double(), C.c_double()
    args = [C.c_void_p(int(a)) for a in (ad, ali, alj, alk, aui, auj, auk, bb, x0, indc)]
    _check(tank.lib, tank.lib.cadmas_m1bcgs_dev(tank.h, *args, C.byref(it), C.byref(bn), C.byref(xn)))
    return it.value, bn.value, xn.value


def divnorm_noalloc(dims, xx, yy, zz, ggx, ggy, ggz, uu, vv, ww, indc, stream=0, lib=None):
    """|VD| of VF_CDIV00 on device arrays (integer device addresses, e.g.
    torch.Tensor.data_ptr(); reference layout) without a handle and without
    allocating: cadmas_divnorm_noalloc.  dims = (NUMI, NUMJ, NUMK)."""
    lib = lib or load_library()
    d = Dims(int(dims[0]), int(dims[1]), int(dims[2]), 0)
    v = C.c_double()
    args = [C.c_void_p(int(a)) for a in (xx, yy, zz, ggx, ggy, ggz, uu, vv, ww, indc)]
    _check(lib, lib.cadmas_divnorm_noalloc(C.byref(d), *args, C.c_void_p(int(stream)), C.byref(v)))
    return v.value


def open_speed(depth, period, grav=9.8, lib=None) -> float:
    """Phase speed C = L/T of an open side (cadmas_open_speed; host only)."""
    lib = lib or load_library()
    c = C.c_double()
    _check(lib, lib.cadmas_open_speed(float(depth), float(period), float(grav), C.byref(c)))
    return c.value


class Batch:
    """Tanks of the mixed solver whose pressure solves run together, one
    launch per solver kernel for all of them (cadmas_batch_*).  The tanks
    stay owned by the caller and must outlive the batch."""

    def __init__(self, tanks, lib=None):
        self.lib = lib or load_library()
        self.tanks = list(tanks)
        n = len(self.tanks)
        hs = (C.c_void_p * n)(*[t.h.value for t in self.tanks])
        self.h = C.c_void_p()
        self.lib.cadmas_batch_create.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_void_p)]
        _check(self.lib, self.lib.cadmas_batch_create(hs, n, C.byref(self.h)))

    def step(self, dts=None):
        """One SMAC step of every tank; returns the per-tank statuses."""
        n = len(self.tanks)
        dt = (C.c_double * n)(*[float(d) for d in (dts if dts is not None else [t.case.dt for t in self.tanks])])
        st = (C.c_int * n)()
        self.lib.cadmas_batch_step.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        rc = self.lib.cadmas_batch_step(self.h, dt, st)
        if rc != OK:
            raise CadmasError(rc, self.lib.cadmas_strerror(rc).decode())
        return list(st)

    def close(self):
        if self.h:
            self.lib.cadmas_batch_destroy.argtypes = [C.c_void_p]
            self.lib.cadmas_batch_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def step_ensemble(tanks, dts=None, lib=None):
    """One SMAC step of every tank, the tanks running side by side on the
    GPU (cadmas_step_ensemble).  Returns the per-tank statuses."""
    lib = lib or load_library()
    n = len(tanks)
    hs = (C.c_void_p * n)(*[t.h.value for t in tanks])
    dt = (C.c_double * n)(*[float(d) for d in (dts if dts is not None else [t.case.dt for t in tanks])])
    st = (C.c_int * n)()
    rc = lib.cadmas_step_ensemble(hs, n, dt, st)
    if rc != OK:
        raise CadmasError(rc, lib.cadmas_strerror(rc).decode())
    return list(st)
