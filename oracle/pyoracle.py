"""ctypes binding of the CPU oracle (test infrastructure only).

Loaded by tests/, __graft_entry__.smoke() and the CPU arms of bench.py to
check or time the GPU library; never by the library itself.
"""
from __future__ import annotations

import ctypes as C
import pathlib
import sys

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
SUM_REF, SUM_GPU = 0, 1


def _pkg():
    mod = sys.modules.get("cadmas_b200")
    if mod is None:
        import importlib.util
        d = HERE.parent / "multiscale-and-multiphysics-integrated-simulator-for-tsunami_b200"
        spec = importlib.util.spec_from_file_location("cadmas_b200", d / "__init__.py",
                                                      submodule_search_locations=[str(d)])
        mod = importlib.util.module_from_spec(spec)
        sys.modules["cadmas_b200"] = mod
        spec.loader.exec_module(mod)
    return mod


_lib = None


def _load_lib():
    global _lib
    if _lib is not None:
        return _lib
    # oracle/build.py under its own module name: the package has a build.py
    # too, and whichever is imported first as `build` would shadow the other
    import importlib.util
    spec = importlib.util.spec_from_file_location("cadmas_oracle_build", HERE / "build.py")
    obuild = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(obuild)
    obuild.build()
    P = _pkg()
    lib = C.CDLL(str(HERE / "liboracle.so"))
    lib.orc_create.argtypes = [C.POINTER(P.Dims), C.POINTER(P.Params), C.c_int]
    lib.orc_create.restype = C.c_void_p
    lib.orc_destroy.argtypes = [C.c_void_p]
    lib.orc_destroy.restype = None
    lib.orc_upload_static.argtypes = [C.c_void_p, C.POINTER(P.Static)]
    lib.orc_set_state.argtypes = [C.c_void_p, C.POINTER(P.State)]
    lib.orc_get_state.argtypes = [C.c_void_p, C.POINTER(P.State)]
    lib.orc_init_state.argtypes = [C.c_void_p, C.c_int]
    lib.orc_step.argtypes = [C.c_void_p, C.c_double]
    lib.orc_get_stats.argtypes = [C.c_void_p, C.POINTER(P.Stats)]
    lib.orc_divnorm.argtypes = [C.c_void_p, C.POINTER(C.c_double)]
    dp = C.POINTER(C.c_double)
    lib.orc_m1bcgs.argtypes = [C.c_void_p] + [dp] * 9 + [C.POINTER(C.c_int), C.POINTER(C.c_int), dp, dp]
    lib.orc_get_poisson.argtypes = [C.c_void_p, C.c_int, dp]
    lib.orc_get_timers.argtypes = [C.c_void_p, dp]
    lib.orc_get_drop.argtypes = [C.c_void_p] + [dp] * 6
    lib.orc_set_drop.argtypes = [C.c_void_p] + [dp] * 6
    lib.orc_cdtcal.argtypes = [C.c_void_p] + [C.c_double] * 4 + [dp]
    lib.orc_set_time.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_int]
    lib.orc_get_turb.argtypes = [C.c_void_p] + [dp] * 6
    lib.orc_set_turb.argtypes = [C.c_void_p] + [dp] * 4
    lib.orc_slope_counts.argtypes = [C.c_void_p, C.POINTER(C.c_int)]
    lib.orc_slope_fn.argtypes = [C.c_int, C.c_double]
    lib.orc_slope_fn.restype = C.c_double
    lib.orc_fslp.argtypes = [C.c_int, dp, dp, C.c_double, dp, dp]
    lib.orc_croot3.argtypes = [C.c_double] * 4 + [dp, C.POINTER(C.c_int)]
    lib.orc_num_threads.argtypes = []
    lib.orc_num_threads.restype = C.c_int
    _lib = lib
    return lib


class Oracle:
    """CPU restatement of the SMAC step on the same inputs as cadmas_b200.Tank."""

    def __init__(self, case, sum_mode=SUM_GPU, **over):
        self.lib = _load_lib()
        P = _pkg()
        self.P = P
        self.case = case
        # defaults of the library header restated (vf_a2dflt.f)
        base = P.Params()
        base.rho0, base.grz0, base.vvmax = 1.0e3, 9.8, 30.0
        base.cgpara, base.cgepsa, base.cgepsr, base.cgdiv = 0.95, 1.0e-15, 1.0e-12, 1.0e30
        base.flower, base.fupper, base.plower, base.scmvp = 1.0e-6, 1.0 - 1.0e-6, 1.0e-4, 1.0
        base.wvlvl, base.wbub = 0.0, 0.2
        for d in range(4):
            base.idamp[d] = -1
            base.damp[d][0], base.damp[d][1], base.damp[d][2], base.damp[d][3] = 0.6, 0.6, 0.0, 0.0
        base.icgtyp, base.icgmax, base.ibsuw0 = 1, 500, 0
        base.idrop = 1
        base.anu0, base.scmk = 1.0e-6, 1.0
        base.akmink = base.akmine = base.akinik = base.akinie = 1.0e-20
        base.akcmu, base.aksgk, base.aksge, base.akc1, base.akc2, base.akc3 = 0.09, 1.0, 1.3, 1.44, 1.92, 0.0
        base.akk0, base.aka0 = 0.4, 5.5
        self.params = P.make_params(case, base, **over)
        d = P.Dims(case.ni, case.nj, case.nk, case.numb)
        self.h = self.lib.orc_create(C.byref(d), C.byref(self.params), int(sum_mode))
        if not self.h:
            raise RuntimeError("orc_create failed")
        self._static = P.static_of(case)
        self._rc(self.lib.orc_upload_static(self.h, C.byref(self._static)))
        wv = getattr(case, "wave", None)
        if wv:
            bc = P.WaveBC(int(wv["side"]), int(wv["first"]), int(wv["last"]), 0, float(wv["depth"]),
                          float(wv["period"]), float(wv.get("ramp", 0.0)))
            if wv.get("theory") is not None:
                self.lib.orc_set_wave_func.argtypes = [C.c_void_p, C.POINTER(P.WaveBC), C.POINTER(P.WaveTheory)]
                self._rc(self.lib.orc_set_wave_func(self.h, C.byref(bc), C.byref(wv["theory"])))
            elif wv.get("stream") is not None:
                self.lib.orc_set_wave_theory.argtypes = [C.c_void_p, C.POINTER(P.WaveBC), C.POINTER(P.StreamWave)]
                self._rc(self.lib.orc_set_wave_theory(self.h, C.byref(bc), C.byref(wv["stream"])))
            else:
                bc, tab, keep = P.wave_structs(wv)
                self.lib.orc_set_wave.argtypes = [C.c_void_p, C.POINTER(P.WaveBC), C.POINTER(P.WaveTable)]
                self._rc(self.lib.orc_set_wave(self.h, C.byref(bc), C.byref(tab)))
            if wv.get("angle") is not None:
                a, sx, sy = (float(v) for v in wv["angle"])
                self.lib.orc_set_wave_angle.argtypes = [C.c_void_p, C.c_int] + [C.c_double] * 3
                self._rc(self.lib.orc_set_wave_angle(self.h, int(wv["side"]), a, sx, sy))
        for op in getattr(case, "open", None) or []:
            self.lib.orc_set_open.argtypes = [C.c_void_p, C.c_int, C.c_double, C.c_double]
            self._rc(self.lib.orc_set_open(self.h, int(op["side"]), float(op["depth"]), float(op["period"])))
        if getattr(case, "source", None):
            ws, tab, keep = P.source_structs(case.source)
            if case.source.get("theory") is not None:
                self.lib.orc_set_wave_source_func.argtypes = [C.c_void_p, C.POINTER(P.WaveSrc),
                                                              C.POINTER(P.WaveTheory)]
                self._rc(self.lib.orc_set_wave_source_func(self.h, C.byref(ws), C.byref(case.source["theory"])))
            else:
                self.lib.orc_set_wave_source.argtypes = [C.c_void_p, C.POINTER(P.WaveSrc), C.POINTER(P.WaveTable)]
                self._rc(self.lib.orc_set_wave_source(self.h, C.byref(ws), C.byref(tab) if tab else None))
        self.set_state(P.initial_state(case))

    def _rc(self, rc):
        if rc != 0:
            raise self.P.CadmasError(rc, f"oracle status {rc}")

    def set_state(self, arrs):
        s = self.P.state_struct(arrs)
        self._rc(self.lib.orc_set_state(self.h, C.byref(s)))

    def get_state(self):
        c = self.case
        arrs = self.P.new_state_arrays(c.ni, c.nj, c.nk, c.numb)
        s = self.P.state_struct(arrs)
        self._rc(self.lib.orc_get_state(self.h, C.byref(s)))
        arrs["tnow"], arrs["nnow"] = s.tnow, s.nnow
        return arrs

    def init_state(self, hydrostatic=True):
        self._rc(self.lib.orc_init_state(self.h, int(bool(hydrostatic))))

    def set_time(self, tnow, dtnow, nnow):
        self._rc(self.lib.orc_set_time(self.h, float(tnow), float(dtnow), int(nnow)))

    def cdtcal(self, dtinit=1.0e-6, dtmin=0.0, dtmax=1.0e20, dtsafe=0.1):
        """VF_CDTCAL in the handle's order (reference: running minimum)."""
        dt = C.c_double()
        self._rc(self.lib.orc_cdtcal(self.h, dtinit, dtmin, dtmax, dtsafe, C.byref(dt)))
        return dt.value

    def get_drop(self):
        """DROPTX..DROPWW as {droptx, ..., dropww}."""
        c = self.case
        arrs = {n: np.zeros(c.ni * c.nj * c.nk) for n in self.P.DROP_ARRAYS}
        dp = C.POINTER(C.c_double)
        self._rc(self.lib.orc_get_drop(self.h, *(arrs[n].ctypes.data_as(dp) for n in self.P.DROP_ARRAYS)))
        return arrs

    def set_drop(self, arrs):
        keep = {n: np.ascontiguousarray(arrs[n], dtype=np.float64) for n in self.P.DROP_ARRAYS}
        dp = C.POINTER(C.c_double)
        self._rc(self.lib.orc_set_drop(self.h, *(keep[n].ctypes.data_as(dp) for n in self.P.DROP_ARRAYS)))

    def get_turb(self):
        """The k-epsilon state {ak, ae, anut, anu} (flat) and {bck, bce}."""
        c = self.case
        cells, faces = self.P.TURB_CELLS, self.P.TURB_FACES
        arrs = {n: np.zeros(c.ni * c.nj * c.nk) for n in cells}
        arrs.update({n: np.zeros(max(c.numb, 1)) for n in faces})
        dp = C.POINTER(C.c_double)
        self._rc(self.lib.orc_get_turb(self.h, *(arrs[n].ctypes.data_as(dp) for n in cells + faces)))
        return arrs

    def set_turb(self, arrs):
        keep = {n: np.ascontiguousarray(arrs[n], dtype=np.float64).reshape(-1, order="F")
                for n in ("ak", "ae", "bck", "bce")}
        dp = C.POINTER(C.c_double)
        self._rc(self.lib.orc_set_turb(self.h, *(keep[n].ctypes.data_as(dp) for n in ("ak", "ae", "bck", "bce"))))

    def slope_counts(self):
        """Cells of each slope type 0..7 seen by VF_FCONVS so far."""
        n = (C.c_int * 8)()
        self._rc(self.lib.orc_slope_counts(self.h, n))
        return list(n)

    def step(self, dt=None):
        self._rc(self.lib.orc_step(self.h, float(dt if dt is not None else self.case.dt)))

    def stats(self):
        st = self.P.Stats()
        self._rc(self.lib.orc_get_stats(self.h, C.byref(st)))
        return {n: getattr(st, n) for n, _ in self.P.Stats._fields_ if n != "pad"}

    def divnorm(self):
        v = C.c_double()
        self._rc(self.lib.orc_divnorm(self.h, C.byref(v)))
        return v.value

    def timers(self):
        t = (C.c_double * 5)()
        self.lib.orc_get_timers(self.h, t)
        return list(t)

    def poisson(self, which):
        c = self.case
        out = np.zeros((c.ni, c.nj, c.nk), order="F")
        self._rc(self.lib.orc_get_poisson(self.h, which, out.ctypes.data_as(C.POINTER(C.c_double))))
        return out

    def m1bcgs(self, ad, ali, alj, alk, aui, auj, auk, bb, x0, indc):
        dp = C.POINTER(C.c_double)
        it, bn, xn = C.c_int(), C.c_double(), C.c_double()
        arrs = [np.asfortranarray(a, dtype=np.float64) for a in (ad, ali, alj, alk, aui, auj, auk, bb)]
        x = np.array(x0, dtype=np.float64, order="F")
        ic = np.asfortranarray(indc, dtype=np.int32)
        self._rc(self.lib.orc_m1bcgs(self.h, *[a.ctypes.data_as(dp) for a in arrs], x.ctypes.data_as(dp),
                                     ic.ctypes.data_as(C.POINTER(C.c_int)), C.byref(it), C.byref(bn),
                                     C.byref(xn)))
        return x, it.value, bn.value, xn.value

    def close(self):
        if getattr(self, "h", None):
            self.lib.orc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def num_threads() -> int:
    """Threads of the oracle's parallel loops (OpenMP; OMP_NUM_THREADS)."""
    return int(_load_lib().orc_num_threads())


def slope_fn(fn: int, x: float) -> float:
    """The oracle's cube root (0), arctangent (1) or cosine (2) of VF_CROOT3."""
    return float(_load_lib().orc_slope_fn(int(fn), float(x)))


def fslp(s, d, fval):
    """VF_FSLP2A/3A then VF_FSLP2F/3F for normal s and cell widths d:
    (plane offset, water fraction recovered), or None on P.G ERROR."""
    dim = len(s)
    sa = (C.c_double * dim)(*s)
    da = (C.c_double * dim)(*d)
    aa, fb = C.c_double(), C.c_double()
    rc = _load_lib().orc_fslp(dim, sa, da, float(fval), C.byref(aa), C.byref(fb))
    return None if rc else (aa.value, fb.value)


def wave_eval(th, phase, z=0.0):
    """(eta, u, w) of a solved wave theory (the package's WaveTheory) by the
    oracle's restatement of VF_CWMAK1/VF_CWMAK2."""
    lib = _load_lib()
    P = _pkg()
    e, u, w = C.c_double(), C.c_double(), C.c_double()
    dp = C.POINTER(C.c_double)
    lib.orc_wave_eval.argtypes = [C.POINTER(P.WaveTheory), C.c_double, C.c_double, dp, dp, dp]
    rc = lib.orc_wave_eval(C.byref(th), float(phase), float(z), C.byref(e), C.byref(u), C.byref(w))
    if rc != 0:
        raise P.CadmasError(rc, f"oracle status {rc}")
    return e.value, u.value, w.value


def open_speed(depth, period, grav=9.8):
    """VF_COMAK0's wave length over the period (BCTYP(6,JD)), or None."""
    c = C.c_double()
    lib = _load_lib()
    lib.orc_open_speed.argtypes = [C.c_double, C.c_double, C.c_double, C.POINTER(C.c_double)]
    rc = lib.orc_open_speed(float(depth), float(period), float(grav), C.byref(c))
    return None if rc else c.value


def ln(x):
    """The logarithm of the log-law wall functions."""
    lib = _load_lib()
    lib.orc_ln.argtypes = [C.c_double]
    lib.orc_ln.restype = C.c_double
    return lib.orc_ln(float(x))


def cloglw(dl, va, anu0=1.0e-6, akk0=0.4, aka0=5.5):
    """VF_CLOGLW's friction velocity, or None when it does not converge."""
    lib = _load_lib()
    lib.orc_cloglw.argtypes = [C.c_double] * 5 + [C.POINTER(C.c_double)]
    vt = C.c_double()
    rc = lib.orc_cloglw(float(dl), float(va), float(anu0), float(akk0), float(aka0), C.byref(vt))
    return None if rc else vt.value


def clogks(dl, va, ks, anu0=1.0e-6, akk0=0.4, aka0=5.5):
    """VF_CLOGKS's friction velocity on a rough wall of roughness ks."""
    lib = _load_lib()
    lib.orc_clogks.argtypes = [C.c_double] * 6
    lib.orc_clogks.restype = C.c_double
    return lib.orc_clogks(float(dl), float(va), float(ks), float(anu0), float(akk0), float(aka0))


def croot3(a, b, c, d):
    """VF_CROOT3: (roots, number of roots)."""
    x = (C.c_double * 3)()
    n = C.c_int()
    _load_lib().orc_croot3(a, b, c, d, x, C.byref(n))
    return list(x)[:n.value], n.value
