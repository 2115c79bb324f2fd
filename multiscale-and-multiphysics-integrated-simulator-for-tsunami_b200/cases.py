"""Synthetic wave-tank cases: the host-side set-up of CADMAS-SURF/3D in numpy.

The Fortran program prepares the static fields of a run once, before the time
loop, from its text input.  This module does the same from Python arguments,
restating the set-up routines (Simulators/CADMAS-SURF-3D/Source code/):

  grid metrics XX/YY/ZZ(6,N)       VF_CGRID   vf_cgrid.f:44-67
  ghost cells and obstacles NF=-1  VF_CNFDFL  vf_cnfdfl.f:37-50, VF_IIOBST vf_iiobst.f:50
  porosity GGV/GGX/GGY/GGZ, CM, CD VF_IIPORO  vf_iiporo.f:80-245
  face indices INDX/INDY/INDZ      VF_CINDX   vf_cindx.f:30-140
  boundary list INDB(4,NUMB)       VF_CINDB   vf_cindb.f:30-95
  GLV, GLX/GLY/GLZ                 VF_CGLV    vf_cglv.f:34, VF_CGLXYZ vf_cglxyz.f:65-105
  ANU                              VF_CNU00   vf_cnu00.f:30-45
  initial F (still water + F box)  VF_CINIT   vf_cinit.f:150-190

Every 3-D array is a numpy array of shape (NUMI, NUMJ, NUMK) in Fortran
order, so ``a.ctypes.data`` is the Fortran array the library expects.
Indices in the arguments below are the Fortran array indices (1-based, ghost
layer included): interior cells are 2..NUMI-1.

Randomness (obstacle boxes, porosity) comes from numpy's Philox generator
seeded with the case seed, so the GPU library and the oracle see the same
bytes.
"""
from __future__ import annotations

import dataclasses
import numpy as np

# Velocity/pressure boundary types INDB(3,L) and F boundary types INDB(4,L)
# (vf_a1main.f:151-170).
VP_SLIP, VP_NOSLIP, VP_FIXED, VP_FREE, VP_WAVE, VP_LOGLAW, VP_OPEN, VP_ROUGH = 1, 2, 3, 4, 5, 6, 7, 8
F_FIXED, F_FREE, F_WAVE, F_OPEN = 1, 2, 5, 7


def grid_metrics(coords: np.ndarray) -> np.ndarray:
    """VF_CGRID (vf_cgrid.f:44-67) for one axis of a serial run.

    coords: the NUML-1 face coordinates of the interior, XYZ(1,2..NUML).
    Returns XYZ(6,NUML) in Fortran order, flattened as the library expects.
    """
    coords = np.asarray(coords, dtype=np.float64)
    nl = coords.size + 1
    x = np.zeros((6, nl), order="F")
    x[0, 1:] = coords
    for i in range(1, nl - 1):            # I = 2..NUML-1
        x[1, i] = x[0, i + 1] - x[0, i]
        x[3, i] = 1.0 / x[1, i]
    x[1, 0] = x[1, 1]                     # LG1 == 2
    x[3, 0] = 1.0 / x[1, 0]
    x[0, 0] = x[0, 1] - x[1, 0]
    x[1, nl - 1] = x[1, nl - 2]           # LG2 == NUML0
    x[3, nl - 1] = 1.0 / x[1, nl - 1]
    for i in range(1, nl):                # I = 2..NUML
        x[2, i] = (x[1, i] + x[1, i - 1]) / 2.0
        x[4, i] = 1.0 / x[2, i]
        x[5, i] = 1.0 / (x[1, i] + x[1, i - 1])
    x[2, 0] = x[4, 0] = x[5, 0] = 0.0
    return x


@dataclasses.dataclass
class Case:
    """Static fields, initial state and parameters of one run."""
    name: str
    ni: int
    nj: int
    nk: int
    xx: np.ndarray
    yy: np.ndarray
    zz: np.ndarray
    nf: np.ndarray
    ggv: np.ndarray
    ggx: np.ndarray
    ggy: np.ndarray
    ggz: np.ndarray
    cm0: np.ndarray
    cd0: np.ndarray
    glv: np.ndarray = None
    glx: np.ndarray = None
    gly: np.ndarray = None
    glz: np.ndarray = None
    anu: np.ndarray = None
    indx: np.ndarray = None
    indy: np.ndarray = None
    indz: np.ndarray = None
    indb: np.ndarray = None
    numb: int = 0
    ff: np.ndarray = None
    uu: np.ndarray = None
    vv: np.ndarray = None
    ww: np.ndarray = None
    pp: np.ndarray = None
    bcu: np.ndarray = None
    bcv: np.ndarray = None
    bcw: np.ndarray = None
    bcp: np.ndarray = None
    bcf: np.ndarray = None
    params: dict = dataclasses.field(default_factory=dict)
    wave: dict = None          # wave-maker side (wave_maker), or None
    open: list = None          # open (radiation) sides (open_boundary), or None
    source: dict = None        # wave source line (wave_source), or None
    dt: float = 1e-3
    hydrostatic: bool = True

    @property
    def interior_cells(self) -> int:
        return (self.ni - 2) * (self.nj - 2) * (self.nk - 2)


def _z3(ni, nj, nk, val=0.0, dtype=np.float64):
    return np.full((ni, nj, nk), val, dtype=dtype, order="F")


def new_case(name, xs, ys, zs) -> Case:
    """Grid from face coordinates; all cells fluid-capable, porosity 1
    (vf_a1main.f:495-510), ghost layer obstacle (VF_CNFDFL)."""
    xx, yy, zz = grid_metrics(xs), grid_metrics(ys), grid_metrics(zs)
    ni, nj, nk = xx.shape[1], yy.shape[1], zz.shape[1]
    nf = np.zeros((ni, nj, nk), dtype=np.int32, order="F")
    nf[0, :, :] = nf[-1, :, :] = -1
    nf[:, 0, :] = nf[:, -1, :] = -1
    nf[:, :, 0] = nf[:, :, -1] = -1
    return Case(name=name, ni=ni, nj=nj, nk=nk, xx=xx, yy=yy, zz=zz, nf=nf,
                ggv=_z3(ni, nj, nk, 1.0), ggx=_z3(ni, nj, nk, 1.0),
                ggy=_z3(ni, nj, nk, 1.0), ggz=_z3(ni, nj, nk, 1.0),
                cm0=_z3(ni, nj, nk), cd0=_z3(ni, nj, nk))


def add_obstacle(c: Case, i1, j1, k1, i2, j2, k2):
    """OBST box over array cells I1..I2, J1..J2, K1..K2 (vf_iiobst.f:42-53)."""
    c.nf[i1 - 1:i2, j1 - 1:j2, k1 - 1:k2] = -1


def add_porous(c: Case, i1, j1, k1, i2, j2, k2, gamma, cm=0.0, cd=0.0,
               plower=1.0e-4):
    """POROUS V/X/Y/Z/CM/CD over array cells I1..I2 x J1..J2 x K1..K2
    (vf_iiporo.f): cells get GGV; the faces of those cells, both sides
    included, get GGX/GGY/GGZ; CM/CD on non-obstacle cells."""
    val = max(gamma, plower)  # VAL=MAX(V2+(1-V2)*V1,PLOWER) with V2=0
    sl = (slice(i1 - 1, i2), slice(j1 - 1, j2), slice(k1 - 1, k2))
    obst = c.nf[sl] == -1
    c.ggv[sl] = np.where(obst, c.ggv[sl], val)
    c.cm0[sl] = np.where(obst, c.cm0[sl], cm)
    c.cd0[sl] = np.where(obst, c.cd0[sl], cd)
    c._porous_faces = getattr(c, "_porous_faces", [])
    c._porous_faces.append((i1, j1, k1, i2, j2, k2, val))


def _apply_porous_faces(c: Case):
    # Face permeabilities need INDX/INDY/INDZ (set only where not -1).
    for (i1, j1, k1, i2, j2, k2, val) in getattr(c, "_porous_faces", []):
        sx = (slice(i1 - 1, i2 + 1), slice(j1 - 1, j2), slice(k1 - 1, k2))
        sy = (slice(i1 - 1, i2), slice(j1 - 1, j2 + 1), slice(k1 - 1, k2))
        sz = (slice(i1 - 1, i2), slice(j1 - 1, j2), slice(k1 - 1, k2 + 1))
        c.ggx[sx] = np.where(c.indx[sx] != -1, val, c.ggx[sx])
        c.ggy[sy] = np.where(c.indy[sy] != -1, val, c.ggy[sy])
        c.ggz[sz] = np.where(c.indz[sz] != -1, val, c.ggz[sz])


def build_faces(c: Case):
    """VF_CINDX (vf_cindx.f:30-140): -1 between two obstacles, a boundary
    number (1-based, numbered x, then y, then z faces, each in K,J,I order)
    where exactly one side is obstacle, 0 otherwise."""
    ni, nj, nk, nf = c.ni, c.nj, c.nk, c.nf
    indx = np.zeros((ni, nj, nk), dtype=np.int32, order="F")
    indy = np.zeros_like(indx)
    indz = np.zeros_like(indx)
    ob = nf == -1
    indx[0, :, :] = -1
    indx[1:, :, :] = np.where(ob[:-1, :, :] & ob[1:, :, :], -1, 0)
    indy[:, 0, :] = -1
    indy[:, 1:, :] = np.where(ob[:, :-1, :] & ob[:, 1:, :], -1, 0)
    indz[:, :, 0] = -1
    indz[:, :, 1:] = np.where(ob[:, :, :-1] & ob[:, :, 1:], -1, 0)
    numb = 0
    # x faces: K=2..NK-1, J=2..NJ-1, I=2..NI
    cand = np.zeros_like(indx, dtype=bool)
    n1 = ob[:-1, :, :]
    n2 = ob[1:, :, :]
    cx = (n1 | n2) & (indx[1:, :, :] != -1)
    cand[1:, :, :] = cx
    cand[:, 0, :] = cand[:, -1, :] = False
    cand[:, :, 0] = cand[:, :, -1] = False
    # exceptions: I==2 and N2==-1, I==NUMI and N1==-1
    cand[1, :, :] &= ~ob[1, :, :]
    cand[ni - 1, :, :] &= ~ob[ni - 2, :, :]
    idx = np.nonzero(cand.ravel(order="F"))[0]
    vals = np.arange(numb + 1, numb + 1 + idx.size, dtype=np.int32)
    flat = indx.reshape(-1, order="F")
    flat[idx] = vals
    indx = flat.reshape((ni, nj, nk), order="F")
    numb += idx.size
    # y faces: K=2..NK-1, J=2..NJ, I=2..NI-1
    cand = np.zeros_like(indy, dtype=bool)
    cy = (ob[:, :-1, :] | ob[:, 1:, :]) & (indy[:, 1:, :] != -1)
    cand[:, 1:, :] = cy
    cand[0, :, :] = cand[-1, :, :] = False
    cand[:, :, 0] = cand[:, :, -1] = False
    cand[:, 1, :] &= ~ob[:, 1, :]
    cand[:, nj - 1, :] &= ~ob[:, nj - 2, :]
    idx = np.nonzero(cand.ravel(order="F"))[0]
    flat = indy.reshape(-1, order="F")
    flat[idx] = np.arange(numb + 1, numb + 1 + idx.size, dtype=np.int32)
    indy = flat.reshape((ni, nj, nk), order="F")
    numb += idx.size
    # z faces: K=2..NK, J=2..NJ-1, I=2..NI-1 (no end exceptions)
    cand = np.zeros_like(indz, dtype=bool)
    cz = (ob[:, :, :-1] | ob[:, :, 1:]) & (indz[:, :, 1:] != -1)
    cand[:, :, 1:] = cz
    cand[0, :, :] = cand[-1, :, :] = False
    cand[:, 0, :] = cand[:, -1, :] = False
    idx = np.nonzero(cand.ravel(order="F"))[0]
    flat = indz.reshape(-1, order="F")
    flat[idx] = np.arange(numb + 1, numb + 1 + idx.size, dtype=np.int32)
    indz = flat.reshape((ni, nj, nk), order="F")
    numb += idx.size
    c.indx, c.indy, c.indz, c.numb = indx, indy, indz, numb


def build_boundary_list(c: Case, vp_type=VP_SLIP, f_type=F_FREE, faces=None):
    """VF_CINDB (vf_cindb.f:30-95) plus the B.C. types.

    faces: optional callable (axis, i, j, k, side) -> (vp, f) overriding the
    default types for individual faces (1-based array indices)."""
    nb = max(c.numb, 1)
    indb = np.zeros((4, nb), dtype=np.int32, order="F")
    ni, nj = c.ni, c.nj
    for axis, ind, ns_lo, ns_hi in ((0, c.indx, 1, 2), (1, c.indy, 3, 4), (2, c.indz, 5, 6)):
        flat = ind.reshape(-1, order="F")
        pos = np.nonzero(flat >= 1)[0]
        for p in pos:
            nb_ = flat[p]
            i = p % ni + 1
            j = (p // ni) % nj + 1
            k = p // (ni * nj) + 1
            indb[0, nb_ - 1] = i + ni * (j - 1) + ni * nj * (k - 1)
            n2 = c.nf[i - 1, j - 1, k - 1]
            indb[1, nb_ - 1] = ns_lo if n2 != -1 else ns_hi
            vp, ft = vp_type, f_type
            if faces is not None:
                o = faces(axis, i, j, k, indb[1, nb_ - 1])
                if o is not None:
                    vp, ft = o
            indb[2, nb_ - 1] = vp
            indb[3, nb_ - 1] = ft
    c.indb = indb
    zb = np.zeros(nb, dtype=np.float64)
    c.bcu, c.bcv, c.bcw, c.bcp, c.bcf = (zb.copy() for _ in range(5))


def build_inertia(c: Case):
    """VF_CGLV (vf_cglv.f:34) and VF_CGLXYZ (vf_cglxyz.f:65-105)."""
    ni, nj, nk = c.ni, c.nj, c.nk
    c.glv = np.where(c.nf == -1, 1.0, c.ggv + (1.0 - c.ggv) * c.cm0)
    c.glv = np.asfortranarray(c.glv)
    glx = _z3(ni, nj, nk, 1.0)
    gly = _z3(ni, nj, nk, 1.0)
    glz = _z3(ni, nj, nk, 1.0)
    x6, x2 = c.xx[5], c.xx[1]
    y6, y2 = c.yy[5], c.yy[1]
    z6, z2 = c.zz[5], c.zz[1]
    cm, nf = c.cm0, c.nf
    for k in range(nk):
        for j in range(nj):
            for i in range(ni):
                # GLX
                v = c.indx[i, j, k]
                if v == -1:
                    glx[i, j, k] = 1.0
                elif v == 0:
                    m = x6[i] * (x2[i] * cm[i, j, k] + x2[i - 1] * cm[i - 1, j, k])
                    glx[i, j, k] = c.ggx[i, j, k] + (1.0 - c.ggx[i, j, k]) * m
                elif nf[i, j, k] != -1:
                    glx[i, j, k] = c.ggx[i, j, k] + (1.0 - c.ggx[i, j, k]) * cm[i, j, k]
                else:
                    glx[i, j, k] = c.ggx[i, j, k] + (1.0 - c.ggx[i, j, k]) * cm[i - 1, j, k]
                v = c.indy[i, j, k]
                if v == -1:
                    gly[i, j, k] = 1.0
                elif v == 0:
                    m = y6[j] * (y2[j] * cm[i, j, k] + y2[j - 1] * cm[i, j - 1, k])
                    gly[i, j, k] = c.ggy[i, j, k] + (1.0 - c.ggy[i, j, k]) * m
                elif nf[i, j, k] != -1:
                    gly[i, j, k] = c.ggy[i, j, k] + (1.0 - c.ggy[i, j, k]) * cm[i, j, k]
                else:
                    gly[i, j, k] = c.ggy[i, j, k] + (1.0 - c.ggy[i, j, k]) * cm[i, j - 1, k]
                v = c.indz[i, j, k]
                if v == -1:
                    glz[i, j, k] = 1.0
                elif v == 0:
                    m = z6[k] * (z2[k] * cm[i, j, k] + z2[k - 1] * cm[i, j, k - 1])
                    glz[i, j, k] = c.ggz[i, j, k] + (1.0 - c.ggz[i, j, k]) * m
                elif nf[i, j, k] != -1:
                    glz[i, j, k] = c.ggz[i, j, k] + (1.0 - c.ggz[i, j, k]) * cm[i, j, k]
                else:
                    glz[i, j, k] = c.ggz[i, j, k] + (1.0 - c.ggz[i, j, k]) * cm[i, j, k - 1]
    c.glx, c.gly, c.glz = glx, gly, glz


def build_inertia_fast(c: Case):
    """Vectorised VF_CGLXYZ for large grids; same arithmetic per element."""
    c.glv = np.asfortranarray(np.where(c.nf == -1, 1.0, c.ggv + (1.0 - c.ggv) * c.cm0))
    cm, nf = c.cm0, c.nf

    def one(ind, gg, d6, d2, axis):
        sh = [1, 1, 1]
        sh[axis] = -1
        d6b = d6.reshape(sh)
        d2b = d2.reshape(sh)
        d2m = np.roll(d2, 1).reshape(sh)
        cmm = np.roll(cm, 1, axis=axis)
        m = d6b * (d2b * cm + d2m * cmm)
        normal = gg + (1.0 - gg) * m
        own = gg + (1.0 - gg) * cm
        oth = gg + (1.0 - gg) * cmm
        out = np.where(ind == -1, 1.0, np.where(ind == 0, normal, np.where(nf != -1, own, oth)))
        return np.asfortranarray(out)

    c.glx = one(c.indx, c.ggx, c.xx[5], c.xx[1], 0)
    c.gly = one(c.indy, c.ggy, c.yy[5], c.yy[1], 1)
    c.glz = one(c.indz, c.ggz, c.zz[5], c.zz[1], 2)


def build_viscosity(c: Case, anu0=1.0e-6):
    """VF_CNU00 without k-epsilon (vf_cnu00.f:30-45)."""
    anu = _z3(c.ni, c.nj, c.nk)
    inner = (slice(1, -1), slice(1, -1), slice(1, -1))
    anu[inner] = np.where(c.nf[inner] != -1, anu0, 0.0)
    c.anu = anu


def init_f_still_water(c: Case, wvlvl: float):
    """VF_CINIT F from the still-water level (vf_cinit.f:150-160)."""
    ff = _z3(c.ni, c.nj, c.nk)
    z1 = c.zz[0]
    for k in range(1, c.nk - 1):          # K = 2..NK-1
        if z1[k] > wvlvl:
            val = 0.0
        elif z1[k + 1] < wvlvl:
            val = 1.0
        else:
            val = (wvlvl - z1[k]) / (z1[k + 1] - z1[k])
        sl = c.nf[1:-1, 1:-1, k] != -1
        ff[1:-1, 1:-1, k] = np.where(sl, val, 0.0)
    c.ff = ff


def f_box(c: Case, i1, j1, k1, i2, j2, k2, val):
    """DEBUG F-BOX (vf_cinit.f:171-182), array indices."""
    sl = (slice(i1 - 1, i2), slice(j1 - 1, j2), slice(k1 - 1, k2))
    c.ff[sl] = np.where(c.nf[sl] != -1, val, c.ff[sl])


def finish(c: Case, vp_type=VP_SLIP, f_type=F_FREE, faces=None, fast=None):
    """Faces, boundary list, porous faces, inertia, viscosity, zero state."""
    build_faces(c)
    _apply_porous_faces(c)
    build_boundary_list(c, vp_type, f_type, faces)
    if fast is None:
        fast = c.ni * c.nj * c.nk > 200_000
    (build_inertia_fast if fast else build_inertia)(c)
    build_viscosity(c, c.params.get("anu0", 1.0e-6))
    # k-epsilon boundaries: zero gradient ('K FREE+A', 'E FREE+A') on every
    # face (read only when leqk != 0)
    nb = max(c.numb, 1)
    c.indbk = np.full(nb, 2, dtype=np.int32)
    c.indbe = np.full(nb, 2, dtype=np.int32)
    c.bck = np.zeros(nb)
    c.bce = np.zeros(nb)
    shape = (c.ni, c.nj, c.nk)
    c.uu = _z3(*shape)
    c.vv = _z3(*shape)
    c.ww = _z3(*shape)
    c.pp = _z3(*shape)
    if c.ff is None:
        c.ff = _z3(*shape)
    return c


# ----------------------------------------------------------------- the cases
def dam_break(nx=64, ny=8, nz=32, d=0.01, column=(16, 16), dt=1.0e-4):
    """Plain FP64 dam break in a closed free-slip box.

    64x8x32 cells of 0.01 m; water where x < 0.16 m and z < 0.16 m: still
    water level 0.16 m plus an F box of F=0 over interior cells
    i = 17..64, all j, k = 1..16 (DEBUG F-BOX)."""
    c = new_case("dam_break", np.arange(nx + 1) * d, np.arange(ny + 1) * d,
                 np.arange(nz + 1) * d)
    c.params.update(wvlvl=column[1] * d, wbub=-1.0, idrop=0, cgepsr=1.0e-10)  # BUB OFF, DROP OFF
    init_f_still_water(c, column[1] * d)
    f_box(c, column[0] + 2, 2, 2, nx + 1, ny + 1, column[1] + 1, 0.0)
    c.dt = dt
    return finish(c)


def porous_flume(nx=512, ny=32, nz=96, dx=0.02, dy=0.02, dz=0.01, depth=0.5,
                 block=(6.0, 7.0, 0.6), gamma=0.4, cm=1.2, cd=1.0,
                 sponge_width=2.0, sponge_degree=2, dt=2.0e-3):
    """Wave flume with a porous breakwater and an outlet sponge.

    Still-water depth 0.5 m; porous block x in [6,7] m, full width,
    z < 0.6 m, porosity 0.4, CM 1.2, CD 1.0; 2 m damping zone at x+
    (MODEL DAMP X+).  Walls are free-slip."""
    c = new_case("porous_flume", np.arange(nx + 1) * dx, np.arange(ny + 1) * dy,
                 np.arange(nz + 1) * dz)
    i1 = int(round(block[0] / dx)) + 2
    i2 = int(round(block[1] / dx)) + 1
    k2 = min(int(round(block[2] / dz)) + 1, nz + 1)
    add_porous(c, i1, 2, 2, i2, ny + 1, k2, gamma, cm, cd)
    c.params.update(wvlvl=depth, wbub=-1.0, cgepsr=1.0e-10,
                    glxmin=0.0, glxmax=nx * dx, glymin=0.0, glymax=ny * dy,
                    idamp=[-1, sponge_degree, -1, -1],
                    damp_xp=[0.6, 0.6, sponge_width, depth])
    init_f_still_water(c, depth)
    c.dt = dt
    return finish(c)


def solitary_beach(nx=1024, ny=128, nz=128, dx=0.02, dy=0.02, dz=0.01,
                   depth=0.6, x_toe=10.0, slope=1.0 / 20.0, amp=0.15,
                   x0=5.0, nbox=40, seed=0, dt=1.0e-3):
    """Solitary wave on a 1:20 beach with 40 seeded porous boxes.

    Beach: staircase obstacle cells below z = (x - x_toe)*slope.  Boxes:
    sides U(0.1,0.5) m, porosity U(0.3,1.0), resting on the bed.  The first
    order solitary wave eta = A sech^2(k (x-x0)), k = sqrt(3A/(4h^3)),
    u = sqrt(g/h) eta, is injected as the initial F and u."""
    rng = np.random.Generator(np.random.Philox(seed))
    c = new_case("solitary_beach", np.arange(nx + 1) * dx, np.arange(ny + 1) * dy,
                 np.arange(nz + 1) * dz)
    xc = (np.arange(nx) + 0.5) * dx
    zb = np.clip((xc - x_toe) * slope, 0.0, None)
    for i in range(nx):
        kk = int(np.floor(zb[i] / dz + 1e-9))
        if kk > 0:
            c.nf[i + 1, 1:-1, 1:kk + 1] = -1
    for _ in range(nbox):
        sx, sy, sz = rng.uniform(0.1, 0.5, size=3)
        g = rng.uniform(0.3, 1.0)
        bx = rng.uniform(0.0, nx * dx - sx)
        by = rng.uniform(0.0, ny * dy - sy)
        i1 = int(bx / dx) + 2
        i2 = min(int((bx + sx) / dx) + 1, nx + 1)
        j1 = int(by / dy) + 2
        j2 = min(int((by + sy) / dy) + 1, ny + 1)
        ic = min(max((i1 + i2) // 2 - 2, 0), nx - 1)
        kb = int(np.floor(zb[ic] / dz + 1e-9)) + 2
        k2 = min(kb + int(sz / dz) - 1, nz + 1)
        if i2 >= i1 and j2 >= j1 and k2 >= kb:
            add_porous(c, i1, j1, kb, i2, j2, k2, g)
    g0 = 9.8
    k_s = np.sqrt(3.0 * amp / (4.0 * depth ** 3))
    eta = amp / np.cosh(k_s * (xc - x0)) ** 2
    c.params.update(wvlvl=depth, wbub=-1.0, cgepsr=1.0e-8)
    init_f_still_water(c, depth)
    ff = c.ff
    z1 = c.zz[0]
    for i in range(nx):
        lvl = depth + eta[i]
        for k in range(1, nz + 1):
            if z1[k] > lvl:
                v = 0.0
            elif z1[k + 1] < lvl:
                v = 1.0
            else:
                v = (lvl - z1[k]) / (z1[k + 1] - z1[k])
            ff[i + 1, 1:-1, k] = np.where(c.nf[i + 1, 1:-1, k] != -1, v, 0.0)
    c.dt = dt
    finish(c)
    xf = c.xx[0]                                   # XX(1,I): face I position
    u_face = np.sqrt(g0 / depth) * amp / np.cosh(k_s * (xf - x0)) ** 2
    nf, ff, uu = c.nf, c.ff, c.uu
    for i0 in range(2, c.ni - 1):                  # faces I = 3..NUMI-1
        m = (nf[i0 - 1] != -1) & (nf[i0] != -1) & ((ff[i0 - 1] > 0.0) | (ff[i0] > 0.0))
        uu[i0] = np.where(m, u_face[i0], 0.0)
    c.hydrostatic = True
    return c


def random_tank(seed=0, nx=12, ny=6, nz=10, d=0.01, nobst=2, nporous=2,
                level=0.55, nbox=2, dt=2.0e-4, slip=True):
    """Small random tank for parity tests: obstacles, porous blocks, a still
    water level and random F boxes, with random face spacing."""
    rng = np.random.Generator(np.random.Philox(seed))

    def axis(n):
        w = rng.uniform(0.8, 1.25, size=n) * d
        return np.concatenate([[0.0], np.cumsum(w)])

    c = new_case(f"random_tank_{seed}", axis(nx), axis(ny), axis(nz))
    for _ in range(nobst):
        i1 = int(rng.integers(3, nx)); j1 = int(rng.integers(2, ny + 1))
        i2 = min(i1 + int(rng.integers(0, 3)), nx + 1)
        j2 = min(j1 + int(rng.integers(0, 3)), ny + 1)
        k2 = int(rng.integers(2, max(3, nz // 3)))
        add_obstacle(c, i1, j1, 2, i2, j2, k2)
    for _ in range(nporous):
        i1 = int(rng.integers(2, nx)); j1 = int(rng.integers(2, ny))
        k1 = int(rng.integers(2, nz))
        i2 = min(i1 + int(rng.integers(1, 4)), nx + 1)
        j2 = min(j1 + int(rng.integers(1, 4)), ny + 1)
        k2 = min(k1 + int(rng.integers(1, 4)), nz + 1)
        add_porous(c, i1, j1, k1, i2, j2, k2, float(rng.uniform(0.3, 0.9)),
                   float(rng.uniform(0.0, 1.5)), float(rng.uniform(0.0, 2.0)))
    ztop = c.zz[0, -1]
    wv = level * ztop
    c.params.update(wvlvl=wv, wbub=-1.0, cgepsr=1.0e-12)
    init_f_still_water(c, wv)
    for _ in range(nbox):
        i1 = int(rng.integers(2, nx + 1)); i2 = min(i1 + int(rng.integers(1, 5)), nx + 1)
        j1 = int(rng.integers(2, ny + 1)); j2 = min(j1 + int(rng.integers(1, 4)), ny + 1)
        k1 = int(rng.integers(2, nz + 1)); k2 = min(k1 + int(rng.integers(1, 4)), nz + 1)
        f_box(c, i1, j1, k1, i2, j2, k2, float(rng.choice([0.0, 1.0, rng.uniform()])))
    c.dt = dt
    finish(c, vp_type=VP_SLIP if slip else VP_NOSLIP)
    return c


def turbulence(c: Case, k0=1.0e-4, e0=1.0e-5, seed=None, **consts):
    """Switch the k-epsilon model on (LEQK = 1) with initial k0, e0
    (AKINIK, AKINIE).  With a seed, each boundary face gets a random k and
    e type among fixed/zero gradient with and without convective inflow
    (1, 2, -1, -2: 'FIX+A', 'FREE+A', 'FIX-A', 'FREE-A') and fixed values
    near k0, e0."""
    c.params.update(leqk=1, akinik=k0, akinie=e0, **consts)
    if seed is not None:
        rng = np.random.Generator(np.random.Philox(seed + 1000))
        nb = c.indbk.size
        c.indbk = rng.choice(np.array([1, 2, -1, -2], dtype=np.int32), size=nb)
        c.indbe = rng.choice(np.array([1, 2, -1, -2], dtype=np.int32), size=nb)
        c.bck = rng.uniform(0.5, 2.0, size=nb) * k0
        c.bce = rng.uniform(0.5, 2.0, size=nb) * e0
    return c


def turbulent_tank(seed=0, k0=1.0e-4, e0=1.0e-5, **kw):
    """A random tank (obstacles, porous blocks, F boxes) with the k-epsilon
    model on and random k, e boundary types."""
    c = random_tank(seed, **kw)
    c.name = f"turbulent_tank_{seed}"
    return turbulence(c, k0, e0, seed=seed)


def loglaw_walls(c: Case, seed=0, frac=0.6, ks=(2.0e-4, 2.0e-3)) -> Case:
    """Turn a seeded fraction `frac` of the slip and no-slip faces into
    log-law (6) or fully rough (8) walls, half each, the rough ones with a
    roughness BCVI uniform in `ks` (input 'B.C. LOG-LAW', 'B.C. ROUGH'); the
    k and e types of those faces follow the velocity type, as VF_IIBOUN
    sets them."""
    rng = np.random.Generator(np.random.Philox(seed + 2000))
    nb = c.indb.shape[1]
    c.bcvi = np.zeros(max(nb, 1))
    for L in range(nb):
        if c.indb[2, L] not in (VP_SLIP, VP_NOSLIP) or rng.uniform() >= frac:
            continue
        t = VP_LOGLAW if rng.uniform() < 0.5 else VP_ROUGH
        c.indb[2, L] = t
        if t == VP_ROUGH:
            c.bcvi[L] = rng.uniform(*ks)
        c.indbk[L] = t
        c.indbe[L] = t
    return c


def loglaw_tank(seed=0, turb=False, speed=0.05, **kw):
    """A random tank whose walls are partly log-law and rough walls, with
    a seeded flow (|u|, |v|, |w| up to `speed`) in the water so that the
    walls shear from the first step; `turb` switches the k-epsilon model on
    (so that the cells next to those walls take VF_BWKELG's k and e)."""
    c = random_tank(seed, **kw)
    c.name = f"loglaw_tank_{seed}"
    if turb:
        turbulence(c, seed=None)
    loglaw_walls(c, seed)
    rng = np.random.Generator(np.random.Philox(seed + 3000))
    wet = c.ff > 0.0
    for a in (c.uu, c.vv, c.ww):
        a += rng.uniform(-speed, speed, a.shape) * wet
    return c


def droplet_tank(seed=0, nx=24, ny=6, nz=20, d=0.01, ndrop=8, level=0.3, dt=2.0e-3, speed=1.0):
    """Droplets over a pool (the TimerDoor droplet model VF_FDROPF): single
    water cells (F in 0.3..1) in the air, each isolated, so the flag update
    turns them into gas cells that hold water.  An obstacle step and a
    porous block stand in the pool; droplets above the step land on it.
    c.drop_state holds droplet arrays (DROPTX..DROPWW, flat, column-major)
    that make the droplets old ones (time 0) already moving with random
    velocities (|u|, |w| up to `speed`, |v| up to speed/2), for
    cadmas_set_drop: they then fly sideways, rise and fall from the first
    steps."""
    rng = np.random.Generator(np.random.Philox(seed))

    def axis(n):
        w = rng.uniform(0.85, 1.2, size=n) * d
        return np.concatenate([[0.0], np.cumsum(w)])

    c = new_case(f"droplet_tank_{seed}", axis(nx), axis(ny), axis(nz))
    kw = max(3, int(level * nz))          # last water layer
    ks = kw + 3                           # top of the obstacle step
    i1s = nx // 2 + 2
    add_obstacle(c, i1s, 2, 2, nx + 1, ny + 1, ks)
    add_porous(c, 3, 2, 2, 5, ny + 1, kw, 0.5, 0.8, 1.0)
    wv = c.zz[0, kw]
    c.params.update(wvlvl=wv, wbub=-1.0, cgepsr=1.0e-12, idrop=1)
    init_f_still_water(c, wv)
    placed = []
    tries = 0
    while len(placed) < ndrop and tries < 1000:
        tries += 1
        i = int(rng.integers(3, nx + 1)); j = int(rng.integers(2, ny + 2))
        k = int(rng.integers(ks + 2, nz))
        if c.nf[i - 1, j - 1, k - 1] == -1 or any(abs(i - a) + abs(j - b) + abs(k - e) < 4 for a, b, e in placed):
            continue
        placed.append((i, j, k))
        c.ff[i - 1, j - 1, k - 1] = float(rng.uniform(0.3, 1.0))
    c.dt = dt
    finish(c)
    shape = (c.ni, c.nj, c.nk)
    ds = {"droptx": _z3(*shape, -1.0e10)}
    for nm in ("dropty", "droptz", "dropuu", "dropvv", "dropww"):
        ds[nm] = _z3(*shape)
    for i, j, k in placed:
        u, v, w = (float(rng.uniform(-speed, speed)) for _ in range(3))
        c0 = (i - 1, j - 1, k - 1)
        ds["droptx"][c0] = ds["dropty"][c0] = ds["droptz"][c0] = 0.0
        ds["dropuu"][c0], ds["dropvv"][c0], ds["dropww"][c0] = u, 0.5 * v, w
    c.drop_state = {nm: a.reshape(-1, order="F") for nm, a in ds.items()}
    return c


def linear_wave_initial(c: Case, H: float, T: float, depth: float, g0: float = 9.8, phase0: float = 0.0):
    """Fill the tank with a first-order (Airy) progressive wave train,
    eta = H/2 cos(kx + 2 pi phase0), u = H/2 w cosh(kz)/sinh(kh) cos(kx + 2 pi phase0),
    w = H/2 w sinh(kz)/sinh(kh) sin(kx + 2 pi phase0) (z from the bed), with
    w^2 = g k tanh(k h): the train a wave maker at x = 0 whose phase at
    TNOW = 0 is phase0 would have made (phase 0: a crest at x = 0)."""
    ph = 2.0 * np.pi * phase0
    om = 2.0 * np.pi / T
    k = om * om / g0
    for _ in range(60):  # Newton on f(k) = g k tanh(kh) - w^2
        th = np.tanh(k * depth)
        fk = g0 * k * th - om * om
        dk = g0 * th + g0 * k * depth * (1.0 - th * th)
        k -= fk / dk
    a = 0.5 * H
    x1, z1 = c.xx[0], c.zz[0]
    xc = 0.5 * (x1[1:-1] + x1[2:])                    # cell centres I = 2..NI-1
    level = depth + a * np.cos(k * xc + ph)
    for i in range(1, c.ni - 1):
        lv = level[i - 1]
        for kk in range(1, c.nk - 1):
            if z1[kk] > lv:
                v = 0.0
            elif z1[kk + 1] < lv:
                v = 1.0
            else:
                v = (lv - z1[kk]) / (z1[kk + 1] - z1[kk])
            c.ff[i, 1:-1, kk] = np.where(c.nf[i, 1:-1, kk] != -1, v, 0.0)
    zc = 0.5 * (z1[1:-1] + z1[2:])                    # cell-centre heights K = 2..NK-1
    sk = np.sinh(k * depth)
    wet = c.ff > 0.0
    for i0 in range(2, c.ni - 1):                     # x faces between interior cells
        prof = a * om * np.cosh(k * zc) / sk * np.cos(k * x1[i0] + ph)
        m = (c.nf[i0 - 1, 1:-1, 1:-1] != -1) & (c.nf[i0, 1:-1, 1:-1] != -1) & \
            (wet[i0 - 1, 1:-1, 1:-1] | wet[i0, 1:-1, 1:-1])
        c.uu[i0, 1:-1, 1:-1] = np.where(m, prof[None, :], 0.0)
    for kk in range(2, c.nk - 1):                     # z faces between interior cells
        prof = a * om * np.sinh(k * z1[kk]) / sk * np.sin(k * xc + ph)
        m = (c.nf[1:-1, 1:-1, kk - 1] != -1) & (c.nf[1:-1, 1:-1, kk] != -1) & \
            (wet[1:-1, 1:-1, kk - 1] | wet[1:-1, 1:-1, kk])
        c.ww[1:-1, 1:-1, kk] = np.where(m, prof[:, None], 0.0)
    return k


def _wavenumber(T: float, depth: float, g0: float = 9.8) -> float:
    """k of w^2 = g k tanh(k h) by Newton from the deep-water value."""
    om = 2.0 * np.pi / T
    k = om * om / g0
    for _ in range(60):
        th = np.tanh(k * depth)
        fk = g0 * k * th - om * om
        dk = g0 * th + g0 * k * depth * (1.0 - th * th)
        k -= fk / dk
    return k


def first_order_wave_table(H: float, T: float, depth: float, g0: float = 9.8, ntt: int = 121,
                           nzz: int = 81, ztop: float | None = None) -> dict:
    """Matrix table (the input of WAVE-BC ... FUNC MATRIX) of a first-order
    progressive wave at the boundary, eta = H/2 cos(2 pi p),
    u = H/2 w cosh(k(z+h))/sinh(kh) cos(2 pi p),
    w = H/2 w sinh(k(z+h))/sinh(kh) sin(2 pi p), at phases p = 0..1 and
    heights z = -h..ztop above the still water level; the reference's
    phase at time t is p = frac(p0 - t/T), so p0 = 0 puts a crest at
    the boundary at t = 0."""
    k = _wavenumber(T, depth, g0)
    om = 2.0 * np.pi / T
    a = 0.5 * H
    tt = np.linspace(0.0, 1.0, ntt)
    zt = ztop if ztop is not None else 1.5 * a
    zz = np.linspace(-depth, zt, nzz)
    sk = np.sinh(k * depth)
    ph = 2.0 * np.pi * tt
    un = a * om * np.cosh(k * (zz[:, None] + depth)) / sk * np.cos(ph)[None, :]
    ut = a * om * np.sinh(k * (zz[:, None] + depth)) / sk * np.sin(ph)[None, :]
    return dict(tt=tt, hh=a * np.cos(ph), zz=zz, un=np.asfortranarray(un), ut=np.asfortranarray(ut),
                phase0=0.0, mtbtyp=1, wavenumber=k)


def wave_maker(c: Case, H: float, T: float, depth: float, side: int = 1, ramp: float = 0.0,
               table: dict | None = None, stream: int = 0, func: str | None = None,
               angle: tuple | None = None) -> Case:
    """Make side `side` (1 X-, 2 X+, 3 Y-, 4 Y+) a wave-maker boundary:
    its domain-boundary faces get B.C. type 5 for velocity and F
    (WAVE-BC, INDB(3,L) = INDB(4,L) = 5) over the whole side, driven by
    the stream-function wave of order `stream` (WAVE-BC ... FUNC STREAM N)
    when stream >= 1, by the theory `func` ("stokes", "cnoidal",
    "stk-cnd": FUNC STOKES | CNOIDAL | STK-CND), else by a first-order wave
    table unless `table` is given.  `angle` = (degrees, x, y) makes the
    incidence oblique (WAVE-BC ... ANGLE; wave theories only)."""
    ns = {1: 1, 2: 2, 3: 3, 4: 4}[side]
    for L in range(c.indb.shape[1]):
        ijk, NS = int(c.indb[0, L]), int(c.indb[1, L])
        if NS != ns:
            continue
        i = (ijk - 1) % c.ni + 1
        j = ((ijk - 1) // c.ni) % c.nj + 1
        if (side == 1 and i == 2) or (side == 2 and i == c.ni) or (side == 3 and j == 2) or \
                (side == 4 and j == c.nj):
            c.indb[2, L] = VP_WAVE
            c.indb[3, L] = F_WAVE
    first, last = 2, (c.nj - 1 if side <= 2 else c.ni - 1)
    if func is not None:
        from . import wave_solve
        c.wave = dict(side=side, first=first, last=last, depth=depth, period=T, ramp=ramp, table=None,
                      theory=wave_solve(func, depth, T, H, c.params.get("grz0", 9.8)), angle=angle)
        return c
    if stream >= 1:
        from . import stream_solve
        c.wave = dict(side=side, first=first, last=last, depth=depth, period=T, ramp=ramp, table=None,
                      stream=stream_solve(stream, depth, T, H, c.params.get("grz0", 9.8)), angle=angle)
        return c
    if angle is not None:
        raise ValueError("(WAVE-BC ANGLE) CAN NOT USE.: an angle needs a wave theory")
    c.wave = dict(side=side, first=first, last=last, depth=depth, period=T, ramp=ramp,
                  table=table if table is not None else first_order_wave_table(H, T, depth))
    return c


def wave_source(c: Case, line: int, H: float, T: float, depth: float, ramp: float = 0.0, axis: str = "x",
                table: dict | None = None, func=None) -> Case:
    """A wave source line (MODEL WAVE-SRC X|Y ...): the cell column
    I = `line` (axis x, 1-based with ghosts) or row J = `line` (axis y)
    emits waves to both sides, its strength the velocity of the wave theory
    `func` (a stream-function order N, "stokes", "cnoidal" or "stk-cnd":
    FUNC STREAM N | STOKES | CNOIDAL | STK-CND) or else of a first-order
    wave table unless `table` is given (FUNC MATRIX; the table is the one
    of a wave maker, if the case has one)."""
    ln = int(line) if axis == "x" else -int(line)
    if func is not None:
        from . import wave_solve
        c.source = dict(line=ln, depth=depth, period=T, ramp=ramp, table=None,
                        theory=wave_solve(func, depth, T, H, c.params.get("grz0", 9.8)))
        return c
    if table is None and getattr(c, "wave", None) is None:
        table = first_order_wave_table(H, T, depth)
    c.source = dict(line=ln, depth=depth, period=T, ramp=ramp, table=table)
    return c


def source_flume(nx=120, ny=4, nz=40, dx=0.05, dz=0.01, depth=0.25, H=0.03, T=1.2, ramp=0.5,
                 axis="x", sponge_width=1.0, dt=2.0e-3, func=None) -> Case:
    """Still water between two damping zones with a wave source line in
    the middle: along x, the column I = nx/2 + 2 of an nx x ny x nz flume;
    along y, the row J = nx/2 + 2 of the same flume turned by 90 degrees
    (ny x nx x nz).  The source is faded in over `ramp` periods."""
    L, W = np.arange(nx + 1) * dx, np.arange(ny + 1) * dx
    zs = np.arange(nz + 1) * dz
    damp = [0.6, 0.6, sponge_width, depth]
    if axis == "x":
        c = new_case("source_flume_x", L, W, zs)
        c.params.update(glxmin=0.0, glxmax=nx * dx, glymin=0.0, glymax=ny * dx, idamp=[2, 2, -1, -1],
                        damp_xm=damp, damp_xp=damp)
    else:
        c = new_case("source_flume_y", W, L, zs)
        c.params.update(glxmin=0.0, glxmax=ny * dx, glymin=0.0, glymax=nx * dx, idamp=[-1, -1, 2, 2],
                        damp_ym=damp, damp_yp=damp)
    c.params.update(wvlvl=depth, wbub=-1.0, cgepsr=1.0e-10)
    init_f_still_water(c, depth)
    c.dt = dt
    finish(c)
    wave_source(c, nx // 2 + 2, H, T, depth, ramp=ramp, axis=axis, func=func)
    return c


def level_table(amp: float, ntt: int = 121, depth: float = 1.0) -> dict:
    """A matrix table of type MTBTYP 3 (fixed water level): the level
    above WVLVL over one period, amp sin^2(pi p) (a single long crest, as a
    tsunami's leading wave), p the phase in [0,1].  The velocity columns
    are placeholders; a level table sets no velocities."""
    tt = np.linspace(0.0, 1.0, ntt)
    zz = np.array([-depth, 0.0])
    return dict(tt=tt, hh=amp * np.sin(np.pi * tt) ** 2, zz=zz, un=np.zeros((2, ntt), order="F"),
                ut=np.zeros((2, ntt), order="F"), phase0=0.0, mtbtyp=3)


def fixed_level_flume(nx=96, ny=4, nz=48, dx=0.05, dz=0.01, depth=0.3, amp=0.05, T=4.0, ramp=0.0,
                      open_end=True, side=1) -> Case:
    """Flume driven on side `side` (1 = X-) by a fixed water level (WAVE-BC
    ... FUNC MATRIX with MTBTYP 3) following `level_table`: the boundary faces act as free
    faces and the column next to the side takes the level (VF_BWFFSF);
    with `open_end` the X+ side radiates (MODEL OPEN-BC)."""
    c = porous_flume(nx=nx, ny=ny, nz=nz, dx=dx, dy=dx, dz=dz, depth=depth,
                     block=(0.6 * nx * dx, 0.6 * nx * dx + 0.2, depth + amp), gamma=0.5)
    c.params.update(idamp=[-1, -1, -1, -1])
    wave_maker(c, 2.0 * amp, T, depth, side=side, ramp=ramp, table=level_table(amp, depth=depth))
    if open_end:
        open_boundary(c, depth, T, side=2)
    c.name = "fixed_level_flume"
    return c


def open_boundary(c: Case, depth: float, T: float, side: int = 2) -> Case:
    """Make side `side` (1 X-, 2 X+, 3 Y-, 4 Y+) an open (radiation)
    boundary for waves of period T in still-water depth `depth` (MODEL
    OPEN-BC, vf_iimdl.f:176-213): its domain-boundary faces get B.C. type 7
    for velocity and F with zero values (vf_csetup.f:146-213)."""
    for L in range(c.indb.shape[1]):
        ijk, NS = int(c.indb[0, L]), int(c.indb[1, L])
        if NS != side:
            continue
        i = (ijk - 1) % c.ni + 1
        j = ((ijk - 1) // c.ni) % c.nj + 1
        if (side == 1 and i == 2) or (side == 2 and i == c.ni) or (side == 3 and j == 2) or \
                (side == 4 and j == c.nj):
            c.indb[2, L] = VP_OPEN
            c.indb[3, L] = F_OPEN
            for a in (c.bcu, c.bcv, c.bcw, c.bcp, c.bcf):
                if a is not None:
                    a[L] = 0.0
    c.open = (c.open or []) + [dict(side=side, depth=depth, period=T)]
    return c


def open_flume(nx=160, ny=4, nz=64, dx=0.02, dz=0.01, depth=0.4, H=0.06, T=1.2, seed=0,
               y_open=False) -> Case:
    """Wave flume with a wave maker at X- and a radiation outlet at X+ in
    place of a damping zone, a developed wave train already in it and
    seeded noise (Philox) on the velocities; `y_open` opens the Y+ side too."""
    c = porous_flume(nx=nx, ny=ny, nz=nz, dx=dx, dy=dx, dz=dz, depth=depth,
                     block=(0.6 * nx * dx, 0.6 * nx * dx + 0.2, depth + H), gamma=0.5)
    c.params.update(idamp=[-1, -1, -1, -1])  # no damping zone
    linear_wave_initial(c, H, T, depth)
    rng = np.random.Generator(np.random.Philox(seed))
    for a in (c.uu, c.vv, c.ww):
        a += rng.normal(0.0, 0.002, a.shape) * (c.ff > 0.0)
    wave_maker(c, H, T, depth, side=1)
    open_boundary(c, depth, T, side=2)
    if y_open:
        open_boundary(c, depth, T, side=4)
    c.name = "open_flume"
    return c


def ensemble_flumes(members: int = 64, seed: int = 0, dx: float = 0.02, dz: float = 0.01,
                    scale: float = 1.0) -> list:
    """Independent wave flumes of uneven size: nx in U{256..1024},
    ny in U{16..64}, nz in U{64..128} (times `scale` in x), depth U(0.4,0.8)
    m (kept below 0.75 of the flume height), regular waves H U(0.05,0.2) m,
    T U(1,3) s from a wave maker on a developed wave train, one porous block
    of porosity U(0.3,0.6) per flume (seeded, Philox)."""
    rng = np.random.Generator(np.random.Philox(seed))
    out = []
    for m in range(members):
        nx = max(16, int(rng.integers(256, 1025) * scale))
        ny = int(rng.integers(16, 65))
        nz = int(rng.integers(64, 129))
        depth = min(float(rng.uniform(0.4, 0.8)), 0.75 * nz * dz)
        H = min(float(rng.uniform(0.05, 0.2)), 0.3 * depth)
        T = float(rng.uniform(1.0, 3.0))
        gam = float(rng.uniform(0.3, 0.6))
        x0 = float(rng.uniform(0.3, 0.6)) * nx * dx
        c = porous_flume(nx=nx, ny=ny, nz=nz, dx=dx, dy=dx, dz=dz, depth=depth,
                         block=(x0, x0 + 1.0, depth + H), gamma=gam,
                         sponge_width=min(2.0, 0.2 * nx * dx))
        linear_wave_initial(c, H, T, depth)
        wave_maker(c, H, T, depth)
        c.name = f"ensemble_{m}"
        out.append(c)
    return out