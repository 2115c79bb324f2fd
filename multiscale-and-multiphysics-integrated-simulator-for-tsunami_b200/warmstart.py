"""Training of the learned initial guess of the pressure solve (warm_start=2).

The network (cadmas_unet_*, tcgen05 convolutions) maps, per cell,
(BB/s, F, GGV, INDC != -1) to PT/s, s the RMS of BB over computed cells.
Its training pairs are the solver's own: each step of a run with the plain
zero guess gives the right-hand side BB and the converged correction PT of
its pressure solve, with F and INDC as they were when the system was
assembled.  Training minimises the mean square error of PT/s over computed
cells plus the residual |BB - A PT| of the guess in the sample's own
pressure system, with Adam on the GPU.

    samples = collect(case, steps=200)            # (x, t, m, a7) per step
    params, c = train(samples, epochs=20)         # FP32 parameters, scale
    tank = Tank(case, warm_start=2); tank.set_warm_net(params, c)
"""
from __future__ import annotations

import numpy as np

from . import Tank, UNet


def volume_dims(case):
    """The network's volume (X, Y, Z): the grid rounded up to multiples of 4."""
    r = lambda n: (n + 3) & ~3
    return r(case.ni), r(case.nj), r(case.nk)


def features(case, ff, indc, bb):
    """(x, s): x the (Z, Y, X, 4) float32 input as the device builds it
    (warmstart.cu, k_ws_features), s the scale of BB."""
    X, Y, Z = volume_dims(case)
    live = indc != -1
    inner = np.zeros(live.shape, bool)
    inner[1:-1, 1:-1, 1:-1] = True
    sel = live & inner
    n = int(sel.sum())
    s = float(np.sqrt((bb[sel] ** 2).sum() / n)) if n and (bb[sel] ** 2).sum() > 0 else 1.0
    x = np.zeros((Z, Y, X, 4), np.float32)
    ni, nj, nk = case.ni, case.nj, case.nk
    T = lambda a: np.transpose(a, (2, 1, 0))  # (ni,nj,nk) -> (nk,nj,ni)
    x[:nk, :nj, :ni, 0] = T(np.where(live, bb / s, 0.0))
    x[:nk, :nj, :ni, 1] = T(ff)
    x[:nk, :nj, :ni, 2] = T(case.ggv)
    x[:nk, :nj, :ni, 3] = T(live.astype(np.float64))
    return x, s


def target(case, indc, pt, s):
    """(t, m): PT/s and the mask of interior computed cells, (Z, Y, X)."""
    X, Y, Z = volume_dims(case)
    sel = indc != -1
    inner = np.zeros(sel.shape, bool)
    inner[1:-1, 1:-1, 1:-1] = True
    sel &= inner
    T = lambda a: np.transpose(a, (2, 1, 0))
    t = np.zeros((Z, Y, X), np.float32)
    m = np.zeros((Z, Y, X), np.float32)
    t[:case.nk, :case.nj, :case.ni] = T(np.where(sel, pt / s, 0.0))
    m[:case.nk, :case.nj, :case.ni] = T(sel.astype(np.float64))
    return t, m


def system_volume(case, sysd):
    """(Z, Y, X, 7) float32: AD, ALI, ALJ, ALK, AUI, AUJ, AUK per voxel."""
    X, Y, Z = volume_dims(case)
    a = np.zeros((Z, Y, X, 7), np.float32)
    for k, n in enumerate(("ad", "ali", "alj", "alk", "aui", "auj", "auk")):
        a[:case.nk, :case.nj, :case.ni, k] = np.transpose(sysd[n], (2, 1, 0))
    return a


def collect(case, steps, every=1, skip=0, **tank_kw):
    """Training samples (x, t, m, a7) from a run of `steps` steps with the
    zero guess: one per `every` steps after the first `skip`; t = PT/s."""
    tank = Tank(case, **tank_kw)
    tank.init_state(case.hydrostatic)
    out = []
    for n in range(steps):
        st = tank.get_state()
        tank.set_time(st["tnow"] + case.dt, case.dt, st["nnow"] + 1)
        tank.v1cal()
        take = n >= skip and (n - skip) % every == 0
        if take:
            sysd = tank.get_system()
            bb, pt = tank.get_solve()
        tank.f1cal()
        if take:
            x, s = features(case, st["ff"], st["indc"], bb)
            t, m = target(case, st["indc"], pt, s)
            out.append((x, t, m, system_volume(case, sysd)))
    return out


def output_scale(samples):
    """RMS of PT/s over the counted cells of the samples: the network
    predicts PT/(s c) with this c."""
    num = sum(float((t ** 2 * m).sum()) for _, t, m, _ in samples)
    den = sum(float(m.sum()) for _, _, m, _ in samples)
    return float(np.sqrt(num / den)) if den > 0 and num > 0 else 1.0


# (cin, cout) of the ten 3x3x3 convolutions, in parameter order
LAYERS = [(16, 16), (16, 16), (16, 32), (32, 32), (32, 64), (64, 64), (96, 32), (32, 32), (48, 16), (16, 16)]


def init_params(seed=0):
    """He initialisation (FP32) of the network's parameters in the library's
    order (per convolution W[cout][27][cin] then b[cout]; head 16 + 1),
    zero on the 12 unused input channels of the first layer."""
    rng = np.random.default_rng(seed)
    out = []
    for l, (cin, cout) in enumerate(LAYERS):
        fan = 27 * (4 if l == 0 else cin)
        w = rng.normal(0.0, np.sqrt(2.0 / fan), (cout, 27, cin))
        if l == 0:
            w[:, :, 4:] = 0.0
        out += [w.ravel(), rng.normal(0.0, 0.01, cout)]
    out += [rng.normal(0.0, 0.25, 16), np.zeros(1)]
    return np.concatenate(out).astype(np.float32)


def train(samples, epochs=20, batch=1, lr=1.0e-3, seed=0, params=None, w_mse=1.0, w_res=1.0, c=None, log=None):
    """Adam on the GPU over the samples (x, t, m, a7) with the loss
    w_mse |m (y - t/c)|^2 / n + w_res |m (b - c A (m y))|^2 / n;
    returns (FP32 parameters, c)."""
    x0 = samples[0][0]
    Z, Y, X, _ = x0.shape
    c = output_scale(samples) if c is None else c
    net = UNet(X, Y, Z, batch)
    net.set_params(params if params is not None else init_params(seed))
    rng = np.random.default_rng(seed)
    for ep in range(epochs):
        order = rng.permutation(len(samples))
        tot, nb = 0.0, 0
        for i in range(0, len(order) - batch + 1, batch):
            idx = order[i:i + batch]
            xb = np.stack([samples[j][0] for j in idx])
            tb = np.stack([samples[j][1] for j in idx]) / c
            mb = np.stack([samples[j][2] for j in idx])
            ab = np.stack([samples[j][3] for j in idx])
            loss, _ = net.train_sys(xb, tb, mb, ab, c=c, w_mse=w_mse, w_res=w_res, lr=lr)
            tot += loss
            nb += 1
        if log is not None:
            log(ep, tot / max(1, nb))
    p = net.get_params()
    net.close()
    return p, c
