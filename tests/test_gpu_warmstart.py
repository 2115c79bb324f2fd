"""The learned initial guess of the pressure solve (warm_start = 2).

- The training loss with the residual term (cadmas_unet_train_sys) has the
  gradient of the FP64 reference (oracle/unet_ref.py), per layer cosine
  >= 0.99.
- A network whose guess does not lower |BB - A PT0| is dropped on every
  step, and the run is then bit for bit the zero-guess run.
- A network trained on a dam break's own solves gives guesses that are
  kept, and the run with them meets the same stopping test: every solve's
  true relative residual stays within 10x of the zero-guess run's largest,
  and the fluid volume matches it to 1e-9.
"""
import importlib
import pathlib
import sys

import numpy as np
import pytest

sys.path.insert(0, str(pathlib.Path(__file__).resolve().parents[1] / "oracle"))
import unet_ref as R  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ws(pkg):
    return importlib.import_module("cadmas_b200.warmstart")


def test_residual_loss_gradient_matches_reference(gpu_lib, pkg):
    B, Z, Y, X = 2, 8, 4, 8
    rng = np.random.default_rng(11)
    x = rng.normal(size=(B, Z, Y, X, 4)).astype(np.float32)
    t = rng.normal(size=(B, Z, Y, X)).astype(np.float32)
    m = (rng.uniform(size=(B, Z, Y, X)) < 0.8).astype(np.float32)
    a7 = rng.normal(size=(B, Z, Y, X, 7)).astype(np.float32)
    a7[..., 0] += 6.0
    p = R.he_init(12).astype(np.float32)
    net = pkg.UNet(X, Y, Z, B)
    net.set_params(p)
    kw = dict(c=0.7, w_mse=0.3, w_res=1.0)
    loss, g = net.train_sys(x, t, m, a7, update=False, want_grad=True, **kw)
    l_ex, g_ex = R.loss_grad(p.astype(np.float64), x.astype(np.float64), t.astype(np.float64),
                             m.astype(np.float64), a7=a7.astype(np.float64), **kw)
    assert abs(loss - l_ex) <= 3e-2 * l_ex
    for l in range(len(R.LAYERS)):
        a, b = R.OFFS[l][0], R.OFFS[l][1] + R.LAYERS[l][1]
        ga, ge = g[a:b].astype(np.float64), g_ex[a:b]
        if l == 0:
            keep = np.zeros((16, 27, 16), bool)
            keep[:, :, :4] = True
            keep = np.concatenate([keep.ravel(), np.ones(16, bool)])
            ga, ge = ga[keep], ge[keep]
        cos = ga @ ge / (np.linalg.norm(ga) * np.linalg.norm(ge))
        assert cos >= 0.99, (l, cos)


def test_bad_network_is_dropped(gpu_lib, pkg, ws):
    c = pkg.cases.dam_break()
    a = pkg.Tank(c)
    b = pkg.Tank(c, warm_start=2)
    b.set_warm_net(ws.init_params(0) * 30.0, 50.0)
    a.init_state(True)
    b.init_state(True)
    for _ in range(6):
        a.step(c.dt)
        b.step(c.dt)
    assert b.warm_stats() == (0, 6)
    sa, sb = a.get_state(), b.get_state()
    for k in ("uu", "vv", "ww", "pp", "ff", "nf"):
        assert sa[k].tobytes() == sb[k].tobytes(), k


def test_trained_guess_is_used_and_meets_the_tolerance(gpu_lib, pkg, ws):
    c = pkg.cases.dam_break()
    samples = ws.collect(c, 60)
    params, scale = ws.train(samples, epochs=25, batch=4, lr=1e-3, w_mse=0.1, w_res=1.0)
    runs = {}
    for mode in (0, 2):
        t = pkg.Tank(c, warm_start=mode, diag_relres=1)
        if mode == 2:
            t.set_warm_net(params, scale)
        t.init_state(True)
        it, rel = [], []
        for _ in range(60):
            t.step(c.dt)
            s = t.stats()
            it.append(s["icgitr"])
            rel.append(s["true_relres"])
        runs[mode] = (it, rel, t.stats()["fsum"], t.warm_stats() if mode == 2 else None)
    kept, dropped = runs[2][3]
    assert kept + dropped == 60 and kept > 0
    assert max(runs[2][1]) <= 10.0 * max(runs[0][1])
    assert abs(runs[2][2] - runs[0][2]) <= 1e-9 * runs[0][2]
    print(f"iterations zero {sum(runs[0][0])} learned {sum(runs[2][0])}, kept {kept}/60")
