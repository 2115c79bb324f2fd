"""The CPU reference of the warm-start U-Net (oracle/unet_ref.py) against
central finite differences of its own loss: directional derivatives along
random directions agree with the analytic gradient to 1e-6 relative in
FP64.  This pins the reference that the GPU's gradients are checked
against."""
import pathlib
import sys

import numpy as np

sys.path.insert(0, str(pathlib.Path(__file__).resolve().parents[1] / "oracle"))
import unet_ref as R  # noqa: E402


def sample(seed, B=1, Z=4, Y=4, X=8):
    rng = np.random.default_rng(seed)
    x = rng.normal(size=(B, Z, Y, X, 4))
    t = rng.normal(size=(B, Z, Y, X))
    m = (rng.uniform(size=(B, Z, Y, X)) < 0.8).astype(float)
    return x, t, m


def test_reference_gradient_matches_finite_differences():
    p = R.he_init(1)
    x, t, m = sample(2)
    loss, g = R.loss_grad(p, x, t, m)
    rng = np.random.default_rng(3)
    h = 1e-6
    for _ in range(4):
        v = rng.normal(size=p.size)
        v /= np.linalg.norm(v)
        lp, _ = R.loss_grad(p + h * v, x, t, m)
        lm, _ = R.loss_grad(p - h * v, x, t, m)
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g @ v) <= 1e-6 * max(abs(fd), 1e-3 * abs(loss)), (fd, g @ v)


def test_reference_layer_shapes_and_count():
    assert R.NPARAM == sum(27 * a * b + b for a, b, _ in R.LAYERS) + 17
    p = R.he_init(0)
    x, _, _ = sample(0, B=2, Z=8, Y=4, X=4)
    y, A = R.forward(p, x)
    assert y.shape == (2, 8, 4, 4)
    assert A["u2"].shape[-1] == 96 and A["u1"].shape[-1] == 48


def test_bf16_rounding():
    v = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -9, -3.14159, 1e-30])
    r = R.bf16(v)
    assert r[0] == 1.0 and r[1] == 1.0  # tie to even
    assert r[2] == 1.0 + 2 ** -7
    assert abs(r[3] + 3.140625) < 1e-12


def test_residual_loss_gradient_matches_finite_differences():
    p = R.he_init(4)
    x, t, m = sample(5)
    rng = np.random.default_rng(6)
    a7 = rng.normal(size=x.shape[:4] + (7,))
    a7[..., 0] += 6.0
    kw = dict(a7=a7, c=0.7, w_mse=0.3, w_res=1.0)
    loss, g = R.loss_grad(p, x, t, m, **kw)
    h = 1e-6
    for _ in range(3):
        v = rng.normal(size=p.size)
        v /= np.linalg.norm(v)
        fd = (R.loss_grad(p + h * v, x, t, m, **kw)[0] - R.loss_grad(p - h * v, x, t, m, **kw)[0]) / (2 * h)
        assert abs(fd - g @ v) <= 1e-6 * max(abs(fd), 1e-3 * abs(loss)), (fd, g @ v)


def test_transposed_system_is_the_adjoint():
    rng = np.random.default_rng(7)
    a7 = rng.normal(size=(2, 4, 4, 8, 7))
    f, r = rng.normal(size=(2, 4, 4, 8)), rng.normal(size=(2, 4, 4, 8))
    assert abs((R.apply_sys(a7, f) * r).sum() - (f * R.apply_sys_t(a7, r)).sum()) < 1e-10
