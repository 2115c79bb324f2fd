"""CPU reference of the learned warm start's U-Net (test infrastructure).

The same network as the library's cadmas_unet (csrc/unet.cu): 3x3x3
convolutions with bias and ReLU over channels 16/32/64, 2x2x2 average
pooling, nearest upsampling with skip concatenation, a 1x1x1 head, masked
mean-square loss; forward and backward in numpy FP64.

  q=None      exact FP64 (the gradient reference; itself checked against
              central finite differences in tests/test_unet_ref.py)
  q=bf16      rounds weights, activations and the stored gradients to
              BF16 where the GPU stores BF16, so the GPU differs from it
              only by FP32 versus FP64 accumulation

Arrays: volumes (B, Z, Y, X, C) C-ordered (x fastest), as the library's
host arrays; parameters one flat vector in the library's order (per
convolution W[cout][27][cin] then b[cout]; head 16 weights, bias).
"""
import numpy as np

LAYERS = [(16, 16, 0), (16, 16, 0), (16, 32, 1), (32, 32, 1), (32, 64, 2),
          (64, 64, 2), (96, 32, 1), (32, 32, 1), (48, 16, 0), (16, 16, 0)]


def offsets():
    out, o = [], 0
    for cin, cout, _ in LAYERS:
        out.append((o, o + 27 * cin * cout))
        o += 27 * cin * cout + cout
    return out, o, o + 16, o + 17


OFFS, HEAD_W, HEAD_B, NPARAM = offsets()


def bf16(a):
    """Round to the nearest BF16 (ties to even), as __float2bfloat16."""
    x = np.asarray(a, dtype=np.float32)
    u = x.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return r.view(np.float32).astype(np.float64)


def ident(a):
    return np.asarray(a, dtype=np.float64)


def unpack(p):
    ws = []
    for (cin, cout, _), (w, b) in zip(LAYERS, OFFS):
        ws.append((p[w:b].reshape(cout, 27, cin), p[b:b + cout]))
    return ws, p[HEAD_W:HEAD_B], p[HEAD_B]


def he_init(seed=0):
    rng = np.random.default_rng(seed)
    p = np.zeros(NPARAM)
    for (cin, cout, _), (w, b) in zip(LAYERS, OFFS):
        fan = 27 * (4 if (cin, cout) == (16, 16) and w == 0 else cin)
        p[w:b] = rng.normal(0.0, np.sqrt(2.0 / fan), 27 * cin * cout)
        if w == 0:  # only the 4 real input channels of the first layer
            p[w:b].reshape(cout, 27, cin)[:, :, 4:] = 0.0
        p[b:b + cout] = rng.normal(0.0, 0.01, cout)
    p[HEAD_W:HEAD_B] = rng.normal(0.0, np.sqrt(1.0 / 16), 16)
    return p


def _taps():
    return [(t // 9 - 1, (t // 3) % 3 - 1, t % 3 - 1) for t in range(27)]


def _shift(x, dz, dy, dx):
    """x[b, z+dz, y+dy, x+dx, :] with zeros outside."""
    B, Z, Y, X, C = x.shape
    p = np.zeros((B, Z + 2, Y + 2, X + 2, C))
    p[:, 1:-1, 1:-1, 1:-1] = x
    return p[:, 1 + dz:1 + dz + Z, 1 + dy:1 + dy + Y, 1 + dx:1 + dx + X]


def conv(x, W, b):
    y = np.broadcast_to(b, x.shape[:4] + (W.shape[0],)).copy()
    for t, (dz, dy, dx) in enumerate(_taps()):
        y += _shift(x, dz, dy, dx) @ W[:, t, :].T
    return y


def conv_back(x, W, dy):
    """(dx, dW, db) of y = conv(x, W, b) for output gradient dy."""
    dW = np.zeros_like(W)
    dx = np.zeros_like(x)
    for t, (dz, dyy, dxx) in enumerate(_taps()):
        xs = _shift(x, dz, dyy, dxx)
        dW[:, t, :] = np.einsum("bzyxo,bzyxc->oc", dy, xs)
        dx += _shift(dy @ W[:, t, :], -dz, -dyy, -dxx)
    return dx, dW, dy.sum(axis=(0, 1, 2, 3))


def pool(x):
    B, Z, Y, X, C = x.shape
    return x.reshape(B, Z // 2, 2, Y // 2, 2, X // 2, 2, C).mean(axis=(2, 4, 6))


def pool_back(d):
    return np.repeat(np.repeat(np.repeat(d, 2, 1), 2, 2), 2, 3) / 8.0


def up(x):
    return np.repeat(np.repeat(np.repeat(x, 2, 1), 2, 2), 2, 3)


def up_back(d):
    B, Z, Y, X, C = d.shape
    return d.reshape(B, Z // 2, 2, Y // 2, 2, X // 2, 2, C).sum(axis=(2, 4, 6))


def forward(p, x4, q=ident):
    """Output (B,Z,Y,X) and the saved activations."""
    ws, wh, bh = unpack(p)
    ws = [(q(W), b) for W, b in ws]
    B, Z, Y, X, _ = x4.shape
    xin = np.zeros((B, Z, Y, X, 16))
    xin[..., :4] = q(x4)
    A = {"xin": xin}
    relu = lambda v: q(np.maximum(v, 0.0))
    A["a0"] = relu(conv(xin, *ws[0]))
    A["a1"] = relu(conv(A["a0"], *ws[1]))
    A["p1"] = q(pool(A["a1"]))
    A["a2"] = relu(conv(A["p1"], *ws[2]))
    A["a3"] = relu(conv(A["a2"], *ws[3]))
    A["p2"] = q(pool(A["a3"]))
    A["a4"] = relu(conv(A["p2"], *ws[4]))
    A["a5"] = relu(conv(A["a4"], *ws[5]))
    A["u2"] = np.concatenate([up(A["a5"]), A["a3"]], axis=-1)
    A["a6"] = relu(conv(A["u2"], *ws[6]))
    A["a7"] = relu(conv(A["a6"], *ws[7]))
    A["u1"] = np.concatenate([up(A["a7"]), A["a1"]], axis=-1)
    A["a8"] = relu(conv(A["u1"], *ws[8]))
    A["a9"] = relu(conv(A["a8"], *ws[9]))
    y = A["a9"] @ wh + bh
    return y, A


def apply_sys(a7, f):
    """A f with the 7 coefficients (AD, ALI, ALJ, ALK, AUI, AUJ, AUK) per
    voxel, zero outside the volume (VF_MZAX)."""
    s = lambda dz, dy, dx: _shift(f[..., None], dz, dy, dx)[..., 0]
    return (a7[..., 0] * f + a7[..., 1] * s(0, 0, -1) + a7[..., 2] * s(0, -1, 0) + a7[..., 3] * s(-1, 0, 0) +
            a7[..., 4] * s(0, 0, 1) + a7[..., 5] * s(0, 1, 0) + a7[..., 6] * s(1, 0, 0))


def apply_sys_t(a7, r):
    """A^T r for the same coefficients."""
    s = lambda f, dz, dy, dx: _shift(f[..., None], dz, dy, dx)[..., 0]
    return (a7[..., 0] * r + s(a7[..., 1] * r, 0, 0, 1) + s(a7[..., 2] * r, 0, 1, 0) + s(a7[..., 3] * r, 1, 0, 0) +
            s(a7[..., 4] * r, 0, 0, -1) + s(a7[..., 5] * r, 0, -1, 0) + s(a7[..., 6] * r, -1, 0, 0))


def loss_grad(p, x4, t, m, q=ident, a7=None, c=1.0, w_mse=1.0, w_res=0.0):
    """w_mse |m (y - t)|^2 / n + w_res |m (b - c A (m y))|^2 / n (n = sum m,
    b = x4[..., 0], A from a7) and its gradient over the parameters."""
    ws, wh, bh = unpack(p)
    wq = [q(W) for W, _ in ws]
    y, A = forward(p, x4, q)
    cnt = m.sum()
    e = (y - t) * m
    loss = w_mse * (e * e).sum() / cnt
    dy = w_mse * 2.0 * e / cnt
    if a7 is not None and w_res != 0.0:
        r = m * (x4[..., 0] - c * apply_sys(a7, m * y))
        loss += w_res * (r * r).sum() / cnt
        dy += -2.0 * c * w_res / cnt * m * apply_sys_t(a7, r)
    g = np.zeros_like(p)
    g[HEAD_W:HEAD_B] = np.einsum("bzyx,bzyxc->c", dy, A["a9"])
    g[HEAD_B] = dy.sum()
    mask = lambda d, a: d * (a > 0)

    def grads(l, x, d):
        _, dW, db = conv_back(x, wq[l], d)
        g[OFFS[l][0]:OFFS[l][1]] = dW.ravel()
        g[OFFS[l][1]:OFFS[l][1] + LAYERS[l][1]] = db

    def dgrad(l, d):
        return conv_back(np.zeros(d.shape[:4] + (LAYERS[l][0],)), wq[l], d)[0]

    d9 = q(mask(dy[..., None] * wh, A["a9"]))
    grads(9, A["a8"], d9)
    d8 = q(mask(dgrad(9, d9), A["a8"]))
    grads(8, A["u1"], d8)
    du1 = q(mask(dgrad(8, d8), A["u1"]))
    d7 = q(up_back(du1[..., :32]))
    d1 = du1[..., 32:]
    grads(7, A["a6"], d7)
    d6 = q(mask(dgrad(7, d7), A["a6"]))
    grads(6, A["u2"], d6)
    du2 = q(mask(dgrad(6, d6), A["u2"]))
    d5 = q(up_back(du2[..., :64]))
    d3 = du2[..., 64:]
    grads(5, A["a4"], d5)
    d4 = q(mask(dgrad(5, d5), A["a4"]))
    grads(4, A["p2"], d4)
    dp2 = q(dgrad(4, d4))
    d3 = q(mask(q(d3 + pool_back(dp2)), A["a3"]))
    grads(3, A["a2"], d3)
    d2 = q(mask(dgrad(3, d3), A["a2"]))
    grads(2, A["p1"], d2)
    dp1 = q(dgrad(2, d2))
    d1 = q(mask(q(d1 + pool_back(dp1)), A["a1"]))
    grads(1, A["a0"], d1)
    d0 = q(mask(dgrad(1, d1), A["a0"]))
    grads(0, A["xin"], d0)
    return loss, g
