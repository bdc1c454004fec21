"""CPU oracle of the surrogate U-Net (test infrastructure only).

A numpy restatement of the network of multi-block-lbm-gpu_b200/csrc/unet.cu
(the learned warm start has no counterpart in the reference project): the
same layers, parameter layout and loss, with BF16 rounding (round to nearest
even) at the same points as the device code, so that its forward values and
gradients agree with the GPU's up to FP32 summation order.
"""
import numpy as np

LAYERS = [(16, 32, 0), (32, 32, 0), (32, 64, 1), (64, 64, 1), (64, 128, 2), (128, 128, 2), (128, 256, 3),
          (256, 256, 3), (384, 128, 2), (128, 128, 2), (192, 64, 1), (64, 64, 1), (96, 32, 0), (32, 32, 0)]


ROUND = True  # False: exact float64 arithmetic (for finite-difference checks of the oracle itself)


def bf(x):
    """float32 -> nearest BF16 (ties to even) -> float32."""
    if not ROUND:
        return np.asarray(x, dtype=np.float64)
    x = np.ascontiguousarray(x, dtype=np.float32)
    u = x.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return (r & 0xFFFFFFFF).astype(np.uint32).view(np.float32).reshape(x.shape)


def unpack(p):
    out, off = [], 0
    for cin, cout, _ in LAYERS:
        w = p[off:off + cout * 9 * cin].reshape(cout, 9, cin)
        off += cout * 9 * cin
        b = p[off:off + cout]
        off += cout
        out.append((w, b))
    hw = p[off:off + 96].reshape(3, 32)
    off += 96
    hb = p[off:off + 3]
    return out, hw, hb


def conv(x, w):
    """3x3, zero padding 1: x [N,H,W,Cin], w [Cout,9,Cin] -> [N,H,W,Cout] (float64 sums)."""
    N, H, W, _ = x.shape
    xp = np.pad(x.astype(np.float64), ((0, 0), (1, 1), (1, 1), (0, 0)))
    y = np.zeros((N, H, W, w.shape[0]))
    for t in range(9):
        dy, dx = t // 3 - 1, t % 3 - 1
        y += xp[:, 1 + dy:1 + dy + H, 1 + dx:1 + dx + W, :] @ w[:, t, :].T.astype(np.float64)
    return y


def conv_dgrad(g, w):
    N, H, W, _ = g.shape
    dxp = np.zeros((N, H + 2, W + 2, w.shape[2]))
    for t in range(9):
        dy, dx = t // 3 - 1, t % 3 - 1
        dxp[:, 1 + dy:1 + dy + H, 1 + dx:1 + dx + W, :] += g.astype(np.float64) @ w[:, t, :].astype(np.float64)
    return dxp[:, 1:-1, 1:-1, :]


def conv_wgrad(g, x):
    N, H, W, cin = x.shape
    xp = np.pad(x.astype(np.float64), ((0, 0), (1, 1), (1, 1), (0, 0)))
    dw = np.zeros((g.shape[3], 9, cin))
    gf = g.reshape(-1, g.shape[3]).astype(np.float64)
    for t in range(9):
        dy, dx = t // 3 - 1, t % 3 - 1
        dw[:, t, :] = gf.T @ xp[:, 1 + dy:1 + dy + H, 1 + dx:1 + dx + W, :].reshape(-1, cin)
    return dw


def pool(x):
    return bf(0.25 * (x[:, 0::2, 0::2] + x[:, 0::2, 1::2] + x[:, 1::2, 0::2] + x[:, 1::2, 1::2]))


def up(x):
    return np.repeat(np.repeat(x, 2, axis=1), 2, axis=2)


def forward_backward(p, inp, target=None, mask=None):
    """inp [N,H,W,4]; returns (out [N,H,W,3], loss, grads in the parameter layout)."""
    layers, hw, hb = unpack(p)
    N, H, W, _ = inp.shape
    x0 = np.zeros((N, H, W, 16), np.float32 if ROUND else np.float64)
    x0[..., :4] = inp
    x0 = bf(x0)
    wb = [bf(w) for w, _ in layers]
    act, xin = [None] * 14, [None] * 14

    def run(i, x):
        xin[i] = x
        act[i] = bf(np.maximum(conv(x, wb[i]) + layers[i][1], 0.0))
        return act[i]

    h = run(1, run(0, x0))
    pools = [pool(act[1])]
    run(3, run(2, pools[0]))
    pools.append(pool(act[3]))
    run(5, run(4, pools[1]))
    pools.append(pool(act[5]))
    run(7, run(6, pools[2]))
    cats = []
    for prev, skip, la in ((7, 5, 8), (9, 3, 10), (11, 1, 12)):
        c = np.concatenate([up(act[prev]), act[skip]], axis=3)
        cats.append(c)
        run(la + 1, run(la, c))
    feat = act[13].astype(np.float64)
    out = feat @ hw.T.astype(np.float64) + hb
    if target is None:
        return out.astype(np.float32), None, None
    denom = 3.0 * N * H * W
    d = out - target
    loss = float(np.sum(mask[..., None] * d * d) / denom)
    gy = 2.0 * mask[..., None] * d / denom
    grads = []
    ghw = gy.reshape(-1, 3).T @ feat.reshape(-1, 32)
    ghb = gy.reshape(-1, 3).sum(0)
    g = [None] * 14
    g[13] = gy @ hw.astype(np.float64)
    gl = [None] * 14

    def back(i, need_x=True):
        gb = bf(np.where(act[i] > 0, g[i], 0.0))
        gl[i] = (conv_wgrad(gb, xin[i]), gb.reshape(-1, gb.shape[3]).astype(np.float64).sum(0))
        return conv_dgrad(gb, wb[i]) if need_x else None

    for prev, skip, la, cs in ((11, 1, 12, 64), (9, 3, 10, 128), (7, 5, 8, 256)):
        g[la] = back(la + 1)
        gc = back(la)
        gup = gc[..., :cs]
        gp = gup[:, 0::2, 0::2] + gup[:, 0::2, 1::2] + gup[:, 1::2, 0::2] + gup[:, 1::2, 1::2]
        g[prev] = gp if g[prev] is None else g[prev] + gp
        g[skip] = gc[..., cs:] if g[skip] is None else g[skip] + gc[..., cs:]
    for lv in (3, 2, 1, 0):
        la, lb = 2 * lv, 2 * lv + 1
        g[la] = back(lb)
        if lv == 0:
            back(la, need_x=False)
        else:
            gpool = back(la)
            g[la - 1] = g[la - 1] + 0.25 * up(gpool)
    flat = []
    for i in range(14):
        flat += [gl[i][0].ravel(), gl[i][1].ravel()]
    flat += [ghw.ravel(), ghb.ravel()]
    if not ROUND:
        return out, loss, np.concatenate(flat)
    return out.astype(np.float32), loss, np.concatenate(flat).astype(np.float32)
