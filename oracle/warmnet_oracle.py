"""NumPy restatement of the learned warm-start network (homo3d_b200/csrc/k_warmnet.cu).

TEST INFRASTRUCTURE ONLY: the oracle for the CUDA forward pass and gradients.
There is no reference counterpart; this file is pinned by central finite
differences of its own loss (tests/test_warmnet_oracle.py).

Layout shared with the CUDA code: activations [batch, channel, R^3] with voxel
x + R*(y + R*z); parameters one flat float vector holding, for the seven 3x3x3
convolutions e0 e1 e2 e3 d2 d1 d0 and then the 1x1 output layer, the weights
[cout][cin][27] (tap (dx+1) + 3(dy+1) + 9(dz+1)) followed by the biases [cout].
"""
import numpy as np

LAYERS = [(1, 16, 0), (16, 32, 1), (32, 64, 2), (64, 64, 3), (64, 32, 2), (32, 16, 1), (16, 16, 0)]
NOUT, NOUT_IN = 18, 16
TAPS = [(t % 3 - 1, t // 3 % 3 - 1, t // 9 - 1) for t in range(27)]


def unpack(p):
    p = np.asarray(p, np.float64)
    out, off = [], 0
    for ci, co, _ in LAYERS:
        w = p[off:off + co * ci * 27].reshape(co, ci, 27)
        off += co * ci * 27
        b = p[off:off + co]
        off += co
        out.append((w, b))
    w = p[off:off + NOUT * NOUT_IN].reshape(NOUT, NOUT_IN)
    off += NOUT * NOUT_IN
    b = p[off:off + NOUT]
    off += NOUT
    out.append((w, b))
    assert off == p.size
    return out


def num_params():
    return sum(co * ci * 27 + co for ci, co, _ in LAYERS) + NOUT * NOUT_IN + NOUT


def _shift(x, d):
    """x[..., z, y, x] -> its value at voxel v + d (periodic)"""
    dx, dy, dz = d
    return np.roll(x, shift=(-dz, -dy, -dx), axis=(-3, -2, -1))


def conv(x, w, b):
    """x [B, ci, R, R, R] -> [B, co, R, R, R], periodic 3x3x3"""
    y = np.zeros((x.shape[0], w.shape[0]) + x.shape[2:])
    for t, d in enumerate(TAPS):
        y += np.einsum("oi,bizyx->bozyx", w[:, :, t], _shift(x, d))
    return y + b[None, :, None, None, None]


def conv_wgrad(x, gz):
    gw = np.zeros((gz.shape[1], x.shape[1], 27))
    for t, d in enumerate(TAPS):
        gw[:, :, t] = np.einsum("bozyx,bizyx->oi", gz, _shift(x, d))
    return gw, gz.sum(axis=(0, 2, 3, 4))


def conv_dgrad(gz, w):
    gx = np.zeros((gz.shape[0], w.shape[1]) + gz.shape[2:])
    for t, d in enumerate(TAPS):
        gx += _shift(np.einsum("oi,bozyx->bizyx", w[:, :, t], gz), tuple(-c for c in d))
    return gx


def pool(x):
    B, C, R = x.shape[0], x.shape[1], x.shape[2]
    return x.reshape(B, C, R // 2, 2, R // 2, 2, R // 2, 2).mean(axis=(3, 5, 7))


def up(x):
    return x.repeat(2, axis=2).repeat(2, axis=3).repeat(2, axis=4)


def up_grad(g):
    s = g.shape
    return g.reshape(s[:2] + (s[2] // 2, 2, s[3] // 2, 2, s[4] // 2, 2)).sum(axis=(3, 5, 7))


def relu(x):
    return np.maximum(x, 0.0)


def forward(p, x, keep=False):
    """x [B, R^3] -> y [B, 18, R^3]"""
    P = unpack(p)
    B = x.shape[0]
    R = round(x.shape[1] ** (1 / 3))
    x5 = np.asarray(x, np.float64).reshape(B, 1, R, R, R)
    a0 = relu(conv(x5, *P[0]))
    p1 = pool(a0)
    a1 = relu(conv(p1, *P[1]))
    p2 = pool(a1)
    a2 = relu(conv(p2, *P[2]))
    p3 = pool(a2)
    a3 = relu(conv(p3, *P[3]))
    u2 = up(a3) + a2
    d2 = relu(conv(u2, *P[4]))
    u1 = up(d2) + a1
    d1 = relu(conv(u1, *P[5]))
    u0 = up(d1) + a0
    d0 = relu(conv(u0, *P[6]))
    W, b = P[7]
    y = np.einsum("oc,bczyx->bozyx", W, d0) + b[None, :, None, None, None]
    if keep:
        return y.reshape(B, NOUT, -1), dict(x=x5, a0=a0, p1=p1, a1=a1, p2=p2, a2=a2, p3=p3, a3=a3, u2=u2, d2=d2,
                                            u1=u1, d1=d1, u0=u0, d0=d0, y=y)
    return y.reshape(B, NOUT, -1)


def loss_and_grad(p, x, t):
    """mean squared error of the prediction against t [B, 18, R^3] and its gradient"""
    P = unpack(p)
    _, A = forward(p, x, keep=True)
    t5 = np.asarray(t, np.float64).reshape(A["y"].shape)
    n = t5.size
    loss = ((A["y"] - t5) ** 2).sum() / n
    gy = 2 * (A["y"] - t5) / n
    grads = [None] * 8
    grads[7] = (np.einsum("bozyx,bczyx->oc", gy, A["d0"]), gy.sum(axis=(0, 2, 3, 4)))
    gd0 = np.einsum("oc,bozyx->bczyx", P[7][0], gy) * (A["d0"] > 0)
    grads[6] = conv_wgrad(A["u0"], gd0)
    gu0 = conv_dgrad(gd0, P[6][0])
    gd1 = up_grad(gu0) * (A["d1"] > 0)
    grads[5] = conv_wgrad(A["u1"], gd1)
    gu1 = conv_dgrad(gd1, P[5][0])
    gd2 = up_grad(gu1) * (A["d2"] > 0)
    grads[4] = conv_wgrad(A["u2"], gd2)
    gu2 = conv_dgrad(gd2, P[4][0])
    ga3 = up_grad(gu2) * (A["a3"] > 0)
    grads[3] = conv_wgrad(A["p3"], ga3)
    ga2 = (gu2 + up(conv_dgrad(ga3, P[3][0])) / 8) * (A["a2"] > 0)
    grads[2] = conv_wgrad(A["p2"], ga2)
    ga1 = (gu1 + up(conv_dgrad(ga2, P[2][0])) / 8) * (A["a1"] > 0)
    grads[1] = conv_wgrad(A["p1"], ga1)
    ga0 = (gu0 + up(conv_dgrad(ga1, P[1][0])) / 8) * (A["a0"] > 0)
    grads[0] = conv_wgrad(A["x"], ga0)
    flat = np.concatenate([np.concatenate([gw.ravel(), gb]) for gw, gb in grads])
    return loss, flat


def init_params(seed=0):
    """random parameters with nonzero biases (every ReLU path gets exercised)"""
    rng = np.random.default_rng(seed)
    parts = []
    for ci, co, _ in LAYERS:
        parts.append(rng.standard_normal(co * ci * 27) * np.sqrt(2.0 / (ci * 27)))
        parts.append(rng.standard_normal(co) * 0.1)
    parts.append(rng.standard_normal(NOUT * NOUT_IN) * 0.3)
    parts.append(rng.standard_normal(NOUT) * 0.1)
    return np.concatenate(parts)
