"""FP64 numpy restatement of the reference expression layer's radial convolution.

TEST INFRASTRUCTURE ONLY (imported by tests/): the oracle for h3d_conv_radial and for
the shear-isotropy MMA loop.  Follows homo3d AutoDiff/TensorExpression.h:1002-1044
(the Spline4 weight w = 1 - 6 q + 8 q^1.5 - 3 q^2, q = |o|^2 / r^2 < 1, window
half-width (int)(r + 0.5)) and AutoDiff/TensorExpression.cuh:288-369 (conv_kernel:
the sum over in-grid offsets divided by their weight sum; conv_backward_kernel: the
transpose).  Arrays are lexicographic (x fastest), shape (nz, ny, nx).
"""
import numpy as np


def _weights(r):
    hw = int(r + 0.5)
    o = np.arange(-hw, hw + 1)
    oz, oy, ox = np.meshgrid(o, o, o, indexing="ij")
    q = (ox * ox + oy * oy + oz * oz) / (r * r)
    w = np.where(q < 1, 1 - 6 * q + 8 * q * np.sqrt(q) - 3 * q * q, 0.0)
    return hw, w


def _shifted(a, dz, dy, dx, periodic):
    """b[p] = a[p + d] (zero outside unless periodic), and the in-grid mask"""
    n = a.shape
    if periodic:
        return np.roll(a, (-dz, -dy, -dx), axis=(0, 1, 2)), np.ones(n, bool)
    b = np.zeros(n)
    m = np.zeros(n, bool)
    sl = lambda d, k: (slice(max(0, -d), min(k, k - d)), slice(max(0, d), min(k, k + d)))
    (zd, zs), (yd, ys), (xd, xs) = sl(dz, n[0]), sl(dy, n[1]), sl(dx, n[2])
    b[zd, yd, xd] = a[zs, ys, xs]
    m[zd, yd, xd] = True
    return b, m


def conv(a, r, periodic=False):
    """out, ws (the in-grid weight sums)"""
    hw, w = _weights(r)
    a = np.asarray(a, np.float64)
    s = np.zeros(a.shape)
    ws = np.zeros(a.shape)
    for dz in range(-hw, hw + 1):
        for dy in range(-hw, hw + 1):
            for dx in range(-hw, hw + 1):
                wt = w[dz + hw, dy + hw, dx + hw]
                b, m = _shifted(a, dz, dy, dx, periodic)
                s += wt * b
                ws += wt * m
    return s / ws, ws


def conv_adjoint(g, r, periodic=False):
    hw, w = _weights(r)
    _, ws = conv(np.zeros_like(g, dtype=np.float64), r, periodic)
    gw = np.asarray(g, np.float64) / ws
    out = np.zeros(gw.shape)
    for dz in range(-hw, hw + 1):
        for dy in range(-hw, hw + 1):
            for dx in range(-hw, hw + 1):
                b, _ = _shifted(gw, -dz, -dy, -dx, periodic)
                out += w[dz + hw, dy + hw, dx + hw] * b
    return out
