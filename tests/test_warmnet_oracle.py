"""The NumPy restatement of the warm-start network (oracle/warmnet_oracle.py)
pinned by central finite differences of its own loss."""
import numpy as np

import oracle.warmnet_oracle as W


def test_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    R, B = 8, 2
    p = W.init_params(1)
    x = rng.uniform(0.0, 1.0, (B, R ** 3))
    t = rng.standard_normal((B, W.NOUT, R ** 3))
    _, g = W.loss_and_grad(p, x, t)
    assert g.size == p.size == W.num_params()
    h = 1e-5
    for i in rng.choice(p.size, 40, replace=False):
        e = np.zeros_like(p)
        e[i] = h
        fd = (W.loss_and_grad(p + e, x, t)[0] - W.loss_and_grad(p - e, x, t)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 + 1e-4 * abs(fd), (i, fd, g[i])


def test_forward_is_translation_equivariant():
    """periodic convolutions, pooling and upsampling commute with shifts by 8 voxels"""
    rng = np.random.default_rng(2)
    R = 16
    p = W.init_params(3)
    x = rng.uniform(0.0, 1.0, (1, R ** 3))
    y = W.forward(p, x).reshape(1, W.NOUT, R, R, R)
    xs = np.roll(x.reshape(1, R, R, R), 8, axis=3).reshape(1, -1)
    ys = W.forward(p, xs).reshape(1, W.NOUT, R, R, R)
    assert np.allclose(np.roll(y, 8, axis=4), ys, atol=1e-10)
