"""The learned warm start: the CUDA network against its NumPy oracle (forward
pass and gradients), training on solver-generated pairs, the solver hook, and
the fallback from a bad starting guess."""
import numpy as np
import pytest

import homo3d_b200 as H
import oracle.warmnet_oracle as W
from homo3d_b200 import warmnet as WN
from tests.conftest import smooth_density

pytestmark = pytest.mark.gpu


def test_forward_and_gradients_match_oracle(torch_cuda):
    torch = torch_cuda
    R, B = 8, 2
    net = H.WarmNet(R, max_batch=B, seed=3)
    p = W.init_params(5)
    net.set_params(p.astype(np.float32))
    rng = np.random.default_rng(0)
    x = rng.uniform(0.0, 1.0, (B, R ** 3)).astype(np.float32)
    t = rng.standard_normal((B, W.NOUT, R ** 3)).astype(np.float32)
    y = net.forward(torch.tensor(x, device="cuda")).cpu().numpy()
    p32 = p.astype(np.float32).astype(np.float64)
    yref = W.forward(p32, x.astype(np.float64))
    assert np.abs(y - yref).max() <= 1e-4 * np.abs(yref).max()
    loss = net.gradients(torch.tensor(x, device="cuda"), torch.tensor(t, device="cuda"))
    lref, gref = W.loss_and_grad(p32, x.astype(np.float64), t.astype(np.float64))
    g = net.grads().astype(np.float64)
    assert abs(loss - lref) <= 1e-5 * abs(lref)
    assert np.abs(g - gref).max() <= 1e-4 * np.abs(gref).max()


def test_training_fits_solver_pairs_and_the_hook_starts_the_solve(torch_cuda):
    n, R = 32, 16
    x, t = WN.solver_pairs(n, R, seeds=[0, 1, 2, 3], iters=4, relthres=1e-3)
    assert x.shape == (16, R ** 3) and t.shape == (16, 18, R ** 3)
    net = H.WarmNet(R, max_batch=4, seed=0)
    hist = WN.train(net, x, t, steps=300, batch=4, lr=2e-3)
    assert np.mean(hist[-10:]) < 0.5 * hist[0]
    rows = WN.compare_starts(net, n, seeds=[100, 101], relthres=1e-5)
    for r in rows:
        assert abs(r["learned_C00"] - r["zero_C00"]) <= 1e-5 * abs(r["zero_C00"])
        assert r["learned_vcycles"] <= r["zero_vcycles"] + 1


def test_bad_guess_falls_back_to_zero_start(torch_cuda):
    torch = torch_cuda
    n = 16
    hd = H.Homogenization(n)
    rho = smooth_density(n, seed=4)
    hd.update(torch.tensor(rho, dtype=torch.float32, device="cuda"))
    hd.reset_solutions()
    hd.elasticMatrix(1e-5)
    k0 = hd.last_stats["vcycles"]
    wild = np.random.default_rng(1).standard_normal((6, n ** 3, 3)).astype(np.float32) * 1e3
    hd.grid.set(H.FIELD_CHI, wild)
    hd.elasticMatrix(1e-5)
    assert hd.last_stats["vcycles"] == k0
