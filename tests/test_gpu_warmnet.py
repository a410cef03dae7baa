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
        # the solver drops a starting guess whose residual exceeds a zero start's,
        # so a learned start never costs V-cycles
        assert r["learned_vcycles"] <= r["zero_vcycles"]


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


@pytest.mark.parametrize("n", [64, 128])
def test_coarse_resolution_start_cannot_save_vcycles(torch_cuda, n):
    """The bound on any warm start predicted at a coarser resolution: the converged
    solution itself, sampled at the even vertices (half resolution) and
    interpolated back trilinearly, starts the relthres-1e-5 solve no better than
    zero (its interpolation error leaves a residual above ||f||), and the same
    solution with 1 % random noise neither; only the full-resolution solution
    itself saves V-cycles.  A learned network at the solve's resolution would have
    to be accurate to well under 1 % per vertex to pay."""
    torch = torch_cuda
    rho = smooth_density(n, seed=0).astype(np.float32)
    hd = H.Homogenization(n)
    hd.update(torch.tensor(rho, device="cuda"))
    hd.elasticMatrix(1e-9)
    chi = hd.grid.get(H.FIELD_CHI)
    hd.reset_solutions()
    hd.elasticMatrix(1e-5)
    zero = hd.last_stats["vcycles"]
    c = torch.tensor(chi.reshape(6, n, n, n, 3).astype(np.float64))
    R = n // 2
    cm = c[:, ::2, ::2, ::2].permute(0, 4, 1, 2, 3)  # the even vertices: coarse node k is fine vertex 2k
    big = torch.cat([cm, cm[:, :, :1]], 2)
    big = torch.cat([big, big[:, :, :, :1]], 3)
    big = torch.cat([big, big[:, :, :, :, :1]], 4)
    up = torch.nn.functional.interpolate(big, size=(n + 2,) * 3, mode="trilinear", align_corners=True)[:, :, :n, :n, :n]
    guess = up.permute(0, 2, 3, 4, 1).numpy().reshape(6, n ** 3, 3).astype(np.float32)
    noisy = (chi * (1 + 0.01 * np.random.default_rng(0).standard_normal(chi.shape))).astype(np.float32)
    counts = {}
    for name, g in (("half", guess), ("noisy", noisy), ("exact", chi)):
        hd.grid.set(H.FIELD_CHI, g)
        hd.elasticMatrix(1e-5)
        counts[name] = hd.last_stats["vcycles"]
    hd.close()
    assert counts["half"] >= zero and counts["noisy"] >= zero, (zero, counts)
    assert counts["exact"] < zero, (zero, counts)
