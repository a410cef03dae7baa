"""The device MMA update (h3d_mma_*) against the FP64 oracle restatement."""
import numpy as np
import pytest

import homo3d_b200 as H
import oracle.oracle as O

pytestmark = pytest.mark.gpu


def run_both(torch, m, n, iters, seed):
    """the same design problem driven through the library and the oracle, feeding
    each the float design the library returned (the reference's float boundary)"""
    rng = np.random.default_rng(seed)
    w = rng.uniform(0.2, 1.0, n)
    A = rng.uniform(0.5, 1.5, (m, n)) / n
    gpu = H.MMAOptimizer(m, n, 1.0, 0.0, 1000.0, 1.0)
    gpu.setBound(0.001, 1.0)
    ora = O.MMA(m, n, 1.0, 0.0, 1000.0, 1.0)
    ora.set_bound(0.001, 1.0)
    x = np.full(n, 0.3, np.float32)
    worst = 0.0
    for it in range(iters):
        xd = x.astype(np.float64)
        df = (-w / xd ** 2).astype(np.float32)
        g = (A @ xd - 0.3 * A.sum(axis=1)).astype(np.float32)
        dg = A.astype(np.float32)
        xt = torch.tensor(x, device="cuda")
        gpu.update(it, xt, torch.tensor(df, device="cuda"), torch.tensor(g, device="cuda"),
                   [torch.tensor(dg[i], device="cuda") for i in range(m)])
        xg = xt.cpu().numpy()
        xo = ora.update(it, x.astype(np.float64), df.astype(np.float64), g.astype(np.float64),
                        dg.astype(np.float64))
        worst = max(worst, float(np.abs(xg.astype(np.float64) - xo).max()))
        x = xg
    return worst, gpu, ora


@pytest.mark.parametrize("m", [1, 2])
def test_mma_matches_oracle(torch_cuda, m):
    worst, gpu, ora = run_both(torch_cuda, m, 5000, 6, seed=m)
    assert worst < 2e-6, worst
    assert abs(gpu.newton_steps - ora.newton) <= 2


def test_mma_large_design(torch_cuda):
    """a 64^3 design vector: the grid-stride kernels and the block partials"""
    worst, _, _ = run_both(torch_cuda, 1, 64 ** 3, 3, seed=7)
    assert worst < 2e-6, worst


def test_mma_toy_problem_converges(torch_cuda):
    torch = torch_cuda
    c1, c2 = np.array([5.0, 2.0, 1.0]), np.array([3.0, 4.0, 3.0])
    mma = H.MMAOptimizer(2, 3)
    mma.setBound(0.0, 5.0)
    x = torch.tensor([4.0, 3.0, 2.0], device="cuda")
    for it in range(1, 31):
        xh = x.cpu().numpy().astype(np.float64)
        g = np.array([((xh - c1) ** 2).sum() - 9, ((xh - c2) ** 2).sum() - 9], np.float32)
        dg = [torch.tensor(2 * (xh - c), dtype=torch.float32, device="cuda") for c in (c1, c2)]
        mma.update(it, x, 2 * x, torch.tensor(g, device="cuda"), dg)
    assert np.allclose(x.cpu().numpy(), [2.0175, 1.7800, 1.2375], atol=2e-3)


def test_mma_rejects_bad_arguments(torch_cuda):
    with pytest.raises(H.H3DError):
        H.MMAOptimizer(5, 100)
    mma = H.MMAOptimizer(1, 10)
    x = torch_cuda.zeros(10, device="cuda")
    with pytest.raises(H.H3DError):  # bounds not set
        mma.update(0, x, x, x[:1], [x])
