"""The cooperative V-cycle bottom (h3d_set_vcycle_bottom, k_vcycle_bottom): the
small levels of a V-cycle in one launch give the same iterates as the separate
launches, to the last bit."""
import numpy as np
import pytest

import homo3d_b200 as H
from tests.conftest import random_field, smooth_density, to_lib_field

pytestmark = pytest.mark.gpu


def _cycles(torch, n, bottom, ncycle=3, **kw):
    hd = H.Homogenization(n, **kw)
    hd.update(torch.tensor(smooth_density(n, seed=4), dtype=torch.float32, device="cuda"))
    hd.set_vcycle_bottom(bottom)
    hd.grid.set(H.FIELD_U, to_lib_field(random_field(n ** 3, 1, 0.1)))
    hd.grid.set(H.FIELD_F, to_lib_field(random_field(n ** 3, 2)))
    for _ in range(ncycle):
        hd.mg.v_cycle()
    out = [hd.mg.grids[l].get(H.FIELD_U) for l in range(hd.nlevels)]
    out += [hd.mg.grids[l].get(H.FIELD_R) for l in range(hd.nlevels - 1)]
    hd.close()
    return out


@pytest.mark.parametrize("n,kw", [(16, {}), (64, {}), (128, {}), (64, {"stencil": H.STENCIL_FP32}),
                                  (64, {"coarse_mode": H.COARSE_PROJECT})])
def test_bottom_is_bit_identical_to_separate_launches(torch_cuda, n, kw):
    a = _cycles(torch_cuda, n, 0, **kw)
    b = _cycles(torch_cuda, n, 32768, **kw)
    for i, (x, y) in enumerate(zip(a, b)):
        assert np.array_equal(x, y), i


def test_bottom_solve_matches(torch_cuda):
    torch = torch_cuda
    n = 64
    t = torch.tensor(smooth_density(n, seed=6), dtype=torch.float32, device="cuda")
    res = []
    for bottom in (0, 32768, 1 << 20):
        hd = H.Homogenization(n)
        hd.set_vcycle_bottom(bottom)
        hd.update(t)
        res.append((hd.elasticMatrix(1e-5), hd.last_stats))
        hd.close()
    for C, st in res[1:]:
        assert np.array_equal(C, res[0][0])
        assert st["vcycles"] == res[0][1]["vcycles"] and st["rel_res"] == res[0][1]["rel_res"]
