"""The autotuner's launch shapes give the same results to the last bit, the first
solve picks one per level, and the tuning entry points check their arguments."""
import numpy as np
import pytest

import homo3d_b200 as H
from tests.conftest import smooth_density

pytestmark = pytest.mark.gpu


def _solve(torch, n, shapes, precision, stencil=H.STENCIL_FP16):
    hd = H.Homogenization(n, precision=precision, stencil=stencil)
    hd.update(torch.tensor(smooth_density(n, seed=7, vol=0.3), dtype=torch.float32, device="cuda"))
    for l in range(hd.nlevels):
        hd.set_tuning(l, shapes, shapes)
    C = hd.elasticMatrix(1e-6)
    st = hd.last_stats
    hd.close()
    return C, st


@pytest.mark.parametrize("precision,stencil", [(H.PREC_REFINE, H.STENCIL_FP16), (H.PREC_FP32, H.STENCIL_FP16),
                                               (H.PREC_REFINE, H.STENCIL_FP32)])
def test_launch_shapes_are_bit_identical(torch_cuda, precision, stencil):
    C0, s0 = _solve(torch_cuda, 32, 0, precision, stencil)
    for shape in range(1, H.NUM_SHAPES):
        C1, s1 = _solve(torch_cuda, 32, shape, precision, stencil)
        assert np.array_equal(C0, C1), shape
        assert s0["vcycles"] == s1["vcycles"] and s0["rel_res"] == s1["rel_res"], shape


def test_first_solve_tunes_and_tuning_entry_points(torch_cuda):
    torch = torch_cuda
    n = 32
    hd = H.Homogenization(n)
    with pytest.raises(H.H3DError):  # nothing to time before the stencils exist
        hd.autotune()
    hd.update(torch.tensor(smooth_density(n, seed=1), dtype=torch.float32, device="cuda"))
    assert all(t == (0, 0) for t in hd.tuning())
    C = hd.elasticMatrix(1e-5)
    shapes = hd.tuning()
    assert len(shapes) == hd.nlevels and all(0 <= g < H.NUM_SHAPES and 0 <= r < H.NUM_SHAPES for g, r in shapes)
    # re-tuning and forcing shapes keep the same C
    hd.autotune()
    hd.reset_solutions()
    assert np.array_equal(hd.elasticMatrix(1e-5), C)
    for bad in [(-1, 0, 0), (hd.nlevels, 0, 0), (0, H.NUM_SHAPES, 0), (1, 0, 5)]:
        with pytest.raises(H.H3DError):
            hd.set_tuning(*bad)
    hd.close()
