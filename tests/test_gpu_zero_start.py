"""A solve from zero stored solutions (a new handle, or after reset_solutions)
skips the copy and centring of the FP64 solution and, in its first refinement
step, the FP64 residual of a zero solution.  The shortcut must be exact: the same
C to the last bit, the same V-cycle count and residual estimates as the full path,
which runs when the zero solutions are written through set_field instead."""
import numpy as np
import pytest

import homo3d_b200 as H
from tests.conftest import smooth_density

pytestmark = pytest.mark.gpu


def _solve(torch, n, rho, via_set_field, tol):
    hd = H.Homogenization(n)
    hd.update(torch.tensor(rho, dtype=torch.float32, device="cuda"))
    if via_set_field:  # zeros written by the caller: the handle cannot assume them
        hd.grid.set(H.FIELD_CHI, np.zeros((6, hd.nv(0), 3), np.float32))
    else:
        hd.reset_solutions()
    C = hd.elasticMatrix(tol)
    st = hd.last_stats
    # a second design evaluation warm-starts from the stored solutions (full path)
    C2 = hd.elasticMatrix(tol)
    st2 = hd.last_stats
    hd.close()
    return C, st, C2, st2


@pytest.mark.parametrize("n,tol", [(32, 1e-6), (48, 1e-5)])
def test_zero_start_shortcut_is_exact(torch_cuda, n, tol):
    rho = smooth_density(n, seed=3, vol=0.3)
    Ca, sa, Ca2, sa2 = _solve(torch_cuda, n, rho, False, tol)
    Cb, sb, Cb2, sb2 = _solve(torch_cuda, n, rho, True, tol)
    assert np.array_equal(Ca, Cb)
    assert sa["vcycles"] == sb["vcycles"] and sa["rel_res"] == sb["rel_res"]
    assert np.array_equal(Ca2, Cb2) and sa2["vcycles"] == sb2["vcycles"]
