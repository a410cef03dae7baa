"""h3d_field_norms_static (no reference counterpart): the per-case weighted norms
with reduction scratch in a fixed per-device array must equal h3d_field_norms,
which uses the handle's scratch, on consecutive calls.  Kept in the last-collected
file so that it also runs after every other GPU test has used the device."""
import numpy as np
import pytest

import homo3d_b200 as H
from tests.conftest import smooth_density

pytestmark = pytest.mark.gpu


def test_static_scratch_norms_equal_handle_scratch_norms(torch_cuda):
    n = 32
    rho = smooth_density(n, seed=21)
    hd = H.Homogenization(n, precision=H.PREC_FP32)  # level-0 U holds the solution
    hd.update(torch_cuda.tensor(rho, dtype=torch_cuda.float32, device="cuda"))
    hd.elasticMatrix(1e-3)
    for field in (H.FIELD_U, H.FIELD_F, H.FIELD_R):
        ref = hd.field_norms(field)
        first = hd.field_norms_static(field)
        second = hd.field_norms_static(field)
        assert np.all(np.isfinite(ref)) and np.any(ref > 0)
        assert np.array_equal(first, ref), (field, first, ref)
        assert np.array_equal(second, first)


def test_static_scratch_norms_reject_fp64_fields(torch_cuda):
    hd = H.Homogenization(16)
    with pytest.raises(H.H3DError):
        hd.field_norms_static(H.FIELD_CHI)
