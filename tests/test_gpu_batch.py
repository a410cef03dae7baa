"""Batched designs through the C-ABI: designs of uneven resolution and mixed
precision modes solved together give the same C, V-cycle counts and statuses as
the same designs solved one at a time, and per-design failures stay per design."""
import numpy as np
import pytest

import homo3d_b200 as H
from tests.conftest import smooth_density

pytestmark = pytest.mark.gpu

DESIGNS = [(16, 0, 0.2, H.PREC_REFINE), (32, 1, 0.4, H.PREC_FP32), (24, 2, 0.3, H.PREC_REFINE),
           (32, 3, 0.15, H.PREC_FP32), (16, 4, 0.5, H.PREC_FP32)]


def _rho(torch, n, seed, vol):
    return torch.tensor(smooth_density(n, seed=seed, vol=vol), dtype=torch.float32, device="cuda")


@pytest.mark.parametrize("tol", [1e-3, 1e-5])
def test_batch_matches_sequential(torch_cuda, tol):
    torch = torch_cuda
    seq_C, seq_st = [], []
    for n, seed, vol, prec in DESIGNS:
        hd = H.Homogenization(n, precision=prec)
        hd.update(_rho(torch, n, seed, vol))
        seq_C.append(hd.elasticMatrix(tol))
        seq_st.append(hd.last_stats)
        hd.close()
    homs = [H.Homogenization(n, precision=prec) for n, _, _, prec in DESIGNS]
    H.batch_update(homs, [_rho(torch, n, seed, vol) for n, seed, vol, _ in DESIGNS])
    C = H.batch_elasticMatrix(homs, tol)
    for i, hd in enumerate(homs):
        st = hd.last_stats
        assert st["status"] == seq_st[i]["status"] == H.H3D_OK
        assert st["vcycles"] == seq_st[i]["vcycles"]
        assert st["refinements"] == seq_st[i]["refinements"]
        np.testing.assert_allclose(C[i], seq_C[i], rtol=1e-12, atol=1e-12 * np.abs(seq_C[i]).max())
    # a second batched call warm-starts every design from its stored solutions
    C2 = H.batch_elasticMatrix(homs, tol)
    for i, hd in enumerate(homs):
        assert hd.last_stats["vcycles"] <= seq_st[i]["vcycles"]
        assert np.abs(C2[i] - C[i]).max() <= 10 * tol * np.abs(C[i]).max()
    for hd in homs:
        hd.close()


def test_batch_errors_stay_per_design(torch_cuda):
    torch = torch_cuda
    a, b = H.Homogenization(16), H.Homogenization(16)
    a.update(_rho(torch, 16, 0, 0.3))
    # the same handle twice is refused before any work
    with pytest.raises(H.H3DError) as ei:
        H.batch_elasticMatrix([a, a], 1e-3)
    assert ei.value.code == H.H3D_ERR_ARG
    # a design without stencils fails alone; the other still gets its C
    with pytest.raises(H.H3DError) as ei:
        H.batch_elasticMatrix([a, b], 1e-3)
    assert ei.value.code == H.H3D_ERR_STATE
    assert a.last_stats["status"] == H.H3D_OK and a.last_stats["vcycles"] > 0
    ref = H.Homogenization(16)
    ref.update(_rho(torch, 16, 0, 0.3))
    Cr = ref.elasticMatrix(1e-3)
    b.update(_rho(torch, 16, 0, 0.3))
    C = H.batch_elasticMatrix([b], 1e-3)
    np.testing.assert_allclose(C[0], Cr, rtol=1e-12, atol=1e-12 * np.abs(Cr).max())
    # an empty batch is a no-op
    assert H.batch_elasticMatrix([], 1e-3).shape == (0, 6, 6)
    for hd in (a, b, ref):
        hd.close()
