"""The reference's trig-basis initial density (randTri, Framework.cuh:238-310) on
the device (h3d_init_density_trig) against the FP64 numpy restatement
(oracle/init_oracle.py), plain and centred, with and without symmetry."""
import numpy as np
import pytest

import homo3d_b200 as H
from homo3d_b200.density import trig_init_coefficients
from oracle import init_oracle as I
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("P,centered,sym", [(2, False, None), (3, True, None), (4, False, "reflect6")])
def test_trig_init_matches_restatement(torch_cuda, P, centered, sym):
    torch = torch_cuda
    n, vol = 24, 0.3
    hd = H.Homogenization(n)
    rho = torch.zeros(n ** 3, device="cuda")
    c = hd.init_density_trig(rho, n_period=P, vol=vol, sym=sym, centered=centered, seed=P)
    got = rho.cpu().numpy().astype(np.float64)
    v = I.basis_field((n, n, n), P, c, centered)
    if sym:
        v = O.symmetrize_f32((n, n, n), v.ravel().astype(np.float32), sym).astype(np.float64).reshape(v.shape)
    ref, t = I.level_set(v, P, vol)
    assert abs(got.mean() - vol) / vol < 1e-3
    assert got.min() >= 0.001 - 1e-7 and got.max() <= min(1.5 * vol, 1.0) + 1e-6
    # the steep level set (slope 15 M) turns FP32 basis sums into differences of a few 1e-4
    assert np.abs(got - ref.ravel()).max() < 2e-3
    assert np.corrcoef(got, ref.ravel())[0, 1] > 0.9999
    hd.close()


def test_trig_init_rejects_bad_arguments(torch_cuda):
    torch = torch_cuda
    hd = H.Homogenization(8)
    rho = torch.zeros(8 ** 3, device="cuda")
    with pytest.raises(H.H3DError):
        hd.init_density_trig(rho, n_period=2, coeff=np.zeros(5, np.float32))
    with pytest.raises(H.H3DError):
        hd.init_density_trig(rho, n_period=0)
    hd.close()
