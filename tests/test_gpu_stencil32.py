"""FP32 coarse-stencil storage (H3D_STENCIL_FP32, no reference counterpart):
the stencils and the V-cycle against the oracle's FP32-storage mode, and
convergence on a high-contrast design where FP16 storage stalls."""
import numpy as np
import pytest

import homo3d_b200 as H
from tests.conftest import from_lib_field
from tests.test_gpu_parity import copy_stencils_to_oracle, make_pair, rel_err

pytestmark = pytest.mark.gpu


def fp32_pair(torch, n, seed, **kw):
    hd, m, t = make_pair(torch, n=n, seed=seed, stencil=H.STENCIL_FP32, **kw)
    m.set_fp16(3)
    return hd, m, t


def close32(got, ref, rel=2e-5):
    return float(np.abs(got - ref).max()) <= rel * float(np.abs(ref).max())


@pytest.mark.parametrize("n,pin", [(16, 0), (32, 0), (16, 1)])
def test_fp32_level1_stencil(torch_cuda, n, pin):
    hd, m, _ = fp32_pair(torch_cuda, n, n, pin_mode=pin)
    m.galerkin_l1(1)
    got = hd.mg.grids[1].get(H.FIELD_STENCIL).astype(np.float64)
    ref = m.stencil(1)
    assert close32(got, ref), float(np.abs(got - ref).max())
    # FP32 entries are not FP16-representable in general: the storage is really FP32
    assert np.any(got.astype(np.float16).astype(np.float64) != got)


def test_fp32_deeper_stencils(torch_cuda):
    hd, m, _ = fp32_pair(torch_cuda, 32, 1)
    for l in range(2, hd.nlevels):
        m.stencil(l - 1)[:] = hd.mg.grids[l - 1].get(H.FIELD_STENCIL).astype(np.float64)
        m.galerkin(l)
        got = hd.mg.grids[l].get(H.FIELD_STENCIL).astype(np.float64)
        assert close32(got, m.stencil(l)), (l, float(np.abs(got - m.stencil(l)).max()))


def test_fp32_vcycle_matches_oracle(torch_cuda):
    hd, m, _ = fp32_pair(torch_cuda, 32, 5)
    copy_stencils_to_oracle(hd, m)
    hd.grid.enforce_unit_macro_strain()
    m.rhs()
    hd.mg.reset_displacement()
    for it in range(3):
        hd.mg.v_cycle()
        m.vcycle(1.0)
        assert rel_err(from_lib_field(hd.grid.get(H.FIELD_U)), m.u()) < 5e-5, it


def test_fp32_stencils_solve_and_storage_round_trip(torch_cuda):
    torch = torch_cuda
    from tests.conftest import smooth_density
    n = 32
    rho = torch.tensor(smooth_density(n, seed=3, vol=0.3), dtype=torch.float32, device="cuda")
    C = {}
    for st in (H.STENCIL_FP16, H.STENCIL_FP32):
        hd = H.Homogenization(n, stencil=st)
        hd.update(rho)
        C[st] = hd.elasticMatrix(1e-6)
        assert hd.last_stats["status"] == H.H3D_OK
        if st == H.STENCIL_FP32:  # set/get of a level's stencil keeps FP32 values
            g = hd.mg.grids[1]
            s0 = g.get(H.FIELD_STENCIL)
            g.set(H.FIELD_STENCIL, s0)
            assert np.array_equal(g.get(H.FIELD_STENCIL), s0)
        hd.close()
    # the coarse operators only precondition: both converge to the same C
    assert np.abs(C[H.STENCIL_FP16] - C[H.STENCIL_FP32]).max() <= 1e-5 * np.abs(C[H.STENCIL_FP16]).max()


def test_invalid_stencil_precision_is_rejected(torch_cuda):
    with pytest.raises(H.H3DError):
        H.Homogenization(16, stencil=7)
