"""The level-0 residual on the tensor cores (precision H3D_PREC_MIXED_TC, k_fine_tc.cu)
against the FP64 oracle (update_residual_otf_kernel_1, grid.cu:1277-1461), and the
mixed-precision solve against the refined one and the oracle.

Tolerances: the residual is held to 2e-5 of the field's max-norm like the FP32
residual (its TF32 hi + lo operands keep about 21 significant bits, against the
FP32 operator's 24); V-cycles of the mixed mode to 2e-4 of the oracle's field after
three cycles (the FP32 path: 5e-5; the residual's few more rounding bits pass
through the coarse corrections), and C at relthres 1e-5 to 1e-4 of the oracle's C
solved to 1e-10."""
import numpy as np
import pytest

import homo3d_b200 as H
from tests.conftest import from_lib_field, random_field, smooth_density, to_lib_field
from tests.test_gpu_parity import copy_stencils_to_oracle, make_pair, rel_err
from tests.test_gpu_solve import oracle_C

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,scale", [(12, 1.0), (16, 1.0), (28, 1.0), (32, 1e-6), (48, 1e3)])
def test_tc_residual_matches_oracle(torch_cuda, n, scale):
    """random fields of widely different magnitudes; 12 and 28 leave partial 8^3
    bricks (every grid of 32 or more cells per axis is a multiple of 8)"""
    hd, m, _ = make_pair(torch_cuda, n=n, seed=3, precision=H.PREC_MIXED_TC)
    nv = n ** 3
    u0, f0 = random_field(nv, 3, scale), random_field(nv, 4, scale)
    u0[0] = 0
    hd.grid.set(H.FIELD_U, to_lib_field(u0))
    hd.grid.set(H.FIELD_F, to_lib_field(f0))
    m.u()[:] = from_lib_field(to_lib_field(u0))
    m.f()[:] = from_lib_field(to_lib_field(f0))
    hd.grid.update_residual()
    m.residual(0)
    r = from_lib_field(hd.grid.get(H.FIELD_R))
    assert rel_err(r, m.r()) < 2e-5
    assert np.all(r[0] == 0)
    hd.close()


def test_tc_residual_is_deterministic(torch_cuda):
    n = 32
    hd, _, _ = make_pair(torch_cuda, n=n, seed=4, precision=H.PREC_MIXED_TC)
    nv = n ** 3
    hd.grid.set(H.FIELD_U, to_lib_field(random_field(nv, 8)))
    hd.grid.set(H.FIELD_F, to_lib_field(random_field(nv, 9)))
    hd.grid.update_residual()
    a = hd.grid.get(H.FIELD_R)
    hd.grid.update_residual()
    b = hd.grid.get(H.FIELD_R)
    assert np.array_equal(a, b)
    hd.close()


def test_mixed_vcycle_matches_oracle(torch_cuda):
    n = 32
    hd, m, _ = make_pair(torch_cuda, n=n, seed=5, precision=H.PREC_MIXED_TC)
    copy_stencils_to_oracle(hd, m)
    hd.grid.enforce_unit_macro_strain()
    m.rhs()
    hd.mg.reset_displacement()
    for it in range(3):
        hd.mg.v_cycle()
        m.vcycle(1.0)
        u = from_lib_field(hd.grid.get(H.FIELD_U))
        assert rel_err(u, m.u()) < 2e-4, it
    hd.close()


@pytest.mark.parametrize("n,seed,vol", [(32, 11, 0.3), (64, 2, 0.2)])
def test_mixed_solve_matches_refined_and_oracle(torch_cuda, n, seed, vol):
    rho = smooth_density(n, seed=seed, vol=vol)
    t = torch_cuda.tensor(rho, dtype=torch_cuda.float32, device="cuda")
    out = {}
    for prec in (H.PREC_REFINE, H.PREC_MIXED_TC):
        hd = H.Homogenization(n, precision=prec)
        hd.update(t)
        out[prec] = (hd.elasticMatrix(1e-5), hd.last_stats)
        hd.close()
    (Cr, sr), (Cm, sm) = out[H.PREC_REFINE], out[H.PREC_MIXED_TC]
    assert sm["status"] == H.H3D_OK and max(sm["rel_res"]) <= 1e-5
    assert sm["vcycles"] <= sr["vcycles"] + 1, (sm, sr)
    Cref = oracle_C(n, rho).elastic_matrix()
    assert rel_err(Cm, Cref) < 1e-4
    assert rel_err(Cm, Cr) < 1e-5
