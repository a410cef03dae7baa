"""The element-energy contraction on the tensor cores (k_homog_tc.cu) against the
FP64 oracle: sensitivities of arbitrary stored solutions (including a grid whose
element count is not a multiple of the 128-element tile) and C of solved fields."""
import numpy as np
import pytest

import homo3d_b200 as H
from tests.test_gpu_parity import make_pair, rel_err

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [12, 24])
def test_sensitivity_of_arbitrary_solutions_matches_oracle(torch_cuda, n):
    torch = torch_cuda
    hd, m, _ = make_pair(torch, n=n, seed=n)
    rng = np.random.default_rng(n)
    # smooth O(N) displacements plus O(1) noise, like a solution in grid units
    x = np.arange(n) / n
    X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
    base = np.sin(2 * np.pi * X.T.ravel()) + np.cos(2 * np.pi * (Y.T.ravel() + Z.T.ravel()))
    chi = (n * base[None, :, None] * rng.uniform(0.5, 1.5, (6, 1, 3))
           + rng.standard_normal((6, n ** 3, 3))).astype(np.float32)
    hd.grid.set(H.FIELD_CHI, chi)
    dC = rng.standard_normal((6, 6)).astype(np.float32)
    sens = torch.zeros(n ** 3, dtype=torch.float32, device="cuda")
    hd.Sensitivity(dC, sens)
    m.update_stencils()
    ref = m.sensitivity(dC.astype(np.float64), chi=np.transpose(chi, (1, 0, 2)).astype(np.float64))
    assert rel_err(sens.cpu().numpy().astype(np.float64), ref) < 1e-5


def test_elastic_matrix_of_solved_fields_matches_oracle(torch_cuda):
    n = 24
    hd, m, _ = make_pair(torch_cuda, n=n, seed=5)
    C = hd.elasticMatrix(1e-4)
    chi = np.transpose(hd.grid.get(H.FIELD_CHI), (1, 0, 2)).astype(np.float64)
    m.update_stencils()
    Cref = m.elastic_matrix(chi=chi)
    assert rel_err(C, Cref) < 1e-6
    assert np.abs(C - C.T).max() == 0
