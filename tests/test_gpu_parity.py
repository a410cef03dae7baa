"""GPU parity: every grid entry point of libh3d against the FP64 oracle on the same
inputs (called through the C ABI via the homo3d_b200 binding).

Tolerances: FP32 kernels against FP64 are held to 2e-5 of the field's max-norm
(5e-5 for chains of several kernels); FP16 stencil entries to 4 FP16 ulps (the
library and the oracle each round their own FP32/FP64 sums once); the symmetry
maps are bit-exact."""
import numpy as np
import pytest

import homo3d_b200 as H
from oracle import oracle as O
from tests.conftest import from_lib_field, half_ulp, random_field, smooth_density, to_lib_field

pytestmark = pytest.mark.gpu

N = 16


def make_pair(torch, n=N, seed=0, vol=0.3, **kw):
    rho = smooth_density(n, seed=seed, vol=vol)
    hd = H.Homogenization(n, **kw)
    t = torch.tensor(rho, dtype=torch.float32, device="cuda")
    hd.update(t)
    m = O.MG((n, n, n))
    m.set_density(rho.astype(np.float32).astype(np.float64))  # the library sees FP32 densities
    if kw.get("pin_mode", 0) == H.PIN_GALERKIN:
        m.set_pin_identity(False)
    if kw.get("coarse_mode", 0) == H.COARSE_PROJECT:
        m.set_project(True)
    return hd, m, t


def rel_err(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-30)


def copy_stencils_to_oracle(hd, m):
    for l in range(1, hd.nlevels):
        m.stencil(l)[:] = hd.mg.grids[l].get(H.FIELD_STENCIL).astype(np.float64)
    assert m.coarse_factor() == 0


def test_element_matrix(torch_cuda):
    hd = H.Homogenization(8)
    assert np.abs(hd.element_matrix() - O.ke(10.0, 0.3)).max() < 1e-13


def test_hierarchy_matches_reference_rules(torch_cuda):
    for reso in (8, 32, 80, 96, 128):
        hd = H.Homogenization(reso)
        d, r = O.hierarchy((reso,) * 3)
        assert [x[0] for x in hd.dims] == d[:, 0].tolist()
        assert [x[0] for x in hd.ratios] == r[:, 0].tolist()
        hd.close()


def test_rhs(torch_cuda):
    hd, m, _ = make_pair(torch_cuda)
    hd.grid.enforce_unit_macro_strain()
    m.rhs()
    f = from_lib_field(hd.grid.get(H.FIELD_F))
    assert rel_err(f, m.f()) < 2e-6


@pytest.mark.parametrize("w", [1.0, 0.8])
def test_fine_gs(torch_cuda, w):
    hd, m, _ = make_pair(torch_cuda)
    nv = N ** 3
    u0, f0 = random_field(nv, 1), random_field(nv, 2)
    hd.grid.set(H.FIELD_U, to_lib_field(u0))
    hd.grid.set(H.FIELD_F, to_lib_field(f0))
    m.u()[:] = from_lib_field(to_lib_field(u0))
    m.f()[:] = from_lib_field(to_lib_field(f0))
    hd.grid.gs_relaxation(w)
    m.gs(0, w)
    u = from_lib_field(hd.grid.get(H.FIELD_U))
    assert rel_err(u, m.u()) < 2e-5
    assert np.all(u[0] == 0)  # pinned origin


def test_fine_residual(torch_cuda):
    hd, m, _ = make_pair(torch_cuda)
    nv = N ** 3
    u0, f0 = random_field(nv, 3), random_field(nv, 4)
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


def test_weighted_norms(torch_cuda):
    hd, m, _ = make_pair(torch_cuda)
    nv = N ** 3
    f0 = random_field(nv, 5)
    hd.grid.set(H.FIELD_F, to_lib_field(f0))
    got = hd.field_norms(H.FIELD_F)
    ref = O.weighted_norm((N, N, N), from_lib_field(to_lib_field(f0)))
    assert np.abs(got - ref).max() / ref.max() < 1e-12


def test_vcycle_fused_residual_paths_match_separate_launches(torch_cuda):
    """The V-cycle's down leg lets the last colour launch of each level's sweep
    write that colour's residual and runs the residual launch over the other seven
    colours (fine and coarse levels).  The same cycle driven through the per-level
    entry points (a whole sweep, then the residual of all eight colours) must give
    the same residual on every smoothed level and the same final level-0 field, to
    FP32 rounding."""
    n = 32
    hd, _, t = make_pair(torch_cuda, n=n, seed=5)
    h2 = H.Homogenization(n)
    h2.update(t)
    nv = n ** 3
    u0, f0 = to_lib_field(random_field(nv, 21, 0.1)), to_lib_field(random_field(nv, 22))
    for h in (hd, h2):
        h.grid.set(H.FIELD_U, u0)
        h.grid.set(H.FIELD_F, f0)
    hd.mg.v_cycle()  # captured graph: fused last-colour residuals
    g = h2.mg.grids
    nl = h2.nlevels
    for l in range(nl - 1):
        if l > 0:
            g[l].restrict_residual()
            g[l].reset_displacement()
        g[l].gs_relaxation(1.0)
        g[l].update_residual()
    g[nl - 1].restrict_residual()
    g[nl - 1].reset_displacement()
    g[nl - 1].solveHostEquation()
    for l in range(nl - 2, -1, -1):
        g[l].prolongate_correction()
        g[l].gs_relaxation(1.0)
    for l in range(nl - 1):
        ra, rb = hd.mg.grids[l].get(H.FIELD_R), g[l].get(H.FIELD_R)
        assert rel_err(ra, rb) < 2e-5, l
    ua, ub = hd.grid.get(H.FIELD_U), h2.grid.get(H.FIELD_U)
    assert rel_err(ua, ub) < 2e-5
    hd.close()
    h2.close()
