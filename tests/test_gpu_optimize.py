"""GPU: the OC bulk-modulus loop (optiBulk) against the same loop built from the
FP64 oracle's pieces, for a few iterations at tight relthres."""
import numpy as np
import pytest

import homo3d_b200 as H
from homo3d_b200.optimize import OBJECTIVES, bulk_gradient, bulk_objective, optimize_bulk
from homo3d_b200.density import synthetic_density
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def oracle_loop(n, rho, iters, vol=0.3, objective="bulk"):
    obj_fn, grad_fn = OBJECTIVES[objective]
    objs = []
    for it in range(iters):
        m = O.MG((n, n, n))
        m.set_density(rho ** 3)
        m.update_stencils()
        m.rhs()
        m.solve(1e-10, 400)
        C = m.elastic_matrix()
        objs.append(obj_fn(C, it))
        s = m.sensitivity(grad_fn(it).astype(np.float64)) * 3 * rho ** 2
        s = O.symmetrize_f32((n, n, n), s, "reflect6").astype(np.float64)
        s = O.filter_sens((n, n, n), s, rho, 2.0, False)
        rho, _ = O.oc_update(s, rho, vol, 1e-3, 0.05, 0.5)
        rho = O.symmetrize_f32((n, n, n), rho, "reflect6").astype(np.float64)
    return rho, objs


@pytest.mark.parametrize("objective", ["bulk", "shear", "npr"])
def test_oc_loop_matches_oracle(torch_cuda, objective):
    n = 16
    rho0 = synthetic_density(n, seed=5, vol=0.3).ravel().astype(np.float32).astype(np.float64)
    rho, C, rec = optimize_bulk(n, iters=3, rho0=rho0, relthres=1e-8, objective=objective)
    ref_rho, ref_objs = oracle_loop(n, rho0.copy(), 3, objective=objective)
    objs = [r["obj"] for r in rec]
    for a, b in zip(objs, ref_objs):
        assert abs(a - b) / abs(b) < 1e-4, (objs, ref_objs)
    assert np.abs(rho - ref_rho).max() < 1e-3
    assert abs(rho.astype(np.float64).mean() - 0.3) < 2e-4


@pytest.mark.parametrize("seed,vol", [(0, 0.3), (3, 0.4)])
def test_oc_loop_through_high_contrast(torch_cuda, seed, vol):
    """two 128^3 bulk-modulus loops whose fifth solve (densities at their 1e-3 floor
    in places) diverged with the exact coarsest inverse: with the loop's projected
    coarsest solve every solve converges"""
    rho, C, rec = optimize_bulk(128, vol=vol, iters=8, seed=seed, relthres=1e-2)
    assert len(rec) == 8 and all(r["vcycles"] <= 10 for r in rec)
    assert rec[-1]["obj"] < rec[0]["obj"]


def test_oc_loop_improves_bulk_modulus(torch_cuda):
    rho, C, rec = optimize_bulk(32, iters=8, seed=1, relthres=1e-2)
    objs = [r["obj"] for r in rec]
    assert objs[-1] < objs[0]  # obj = -bulk modulus decreases
    assert all(r["vcycles"] >= 1 for r in rec)
    assert rec[-1]["vcycles"] <= rec[0]["vcycles"]  # warm start pays off


def test_shear_loop_raises_shear_modulus(torch_cuda):
    rho, C, rec = optimize_bulk(32, iters=8, seed=3, relthres=1e-2, objective="shear")
    objs = [r["obj"] for r in rec]
    assert objs[-1] < objs[0]  # obj = -shear modulus decreases
    assert abs(rho.astype(np.float64).mean() - 0.3) < 2e-4


def test_npr_loop_lowers_poisson_coupling(torch_cuda):
    torch = torch_cuda
    n = 32
    rho0 = synthetic_density(n, seed=2, vol=0.3).ravel()
    hd = H.Homogenization(n)
    hd.update(torch.tensor((rho0 ** 3).astype(np.float32), device="cuda"))
    C0 = hd.elasticMatrix(1e-4)
    hd.close()
    rho, C, rec = optimize_bulk(n, iters=10, rho0=rho0, relthres=1e-2, objective="npr")
    ratio = lambda c: (c[0, 1] + c[0, 2] + c[1, 2]) / (c[0, 0] + c[1, 1] + c[2, 2])
    assert ratio(C) < ratio(C0)  # the coupling falls relative to the diagonal


@pytest.mark.parametrize("objective", ["bulk", "npr"])
def test_device_design_step_equals_separate_calls(torch_cuda, objective):
    """the captured design-step graph (h3d_design_step) runs the same kernels in the
    same order as the separate entry points: the same densities to the last bit
    (npr changes dC every iteration: the graph reads it at run time)"""
    n = 16
    rho0 = synthetic_density(n, seed=7, vol=0.3).ravel()
    a = optimize_bulk(n, iters=4, rho0=rho0, relthres=1e-6, objective=objective, device_step=True)
    b = optimize_bulk(n, iters=4, rho0=rho0, relthres=1e-6, objective=objective, device_step=False)
    assert np.array_equal(a[0], b[0])
    assert [r["obj"] for r in a[2]] == [r["obj"] for r in b[2]]


def test_design_step_rejects_bad_arguments(torch_cuda):
    torch = torch_cuda
    hd = H.Homogenization(8)
    rho = torch.full((8 ** 3,), 0.3, device="cuda")
    sens = torch.zeros_like(rho)
    with pytest.raises(H.H3DError):
        hd.design_step(np.zeros((6, 6)), rho, sens, 1.5)
    hd.close()


@pytest.mark.parametrize("periodic", [False, True])
def test_conv_radial_and_adjoint_match_restatement(torch_cuda, periodic):
    from oracle import expr_oracle as X
    torch = torch_cuda
    n, r = 16, 2.0
    hd = H.Homogenization(n)
    a = np.random.default_rng(3).uniform(0, 1, (n, n, n))
    t = torch.tensor(a.ravel(), dtype=torch.float32, device="cuda")
    out = torch.empty_like(t)
    hd.conv_radial(t, out, r, periodic)
    ref, _ = X.conv(a, r, periodic)
    assert np.abs(out.cpu().numpy() - ref.ravel()).max() < 1e-6
    hd.conv_radial(t, out, r, periodic, adjoint=True)
    ref = X.conv_adjoint(a, r, periodic)
    assert np.abs(out.cpu().numpy() - ref.ravel()).max() < 1e-5 * np.abs(ref).max()
    # the adjoint is the transpose: <conv a, b> = <a, conv^T b>
    b = np.random.default_rng(4).uniform(-1, 1, (n, n, n))
    lhs = (X.conv(a, r, periodic)[0] * b).sum()
    rhs = (a * X.conv_adjoint(b, r, periodic)).sum()
    assert abs(lhs - rhs) < 1e-9 * abs(lhs)
    hd.close()


def oracle_shear_isotropy(n, rho, iters, vol=0.3, r=2.0):
    """example_opti_shear_isotropy (Framework.cu:274-351) on the FP64 oracle pieces"""
    from homo3d_b200.optimize import SGM_C, SGM_K, ANI_SCALE, VOL_SCALE, shear_isotropy_terms
    from oracle import expr_oracle as X
    ne = n ** 3
    mma = O.MMA(2, ne, 1.0, 0.0, 1000.0, 1.0)
    mma.set_bound(0.001, 1.0)
    objs = []
    for it in range(iters):
        z = X.conv(rho.reshape(n, n, n), r)[0].ravel()
        y = 1.0 / (1.0 + np.exp(-SGM_K * (z - SGM_C)))
        rhop = (y ** 3).astype(np.float32).astype(np.float64)
        m = O.MG((n, n, n))
        m.set_density(rhop)
        m.update_stencils()
        m.rhs()
        m.solve(1e-10, 400)
        C = m.elastic_matrix()
        obj, dC_obj, con, dC_con = shear_isotropy_terms(C)
        objs.append(obj)
        dphys = 3 * y * y * SGM_K * y * (1 - y)
        grads = []
        for dC in (dC_obj, dC_con):
            s = m.sensitivity(dC.astype(np.float64)) * dphys
            g = X.conv_adjoint(s.reshape(n, n, n), r).ravel()
            grads.append(O.symmetrize_f32((n, n, n), g, "reflect6").astype(np.float64))
        gvol = X.conv_adjoint((SGM_K * y * (1 - y) / ne).reshape(n, n, n), r).ravel()
        gval = np.array([(y.mean() - vol) * VOL_SCALE, con * ANI_SCALE - 0.1])
        rho = mma.update(it, rho, grads[0], gval, np.stack([gvol, grads[1]]))
    return rho, objs


def test_shear_isotropy_mma_loop_matches_oracle(torch_cuda):
    from homo3d_b200.optimize import optimize_shear_isotropy
    """from a start whose smoothed, sigmoid-projected density is a connected solid (a
    start below the sigmoid's centre projects to near-void, C ~ 1e-6 E, where the
    1e9 stiffness contrast leaves both solves inaccurate); two iterations: the
    reference's volume scaling (x1000) drives the design towards void after the first
    update, and later iterations meet the same ill-conditioning"""
    n = 16
    rho0 = synthetic_density(n, seed=9, vol=0.6).ravel().astype(np.float32).astype(np.float64)
    rho, C, rec = optimize_shear_isotropy(n, iters=2, rho0=rho0, relthres=1e-8)
    ref_rho, ref_objs = oracle_shear_isotropy(n, rho0.copy(), 2)
    objs = [r["obj"] for r in rec]
    assert objs[0] < -0.5  # a stiff start
    for a, b in zip(objs, ref_objs):
        assert abs(a - b) / abs(b) < 1e-4, (objs, ref_objs)
    # the MMA subproblem amplifies the FP32 rounding of the projected density's
    # gradients near its asymptotes: the designs agree on average, a few elements
    # by ~1e-2
    d = np.abs(rho - ref_rho)
    assert d.mean() < 2e-3 and d.max() < 3e-2, (d.mean(), d.max())
