"""CPU tests of the FP64 oracle: pins it to the reference's hard-coded tables and
to analytic known answers before it is used to check the CUDA library."""
import json
import os

import numpy as np
import pytest

from oracle import oracle as O
from tests.conftest import smooth_density

HERE = os.path.dirname(os.path.abspath(__file__))
E, NU = 10.0, 0.3
LAM = NU * E / ((1 + NU) * (1 - 2 * NU))
MU = E / (2 * (1 + NU))


def base_material(E=E, nu=NU):
    lam = nu * E / ((1 + nu) * (1 - 2 * nu))
    mu = E / (2 * (1 + nu))
    D = np.zeros((6, 6))
    D[:3, :3] = lam
    D[np.arange(3), np.arange(3)] += 2 * mu
    D[np.arange(3, 6), np.arange(3, 6)] = mu
    return D


def test_ke_matches_reference_integer_tables():
    g = json.load(open(os.path.join(HERE, "golden", "ke_lame72.json")))
    kl, km = O.ke_lame()
    assert np.array_equal(np.rint(72 * kl).astype(int).ravel(), np.array(g["kelam72"]))
    assert np.array_equal(np.rint(72 * km).astype(int).ravel(), np.array(g["kemu72"]))
    assert np.abs(72 * kl - np.rint(72 * kl)).max() < 1e-12
    assert np.abs(72 * km - np.rint(72 * km)).max() < 1e-12
    K = O.ke(E, NU)
    assert np.abs(K - (LAM * kl + MU * km)).max() < 1e-12


def test_ke_properties():
    K = O.ke(E, NU)
    assert np.abs(K - K.T).max() == 0
    # rigid translations and rotations are in the null space: 6 zero eigenvalues
    ev = np.sort(np.abs(np.linalg.eigvalsh(K)))
    assert ev[5] < 1e-12 and ev[6] > 0.1
    t = np.tile(np.eye(3), (8, 1))
    assert np.abs(K @ t).max() < 1e-12


@pytest.mark.parametrize("reso,dims,ratios", [
    (8, [8, 4], [0, 2]), (32, [32, 16, 8, 4], [0, 2, 2, 2]), (96, [96, 48, 24, 12, 6], [0, 2, 2, 2, 2]),
    (80, [96, 48, 24, 12, 6], [0, 2, 2, 2, 2]), (320, [320, 160, 80, 40, 20, 10, 5], [0, 2, 2, 2, 2, 2, 2]),
    (256, [256, 128, 64, 32, 16, 8, 4], [0, 2, 2, 2, 2, 2, 2]),
    (512, [512, 128, 64, 32, 16, 8, 4], [0, 4, 2, 2, 2, 2, 2]),
])
def test_hierarchy_rules(reso, dims, ratios):
    d, r = O.hierarchy((reso,) * 3)
    assert d[:, 0].tolist() == dims and r[:, 0].tolist() == ratios


def test_homogeneous_density_gives_base_material():
    m = O.MG((16, 16, 16))
    m.set_density(np.ones(16 ** 3))
    m.rhs()
    assert np.abs(m.f()).max() < 1e-12
    m.update_stencils()
    C = m.elastic_matrix()
    assert np.abs(C - base_material() * (1 + 1e-9)).max() < 1e-10


def laminate_C(phases):
    """Exact homogenized stiffness of layers normal to x (volume fraction, 6x6 Voigt C)."""
    N, T = [0, 4, 5], [1, 2, 3]
    inv_nn = sum(f * np.linalg.inv(C[np.ix_(N, N)]) for f, C in phases)
    Cnn = np.linalg.inv(inv_nn)
    a = sum(f * np.linalg.inv(C[np.ix_(N, N)]) @ C[np.ix_(N, T)] for f, C in phases)
    b = sum(f * C[np.ix_(T, N)] @ np.linalg.inv(C[np.ix_(N, N)]) for f, C in phases)
    c = sum(f * (C[np.ix_(T, T)] - C[np.ix_(T, N)] @ np.linalg.inv(C[np.ix_(N, N)]) @ C[np.ix_(N, T)])
            for f, C in phases)
    out = np.zeros((6, 6))
    out[np.ix_(N, N)] = Cnn
    out[np.ix_(N, T)] = Cnn @ a
    out[np.ix_(T, N)] = (Cnn @ a).T
    out[np.ix_(T, T)] = c + b @ Cnn @ a
    return out


def test_laminate_known_answer():
    n = 16
    x = np.arange(n)
    prof = np.where((x >= 3) & (x < 9), 1.0, 0.2)   # grid-aligned layers along x
    rho = np.broadcast_to(prof[None, None, :], (n, n, n)).ravel()
    m = O.MG((n, n, n))
    m.set_density(rho)
    m.update_stencils()
    m.rhs()
    it, h = m.solve(1e-11, 300)
    assert h[-1].max() <= 1e-11
    C = m.elastic_matrix()
    D = base_material()
    ref = laminate_C([(6 / 16, D * (1 + 1e-9)), (10 / 16, D * (0.2 + 1e-9))])
    assert np.abs(C - ref).max() / np.abs(ref).max() < 1e-8


def test_reflect6_density_gives_cubic_C():
    n = 16
    m = O.MG((n, n, n))
    m.set_density(smooth_density(n, seed=3))
    m.update_stencils()
    m.rhs()
    m.solve(1e-10, 300)
    C = m.elastic_matrix()
    assert np.abs(C - C.T).max() < 1e-9 * np.abs(C).max()
    assert np.all(np.linalg.eigvalsh(C) > 0)
    tol = 1e-6 * np.abs(C).max()
    assert abs(C[0, 0] - C[1, 1]) < tol and abs(C[1, 1] - C[2, 2]) < tol
    assert abs(C[0, 1] - C[0, 2]) < tol and abs(C[0, 1] - C[1, 2]) < tol
    assert abs(C[3, 3] - C[4, 4]) < tol and abs(C[4, 4] - C[5, 5]) < tol
    off = C.copy()
    off[:3, :3] = 0
    off[np.arange(3, 6), np.arange(3, 6)] = 0
    assert np.abs(off).max() < tol


def test_galerkin_fast_equals_reference_loop_nest():
    for n in (8, 16):
        m = O.MG((n, n, n))
        m.set_density(smooth_density(n, seed=1))
        m.galerkin_l1(0)
        a = m.stencil(1).copy()
        m.galerkin_l1(1)
        b = m.stencil(1).copy()
        assert np.abs(a - b).max() == 0.0


def test_galerkin_identity_without_rounding():
    """Level-1 stencil of an interior vertex equals R K P (no FP16, no clamp hit)."""
    n = 8
    m = O.MG((n, n, n))
    m.set_fp16(False)
    rho = np.full(n ** 3, 0.5)
    m.set_density(rho)
    m.galerkin_l1(1)
    st = m.stencil(1)
    K = O.ke(E, NU) * 0.5
    # assemble the periodic fine matrix (unpinned) and P for ratio 2
    nv = n ** 3
    A = np.zeros((3 * nv, 3 * nv))
    idx = lambda x, y, z: (x % n) + n * ((y % n) + n * (z % n))
    for z in range(n):
        for y in range(n):
            for x in range(n):
                nodes = [idx(x + a % 2, y + a // 2 % 2, z + a // 4) for a in range(8)]
                for a in range(8):
                    for b in range(8):
                        A[3 * nodes[a]:3 * nodes[a] + 3, 3 * nodes[b]:3 * nodes[b] + 3] += K[3 * a:3 * a + 3, 3 * b:3 * b + 3]
    nc = n // 2
    P = np.zeros((3 * nv, 3 * nc ** 3))
    for Z in range(nc):
        for Y in range(nc):
            for X in range(nc):
                for oz in range(-1, 2):
                    for oy in range(-1, 2):
                        for ox in range(-1, 2):
                            w = (2 - abs(ox)) * (2 - abs(oy)) * (2 - abs(oz)) / 8
                            f = idx(2 * X + ox, 2 * Y + oy, 2 * Z + oz)
                            c = X + nc * (Y + nc * Z)
                            P[3 * f:3 * f + 3, 3 * c:3 * c + 3] += w * np.eye(3)
    Ac = P.T @ A @ P
    X0 = (2, 2, 2)
    c0 = X0[0] + nc * (X0[1] + nc * X0[2])
    for d in range(27):
        dx, dy, dz = d % 3 - 1, d // 3 % 3 - 1, d // 9 - 1
        c1 = (X0[0] + dx) % nc + nc * ((X0[1] + dy) % nc + nc * ((X0[2] + dz) % nc))
        blk = Ac[3 * c0:3 * c0 + 3, 3 * c1:3 * c1 + 3]
        assert np.abs(st[c0, d].reshape(3, 3) - blk).max() < 1e-12


def test_solve_converges_and_projection_mode_is_slower():
    n = 16
    rho = smooth_density(n, seed=0)
    res = {}
    for proj in (0, 1):
        m = O.MG((n, n, n))
        m.set_project(proj)
        m.set_density(rho)
        m.update_stencils()
        m.rhs()
        it, h = m.solve(1e-5, 40)
        res[proj] = (it, h[-1].max())
    assert res[0][1] <= 1e-5 and res[0][0] < 30
    assert res[1][0] >= res[0][0]  # removing translations from the coarse rhs never helps


def test_sensitivity_matches_finite_differences():
    n = 8
    rho = smooth_density(n, seed=2)
    m = O.MG((n, n, n))
    m.set_density(rho)
    m.update_stencils()
    m.rhs()
    m.solve(1e-12, 400)
    dC = np.zeros((6, 6))
    dC[0, 0] = 1.0
    dC[0, 1] = 0.5
    dC[3, 3] = -2.0
    s = m.sensitivity(dC)
    obj = lambda C: (dC * C).sum()
    for e in (0, 77, 300, 511):
        h = 1e-4
        vals = []
        for sgn in (1, -1):
            r2 = rho.copy()
            r2[e] += sgn * h
            m2 = O.MG((n, n, n))
            m2.set_density(r2)
            m2.update_stencils()
            m2.rhs()
            m2.solve(1e-12, 400)
            vals.append(obj(m2.elastic_matrix()))
        fd = (vals[0] - vals[1]) / (2 * h)
        assert abs(fd - s[e]) <= 1e-6 * max(1.0, abs(fd)) + 1e-7


@pytest.mark.parametrize("sym", ["reflect3", "reflect6", "rotate3"])
def test_symmetrize_is_an_invariant_projection(sym):
    n = 12
    rng = np.random.default_rng(5)
    v = rng.random(n ** 3).astype(np.float32)
    s1 = O.symmetrize_f32((n, n, n), v, sym)
    a = s1.reshape(n, n, n)  # [z, y, x]
    if sym in ("reflect3", "reflect6"):
        for ax in range(3):
            assert np.array_equal(a, np.flip(a, axis=ax))
    if sym == "reflect6":
        assert np.array_equal(a, np.transpose(a, (1, 0, 2)))
        assert np.array_equal(a, np.transpose(a, (2, 1, 0)))
    if sym == "rotate3":
        # 90 degree rotation about z: (x, y) -> (y, -x) about the centre
        assert np.array_equal(a, np.rot90(a, k=1, axes=(1, 2)))
    # the orbit mean preserves the total (up to FP32 rounding)
    assert abs(float(s1.astype(np.float64).sum()) - float(v.astype(np.float64).sum())) < 1e-3


def test_oc_update_hits_volume_and_bounds():
    rng = np.random.default_rng(0)
    n = 16 ** 3
    rho = np.clip(rng.random(n), 1e-3, 1)
    sens = -rng.random(n)
    new, it = O.oc_update(sens, rho, 0.3, 1e-3, 0.05, 0.5)
    assert abs(new.mean() - 0.3) <= 1e-4 or it == 20
    assert np.all(np.abs(new - rho) <= 0.05 + 1e-12)
    assert new.min() >= 1e-3 and new.max() <= 1.0


def test_filter_preserves_constant_ratio():
    n = (10, 10, 10)
    rho = np.full(1000, 0.4)
    sens = np.full(1000, -2.0)
    out = O.filter_sens(n, sens, rho, 2.0, False)
    assert np.abs(out + 2.0).max() < 1e-12
