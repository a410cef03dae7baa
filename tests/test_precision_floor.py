"""Why the level-0 correction is stored in FP32 (CPU, FP64 oracle at 32^3).

Rounding a converged solution chi to a storage format and recomputing its residual
in FP64 leaves ||r||/||f|| far above relthres 1e-5 for FP16 and BF16 (and the floor
grows with the grid, about like N^1.8), while FP32 stays near 1e-6.  Rounding the
element-local differences U - u_0 that the tensor-core residual contracts costs much
less, and an FP16 hi + lo split of them is as accurate as FP32."""
import numpy as np
import pytest

from oracle import oracle as O
from tests.conftest import smooth_density


def rounded(a, kind):
    if kind == "fp32":
        return a.astype(np.float32).astype(np.float64)
    if kind == "fp16":
        return a.astype(np.float16).astype(np.float64)
    if kind == "bf16":  # round to nearest even on the upper 16 bits of the FP32 pattern
        b = a.astype(np.float32).view(np.uint32).astype(np.uint64)
        b = ((b + 0x7FFF + ((b >> 16) & 1)) >> 16) << 16
        return b.astype(np.uint32).view(np.float32).astype(np.float64)
    if kind == "fp16x2":
        hi = a.astype(np.float16).astype(np.float64)
        return hi + (a - hi).astype(np.float16).astype(np.float64)
    return a


@pytest.fixture(scope="module")
def converged():
    n = 32
    m = O.MG((n, n, n))
    rho = smooth_density(n, seed=0, vol=0.3).astype(np.float32).astype(np.float64)
    m.set_density(rho)
    m.update_stencils()
    m.rhs()
    m.solve(1e-10, 400)
    return n, m, rho, m.u(0).copy(), m.f(0).copy()


def rel_res(m, n, u, f):
    m.u(0)[:] = u
    m.residual(0)
    return (O.weighted_norm((n, n, n), m.r(0)) / O.weighted_norm((n, n, n), f)).max()


def test_value_rounding_floor(converged):
    n, m, _, chi, f = converged
    r = {k: rel_res(m, n, rounded(chi, k), f) for k in ("fp32", "fp16", "bf16")}
    assert r["fp32"] < 1e-5
    assert r["fp16"] > 3e-3 and r["bf16"] > 3e-2, r


def ebe_residual(n, rho, u, f, Ke, kind):
    """r = f - sum_e rho_e Ke (U_e - u_0(e)) with the differences rounded to kind"""
    i = np.arange(n)
    ez, ey, ex = [a.ravel() for a in np.meshgrid(i, i, i, indexing="ij")]
    vid = np.stack([((ex + (a & 1)) % n) + n * (((ey + ((a >> 1) & 1)) % n) + n * ((ez + (a >> 2)) % n))
                    for a in range(8)], 1)
    U = u[vid]
    dU = rounded(U - U[:, :1], kind).transpose(0, 2, 1, 3).reshape(-1, 6, 24)
    KU = np.einsum("ij,ecj->eci", Ke, dU) * (1e-9 + rho)[:, None, None]
    Ku = np.zeros_like(u)
    KU = KU.reshape(-1, 6, 8, 3)
    for a in range(8):
        np.add.at(Ku, vid[:, a], KU[:, :, a, :])
    r = f - Ku
    r[0] = 0
    return r


def test_difference_rounding_of_the_element_products(converged):
    n, m, rho, chi, f = converged
    Ke = m.ke()
    fn = O.weighted_norm((n, n, n), f)
    r0 = ebe_residual(n, rho, chi, f, Ke, None)
    d = {k: (O.weighted_norm((n, n, n), ebe_residual(n, rho, chi, f, Ke, k) - r0) / fn).max()
         for k in ("fp16", "fp16x2")}
    assert d["fp16"] < 3e-3 and d["fp16x2"] < 1e-6, d
