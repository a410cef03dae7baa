"""FP64 numpy restatement of the reference's trig-basis initial density.

TEST INFRASTRUCTURE ONLY (imported by tests/): the oracle for the library's
h3d_init_density_trig.  Follows homo3d homogenization/Framework.cuh:106-222
(randTribase_sincos_kernel: the basis sum, positions p = (x, y, z) / (dim - 1),
optionally centred and rotated by a quaternion) and Framework.cuh:238-310 (randTri:
symmetrisation, then the level set m + (M - m) sigmoid(15 (v - t)), M = min(1.5 vol,
1), m = 0.001, t bisected on [-37 P^2, 37 P^2] for at most 60 steps until the mean is
within 1e-3 of vol).  Parity unpinned beyond the formulas: the reference draws its
coefficients from a clock-seeded curand generator, so no run of it can be
reproduced; the coefficients here are the caller's.
"""
import numpy as np


def basis_field(n, P, coeff, centered=False):
    """the basis sum at every voxel, shape (nz, ny, nx), float64"""
    coeff = np.asarray(coeff, np.float64)
    nb = 6 * P + 36 * P * P
    ax = [np.arange(n[d]) / np.float64(n[d] - 1) for d in range(3)]
    z, y, x = np.meshgrid(ax[2], ax[1], ax[0], indexing="ij")
    p = np.stack([x, y, z])                                        # [3, nz, ny, nx]
    if centered:
        w, qx, qy, qz = coeff[nb:nb + 4] / np.linalg.norm(coeff[nb:nb + 4])
        R = np.array([[1 - 2 * (qy * qy + qz * qz), 2 * (qx * qy - w * qz), 2 * (qx * qz + w * qy)],
                      [2 * (qx * qy + w * qz), 1 - 2 * (qx * qx + qz * qz), 2 * (qy * qz - w * qx)],
                      [2 * (qx * qz - w * qy), 2 * (qy * qz + w * qx), 1 - 2 * (qx * qx + qy * qy)]])
        p = np.einsum("ab,b...->a...", R, p - 0.5)
    k = np.arange(1, P + 1).reshape(P, 1, 1, 1)
    cos = [np.cos(2 * np.pi * k * p[a]) for a in range(3)]         # [P, nz, ny, nx] per axis
    sin = [np.sin(2 * np.pi * k * p[a]) for a in range(3)]
    v = np.concatenate(cos + sin)                                  # v(j): j < 3P cos[j/P][j%P], then sin
    s = np.zeros(p.shape[1:])
    for i in range(6 * P):                                         # first order: component fastest
        j = i if i < 3 * P else i - 3 * P
        s += coeff[i] * v[(j % 3) * P + j // 3 + (0 if i < 3 * P else 3 * P)]
    c2 = coeff[6 * P:nb].reshape(6 * P, 6 * P)
    s += np.einsum("j...,jk,k...->...", v, c2, v)
    return s


def level_set(v, P, vol):
    """the volume-matching level-set map of randTri; returns (density, t)"""
    M = min(vol * 1.5, 1.0)
    mp = lambda t: 1.0 / (1 + np.exp(-15.0 * (v - t))) * (M - 0.001) + 0.001
    tu = P * P * 37.0
    tl = -tu
    t = 0.0
    for _ in range(60):
        t = (tu + tl) / 2
        s = mp(t).mean()
        if abs(s - vol) / vol < 1e-3:
            break
        if s > vol:
            tl = t
        if s < vol:
            tu = t
    return mp(t), t
