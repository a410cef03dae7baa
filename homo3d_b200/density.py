"""Seeded synthetic density fields for benchmarks and tests.

rho(x) = clamp(0.3 + 0.25 * sum_{k in {0,1,2}^3} a_k cos(2 pi k.x + phi_k), 1e-3, 1)
with a_k ~ U(-1, 1) and phi_k ~ U(0, 2 pi) drawn from SplitMix64(seed) in the
order k = kx + 3 ky + 9 kz (a_k then phi_k), x the voxel centre (i + 1/2)/N.
The field is then averaged over the 48 symmetries of the cube (reflect6) and
shifted (with the same clamp) until its mean is within 1e-6 of the target volume.

The reference's own initialiser (homogenization/Framework.cuh:238-310, randTri)
is seeded from the clock and cannot be reproduced; this generator replaces it.
Arrays are float64 with shape (nz, ny, nx), i.e. lexicographic order x fastest.
"""
import numpy as np

_M64 = (1 << 64) - 1


class SplitMix64:
    def __init__(self, seed):
        self.state = int(seed) & _M64

    def next_u64(self):
        self.state = (self.state + 0x9E3779B97F4A7C15) & _M64
        z = self.state
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & _M64
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & _M64
        return z ^ (z >> 31)

    def uniform(self):
        return (self.next_u64() >> 11) * (1.0 / (1 << 53))


def trig_init_coefficients(n_period, seed=0, centered=False):
    """coefficients of the reference's randTri initialiser (Framework.cuh:238-310):
    6 P + 36 P^2 (+ 4 for the centred form) values uniform in [-1, 1), drawn here from
    SplitMix64(seed) in place of the reference's clock-seeded curand generator"""
    rng = SplitMix64(seed)
    nb = 6 * n_period + 36 * n_period * n_period + (4 if centered else 0)
    return np.array([2.0 * rng.uniform() - 1.0 for _ in range(nb)], np.float32)


def trig_coefficients(seed):
    rng = SplitMix64(seed)
    a = np.zeros((3, 3, 3))
    phi = np.zeros((3, 3, 3))
    for t in range(27):
        kx, ky, kz = t % 3, t // 3 % 3, t // 9
        a[kz, ky, kx] = 2.0 * rng.uniform() - 1.0
        phi[kz, ky, kx] = 2.0 * np.pi * rng.uniform()
    return a, phi


def trig_field(n, seed):
    """The unclamped trig-basis sum evaluated separably: shape (n, n, n)."""
    a, phi = trig_coefficients(seed)
    x = (np.arange(n) + 0.5) / n
    E = np.exp(2j * np.pi * np.outer(np.arange(3), x))          # [k, i]
    c = a * np.exp(1j * phi)                                     # [kz, ky, kx]
    S = np.einsum("zyx,zk->kyx", c, E)                           # [z, ky, kx]
    T = np.einsum("kyx,yj->kjx", S, E)                           # [z, y, kx]
    field = np.einsum("kjx,xi->kji", T, E).real                  # [z, y, x]
    return 0.3 + 0.25 * field


def reflect6_average(v):
    """Average over the 48 symmetries of the cube (8 mirror flips x 6 axis permutations)."""
    acc = np.zeros_like(v)
    for perm in [(0, 1, 2), (0, 2, 1), (1, 0, 2), (1, 2, 0), (2, 0, 1), (2, 1, 0)]:
        p = np.transpose(v, perm)
        for f in range(8):
            axes = tuple(ax for ax in range(3) if (f >> ax) & 1)
            acc += np.flip(p, axis=axes) if axes else p
    return acc / 48.0


def rescale_volume(v, vol, lo=1e-3, tol=1e-6, iters=200):
    """Shift v (with the clamp to [lo, 1]) so that its mean equals vol."""
    a, b = -2.0, 2.0
    for _ in range(iters):
        t = 0.5 * (a + b)
        m = np.clip(v + t, lo, 1.0).mean()
        if abs(m - vol) <= tol:
            break
        if m < vol:
            a = t
        else:
            b = t
    return np.clip(v + t, lo, 1.0)


def synthetic_density(n, seed=0, vol=0.3, symmetric=True):
    """Design density rho in [1e-3, 1], shape (n, n, n), mean vol."""
    v = np.clip(trig_field(n, seed), 1e-3, 1.0)
    if symmetric:
        v = reflect6_average(v)
    return rescale_volume(v, vol)
