"""Python binding of the FP64 CPU oracle (h3d_oracle.c, mma_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, by ``__graft_entry__.smoke()`` and by
the CPU-baseline leg of ``bench.py``.  The product (``homo3d_b200``) never imports it.

Array conventions (see h3d_oracle.c): vertex fields are float64 ``[nv, 6, 3]`` in
lexicographic vertex order (x fastest); stencils are float64 ``[nv, 27, 9]``.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

_dp = ctypes.POINTER(ctypes.c_double)
_fp = ctypes.POINTER(ctypes.c_float)
_ip = ctypes.POINTER(ctypes.c_int)


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        L.ora_mma_update.restype = ctypes.c_int
        L.ora_mma_update.argtypes = [ctypes.c_int, ctypes.c_long, ctypes.c_int] + [_dp] * 10 + [
            ctypes.c_double, _dp, _dp, _dp, ctypes.c_double]
        L.ora_mg_create.restype = ctypes.c_void_p
        L.ora_mg_create.argtypes = [_ip, ctypes.c_double, ctypes.c_double]
        L.ora_mg_destroy.argtypes = [ctypes.c_void_p]
        L.ora_mg_nlevels.argtypes = [ctypes.c_void_p]
        L.ora_mg_level_info.argtypes = [ctypes.c_void_p, ctypes.c_int, _ip, _ip]
        L.ora_mg_field.restype = _dp
        L.ora_mg_field.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
        L.ora_mg_ke.argtypes = [ctypes.c_void_p, _dp]
        L.ora_mg_set_fp16.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.ora_mg_set_project.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.ora_mg_set_pin_identity.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.ora_mg_set_density.argtypes = [ctypes.c_void_p, _dp]
        L.ora_mg_rhs.argtypes = [ctypes.c_void_p]
        L.ora_mg_gs.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double]
        L.ora_mg_residual.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.ora_mg_restrict.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.ora_mg_prolong.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.ora_mg_galerkin_l1.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.ora_mg_galerkin.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.ora_mg_coarse_matrix.argtypes = [ctypes.c_void_p, _dp]
        L.ora_mg_coarse_factor.argtypes = [ctypes.c_void_p]
        L.ora_mg_coarse_solve.argtypes = [ctypes.c_void_p]
        L.ora_mg_update_stencils.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.ora_mg_vcycle.argtypes = [ctypes.c_void_p, ctypes.c_double]
        L.ora_mg_remove_mean.argtypes = [ctypes.c_void_p]
        L.ora_mg_solve.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_int, _dp]
        L.ora_mg_elastic_matrix.argtypes = [ctypes.c_void_p, _dp, _dp]
        L.ora_mg_sensitivity.argtypes = [ctypes.c_void_p, _dp, _dp, _dp, ctypes.c_int]
        L.ora_weighted_norm.argtypes = [_ip, _dp, _dp]
        L.ora_ke.argtypes = [ctypes.c_double, ctypes.c_double, _dp]
        L.ora_ke_lame.argtypes = [_dp, _dp]
        L.ora_hierarchy.argtypes = [_ip, _ip, _ip]
        L.ora_oc_update.argtypes = [ctypes.c_long, _dp, _dp, ctypes.c_double, ctypes.c_double,
                                    ctypes.c_double, ctypes.c_double]
        L.ora_filter_sens.argtypes = [_ip, _dp, _dp, _dp, ctypes.c_double, ctypes.c_int]
        L.ora_symmetrize_f32.argtypes = [_ip, _fp, ctypes.c_int]
        _LIB = L
    return _LIB


def _d(a):
    return a.ctypes.data_as(_dp)


def _i3(v):
    return (ctypes.c_int * 3)(*[int(x) for x in v])


def ke(E=10.0, nu=0.3):
    out = np.zeros(576)
    lib().ora_ke(E, nu, _d(out))
    return out.reshape(24, 24)


def ke_lame():
    kl = np.zeros(576)
    km = np.zeros(576)
    lib().ora_ke_lame(_d(kl), _d(km))
    return kl.reshape(24, 24), km.reshape(24, 24)


def hierarchy(reso):
    dims = (ctypes.c_int * 48)()
    rat = (ctypes.c_int * 48)()
    nl = lib().ora_hierarchy(_i3(reso), dims, rat)
    if nl < 1:
        raise ValueError("unsupported resolution %r" % (reso,))
    d = np.frombuffer(dims, dtype=np.int32).reshape(16, 3)[:nl].copy()
    r = np.frombuffer(rat, dtype=np.int32).reshape(16, 3)[:nl].copy()
    return d, r


class MMA:
    """State of one MMA optimiser (MMAOptimizer, optimization/mmaOptimizer.h:12-36):
    the FP64 design, the two previous designs and the asymptotes."""

    def __init__(self, m, n, a0=1.0, a=0.0, c=1000.0, d=1.0):
        self.m, self.n, self.a0 = m, n, a0
        self.a = np.full(m, a, np.float64)
        self.c = np.full(m, c, np.float64)
        self.d = np.full(m, d, np.float64)
        self.xmin = np.zeros(n)
        self.xmax = np.ones(n)
        self.xold1 = np.zeros(n)
        self.xold2 = np.zeros(n)
        self.low = np.zeros(n)
        self.upp = np.zeros(n)
        self.newton = 0

    def set_bound(self, xmin, xmax):
        self.xmin = np.broadcast_to(np.asarray(xmin, np.float64), (self.n,)).copy()
        self.xmax = np.broadcast_to(np.asarray(xmax, np.float64), (self.n,)).copy()

    def update(self, itn, x, dfdx, gval, dgdx, move=1.0):
        """returns the new design; x, dfdx are [n], gval [m], dgdx [m, n]"""
        xv = np.ascontiguousarray(x, np.float64).copy()
        df = np.ascontiguousarray(dfdx, np.float64)
        gv = np.ascontiguousarray(gval, np.float64).reshape(self.m)
        dg = np.ascontiguousarray(dgdx, np.float64).reshape(self.m, self.n)
        self.newton = lib().ora_mma_update(self.m, self.n, itn, _d(xv), _d(self.xmin), _d(self.xmax), _d(self.xold1),
                                           _d(self.xold2), _d(df), _d(gv), _d(dg), _d(self.low), _d(self.upp),
                                           self.a0, _d(self.a), _d(self.c), _d(self.d), move)
        return xv


def weighted_norm(n, v):
    v = np.ascontiguousarray(v, dtype=np.float64)
    out = np.zeros(6)
    lib().ora_weighted_norm(_i3(n), _d(v), _d(out))
    return out


def oc_update(sens, rho, volratio, minrho=1e-3, step=0.05, damp=0.5):
    sens = np.ascontiguousarray(sens, dtype=np.float64).ravel()
    r = np.ascontiguousarray(rho, dtype=np.float64).ravel().copy()
    it = lib().ora_oc_update(r.size, _d(sens), _d(r), volratio, minrho, step, damp)
    return r.reshape(np.shape(rho)), it


def filter_sens(n, sens, rho, radius=2.0, periodic=False):
    s = np.ascontiguousarray(sens, dtype=np.float64).ravel()
    r = np.ascontiguousarray(rho, dtype=np.float64).ravel()
    out = np.zeros_like(s)
    lib().ora_filter_sens(_i3(n), _d(s), _d(r), _d(out), float(radius), int(periodic))
    return out


SYM = {"reflect3": 0, "reflect6": 1, "rotate3": 2}


def symmetrize_f32(n, v, sym):
    a = np.ascontiguousarray(v, dtype=np.float32).ravel().copy()
    lib().ora_symmetrize_f32(_i3(n), a.ctypes.data_as(_fp), SYM[sym])
    return a


class MG:
    """FP64 multigrid context: levels, stencils, V-cycles, C and sensitivities."""

    def __init__(self, reso, E=10.0, nu=0.3):
        L = lib()
        self._h = L.ora_mg_create(_i3(reso), E, nu)
        if not self._h:
            raise ValueError("unsupported resolution %r" % (reso,))
        self.nlevels = L.ora_mg_nlevels(self._h)
        self.dims, self.ratios = [], []
        for l in range(self.nlevels):
            d = (ctypes.c_int * 3)()
            r = (ctypes.c_int * 3)()
            L.ora_mg_level_info(self._h, l, d, r)
            self.dims.append(tuple(d))
            self.ratios.append(tuple(r))
        self.E, self.nu = E, nu

    def __del__(self):
        if getattr(self, "_h", None):
            lib().ora_mg_destroy(self._h)
            self._h = None

    def nv(self, l):
        d = self.dims[l]
        return d[0] * d[1] * d[2]

    def field(self, l, which):
        """Live numpy view of u (0), f (1), r (2) or the stencil (3) of level l."""
        p = lib().ora_mg_field(self._h, l, which)
        if which == 3:
            return np.ctypeslib.as_array(p, shape=(self.nv(l), 27, 9))
        return np.ctypeslib.as_array(p, shape=(self.nv(l), 6, 3))

    u = lambda self, l=0: self.field(l, 0)
    f = lambda self, l=0: self.field(l, 1)
    r = lambda self, l=0: self.field(l, 2)
    stencil = lambda self, l: self.field(l, 3)

    def ke(self):
        out = np.zeros(576)
        lib().ora_mg_ke(self._h, _d(out))
        return out.reshape(24, 24)

    def set_fp16(self, on):
        lib().ora_mg_set_fp16(self._h, int(on))

    def set_project(self, on):
        lib().ora_mg_set_project(self._h, int(on))

    def set_pin_identity(self, on):
        lib().ora_mg_set_pin_identity(self._h, int(on))

    def set_density(self, rho_phys):
        a = np.ascontiguousarray(rho_phys, dtype=np.float64).ravel()
        assert a.size == self.nv(0)
        self._rho = a
        lib().ora_mg_set_density(self._h, _d(a))

    def rhs(self):
        lib().ora_mg_rhs(self._h)

    def gs(self, l, w=1.0):
        lib().ora_mg_gs(self._h, l, w)

    def residual(self, l):
        lib().ora_mg_residual(self._h, l)

    def restrict(self, lc):
        lib().ora_mg_restrict(self._h, lc)

    def prolong(self, lf):
        lib().ora_mg_prolong(self._h, lf)

    def galerkin_l1(self, method=1):
        lib().ora_mg_galerkin_l1(self._h, method)

    def galerkin(self, lc):
        lib().ora_mg_galerkin(self._h, lc)

    def update_stencils(self, l1_method=1):
        lib().ora_mg_update_stencils(self._h, l1_method)

    def coarse_matrix(self):
        nd = 3 * self.nv(self.nlevels - 1)
        K = np.zeros((nd, nd))
        lib().ora_mg_coarse_matrix(self._h, _d(K))
        return K

    def coarse_factor(self):
        return lib().ora_mg_coarse_factor(self._h)

    def coarse_solve(self):
        lib().ora_mg_coarse_solve(self._h)

    def vcycle(self, w=1.0):
        lib().ora_mg_vcycle(self._h, w)

    def remove_mean(self):
        lib().ora_mg_remove_mean(self._h)

    def solve(self, tol, maxit=200):
        hist = np.zeros((maxit, 6))
        it = lib().ora_mg_solve(self._h, tol, maxit, _d(hist))
        return it, hist[:it]

    def elastic_matrix(self, chi=None):
        C = np.zeros(36)
        c = None if chi is None else np.ascontiguousarray(chi, dtype=np.float64)
        lib().ora_mg_elastic_matrix(self._h, None if c is None else _d(c), _d(C))
        return C.reshape(6, 6)

    def sensitivity(self, dC, chi=None, pitch=None):
        n = self.dims[0]
        pitch = n[0] if pitch is None else pitch
        out = np.zeros(pitch * n[1] * n[2])
        c = None if chi is None else np.ascontiguousarray(chi, dtype=np.float64)
        dc = np.ascontiguousarray(dC, dtype=np.float64).ravel()
        lib().ora_mg_sensitivity(self._h, None if c is None else _d(c), _d(dc), _d(out), pitch)
        return out
