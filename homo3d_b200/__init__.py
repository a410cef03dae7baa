"""homo3d_b200 -- B200-native periodic-homogenization solver (Python side).

A thin ctypes binding of ``libh3d.so`` (the C ABI declared in include/h3d.h) that
keeps the call surface of lavenklau/homo3d's hot path:

  Homogenization  (homogenization/homogenization.h:17-61): update, elasticMatrix,
                  Sensitivity
  MG              (homogenization/MG.h:14-45): v_cycle, solveEquation,
                  updateStencils, reset_displacement
  Grid            (homogenization/grid.h:104-418): gs_relaxation, update_residual,
                  restrict_residual, prolongate_correction, solveHostEquation,
                  enforce_unit_macro_strain, field access
  OCOptimizer     (optimization/OCOptimizer.h:16-19): update, filterSens
  symmetrize      (AutoDiff/TensorExpression.h:425-445)

Device buffers are passed as CUDA torch tensors (or raw integer device
pointers).  All solver work runs in the CUDA library; importing this package on a
machine without the built library raises ImportError.
"""
import ctypes
import os

import numpy as np

__all__ = ["Homogenization", "MG", "Grid", "OCOptimizer", "MMAOptimizer", "WarmNet", "H3DError", "symmetrize", "lib",
           "LIB_PATH", "batch_update", "batch_elasticMatrix", "Lockstep",
           "reference_resolution"]

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libh3d.so")

H3D_OK, H3D_ERR_ARG, H3D_ERR_CUDA, H3D_ERR_NOMEM, H3D_NOT_CONVERGED, H3D_DIVERGED, H3D_ERR_STATE, \
    H3D_ERR_SINGULAR = range(8)
FIELD_U, FIELD_F, FIELD_R, FIELD_STENCIL, FIELD_CHI, FIELD_SOLUTION = range(6)
COARSE_EXACT, COARSE_PROJECT = 0, 1
PIN_IDENTITY, PIN_GALERKIN = 0, 1
PREC_REFINE, PREC_FP32, PREC_MIXED, PREC_MIXED_TC = 0, 1, 2, 3
NUM_SHAPES = 4  # launch shapes per kernel family the autotuner searches (H3D_NUM_SHAPES)
STENCIL_FP16, STENCIL_FP32 = 0, 1
SYMMETRY = {"reflect3": 0, "reflect6": 1, "rotate3": 2}

_STATUS = {0: "ok", 1: "invalid argument", 2: "CUDA error", 3: "out of device memory", 4: "not converged",
           5: "diverged", 6: "call order", 7: "singular coarsest matrix"}


class H3DError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("h3d error %d (%s): %s" % (code, _STATUS.get(code, "?"), msg))
        self.code = code


class Config(ctypes.Structure):
    _fields_ = [("reso", ctypes.c_int * 3), ("youngs_modulus", ctypes.c_double),
                ("poisson_ratio", ctypes.c_double), ("coarse_mode", ctypes.c_int), ("pin_mode", ctypes.c_int),
                ("precision", ctypes.c_int), ("device", ctypes.c_int), ("stencil_precision", ctypes.c_int)]


class SolveStats(ctypes.Structure):
    _fields_ = [("vcycles", ctypes.c_int), ("status", ctypes.c_int), ("rel_res", ctypes.c_double * 6),
                ("solve_ms", ctypes.c_double), ("refinements", ctypes.c_int)]

    def as_dict(self):
        return {"vcycles": self.vcycles, "status": self.status, "rel_res": list(self.rel_res),
                "solve_ms": self.solve_ms, "refinements": self.refinements}


class DesignParams(ctypes.Structure):
    """h3d_design_params: the update after a solve (h3d_design_step)"""
    _fields_ = [("penal", ctypes.c_float), ("sym", ctypes.c_int), ("filter_radius", ctypes.c_float),
                ("filter_periodic", ctypes.c_int), ("volratio", ctypes.c_float), ("min_rho", ctypes.c_float),
                ("step_limit", ctypes.c_float), ("damp", ctypes.c_float)]


_lib = None
_vp, _ip, _dp, _fp = ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double), \
    ctypes.POINTER(ctypes.c_float)

_SIGS = {
    "h3d_create": [ctypes.POINTER(Config), ctypes.POINTER(ctypes.c_void_p)],
    "h3d_destroy": [_vp],
    "h3d_sync": [_vp],
    "h3d_num_levels": [_vp],
    "h3d_level_dims": [_vp, ctypes.c_int, _ip, _ip],
    "h3d_element_matrix": [_vp, _dp],
    "h3d_update_density": [_vp, _vp, ctypes.c_int],
    "h3d_update_stencils": [_vp],
    "h3d_restrict_stencil": [_vp, ctypes.c_int],
    "h3d_factor_coarsest": [_vp],
    "h3d_enforce_unit_macro_strain": [_vp],
    "h3d_gs_relaxation": [_vp, ctypes.c_int, ctypes.c_float, ctypes.c_int],
    "h3d_update_residual": [_vp, ctypes.c_int],
    "h3d_restrict_residual": [_vp, ctypes.c_int],
    "h3d_prolongate_correction": [_vp, ctypes.c_int],
    "h3d_coarse_solve": [_vp],
    "h3d_reset_displacement": [_vp, ctypes.c_int],
    "h3d_field_norms": [_vp, ctypes.c_int, _dp],
    "h3d_field_norms_static": [_vp, ctypes.c_int, _dp],
    "h3d_v_cycle": [_vp, ctypes.c_float, ctypes.c_int, ctypes.c_int],
    "h3d_solve": [_vp, ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.POINTER(SolveStats)],
    "h3d_elastic_matrix": [_vp, ctypes.c_double, _dp, ctypes.POINTER(SolveStats)],
    "h3d_sensitivity": [_vp, _fp, _vp, ctypes.c_int],
    "h3d_reset_solutions": [_vp],
    "h3d_autotune": [_vp],
    "h3d_get_tuning": [_vp, ctypes.c_int, _ip],
    "h3d_set_tuning": [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_int],
    "h3d_set_vcycle_bottom": [_vp, ctypes.c_int64],
    "h3d_batch_update_density": [ctypes.POINTER(_vp), ctypes.POINTER(_vp), ctypes.c_int],
    "h3d_batch_elastic_matrix": [ctypes.POINTER(_vp), ctypes.c_int, ctypes.c_double, _dp,
                                 ctypes.POINTER(SolveStats), _ip],
    "h3d_lockstep_create": [ctypes.POINTER(_vp), ctypes.c_int, ctypes.POINTER(_vp)],
    "h3d_lockstep_create_groups": [ctypes.POINTER(_vp), ctypes.c_int, ctypes.c_int, ctypes.POINTER(_vp)],
    "h3d_lockstep_elastic_matrix": [_vp, ctypes.c_double, _dp, ctypes.POINTER(SolveStats), _ip],
    "h3d_lockstep_destroy": [_vp],
    "h3d_lockstep_set_shapes": [_vp, ctypes.c_int, ctypes.c_int],
    "h3d_lockstep_autotune": [_vp],
    "h3d_penalize": [_vp, _vp, _vp, ctypes.c_int64, ctypes.c_float],
    "h3d_penalize_backward": [_vp, _vp, _vp, ctypes.c_int64, ctypes.c_float],
    "h3d_oc_update": [_vp, _vp, _vp, ctypes.c_int64, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                      ctypes.c_float],
    "h3d_oc_filter": [_vp, _vp, _vp, _ip, ctypes.c_int, ctypes.c_float, ctypes.c_int],
    "h3d_symmetrize": [_vp, _vp, _ip, ctypes.c_int],
    "h3d_design_step": [_vp, _fp, _vp, _vp, ctypes.POINTER(DesignParams)],
    "h3d_conv_radial": [_vp, _vp, _vp, _ip, ctypes.c_float, ctypes.c_int, ctypes.c_int],
    "h3d_init_density_trig": [_vp, _vp, _ip, ctypes.c_int, _fp, ctypes.c_int, ctypes.c_int, ctypes.c_float,
                              ctypes.c_int],
    "h3d_get_field": [_vp, ctypes.c_int, ctypes.c_int, _fp],
    "h3d_set_field": [_vp, ctypes.c_int, ctypes.c_int, _fp],
    "h3d_mma_create": [ctypes.c_int, ctypes.c_int64, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                       ctypes.c_double, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)],
    "h3d_mma_destroy": [_vp],
    "h3d_mma_set_bounds": [_vp, _vp, _vp],
    "h3d_mma_set_bounds_scalar": [_vp, ctypes.c_float, ctypes.c_float],
    "h3d_mma_update": [_vp, ctypes.c_int, _vp, _vp, _vp, ctypes.POINTER(ctypes.c_void_p), _ip],
    "h3d_warmnet_create": [ctypes.c_int, ctypes.c_int, ctypes.c_uint64, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)],
    "h3d_warmnet_destroy": [_vp],
    "h3d_warmnet_num_params": [_vp, ctypes.POINTER(ctypes.c_int64)],
    "h3d_warmnet_get_params": [_vp, _fp],
    "h3d_warmnet_set_params": [_vp, _fp],
    "h3d_warmnet_get_grads": [_vp, _fp],
    "h3d_warmnet_forward": [_vp, _vp, ctypes.c_int, _vp],
    "h3d_warmnet_gradients": [_vp, _vp, _vp, ctypes.c_int, _dp],
    "h3d_warmnet_train_step": [_vp, _vp, _vp, ctypes.c_int, ctypes.c_float, _dp],
    "h3d_warm_start_learned": [_vp, _vp],
}


def lib():
    """The loaded libh3d.so; raises ImportError when it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError("libh3d.so is not built (run __graft_entry__.build() or homo3d_b200/build.py)")
        L = ctypes.CDLL(LIB_PATH)
        for name, args in _SIGS.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = ctypes.c_int
        L.h3d_last_error.argtypes = [_vp]
        L.h3d_last_error.restype = ctypes.c_char_p
        L.h3d_stream.argtypes = [_vp]
        L.h3d_stream.restype = ctypes.c_void_p
        L.h3d_mma_last_error.argtypes = [_vp]
        L.h3d_mma_last_error.restype = ctypes.c_char_p
        L.h3d_warmnet_last_error.argtypes = [_vp]
        L.h3d_warmnet_last_error.restype = ctypes.c_char_p
        L.h3d_lockstep_last_error.argtypes = [_vp]
        L.h3d_lockstep_last_error.restype = ctypes.c_char_p
        _lib = L
    return _lib


def _ptr(x, need=0, what="buffer"):
    """device address of a CUDA tensor (or an int address, taken as is); need > 0:
    the float32 elements the library will read or write through it (the C-ABI
    cannot check a buffer's size, so a short tensor is refused here)"""
    if x is None:
        return None
    if isinstance(x, int):
        return ctypes.c_void_p(x)
    if hasattr(x, "data_ptr"):
        if not x.is_cuda:
            raise ValueError("expected a CUDA tensor")
        if not x.is_contiguous():
            raise ValueError("expected a contiguous tensor")
        if need:
            if x.element_size() != 4 or not x.is_floating_point():
                raise ValueError("%s: expected a float32 tensor" % what)
            if x.numel() < need:
                raise ValueError("%s holds %d values; %d are needed" % (what, x.numel(), need))
        # the handle's stream does not wait on torch's: finish the tensor's producers first
        import torch
        torch.cuda.current_stream(x.device).synchronize()
        return ctypes.c_void_p(x.data_ptr())
    raise TypeError("expected a CUDA tensor or a device pointer")


def _i3(v):
    return (ctypes.c_int * 3)(*[int(a) for a in v])


def _extent(dims, pitch=-1):
    """elements a lexicographic cell field of dims spans with row pitch `pitch`
    (the x extent when negative): the last cell's index + 1"""
    n0, n1, n2 = (int(a) for a in dims)
    p = n0 if pitch is None or int(pitch) < 0 else int(pitch)
    return (n0 - 1) + p * ((n1 - 1) + n1 * (n2 - 1)) + 1


def reference_resolution(reso):
    """The resolution the reference rounds a requested size to (grid.cpp:21-66)."""
    import math
    out = []
    for r in reso:
        l2 = math.log2(r)
        lcl = max(math.floor(l2) - 2, 0)
        out.append(int(math.ceil(2 ** (l2 - lcl)) * 2 ** lcl))
    return tuple(out)


class _Handle:
    def __init__(self, reso, E=10.0, nu=0.3, coarse_mode=COARSE_EXACT, pin_mode=PIN_IDENTITY,
                 precision=PREC_REFINE, device=0, stencil=STENCIL_FP16):
        L = lib()
        if isinstance(reso, int):
            reso = (reso, reso, reso)
        cfg = Config((ctypes.c_int * 3)(*reso), float(E), float(nu), int(coarse_mode), int(pin_mode),
                     int(precision), int(device), int(stencil))
        self.precision = precision
        self.stencil = stencil
        h = ctypes.c_void_p()
        code = L.h3d_create(ctypes.byref(cfg), ctypes.byref(h))
        if code != H3D_OK:
            raise H3DError(code, "h3d_create failed for resolution %r" % (tuple(reso),))
        self._h = h
        self.nlevels = L.h3d_num_levels(h)
        self.dims, self.ratios = [], []
        for l in range(self.nlevels):
            d, r = (ctypes.c_int * 3)(), (ctypes.c_int * 3)()
            L.h3d_level_dims(h, l, d, r)
            self.dims.append(tuple(d))
            self.ratios.append(tuple(r))

    def check(self, code):
        if code != H3D_OK:
            raise H3DError(code, lib().h3d_last_error(self._h).decode())
        return code

    def close(self):
        if getattr(self, "_h", None):
            lib().h3d_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def sync(self):
        self.check(lib().h3d_sync(self._h))

    @property
    def stream(self):
        return lib().h3d_stream(self._h)

    def nv(self, level=0):
        d = self.dims[level]
        return d[0] * d[1] * d[2]


class Grid:
    """One multigrid level of a handle (grid.h:104-418); all six cases at once."""

    def __init__(self, handle, level):
        self._hd, self.level = handle, level
        self.cellReso = handle.dims[level]
        self.upCoarse = handle.ratios[level]
        self.is_root = level == 0

    def _c(self, code):
        return self._hd.check(code)

    def gs_relaxation(self, w_SOR=1.0, times=1):
        self._c(lib().h3d_gs_relaxation(self._hd._h, self.level, w_SOR, times))

    def update_residual(self):
        self._c(lib().h3d_update_residual(self._hd._h, self.level))

    def restrict_residual(self):
        self._c(lib().h3d_restrict_residual(self._hd._h, self.level))

    def prolongate_correction(self):
        self._c(lib().h3d_prolongate_correction(self._hd._h, self.level))

    def solveHostEquation(self):
        self._c(lib().h3d_coarse_solve(self._hd._h))

    def enforce_unit_macro_strain(self, istrain=None):
        """Right-hand sides of all six unit strains (istrain is accepted for parity)."""
        self._c(lib().h3d_enforce_unit_macro_strain(self._hd._h))

    def reset_displacement(self):
        self._c(lib().h3d_reset_displacement(self._hd._h, self.level))

    def restrict_stencil(self):
        self._c(lib().h3d_restrict_stencil(self._hd._h, self.level))

    def assembleHostMatrix(self):
        self._c(lib().h3d_factor_coarsest(self._hd._h))

    def get(self, field):
        """Host copy of a field: [6, nv, 3] float32 (stencil: [nv, 27, 9])."""
        nv = self._hd.nv(self.level)
        out = np.empty((nv, 27, 9) if field == FIELD_STENCIL else (6, nv, 3), dtype=np.float32)
        self._c(lib().h3d_get_field(self._hd._h, self.level, field, out.ctypes.data_as(_fp)))
        return out

    def set(self, field, values):
        a = np.ascontiguousarray(values, dtype=np.float32)
        nv = self._hd.nv(self.level)
        if a.size != nv * (243 if field == FIELD_STENCIL else 18):
            raise ValueError("wrong field size")
        self._c(lib().h3d_set_field(self._hd._h, self.level, field, a.ctypes.data_as(_fp)))


class MG:
    """Multigrid driver over a handle's levels (MG.h:14-45)."""

    def __init__(self, handle):
        self._hd = handle
        self.grids = [Grid(handle, l) for l in range(handle.nlevels)]

    def v_cycle(self, w_SOR=1.0, pre=1, post=1):
        self._hd.check(lib().h3d_v_cycle(self._hd._h, w_SOR, pre, post))

    def solveEquation(self, tol=1e-2, with_guess=True, case_mask=63):
        st = SolveStats()
        code = lib().h3d_solve(self._hd._h, case_mask, tol, int(with_guess), ctypes.byref(st))
        if code not in (H3D_OK, H3D_NOT_CONVERGED):
            self._hd.check(code)
        return st.as_dict()

    def updateStencils(self):
        self._hd.check(lib().h3d_update_stencils(self._hd._h))

    def reset_displacement(self):
        self._hd.check(lib().h3d_reset_displacement(self._hd._h, -1))

    def getRootGrid(self):
        return self.grids[0]


class Homogenization(_Handle):
    """Homogenized elastic tensor of a periodic unit cell (homogenization.h:17-61)."""

    def __init__(self, reso, E=10.0, nu=0.3, coarse_mode=COARSE_EXACT, pin_mode=PIN_IDENTITY,
                 precision=PREC_REFINE, device=0, stencil=STENCIL_FP16):
        super().__init__(reso, E, nu, coarse_mode, pin_mode, precision, device, stencil)
        self.mg = MG(self)
        self.grid = self.mg.grids[0]
        self.last_stats = None

    def getGrid(self):
        return self.grid

    def element_matrix(self):
        ke = np.zeros(576)
        self.check(lib().h3d_element_matrix(self._h, ke.ctypes.data_as(_dp)))
        return ke.reshape(24, 24)

    def update(self, rho_phys, pitchT=-1):
        """rho_phys: CUDA tensor of the physical (penalised) density, lexicographic on
        the handle's grid (dims[0]: the reference's rounding of the requested size)."""
        need = _extent(self.dims[0], pitchT)
        self.check(lib().h3d_update_density(self._h, _ptr(rho_phys, need, "density"), int(pitchT)))

    def elasticMatrix(self, tol=1e-2):
        C = np.zeros(36)
        st = SolveStats()
        code = lib().h3d_elastic_matrix(self._h, float(tol), C.ctypes.data_as(_dp), ctypes.byref(st))
        self.last_stats = st.as_dict()
        if code not in (H3D_OK, H3D_NOT_CONVERGED):
            self.check(code)
        return C.reshape(6, 6)

    def Sensitivity(self, dC, sens, pitchT=-1):
        d = np.ascontiguousarray(dC, dtype=np.float32).reshape(36)
        self.check(lib().h3d_sensitivity(self._h, d.ctypes.data_as(_fp),
                                         _ptr(sens, _extent(self.dims[0], pitchT), "sensitivity"), int(pitchT)))
        self.sync()  # the caller's buffer is read on other streams

    def reset_solutions(self):
        self.check(lib().h3d_reset_solutions(self._h))

    def autotune(self):
        """time the launch shapes of every level now and keep the fastest"""
        self.check(lib().h3d_autotune(self._h))
        return self.tuning()

    def tuning(self):
        """[(sweep shape, residual shape)] per level"""
        out = []
        for l in range(self.nlevels):
            sh = (ctypes.c_int * 2)()
            self.check(lib().h3d_get_tuning(self._h, l, sh))
            out.append((sh[0], sh[1]))
        return out

    def set_vcycle_bottom(self, max_level_vertices):
        """levels of at most this many vertices run in one cooperative launch (0: off)"""
        self.check(lib().h3d_set_vcycle_bottom(self._h, int(max_level_vertices)))

    def set_tuning(self, level, gs_shape, res_shape=0):
        self.check(lib().h3d_set_tuning(self._h, int(level), int(gs_shape), int(res_shape)))

    def design_step(self, dC, rho, sens, volratio, penal=3.0, sym="reflect6", filter_radius=2.0, periodic=False,
                    min_rho=1e-3, step_limit=0.05, damp=0.5):
        """One OC design update after a solve, as one captured graph on the device
        (h3d_design_step): sens = dObj/drho from dC through rho^penal, symmetrised,
        filtered; rho updated by OC and symmetrised.  rho, sens: CUDA tensors."""
        d = np.ascontiguousarray(dC, dtype=np.float32).reshape(36)
        prm = DesignParams(float(penal), SYMMETRY[sym] if sym else -1, float(filter_radius), int(periodic),
                           float(volratio), float(min_rho), float(step_limit), float(damp))
        ne = _extent(self.dims[0])
        self.check(lib().h3d_design_step(self._h, d.ctypes.data_as(_fp), _ptr(rho, ne, "rho"),
                                         _ptr(sens, ne, "sensitivity"), ctypes.byref(prm)))

    def init_density_trig(self, rho, n_period=10, vol=0.3, sym="reflect6", centered=False, coeff=None, seed=0):
        """the reference's trig-basis initial density (randTri, Framework.cuh:238-310)
        into the CUDA tensor rho (the handle's grid); coefficients drawn uniformly in
        [-1, 1) from SplitMix64(seed) unless given"""
        from .density import trig_init_coefficients
        if coeff is None:
            coeff = trig_init_coefficients(n_period, seed, centered)
        c = np.ascontiguousarray(coeff, dtype=np.float32)
        self.check(lib().h3d_init_density_trig(self._h, _ptr(rho, _extent(self.dims[0]), "rho"), _i3(self.dims[0]),
                                               int(n_period),
                                               c.ctypes.data_as(_fp), c.size, int(centered), float(vol),
                                               SYMMETRY[sym] if sym else -1))
        return c

    def conv_radial(self, x, out, radius, periodic=False, adjoint=False):
        """out = rho.conv(radial_convker_t<Spline4>(radius)) of the reference's
        expression layer (or its transpose), on the handle's grid; CUDA tensors"""
        ne = _extent(self.dims[0])
        self.check(lib().h3d_conv_radial(self._h, _ptr(x, ne, "input"), _ptr(out, ne, "output"), _i3(self.dims[0]),
                                         float(radius),
                                         int(periodic), int(adjoint)))

    def warm_start_learned(self, net):
        """stored solutions from a WarmNet's prediction for the current density"""
        self.check(lib().h3d_warm_start_learned(self._h, net._h))

    def penalize(self, rho, rho_phys, p=3.0):
        """rho_phys = rho^p on the handle's stream (the reference's rho.pow(3))."""
        self.check(lib().h3d_penalize(self._h, _ptr(rho, rho.numel(), "rho"), _ptr(rho_phys, rho.numel(), "rho_phys"),
                                      rho.numel(), float(p)))

    def penalize_backward(self, rho, grad, p=3.0):
        """grad *= p rho^(p-1)."""
        self.check(lib().h3d_penalize_backward(self._h, _ptr(rho, rho.numel(), "rho"),
                                               _ptr(grad, rho.numel(), "gradient"), rho.numel(), float(p)))
        self.sync()

    def field_norms(self, field):
        out = np.zeros(6)
        self.check(lib().h3d_field_norms(self._h, field, out.ctypes.data_as(_dp)))
        return out

    def field_norms_static(self, field):
        """field_norms of U, F or R with the reduction scratch in a fixed per-device
        array (no reference counterpart; calls on one device must not overlap)"""
        out = np.zeros(6)
        self.check(lib().h3d_field_norms_static(self._h, field, out.ctypes.data_as(_dp)))
        return out


class OCOptimizer:
    """Optimality-criteria update and sensitivity filter (OCOptimizer.h:16-19)."""

    def __init__(self, ne, min_density=1e-3, stepLimit=0.02, dampExponent=0.5, handle=None):
        self.ne, self.minRho, self.step_limit, self.damp = int(ne), min_density, stepLimit, dampExponent
        self._hd = handle

    def _handle(self):
        if self._hd is None:
            raise ValueError("OCOptimizer needs the Homogenization handle whose stream it runs on")
        return self._hd

    def update(self, sens, rho, volratio):
        hd = self._handle()
        hd.check(lib().h3d_oc_update(hd._h, _ptr(sens, self.ne, "sensitivity"), _ptr(rho, self.ne, "rho"), self.ne,
                                     volratio, self.minRho,
                                     self.step_limit, self.damp))
        hd.sync()

    def filterSens(self, sens, rho, pitchT, reso, radius=2.0, periodic=False):
        hd = self._handle()
        ne = _extent(reso, pitchT)
        hd.check(lib().h3d_oc_filter(hd._h, _ptr(sens, ne, "sensitivity"), _ptr(rho, ne, "rho"), _i3(reso),
                                     int(pitchT), radius, int(periodic)))
        hd.sync()


class MMAOptimizer:
    """Method of moving asymptotes (MMAOptimizer, optimization/mmaOptimizer.h:12-36):
    ``MMAOptimizer(nconstrain, nvar, a0, a, c, d)``, ``setBound``, ``update``.  The
    design, objective gradient, constraint values and gradients are float32 CUDA
    tensors; the optimiser keeps its FP64 state on the device."""

    def __init__(self, nconstrain, nvar, a0=1.0, a=0.0, c=1000.0, d=1.0, device=0):
        h = ctypes.c_void_p()
        st = lib().h3d_mma_create(int(nconstrain), int(nvar), a0, a, c, d, int(device), ctypes.byref(h))
        if st != H3D_OK:
            raise H3DError(st, "h3d_mma_create failed (1 <= nconstrain <= 4, nvar >= 1)")
        self._h = h
        self.m, self.n = int(nconstrain), int(nvar)
        self.newton_steps = 0

    def close(self):
        if getattr(self, "_h", None):
            lib().h3d_mma_destroy(self._h)
            self._h = None

    __del__ = close

    def check(self, st):
        if st != H3D_OK:
            raise H3DError(st, lib().h3d_mma_last_error(self._h).decode())

    def setBound(self, xmin, xmax):
        if hasattr(xmin, "data_ptr"):
            self.check(lib().h3d_mma_set_bounds(self._h, _ptr(xmin, self.n, "xmin"), _ptr(xmax, self.n, "xmax")))
        else:
            self.check(lib().h3d_mma_set_bounds_scalar(self._h, float(xmin), float(xmax)))

    def update(self, itn, x, dfdx, gval, dgdx):
        """x is replaced in place by the new design; dgdx is a sequence of m tensors"""
        if len(dgdx) != self.m:
            raise ValueError("dgdx needs one gradient per constraint")
        ptrs = (ctypes.c_void_p * self.m)(*[_ptr(g, self.n, "constraint gradient").value for g in dgdx])
        steps = ctypes.c_int(0)
        self.check(lib().h3d_mma_update(self._h, int(itn), _ptr(x, self.n, "design"), _ptr(dfdx, self.n, "gradient"),
                                        _ptr(gval, self.m, "constraint values"), ptrs, ctypes.byref(steps)))
        self.newton_steps = steps.value


class WarmNet:
    """Learned warm start (no reference counterpart): a periodic 3-D conv
    encoder-decoder from the density averaged to ``reso``^3 cells to chi / N at the
    ``reso``^3 coarse vertices, with hand-written CUDA forward, backward and Adam.
    Inputs are float32 CUDA tensors [batch, reso^3]; outputs [batch, 18, reso^3]."""

    NOUT = 18

    def __init__(self, reso=32, max_batch=8, seed=0, device=0):
        h = ctypes.c_void_p()
        st = lib().h3d_warmnet_create(int(reso), int(max_batch), int(seed), int(device), ctypes.byref(h))
        if st != H3D_OK:
            raise H3DError(st, "h3d_warmnet_create failed (reso: multiple of 8 in 8..128, max_batch 1..64)")
        self._h, self.reso, self.max_batch = h, int(reso), int(max_batch)
        n = ctypes.c_int64()
        self.check(lib().h3d_warmnet_num_params(self._h, ctypes.byref(n)))
        self.num_params = n.value

    def close(self):
        if getattr(self, "_h", None):
            lib().h3d_warmnet_destroy(self._h)
            self._h = None

    __del__ = close

    def check(self, st):
        if st != H3D_OK:
            raise H3DError(st, lib().h3d_warmnet_last_error(self._h).decode())

    def params(self):
        out = np.empty(self.num_params, np.float32)
        self.check(lib().h3d_warmnet_get_params(self._h, out.ctypes.data_as(_fp)))
        return out

    def set_params(self, p):
        a = np.ascontiguousarray(p, np.float32)
        if a.size != self.num_params:
            raise ValueError("expected %d parameters" % self.num_params)
        self.check(lib().h3d_warmnet_set_params(self._h, a.ctypes.data_as(_fp)))

    def grads(self):
        out = np.empty(self.num_params, np.float32)
        self.check(lib().h3d_warmnet_get_grads(self._h, out.ctypes.data_as(_fp)))
        return out

    def forward(self, x):
        import torch
        b = x.shape[0]
        y = torch.empty((b, self.NOUT, self.reso ** 3), dtype=torch.float32, device=x.device)
        self.check(lib().h3d_warmnet_forward(self._h, _ptr(x, b * self.reso ** 3, "input"), b, _ptr(y)))
        return y

    def gradients(self, x, t):
        loss = ctypes.c_double()
        b = x.shape[0]
        self.check(lib().h3d_warmnet_gradients(self._h, _ptr(x, b * self.reso ** 3, "input"),
                                               _ptr(t, b * self.NOUT * self.reso ** 3, "target"), b, ctypes.byref(loss)))
        return loss.value

    def train_step(self, x, t, lr=1e-3):
        loss = ctypes.c_double()
        b = x.shape[0]
        self.check(lib().h3d_warmnet_train_step(self._h, _ptr(x, b * self.reso ** 3, "input"),
                                                _ptr(t, b * self.NOUT * self.reso ** 3, "target"), b, float(lr),
                                                ctypes.byref(loss)))
        return loss.value

    def save(self, path):
        self.params().tofile(path)

    def load(self, path):
        self.set_params(np.fromfile(path, dtype=np.float32))


def _handle_array(homs):
    arr = (_vp * len(homs))(*[h._h for h in homs])
    return arr


def batch_update(homs, rho_phys):
    """Homogenization.update on several designs, their stencil assemblies running
    concurrently; rho_phys: one contiguous CUDA tensor per design."""
    if len(homs) != len(rho_phys):
        raise ValueError("one density per design")
    ptrs = (_vp * len(homs))(*[_ptr(r, _extent(h.dims[0]), "density of design %d" % i).value
                               for i, (h, r) in enumerate(zip(homs, rho_phys))])
    code = lib().h3d_batch_update_density(_handle_array(homs), ptrs, len(homs))
    if code != H3D_OK:
        for h in homs:
            msg = lib().h3d_last_error(h._h).decode()
            if msg:
                raise H3DError(code, msg)
        raise H3DError(code, "batch update failed")


def batch_elasticMatrix(homs, tol=1e-2):
    """Homogenization.elasticMatrix on several designs solved together (each on its
    own stream).  Returns the [n, 6, 6] C; each design's solve statistics land in
    its last_stats.  A design that fails raises after all have been attempted."""
    n = len(homs)
    C = np.zeros((n, 36))
    st = (SolveStats * n)()
    status = np.zeros(n, dtype=np.int32)
    status[:] = -1
    code = lib().h3d_batch_elastic_matrix(_handle_array(homs), n, float(tol), C.ctypes.data_as(_dp), st,
                                          status.ctypes.data_as(_ip))
    if code not in (H3D_OK, H3D_NOT_CONVERGED) and (status == -1).any():  # refused before any design ran
        raise H3DError(code, lib().h3d_last_error(homs[0]._h).decode() if n else "")
    for i, h in enumerate(homs):
        h.last_stats = st[i].as_dict()
    for i, h in enumerate(homs):
        if status[i] not in (H3D_OK, H3D_NOT_CONVERGED):
            raise H3DError(int(status[i]), "design %d: %s" % (i, lib().h3d_last_error(h._h).decode()))
    return C.reshape(n, 6, 6)


class Lockstep:
    """Designs solved in lockstep: one launch per V-cycle step over all of them and
    one captured graph per batch V-cycle (h3d_lockstep_*).  The handles must be
    H3D_PREC_FP32 designs on one GPU with the same material, stencil precision and
    coarse mode (resolutions below 512); close the batch before its handles."""

    def __init__(self, homs, groups=None):
        """groups: parallel branches of the batch graph (None: the library's default)"""
        self.homs = list(homs)
        b = _vp()
        if groups is None:
            code = lib().h3d_lockstep_create(_handle_array(self.homs), len(self.homs), ctypes.byref(b))
        else:
            code = lib().h3d_lockstep_create_groups(_handle_array(self.homs), len(self.homs), int(groups),
                                                    ctypes.byref(b))
        if code != H3D_OK:
            msg = lib().h3d_last_error(self.homs[0]._h).decode() if self.homs else ""
            raise H3DError(code, msg or "h3d_lockstep_create failed")
        self._b = b

    def elasticMatrix(self, tol=1e-2):
        """batch_elasticMatrix over the batch's designs; returns the [n, 6, 6] C and
        sets each design's last_stats"""
        if getattr(self, "_b", None) is None:
            raise ValueError("the lockstep batch is closed")
        if any(getattr(h, "_h", None) is None for h in self.homs):
            raise ValueError("a handle of the lockstep batch has been closed")
        n = len(self.homs)
        C = np.zeros((n, 36))
        st = (SolveStats * n)()
        status = np.full(n, -1, dtype=np.int32)
        code = lib().h3d_lockstep_elastic_matrix(self._b, float(tol), C.ctypes.data_as(_dp), st,
                                                 status.ctypes.data_as(_ip))
        if code not in (H3D_OK, H3D_NOT_CONVERGED) and (status == -1).any():
            raise H3DError(code, lib().h3d_lockstep_last_error(self._b).decode())
        for i, h in enumerate(self.homs):
            h.last_stats = st[i].as_dict()
        for i, h in enumerate(self.homs):
            if status[i] not in (H3D_OK, H3D_NOT_CONVERGED):
                raise H3DError(int(status[i]), "design %d: %s" % (i, lib().h3d_last_error(h._h).decode()))
        return C.reshape(n, 6, 6)

    def autotune(self):
        """time both launch shapes of every group and level on scratch fields, keep the faster"""
        code = lib().h3d_lockstep_autotune(self._b)
        if code != H3D_OK:
            raise H3DError(code, lib().h3d_lockstep_last_error(self._b).decode())

    def set_shapes(self, fine_shape, coarse_shape):
        """force the sweeps' launch shapes (0 or 1; 0 and 0 by default)"""
        code = lib().h3d_lockstep_set_shapes(self._b, int(fine_shape), int(coarse_shape))
        if code != H3D_OK:
            raise H3DError(code, lib().h3d_lockstep_last_error(self._b).decode())

    def close(self):
        if getattr(self, "_b", None):
            lib().h3d_lockstep_destroy(self._b)
            self._b = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def symmetrize(handle, field, reso, sym="reflect6"):
    """Orbit-average a lexicographic CUDA field in place (TensorExpression.h:425-445)."""
    handle.check(lib().h3d_symmetrize(handle._h, _ptr(field, _extent(reso), "field"), _i3(reso), SYMMETRY[sym]))
    handle.sync()
