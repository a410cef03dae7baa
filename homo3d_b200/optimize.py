"""OC design loops on the library's entry points: bulk-modulus maximisation (the
loop of homo3d's optiBulk, homogenization/testAutoDiff.cu:282-331), shear-modulus
maximisation (optiShear, homogenization/testAutoDiff.cu:334-381) and the
negative-Poisson-ratio loop (example_opti_npr, Framework.cu:208-272).

Per iteration: rho_phys = rho^3; update the hierarchy; six solves and C (warm
start from the previous iteration); the objective, bulk
-(C00+C11+C22 + 2(C01+C02+C12))/3, shear -(C33+C44+C55)/3 or npr
C01+C02+C12 - (C00+C11+C22) 0.8^iter;
sensitivities wrt rho_phys, chain rule 3 rho^2; symmetrise; filter; OC update;
symmetrise the density.  Every step runs on the handle's stream.

    python -m homo3d_b200.optimize --reso 128 --iters 50 [--objective npr]
"""
import argparse
import json
import time

import numpy as np

from . import (COARSE_PROJECT, PIN_IDENTITY, PREC_REFINE, STENCIL_FP16, Homogenization, OCOptimizer, symmetrize)
from .density import synthetic_density


def bulk_gradient():
    """d obj / d C of obj = -(C00 + C11 + C22 + 2 (C01 + C02 + C12)) / 3 (upper entries only,
    as the expression Ch(0,1) etc. records them)."""
    dC = np.zeros((6, 6), np.float32)
    for i in range(3):
        dC[i, i] = -1.0 / 3.0
    dC[0, 1] = dC[0, 2] = dC[1, 2] = -2.0 / 3.0
    return dC


def bulk_objective(C):
    return -(C[0, 0] + C[1, 1] + C[2, 2] + 2 * (C[0, 1] + C[0, 2] + C[1, 2])) / 3.0


def shear_objective(C):
    """-(C33 + C44 + C55) / 3 (testAutoDiff.cu:343)"""
    return -(C[3, 3] + C[4, 4] + C[5, 5]) / 3.0


def shear_gradient():
    dC = np.zeros((6, 6), np.float32)
    for i in range(3, 6):
        dC[i, i] = -1.0 / 3.0
    return dC


NPR_BETA = 0.8  # Framework.cu:241


def npr_objective(C, it, beta=NPR_BETA):
    return C[0, 1] + C[0, 2] + C[1, 2] - (C[0, 0] + C[1, 1] + C[2, 2]) * beta ** it


def npr_gradient(it, beta=NPR_BETA):
    """d obj / d C of the npr objective (upper entries, as recorded by Ch(0,1) etc.)"""
    dC = np.zeros((6, 6), np.float32)
    dC[0, 1] = dC[0, 2] = dC[1, 2] = 1.0
    for i in range(3):
        dC[i, i] = -np.float32(beta ** it)
    return dC


OBJECTIVES = {"bulk": (lambda C, it: bulk_objective(C), lambda it: bulk_gradient()),
              "shear": (lambda C, it: shear_objective(C), lambda it: shear_gradient()),
              "npr": (npr_objective, npr_gradient)}


class ConvergeChecker:
    """Stops when the relative objective change stays below thres for three
    consecutive iterations after iteration 11 (Framework.cuh:312-343)."""

    def __init__(self, thres=5e-4, length=10):
        self.thres, self.obj, self.length = thres, [0.0] * length, length

    def is_converge(self, it, obj):
        self.obj[it % self.length] = obj
        if it <= 11:
            return False
        g = lambda k: self.obj[(it - k) % self.length]
        return all(abs(g(i) - g(i + 1)) / abs(g(i + 1)) <= self.thres for i in range(3))


def optimize_bulk(reso, vol=0.3, iters=50, seed=0, relthres=1e-2, filter_radius=2.0, step=0.05, damp=0.5,
                  sym="reflect6", finthres=5e-4, stop_on_converge=False, rho0=None, E=10.0, nu=0.3,
                  coarse_mode=COARSE_PROJECT, pin_mode=PIN_IDENTITY, precision=PREC_REFINE, device=0,
                  on_solve=None, stencil=STENCIL_FP16, objective="bulk", device_step=True):
    """The OC loop of testAutoDiff.cu:282-331 (objective "bulk"), of
    testAutoDiff.cu:334-381 ("shear") or of Framework.cu:208-272 ("npr");
    device_step runs the update after each solve (sensitivity, SIMP backward,
    symmetry, filter, OC, symmetry) as one captured graph (h3d_design_step),
    otherwise as separate entry-point calls; on_solve(hom, rho_phys) is called after every
    solve (e.g. to record training pairs).  The coarsest solve projects out the
    mean of its right-hand side (COARSE_PROJECT, as the reference's null-space
    projection at the coarsest grid does): after a few OC steps the densities reach
    their 1e-3 floor (element stiffness contrast ~1e9), where the exact inverse of
    the pinned coarsest matrix made some designs' V-cycles diverge."""
    obj_fn, grad_fn = OBJECTIVES[objective]
    import torch

    hom = Homogenization(reso, E, nu, coarse_mode, pin_mode, precision, device, stencil)
    n = hom.dims[0]
    ne = n[0] * n[1] * n[2]
    dev = torch.device("cuda", device)
    if rho0 is None:
        rho0 = synthetic_density(n[0], seed=seed, vol=vol).ravel()
    rho = torch.tensor(np.asarray(rho0, dtype=np.float32).ravel(), device=dev)
    rhop = torch.empty_like(rho)
    sens = torch.empty_like(rho)
    oc = OCOptimizer(ne, 1e-3, step, damp, handle=hom)
    stream = torch.cuda.ExternalStream(hom.stream, device=dev)
    checker = ConvergeChecker(finthres)
    records = []
    for it in range(iters):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0 = time.perf_counter()
        e0.record(stream)
        hom.penalize(rho, rhop, 3.0)
        hom.update(rhop)
        C = hom.elasticMatrix(relthres)
        st = hom.last_stats
        if on_solve is not None:
            on_solve(hom, rhop)
        obj = float(obj_fn(C, it))
        done = checker.is_converge(it, obj)
        if device_step:
            hom.design_step(grad_fn(it), rho, sens, vol, 3.0, sym, filter_radius, False, 1e-3, step, damp)
        else:
            hom.Sensitivity(grad_fn(it), sens)
            hom.penalize_backward(rho, sens, 3.0)
            symmetrize(hom, sens, n, sym)
            oc.filterSens(sens, rho, n[0], n, filter_radius)
            oc.update(sens, rho, vol)
            symmetrize(hom, rho, n, sym)
        e1.record(stream)
        e1.synchronize()
        records.append({"iter": it, "obj": obj, "vcycles": st["vcycles"], "solve_ms": st["solve_ms"],
                        "iter_ms": e0.elapsed_time(e1), "wall_ms": (time.perf_counter() - t0) * 1e3,
                        "vol": float(rho.double().mean())})
        if done and stop_on_converge:
            break
    C = hom.elasticMatrix(relthres)
    out = rho.cpu().numpy()
    hom.close()
    return out, C, records


SGM_K, SGM_C = 30.0, 0.5            # .sgm() defaults (TensorExpression.h:555)
ANI_SCALE, VOL_SCALE = 1000.0, 1000.0  # Framework.cu:314, 320


def shear_isotropy_terms(C):
    """(objective, dC of it, anisotropy constraint (2S/D - 1)^2 ANI_SCALE, its dC) of
    example_opti_shear_isotropy (Framework.cu:303-318): S = C33 + C44 + C55,
    D = C00 + C11 + C22 - C01 - C02 - C12 (upper entries, as Ch(0,1) records them)"""
    S = C[3, 3] + C[4, 4] + C[5, 5]
    D = C[0, 0] + C[1, 1] + C[2, 2] - C[0, 1] - C[0, 2] - C[1, 2]
    q = 2 * S / D - 1
    con = q * q * ANI_SCALE
    dS, dD = ANI_SCALE * 2 * q * 2 / D, ANI_SCALE * 2 * q * (-2 * S / (D * D))
    dC = np.zeros((6, 6), np.float32)
    for i in range(3):
        dC[3 + i, 3 + i] = dS
        dC[i, i] = dD
    dC[0, 1] = dC[0, 2] = dC[1, 2] = -dD
    return -S / 3.0, shear_gradient(), con, dC


def optimize_shear_isotropy(reso, vol=0.3, iters=20, seed=0, relthres=1e-2, filter_radius=2.0, sym="reflect6",
                            rho0=None, E=10.0, nu=0.3, device=0, precision=PREC_REFINE):
    """example_opti_shear_isotropy (Framework.cu:274-351): maximise the shear modulus
    -(C33 + C44 + C55) / 3 by MMA (2 constraints; a0 = 1, a = 0, c = 1000, d = 1,
    bounds [0.001, 1]) with the physical density rho_phys = sgm(conv(rho))^3 (radial
    Spline4 convolution of radius filter_radius, sigmoid 1 / (1 + exp(-30 (v - 0.5)))):
    g0 = (mean sgm(conv(rho)) - vol) 1000 with the unscaled, unsymmetrised gradient of
    the mean, g1 = (anisotropy) 1000 - 0.1 with the gradient of the anisotropy
    (symmetrised); the objective gradient symmetrised.  The scalings are the
    reference's."""
    import torch

    from . import MMAOptimizer
    hom = Homogenization(reso, E, nu, COARSE_PROJECT, PIN_IDENTITY, precision, device)
    n = hom.dims[0]
    ne = n[0] * n[1] * n[2]
    dev = torch.device("cuda", device)
    if rho0 is None:
        rho0 = synthetic_density(n[0], seed=seed, vol=vol).ravel()
    rho = torch.tensor(np.asarray(rho0, dtype=np.float32).ravel(), device=dev)
    z, tmp, grad_obj, grad_ani, grad_vol = (torch.empty_like(rho) for _ in range(5))
    sens = torch.empty_like(rho)
    mma = MMAOptimizer(2, ne, 1.0, 0.0, 1000.0, 1.0, device=device)
    mma.setBound(0.001, 1.0)
    stream = torch.cuda.ExternalStream(hom.stream, device=dev)
    records = []
    for it in range(iters):
        with torch.cuda.stream(stream):
            hom.conv_radial(rho, z, filter_radius)
            y = torch.sigmoid(SGM_K * (z - SGM_C))
            rhop = y ** 3
            dphys = 3 * y * y * SGM_K * y * (1 - y)           # d rho_phys / d z
        hom.update(rhop)
        C = hom.elasticMatrix(relthres)
        obj, dC_obj, con, dC_con = shear_isotropy_terms(C)
        for dC, out in ((dC_obj, grad_obj), (dC_con, grad_ani)):
            hom.Sensitivity(dC, sens)
            with torch.cuda.stream(stream):
                torch.mul(sens, dphys, out=tmp)
            hom.conv_radial(tmp, out, filter_radius, adjoint=True)
            symmetrize(hom, out, n, sym)
        with torch.cuda.stream(stream):
            volr = float(y.double().mean())
            torch.mul(SGM_K * y * (1 - y), 1.0 / ne, out=tmp)
        hom.conv_radial(tmp, grad_vol, filter_radius, adjoint=True)
        hom.sync()
        gval = torch.tensor([(volr - vol) * VOL_SCALE, con * ANI_SCALE - 0.1], dtype=torch.float32, device=dev)
        mma.update(it, rho, grad_obj, gval, [grad_vol, grad_ani])
        records.append({"iter": it, "obj": float(obj), "anisotropy": float(con), "vol": volr,
                        "zener": float(np.sqrt(con / ANI_SCALE) + 1), "vcycles": hom.last_stats["vcycles"],
                        "newton": mma.newton_steps})
    out = rho.cpu().numpy()
    mma.close()
    hom.close()
    return out, C, records


def main():
    p = argparse.ArgumentParser()
    p.add_argument("--reso", type=int, default=128)
    p.add_argument("--iters", type=int, default=50)
    p.add_argument("--vol", type=float, default=0.3)
    p.add_argument("--seed", type=int, default=0)
    p.add_argument("--relthres", type=float, default=1e-2)
    p.add_argument("--objective", choices=sorted(OBJECTIVES), default="bulk")
    p.add_argument("--out-density", default="", help="write the final density in the binary voxel format")
    a = p.parse_args()
    rho, C, rec = optimize_bulk(a.reso, a.vol, a.iters, a.seed, a.relthres, objective=a.objective)
    if a.out_density:
        from .voxelio import write_density
        n = round(rho.size ** (1 / 3))
        write_density(a.out_density, rho, (n, n, n))
    print(json.dumps({"final_C": C.tolist(), "iterations": rec}))


if __name__ == "__main__":
    main()
