"""The learned warm start: training pairs from the solver, training, and the
V-cycle comparison against the plain start.  No reference counterpart (the
reference starts each design from the previous design's solutions).

Pairs: the density rho_phys averaged to R^3 cells (network input) and the
converged solutions chi at the R^3 coarse vertices (every (n/R)-th vertex, mean
removed, divided by n; 18 channels = case x component) (target).  They come from
OC trajectories (`optimize_bulk`, one pair per solve) of seeded trig-basis
designs, so the training densities look like the ones the solver meets.

    python -m homo3d_b200.warmnet --reso 64 --net-reso 32 --seeds 0-31 --iters 20 \\
        --steps 3000 --out warmnet_r32.bin
"""
import argparse
import json
import time

import numpy as np

from . import FIELD_CHI, STENCIL_FP16, STENCIL_FP32, H3DError, Homogenization, WarmNet
from .density import synthetic_density
from .optimize import optimize_bulk


def pooled_density(rho_phys, n, R):
    """mean of the n^3 lexicographic cells over each of the R^3 coarse cells"""
    s = n // R
    r = np.asarray(rho_phys, np.float64).reshape(R, s, R, s, R, s)
    return r.mean(axis=(1, 3, 5)).reshape(-1).astype(np.float32)


def coarse_target(chi, n, R):
    """chi [6, n^3, 3] (lexicographic vertices) -> [18, R^3] at every (n/R)-th
    vertex, per-channel mean removed, divided by n"""
    s = n // R
    c = np.asarray(chi, np.float64).reshape(6, n, n, n, 3)[:, ::s, ::s, ::s, :]
    c = np.transpose(c, (0, 4, 1, 2, 3)).reshape(18, R ** 3)
    c -= c.mean(axis=1, keepdims=True)
    return (c / n).astype(np.float32)


def solver_pairs(n, R, seeds, iters=20, relthres=1e-3, vol_range=(0.1, 0.5), device=0):
    """(x [P, R^3], t [P, 18, R^3]) from OC trajectories of the given seeds"""
    xs, ts = [], []

    def record(hom, rhop):
        xs.append(pooled_density(rhop.cpu().numpy(), n, R))
        ts.append(coarse_target(hom.grid.get(FIELD_CHI), n, R))

    skipped = []
    for seed in seeds:
        vol = float(np.random.default_rng(10007 + seed).uniform(*vol_range))
        try:
            optimize_bulk(n, vol=vol, iters=iters, seed=seed, relthres=relthres, device=device, on_solve=record)
        except H3DError as e:  # a trajectory whose solve fails keeps the pairs recorded before it
            skipped.append({"seed": seed, "vol": vol, "error": str(e)})
    solver_pairs.skipped = skipped
    return np.stack(xs), np.stack(ts)


def train(net, x, t, steps=2000, batch=8, lr=1e-3, seed=0, log_every=0):
    """Adam on random mini-batches, learning rate decaying to lr / 10; returns the
    loss history"""
    import torch
    dev = torch.device("cuda", 0)
    X = torch.tensor(x, device=dev)
    T = torch.tensor(t, device=dev)
    rng = np.random.default_rng(seed)
    hist = []
    for s in range(steps):
        idx = torch.tensor(rng.choice(len(X), size=min(batch, len(X)), replace=False), device=dev)
        loss = net.train_step(X[idx].contiguous(), T[idx].contiguous(), lr * (0.1 ** (s / max(steps, 1))))
        hist.append(loss)
        if log_every and s % log_every == 0:
            print(json.dumps({"step": s, "loss": loss}), flush=True)
    return hist


def compare_starts(net, n, seeds, relthres=1e-5, vol_range=(0.1, 0.5), device=0, stencil=STENCIL_FP16):
    """V-cycles and solve time of the plain zero start and of the learned start on
    fresh designs (trig-basis densities, rho^3); a solve that fails is recorded in
    the row's "error" and left out of the averages"""
    import torch
    out = []
    hd = Homogenization(n, device=device, stencil=stencil)
    for seed in seeds:
        vol = float(np.random.default_rng(20011 + seed).uniform(*vol_range))
        rho = synthetic_density(n, seed=seed, vol=vol).ravel().astype(np.float64)
        rhop = torch.tensor((rho ** 3).astype(np.float32), device="cuda")
        hd.update(rhop)
        row = {"seed": seed, "vol": vol}
        for mode in ("zero", "learned"):
            hd.reset_solutions()
            t0 = time.perf_counter()
            if mode == "learned":
                hd.warm_start_learned(net)
            try:
                C = hd.elasticMatrix(relthres)
            except H3DError as e:
                row["error"] = "%s start: %s" % (mode, e)
                break
            row[mode + "_ms"] = (time.perf_counter() - t0) * 1e3
            row[mode + "_vcycles"] = hd.last_stats["vcycles"]
            row[mode + "_C00"] = float(C[0, 0])
        out.append(row)
    hd.close()
    return out


def _seeds(spec):
    a, _, b = spec.partition("-")
    return list(range(int(a), int(b) + 1)) if b else [int(a)]


def main():
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--reso", type=int, default=64, help="fine grid of the training solves")
    ap.add_argument("--net-reso", type=int, default=32)
    ap.add_argument("--seeds", default="0-31")
    ap.add_argument("--iters", type=int, default=20, help="OC iterations per trajectory")
    ap.add_argument("--steps", type=int, default=3000)
    ap.add_argument("--batch", type=int, default=8)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--eval-reso", default="", help="compare starts at these sizes after training (e.g. 128,256)")
    ap.add_argument("--eval-tols", default="1e-5", help="relative residual thresholds of the compared solves")
    ap.add_argument("--eval-seeds", default="1000-1003")
    ap.add_argument("--stencils", choices=["fp16", "fp32"], default="fp16", help="coarse stencils of the compared solves")
    ap.add_argument("--out", default="")
    args = ap.parse_args()
    t0 = time.perf_counter()
    x, t = solver_pairs(args.reso, args.net_reso, _seeds(args.seeds), iters=args.iters)
    t1 = time.perf_counter()
    net = WarmNet(args.net_reso, max_batch=args.batch, seed=0)
    hist = train(net, x, t, steps=args.steps, batch=args.batch, lr=args.lr, log_every=max(args.steps // 10, 1))
    t2 = time.perf_counter()
    if args.out:
        net.save(args.out)
    rep = {"pairs": int(len(x)), "skipped_trajectories": solver_pairs.skipped, "params": net.num_params,
           "data_s": round(t1 - t0, 1), "train_s": round(t2 - t1, 1), "loss_first": hist[0],
           "loss_last10": float(np.mean(hist[-10:]))}
    if args.eval_reso:
        rep["eval"] = []
        for n in (int(v) for v in args.eval_reso.split(",")):
            for tol in (float(v) for v in args.eval_tols.split(",")):
                allrows = compare_starts(net, n, _seeds(args.eval_seeds), relthres=tol,
                                         stencil=STENCIL_FP32 if args.stencils == "fp32" else STENCIL_FP16)
                rows = [r for r in allrows if "error" not in r]
                rep["eval"].append({
                    "reso": n, "relthres": tol, "stencils": args.stencils, "designs": len(rows),
                    "failed": [r["error"] for r in allrows if "error" in r],
                    "vcycles_zero": float(np.mean([r["zero_vcycles"] for r in rows])),
                    "vcycles_learned": float(np.mean([r["learned_vcycles"] for r in rows])),
                    "ms_zero": float(np.mean([r["zero_ms"] for r in rows])),
                    "ms_learned": float(np.mean([r["learned_ms"] for r in rows])),
                    "max_rel_C00_diff": float(max(abs(r["learned_C00"] - r["zero_C00"]) / abs(r["zero_C00"])
                                                  for r in rows))})
                print(json.dumps(rep["eval"][-1]), flush=True)
    print(json.dumps(rep), flush=True)


if __name__ == "__main__":
    main()
