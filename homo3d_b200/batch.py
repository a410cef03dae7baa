"""Batched designs: many independent unit cells of uneven resolution homogenized
together, in two forms, against the same designs solved one at a time:
  streams  -- each design's V-cycles on its own stream, the host advancing
              whichever design's step has completed (h3d_batch_elastic_matrix);
  lockstep -- all designs step through their V-cycles together, one launch per
              V-cycle step over every design and one captured graph per batch
              V-cycle (h3d_lockstep_*, FP32 designs only).
No reference counterpart: the reference homogenizes one design per process.

Designs: seeded trig-basis densities (the same generator as every other
workload), volume fraction U(0.1, 0.5) per design, physical density rho^3, all
six load cases, zero starting guess.  One "pass" = stencil assembly + the six
solves + C for every design.

    python -m homo3d_b200.batch --sizes 64x8,96x8,128x8 --tol 1e-3 --precision fp32
"""
import argparse
import json
import time

import numpy as np

from . import PREC_FP32, PREC_REFINE, Homogenization, Lockstep, batch_elasticMatrix, batch_update
from .density import synthetic_density


def parse_sizes(spec):
    """'64x8,96x8' -> [64]*8 + [96]*8"""
    out = []
    for part in spec.split(","):
        n, _, k = part.partition("x")
        out += [int(n)] * (int(k) if k else 1)
    return out


def make_designs(sizes, seed0=0, vol_range=(0.1, 0.5)):
    """per design: (n, seed, vol, rho_phys float32 lexicographic)"""
    out = []
    for i, n in enumerate(sizes):
        seed = seed0 + i
        vol = float(np.random.default_rng(30011 + seed).uniform(*vol_range))
        rho = synthetic_density(n, seed=seed, vol=vol).ravel().astype(np.float64)
        out.append((n, seed, vol, (rho ** 3).astype(np.float32)))
    return out


def shard(n_designs, rank, world):
    """round-robin share of the designs for one rank (no exchange between ranks
    until the final gather)"""
    return list(range(rank, n_designs, world))


def gather_designs(dist, n_designs, local_idx, local_rows):
    """rows of every rank's designs in design order, on every rank (one object
    all-gather; None without a process group)"""
    if dist is None:
        out = [None] * n_designs
        for i, r in zip(local_idx, local_rows):
            out[i] = r
        return out
    parts = [None] * dist.get_world_size()
    dist.all_gather_object(parts, list(zip(local_idx, local_rows)))
    out = [None] * n_designs
    for part in parts:
        for i, r in part:
            out[i] = r
    return out


def max_over_ranks(dist, values):
    """elementwise maximum of a list of floats over the ranks"""
    if dist is None:
        return list(values)
    import torch
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor(list(values), dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.cpu()]


def run_pass(torch, homs, rhos, tol, batched, lockstep=None):
    """one pass over all designs from a zero start; returns (seconds, C [n,6,6], stats).
    batched: stencils of all designs together, then the solves on per-design streams
    or, given a Lockstep over the same handles, in lockstep"""
    for hd in homs:
        hd.reset_solutions()
        hd.sync()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    t_update = 0.0
    if batched:
        batch_update(homs, rhos)
        t_update = time.perf_counter() - t0
        C = lockstep.elasticMatrix(tol) if lockstep is not None else batch_elasticMatrix(homs, tol)
    else:
        C = np.zeros((len(homs), 6, 6))
        for i, hd in enumerate(homs):
            t1 = time.perf_counter()
            hd.update(rhos[i])
            t_update += time.perf_counter() - t1
            C[i] = hd.elasticMatrix(tol)
    dt = time.perf_counter() - t0
    return dt, t_update, C, [dict(hd.last_stats) for hd in homs]


def main():
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--sizes", default="64x8,96x8,128x8")
    ap.add_argument("--tol", type=float, default=1e-3)
    ap.add_argument("--precision", choices=["fp32", "refine"], default="fp32")
    ap.add_argument("--repeat", type=int, default=3, help="timed passes per arm (after one untimed)")
    ap.add_argument("--device", type=int, default=0)
    args = ap.parse_args()
    import os

    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    dist = None
    if world > 1:  # one rank per GPU (torchrun); designs shard round-robin
        import datetime

        import torch.distributed as dist
        args.device = int(os.environ.get("LOCAL_RANK", "0"))
        torch.cuda.set_device(args.device)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    torch.cuda.set_device(args.device)
    sizes_all = parse_sizes(args.sizes)
    mine = shard(len(sizes_all), rank, world)
    sizes = [sizes_all[i] for i in mine]
    designs = [make_designs(sizes_all)[i] for i in mine]
    prec = PREC_FP32 if args.precision == "fp32" else PREC_REFINE
    free0 = torch.cuda.mem_get_info()[0]
    homs = [Homogenization(n, precision=prec, device=args.device) for n in sizes]
    rhos = [torch.tensor(r, device="cuda") for _, _, _, r in designs]
    torch.cuda.synchronize()
    mem_gb = (free0 - torch.cuda.mem_get_info()[0]) / 1e9
    res = {}
    arms = [("sequential", False, None), ("batched", True, None)]
    lock = None
    if prec == PREC_FP32:
        lock = Lockstep(homs)  # device tables and the batch V-cycle graph, once
        arms.append(("lockstep", True, lock))
    for arm, batched, ls in arms:
        run_pass(torch, homs, rhos, args.tol, batched, ls)  # graph captures, first-touch
        times, upd, Cs, stats = [], [], None, None
        for _ in range(args.repeat):
            if dist is not None:
                dist.barrier()
            dt, tu, Cs, stats = run_pass(torch, homs, rhos, args.tol, batched, ls)
            dt, tu = max_over_ranks(dist, [dt, tu])  # the job's pass ends with its slowest rank
            times.append(dt)
            upd.append(tu)
        k = int(np.argmin(times))
        Cs = gather_designs(dist, len(sizes_all), mine, [c for c in Cs])
        stats = gather_designs(dist, len(sizes_all), mine, stats)
        res[arm] = {"s_per_pass": times[k], "s_update": upd[k], "s_all": times, "C": Cs, "stats": stats}
    if lock is not None:
        lock.close()
    for hd in homs:
        hd.close()
    if dist is not None:
        dist.destroy_process_group()
    if rank != 0:
        return
    sizes = sizes_all
    seq, bat = res["sequential"], res["batched"]
    rel = [float(np.abs(bat["C"][i] - seq["C"][i]).max() / np.abs(seq["C"][i]).max()) for i in range(len(sizes))]
    rep = {
        "workload": "%d designs (%s), 6 load cases, relthres %g, %s" % (len(sizes), args.sizes, args.tol,
                                                                        args.precision),
        "n_gpus": world,
        "designs_per_s_batched": len(sizes) / bat["s_per_pass"],
        "designs_per_s_sequential": len(sizes) / seq["s_per_pass"],
        "speedup": seq["s_per_pass"] / bat["s_per_pass"],
        "s_per_pass": {"batched": bat["s_per_pass"], "sequential": seq["s_per_pass"]},
        "s_stencils": {"batched": bat["s_update"], "sequential": seq["s_update"]},
        "sum_solve_ms_sequential": sum(s["solve_ms"] for s in seq["stats"]),
        "max_rel_C_diff_batched_vs_sequential": max(rel),
        "vcycles": [s["vcycles"] for s in bat["stats"]],
        "vcycles_equal": [s["vcycles"] for s in bat["stats"]] == [s["vcycles"] for s in seq["stats"]],
        "status": [s["status"] for s in bat["stats"]],
        "device_mem_gb_rank0": round(mem_gb, 2),
    }
    if "lockstep" in res:
        lk = res["lockstep"]
        rep["designs_per_s_lockstep"] = len(sizes) / lk["s_per_pass"]
        rep["s_per_pass"]["lockstep"] = lk["s_per_pass"]
        rep["s_stencils"]["lockstep"] = lk["s_update"]
        rep["lockstep_C_identical_to_sequential"] = all(
            np.array_equal(lk["C"][i], seq["C"][i]) for i in range(len(sizes)))
        rep["lockstep_vcycles_equal"] = [s["vcycles"] for s in lk["stats"]] == [s["vcycles"] for s in seq["stats"]]
    print(json.dumps(rep), flush=True)


if __name__ == "__main__":
    main()
