"""Generates tests/golden/oracle_C.json: the FP64 oracle's homogenized tensor C and a
sensitivity checksum for the seeded trig-basis designs the GPU tests solve at full
size (128^3 at volumes 0.1 / 0.3 / 0.5 and the benchmark design, 256^3 at volume
0.3, seed 0).

The oracle (oracle/h3d_oracle.c, FP64, OpenMP over the host cores) solves each
design to a relative residual of 1e-8 (at most 60 V-cycles; the residual reached
is recorded), then reduces C (homogenization.cu:464-575) and the sensitivities of
the bulk-modulus objective for dC = the objective's gradient
(homogenization.cu:697-948), summarised raw and weighted by the physical density
(in near-void elements the raw sensitivity depends on how far the solve went:
their displacements barely enter the residual).  The densities are rounded to FP32 before the oracle
sees them, as the library receives them.  Each record also holds the V-cycle
count at which the oracle's solve first met relthres 1e-5.

    python tests/golden/make_oracle_fixtures.py [--only 128|256]

Takes about 20 minutes on 8 host cores (the 256^3 solve dominates) and about
15 GB of host memory.  Results are merged into the existing file, one entry per
(reso, vol, seed).
"""
import argparse
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

OUT = os.path.join(HERE, "oracle_C.json")
CASES = [(128, 0.1, 0), (128, 0.3, 0), (128, 0.5, 0), (256, 0.3, 0)]


def bulk_dC():
    """d(bulk)/dC of -(C00+C11+C22+2(C01+C02+C12))/9 (Framework.cu:164-165)"""
    d = np.zeros((6, 6))
    d[:3, :3] = -1.0 / 9.0
    return d


def sens_checksum(s):
    """order-independent summary of a sensitivity field: sum, sum of squares, and the
    sums over the eight octants of the cell (position-sensitive)"""
    n = round(s.size ** (1 / 3))
    a = s.reshape(n, n, n)
    h = n // 2
    octs = [float(a[z * h:(z + 1) * h, y * h:(y + 1) * h, x * h:(x + 1) * h].sum())
            for z in range(2) for y in range(2) for x in range(2)]
    return {"sum": float(s.sum()), "sumsq": float((s * s).sum()), "octants": octs}


def run_case(n, vol, seed, tol=1e-8, maxit=60):
    from oracle import oracle as O
    from homo3d_b200.density import synthetic_density
    rho = (synthetic_density(n, seed=seed, vol=vol).ravel() ** 3).astype(np.float32).astype(np.float64)
    m = O.MG((n, n, n))
    m.set_density(rho)
    t0 = time.perf_counter()
    m.update_stencils()
    m.rhs()
    cycles, hist = m.solve(tol, maxit)
    C = m.elastic_matrix()
    sens = m.sensitivity(bulk_dC())
    secs = time.perf_counter() - t0
    worst = hist.max(axis=1)
    to_1e5 = int(np.argmax(worst <= 1e-5)) + 1 if (worst <= 1e-5).any() else None
    return {"reso": n, "vol": vol, "seed": seed, "tol": tol, "vcycles": int(cycles), "vcycles_to_1e-5": to_1e5,
            "rel_res": [float(x) for x in hist[-1]], "C": [float(x) for x in C.ravel()],
            "sens_bulk": sens_checksum(sens), "sens_bulk_weighted": sens_checksum(rho * sens), "oracle_s": round(secs, 1), "threads": os.cpu_count()}


def main():
    p = argparse.ArgumentParser()
    p.add_argument("--only", type=int, default=0)
    p.add_argument("--vol", type=float, default=0)
    args = p.parse_args()
    data = json.load(open(OUT)) if os.path.exists(OUT) else {"cases": []}
    for n, vol, seed in CASES:
        if (args.only and n != args.only) or (args.vol and abs(vol - args.vol) > 1e-9):
            continue
        r = run_case(n, vol, seed)
        print(json.dumps({k: r[k] for k in ("reso", "vol", "vcycles", "vcycles_to_1e-5", "rel_res", "oracle_s")}),
              flush=True)
        data["cases"] = [c for c in data["cases"] if (c["reso"], c["vol"], c["seed"]) != (n, vol, seed)] + [r]
        data["cases"].sort(key=lambda c: (c["reso"], c["vol"], c["seed"]))
        data["generator"] = "tests/golden/make_oracle_fixtures.py (FP64 oracle, oracle/h3d_oracle.c)"
        with open(OUT, "w") as f:
            json.dump(data, f, indent=1)


if __name__ == "__main__":
    main()
