"""Benchmark: ms per 6-case homogenization solve to relthres 1e-5 at 256^3 on B200.

One step = the forward pass a design iteration needs: load the physical density
(rho^3 of a seeded trig-basis design, volume 0.3, E = 10, nu = 0.3), build the
Galerkin hierarchy and the coarsest inverse, solve the six unit-strain cases from
a zero start to relthres 1e-5, and reduce the 6x6 homogenized tensor C.

  python bench.py [--gpus N --steps K --warmup W] [--impl reference]

N > 1 runs under torchrun as independent replicas (one design per rank, no
collective on the data path): value = total solves / max-over-ranks time.
--impl reference times the FP64 CPU restatement of the same solve (the oracle) on
all host cores at the full grid size: one V-cycle per step, the setup and the C
reduction once (see reference_arm()).
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "ms per 6-case solve to relthres 1e-5 at 256^3"


def metric_name(args):
    if args.reso == 256 and args.tol == 1e-5:
        return METRIC
    return "ms per 6-case solve to relthres %g at %d^3" % (args.tol, args.reso)


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="h3d", choices=["h3d", "reference"])
    p.add_argument("--reso", type=int, default=256)
    p.add_argument("--tol", type=float, default=1e-5)
    p.add_argument("--vol", type=float, default=0.3)
    p.add_argument("--seed", type=int, default=0)
    p.add_argument("--pin-mode", type=int, default=0)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-precision-arms", action="store_true", help="skip the mixed-precision arms of the same step")
    p.add_argument("--workload", default="solve", choices=["solve", "mma", "batch"],
                   help="solve: the homogenization step (default); mma: one MMA design update; "
                        "batch: designs/s of 24 designs of 64^3-128^3 solved together")
    p.add_argument("--mma-m", type=int, default=1, help="constraints of the mma workload")
    p.add_argument("--profile", action="store_true",
                   help="only warm-up and timed steps (no e2e, setup or sweep side measurements), for ncu")
    p.add_argument("--precision", type=int, default=0,
                   help="0 refined (FP64 solution), 1 FP32, 2 refined with an FP32-accumulated refinement "
                        "residual, 3 as 2 with the tensor-core level-0 residual")
    return p.parse_args()


class ClockSampler:
    """SM clocks, power and clock-event (throttle) reasons sampled in the background
    while the timed region runs: through NVML every 20 ms (read-only queries), or,
    without NVML, through nvidia-smi every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    BITS = [0x8, 0x40, 0x20, 0x4]  # NVML clock-event reason masks, in NAMES order

    def __init__(self, index):
        self.index = index
        self.rows = []  # (sm MHz, max sm MHz, set of reason names)
        self._stop = threading.Event()
        self._t = None
        self._nvml = None
        try:
            import pynvml
            pynvml.nvmlInit()
            h = None
            try:
                import torch
                pr = torch.cuda.get_device_properties(index)
                bus = "%08x:%02x:%02x.0" % (pr.pci_domain_id, pr.pci_bus_id, pr.pci_device_id)
                h = pynvml.nvmlDeviceGetHandleByPciBusId(bus)
            except Exception:
                h = pynvml.nvmlDeviceGetHandleByIndex(index)
            self._nvml = (pynvml, h)
        except Exception:
            self._nvml = None

    def _sample_nvml(self):
        nv, h = self._nvml
        sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
        mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
        get = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or nv.nvmlDeviceGetCurrentClocksThrottleReasons
        bits = get(h)
        return float(sm), float(mx), {n for n, b in zip(self.NAMES, self.BITS) if bits & b}

    def _sample_smi(self):
        out = subprocess.run(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.FIELDS,
                              "--format=csv,noheader,nounits"], capture_output=True, text=True,
                             timeout=5).stdout.strip()
        if not out:
            return None
        r = [c.strip() for c in out.split(",")]
        sm = float(r[1]) if r[1].replace(".", "").isdigit() else None
        mx = float(r[2]) if r[2].replace(".", "").isdigit() else None
        reasons = {self.NAMES[i] for i in range(4) if len(r) > 5 + i and "Active" in r[5 + i] and "Not" not in r[5 + i]}
        return sm, mx, reasons

    def start(self):
        def run():
            while not self._stop.is_set():
                try:
                    row = self._sample_nvml() if self._nvml else self._sample_smi()
                    if row:
                        self.rows.append(row)
                except Exception:
                    pass
                self._stop.wait(0.02 if self._nvml else 0.2)
        self._t = threading.Thread(target=run, daemon=True)
        self._t.start()

    def stop(self):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)
        sm = [r[0] for r in self.rows if r[0] is not None]
        mx = [r[1] for r in self.rows if r[1] is not None]
        reasons = sorted(set().union(*[r[2] for r in self.rows])) if self.rows else []
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows), "source": "nvml" if self._nvml else "nvidia-smi"}


def dist_init(n):
    if n <= 1 or "RANK" not in os.environ:
        return 0, 1, None
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    rank = int(os.environ["RANK"])
    world = int(os.environ["WORLD_SIZE"])
    local = int(os.environ.get("LOCAL_RANK", rank))
    torch.cuda.set_device(local)
    dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=torch.device("cuda", local))
    return rank, world, dist


def max_over_ranks(dist, value):
    """the largest value over the ranks (the job's time is its slowest rank's)"""
    if dist is None:
        return value
    import torch
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([value], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of the eight colour
# launches of one fine sweep: an ncu capture at 128^3 (1.51 GB per sweep: every
# colour launch reads the whole u field, which exceeds L2) scaled by the vertex
# count, 3.3x the algorithmic bytes
SWEEP_TRAFFIC_BYTES = {128: 1_510_000_000, 256: 12_080_000_000}

PRECISION_NAME = {0: "FP32 V-cycles on the correction of an FP64 solution (iterative refinement)",
                  1: "FP32 solution (the reference's scheme)",
                  2: "FP32 V-cycles on the correction of an FP64 solution (iterative refinement) with the "
                     "refinement residual accumulated in FP32",
                  3: "FP32 V-cycles on the correction of an FP64 solution (iterative refinement) with the "
                     "refinement residual accumulated in FP32 and the level-0 V-cycle residual on tcgen05 "
                     "tensor cores (TF32 hi+lo operands, FP32 accumulation)"}


def launches_per_step(nl, vcycles, reso, refine, refinements, coarsest_nv, mixed=False):
    """kernel launches of this library in one step, counted from the code paths
    (equal to the ncu launch list of the 256^3 step); every step starts from zero
    solutions, so the FP64 solution is cleared instead of copied and centred (no
    kernel for 3) and the first refinement step sets f from f0 (1 kernel) instead
    of u64 += u and the FP64 residual (2)"""
    nblk = -(-(reso ** 3 // 8) // 128) * 3 * 8                  # fine residual norm partials
    finish = 2 if nblk > 4096 else 1                            # one- or two-stage norm reduction
    fine = 8 + 1 + finish + 8                                   # GS (last colour with its residual), residual, norms, GS
    if mixed:
        fine = 8 + 1 + 1 + 8                                    # GS, tensor-core residual, norms, GS
    coarse = (nl - 2) * (8 + 1 + 8)                             # GS per colour, residual, GS per colour
    per_cycle = fine + coarse + 2 * (nl - 1) + 1 + 1            # restrict, prolong, coarsest apply, deflation
    per_refine = 1 + 1 + 2 + 3                                  # u64 += u, residual64, norms, deflation restart
    setup = 1 + 1 + 1 + (nl - 2) + 1 + 1 + 3 * coarsest_nv      # density, level 1, pin patch, deeper, assemble,
    #                                                             first pivot, one launch per pivot column
    if refine:
        pre = 1 + 3 + 2                                         # rhs, balance, norms of f
        post = 2                                                # C: energies, reduction
    else:
        pre = 1 + 1 + 3 + 3 + 2 + 3                             # rhs, convert, warm-start mean, balance, norms, deflation start
        post = 1 + 1 + 2                                        # pending shift into u, convert, C
    zero_start = -1 if refine and refinements > 0 else 0
    return setup + pre + vcycles * per_cycle + refinements * per_refine + zero_start + post


def make_density(args, rank):
    import numpy as np
    from homo3d_b200.density import synthetic_density
    rho = synthetic_density(args.reso, seed=args.seed + rank, vol=args.vol)
    return (rho.ravel() ** 3).astype(np.float32)


def gpu_arm(args):
    import numpy as np
    import torch

    import homo3d_b200 as H

    rank, world, dist = dist_init(args.gpus)
    dev = torch.cuda.current_device()
    rho_h = make_density(args, rank)
    hd = H.Homogenization(args.reso, pin_mode=args.pin_mode, precision=args.precision)
    coarsest_nv = int(np.prod(hd.dims[-1]))
    stream = torch.cuda.ExternalStream(hd.stream)
    rho_d = torch.tensor(rho_h, device="cuda")
    rho_pin = torch.from_numpy(rho_h).pin_memory()
    rho_e2e = torch.empty_like(rho_d)

    def step():
        hd.update(rho_d)
        hd.reset_solutions()
        C = hd.elasticMatrix(args.tol)
        return C

    def step_e2e():
        rho_e2e.copy_(rho_pin, non_blocking=True)   # ordered before the solve by the binding
        hd.update(rho_e2e)
        hd.reset_solutions()
        return hd.elasticMatrix(args.tol)

    for _ in range(args.warmup):
        step()
    st = hd.last_stats
    if st["status"] != H.H3D_OK:
        raise RuntimeError("solve did not converge: %r" % (st,))
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    clocks = ClockSampler(dev)
    clocks.start()
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    ev0.record(stream)
    cycles, refs = [], []
    for _ in range(args.steps):
        C = step()
        cycles.append(hd.last_stats["vcycles"])
        refs.append(hd.last_stats["refinements"])
    ev1.record(stream)
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    clk = clocks.stop()
    t_ms = ev0.elapsed_time(ev1)
    t_max = max_over_ranks(dist, t_ms)
    ms_per_solve = t_max / (args.steps * world)
    if args.profile:
        hd.close()
        if dist is not None:
            dist.destroy_process_group()
        return {"metric": metric_name(args), "value": round(ms_per_solve, 3), "unit": "ms", "profile_run": True, "refinements": refs,
                "vcycles": cycles} if rank == 0 else None

    # end to end through the public API with host buffers
    torch.cuda.synchronize()
    e0 = time.perf_counter()
    for _ in range(args.steps):
        Ce = step_e2e()
    torch.cuda.synchronize()
    e2e_ms = (time.perf_counter() - e0) * 1e3
    e2e_ms = max_over_ranks(dist, e2e_ms) / (args.steps * world)
    if hd.last_stats["status"] != H.H3D_OK:
        raise RuntimeError("end-to-end solve did not converge: %r" % (hd.last_stats,))
    e2e_match = bool(np.abs(Ce - C).max() <= 1e-6 * np.abs(C).max())
    if not e2e_match:
        raise RuntimeError("end-to-end C differs from the device-timed C: %r vs %r" % (Ce, C))
    # C against the FP64 oracle's committed solution of the same design
    fx = oracle_fixture(args) if rank == 0 else None
    c_err = None
    if fx is not None:
        Co = np.array(fx["C"]).reshape(6, 6)
        c_err = float(np.abs(C - Co).max() / np.abs(Co).max())

    # setup alone, and the dominant kernel (fine-level Gauss-Seidel sweep) by itself
    s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s0.record(stream)
    for _ in range(args.steps):
        hd.update(rho_d)
    s1.record(stream)
    torch.cuda.synchronize()
    setup_ms = s0.elapsed_time(s1) / args.steps
    nsweep = 10
    hd.grid.gs_relaxation(1.0, 2)
    g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    g0.record(stream)
    hd.grid.gs_relaxation(1.0, nsweep)
    g1.record(stream)
    torch.cuda.synchronize()
    sweep_ms = g0.elapsed_time(g1) / nsweep
    # the level-1 sweep (27-point FP16 stencils) the same way
    hd.mg.grids[1].gs_relaxation(1.0, 2)
    g0.record(stream)
    hd.mg.grids[1].gs_relaxation(1.0, nsweep)
    g1.record(stream)
    torch.cuda.synchronize()
    sweep1_ms = g0.elapsed_time(g1) / nsweep
    nv1 = int(np.prod(hd.dims[1]))
    bpv1 = 243 * 2 + 3 * 72  # FP16 stencil entries + u read and write + f, per vertex
    n3 = args.reso ** 3
    alg_bytes_sweep = 220.0 * n3          # 3L(2 s_u + s_f) + s_rho per vertex, L = 6, FP32
    flops_sweep = 2.0 * (576 + 234 * 6) * n3
    peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))) if os.path.exists(
        os.path.join(ROOT, "MEASURED_PEAKS.json")) else {"hbm_gbs": 6650.0}
    achieved = alg_bytes_sweep / (sweep_ms * 1e-3) / 1e9
    vc = int(round(sum(cycles) / len(cycles)))

    result = None
    if rank == 0:
        result = {
            "metric": metric_name(args), "value": round(ms_per_solve, 3), "unit": "ms", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(t_max / args.steps, 3),
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic: seeded trig-basis density, reflect6, vol %.2f, rho^3 (SIMP p=3)" % args.vol,
            "config": workload_config(args, hd.nlevels),
            "vcycles": vc, "vcycles_per_s": round(vc / (ms_per_solve * world) * 1e3, 2),
            "setup_ms": round(setup_ms, 3),
            "C00": float(C[0, 0]), "C_e2e_match": e2e_match,
            "C_err_vs_oracle": c_err,
            "e2e": {"value": round(e2e_ms, 3), "unit": "ms", "h2d_bytes_per_step": int(rho_h.nbytes),
                    "d2h_bytes_per_step": 36 * 8},
            "refinements": refs[-1],
            "launch_shapes": hd.tuning(),
            "level1_sweep": {"kernel": "k_coarse_gs (8 colour launches = one sweep of level 1)",
                             "vertices": nv1, "bytes_per_vertex": bpv1, "ms": round(sweep1_ms, 4),
                             "achieved": round(bpv1 * nv1 / (sweep1_ms * 1e-3) / 1e9, 1), "unit": "GB/s",
                             "frac": round(bpv1 * nv1 / (sweep1_ms * 1e-3) / 1e9 / peaks.get("hbm_gbs"), 4)},
            "gpu_launches": sum(launches_per_step(hd.nlevels, c, args.reso, args.precision != 1, r, coarsest_nv,
                                                  args.precision == 3) for c, r in zip(cycles, refs)),
            "roofline": {"kernel": "k_fine_gs (8 colour launches = one sweep)", "bound": "hbm",
                         "achieved": round(achieved, 1), "peak": peaks.get("hbm_gbs"), "unit": "GB/s",
                         "frac": round(achieved / peaks.get("hbm_gbs"), 4),
                         "traffic": SWEEP_TRAFFIC_BYTES.get(args.reso) if args.precision == 0 else None,
                         "traffic_unit": "bytes of DRAM read + write per sweep (ncu capture at 128^3, "
                                         "scaled by the vertex count)",
                         "sweep_ms": round(sweep_ms, 4), "fp32_tflops": round(flops_sweep / sweep_ms / 1e9, 2),
                         "peak_source": "measured" if "when" in peaks else "fallback"},
            "clocks": clk,
        }
    hd.close()
    if rank == 0 and world == 1 and args.precision == 0 and not args.no_precision_arms:
        result["precision_arms"] = precision_arms(args, rho_d, ms_per_solve, vc, c_err, fx)
    if dist is not None:
        dist.destroy_process_group()
    return result


def precision_arms(args, rho_d, plain_ms, plain_vc, plain_err, fx):
    """The precision arms of the same step on the same design, device-timed like the
    headline value: the plain arm (the headline: refined FP32 V-cycles, SIMT
    operator, FP64-accumulated refinement residual) against the mixed arms
    (H3D_PREC_MIXED: the refinement residual accumulated in FP32; H3D_PREC_MIXED_TC:
    besides, the level-0 V-cycle residual on the tensor cores).  The learned warm
    start is not in the step: its trained network saves no V-cycles on fresh
    designs (the solver's fallback rejects its prediction), so it would only add
    its forward pass."""
    import numpy as np
    import torch

    import homo3d_b200 as H

    def arm(precision):
        hm = H.Homogenization(args.reso, pin_mode=args.pin_mode, precision=precision)
        stream = torch.cuda.ExternalStream(hm.stream)

        def step():
            hm.update(rho_d)
            hm.reset_solutions()
            return hm.elasticMatrix(args.tol)

        for _ in range(max(1, min(args.warmup, 2))):
            step()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        ev0.record(stream)
        cyc = []
        for _ in range(args.steps):
            C = step()
            cyc.append(hm.last_stats["vcycles"])
        ev1.record(stream)
        torch.cuda.synchronize()
        st = hm.last_stats
        hm.close()
        err = None
        if fx is not None:
            Co = np.array(fx["C"]).reshape(6, 6)
            err = float(np.abs(C - Co).max() / np.abs(Co).max())
        ms = ev0.elapsed_time(ev1) / args.steps
        return {"ms": round(ms, 3), "ratio_over_plain": round(ms / plain_ms, 4),
                "vcycles": int(round(sum(cyc) / len(cyc))), "refinements": st["refinements"],
                "status": st["status"], "C_err": err, "scheme": PRECISION_NAME[precision]}

    mixed, mixed_tc = arm(H.PREC_MIXED), arm(H.PREC_MIXED_TC)
    best = min((mixed, mixed_tc), key=lambda a: a["ms"])
    return {"plain_ms": round(plain_ms, 3), "plain_vcycles": plain_vc, "plain_C_err": plain_err,
            "target_ratio": 0.5, "mixed": mixed, "mixed_tc": mixed_tc,
            "learned_mixed_ms": None, "ratio": best["ratio_over_plain"], "ratio_arm": best["scheme"],
            "learned": "not in the step (saves no V-cycles on fresh designs): ratio is the faster mixed arm "
                       "over the plain one", "plain": PRECISION_NAME[0]}


FIXTURE = os.path.join(ROOT, "tests", "golden", "oracle_C.json")


def workload_config(args, levels):
    return {"workload": "6-case periodic homogenization solve, %d^3, E=10 nu=0.3, relthres %g, zero start, "
                        "MG V(1,1) with 8-colour GS and FP16 coarse stencils, %s" % (
                            args.reso, args.tol, PRECISION_NAME[args.precision]),
            "reso": args.reso, "load_cases": 6, "relthres": args.tol, "vol": args.vol, "seed": args.seed,
            "pin_mode": args.pin_mode, "levels": int(levels),
            "parallelism": "replicas" if args.gpus > 1 else "single",
            "l2": "inputs larger than L2 (level-0 fields %.1f GB)" % (3 * 18 * 4 * args.reso ** 3 / 1e9)}


def oracle_fixture(args):
    """the committed FP64-oracle record of this design (tests/golden/oracle_C.json),
    or None"""
    if not os.path.exists(FIXTURE):
        return None
    for c in json.load(open(FIXTURE))["cases"]:
        if c["reso"] == args.reso and abs(c["vol"] - args.vol) < 1e-9 and c["seed"] == args.seed:
            return c
    return None


def oracle_vcycles(args):
    """(V-cycle count of the FP64 oracle's own solve of this design to relthres,
    where it comes from)"""
    fx = oracle_fixture(args)
    if fx is not None and args.tol == 1e-5 and fx.get("vcycles_to_1e-5"):
        return int(fx["vcycles_to_1e-5"]), "the oracle's own count for this design (tests/golden/oracle_C.json)"
    from oracle import oracle as O
    from homo3d_b200.density import synthetic_density
    m0 = O.MG((64, 64, 64))
    m0.set_density(synthetic_density(64, seed=args.seed, vol=args.vol).ravel() ** 3)
    m0.update_stencils()
    m0.rhs()
    v, _ = m0.solve(args.tol, 200)
    return int(v), "the oracle's own count for this design at 64^3"


class OracleSolve:
    """The FP64 CPU restatement of the solve (oracle/h3d_oracle.c, OpenMP on all
    host cores) at the full grid size, timed piece by piece: hierarchy setup and
    right-hand sides, single V-cycles, and the reduction of C."""

    def __init__(self, args):
        import numpy as np
        from oracle import oracle as O
        from homo3d_b200.density import synthetic_density
        n = args.reso
        self.m = O.MG((n, n, n))
        self.m.set_density((synthetic_density(n, seed=args.seed, vol=args.vol).ravel() ** 3)
                           .astype(np.float32).astype(np.float64))
        self.timed = 0.0

    def _t(self, fn):
        t0 = time.perf_counter()
        fn()
        dt = time.perf_counter() - t0
        self.timed += dt
        return dt

    def setup(self):
        return self._t(lambda: (self.m.update_stencils(), self.m.rhs()))

    def vcycle(self):
        return self._t(lambda: self.m.vcycle(1.0))

    def elastic(self):
        return self._t(lambda: self.m.elastic_matrix())


def cpu_sample(args, vcycles, vsource, cycles_timed=1):
    """Bounded CPU sample of the same workload: the FP64 oracle's setup, one V-cycle
    and the C reduction, each timed at the full grid size on all host cores; the
    solve is the V-cycle time times a stated V-cycle count (cycle-count
    extrapolated: the full oracle solve at 256^3 takes minutes)."""
    threads = os.cpu_count()
    o = OracleSolve(args)
    t_setup = o.setup()
    t_cyc = [o.vcycle() for _ in range(cycles_timed)]
    t_c = o.elastic()
    cyc = statistics.median(t_cyc)
    ms = (t_setup + vcycles * cyc + t_c) * 1e3
    return {"value": round(ms, 1), "unit": "ms", "cores": threads, "kind": "port",
            "sample": "FP64 oracle on %d host threads at %d^3: setup + %d V-cycle(s) + C timed, "
                      "value = setup + %d x V-cycle + C (cycle-count extrapolated; %d V-cycles = %s)"
                      % (threads, args.reso, cycles_timed, vcycles, vcycles, vsource),
            "vcycles": int(vcycles), "ms_per_vcycle": round(cyc * 1e3, 1), "setup_ms": round(t_setup * 1e3, 1),
            "C_ms": round(t_c * 1e3, 1), "timed_s": round(o.timed, 1)}


def reference_arm(args):
    """The reference's path on the host cores: the reference itself cannot be built
    here (its hot path needs Eigen, glm, gflags and OpenVDB), so this times the FP64
    CPU restatement of its solve (the oracle) on all host cores at the full grid
    size.  Each step is one V-cycle; the hierarchy setup and the C reduction are
    timed once; value = setup + V x (median V-cycle) + C, V the oracle's own
    V-cycle count for this design (the same count the GPU line's cpu_baseline uses)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return None
    os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count()))
    vcycles, vsource = oracle_vcycles(args)
    o = OracleSolve(args)
    t_setup = o.setup()
    for _ in range(min(args.warmup, 1)):
        o.vcycle()
    o.timed = t_setup
    cyc = [o.vcycle() for _ in range(args.steps)]
    t_c = o.elastic()
    c_med = statistics.median(cyc)
    value = round((t_setup + vcycles * c_med + t_c) * 1e3, 1)
    threads = os.cpu_count()
    cb = {"value": value, "unit": "ms", "cores": threads, "kind": "port",
          "sample": "FP64 oracle on %d host threads at %d^3: setup once, %d timed V-cycles (one per step), "
                    "C once; value = setup + %d x median V-cycle + C (cycle-count extrapolated; %d V-cycles = %s)"
                    % (threads, args.reso, args.steps, vcycles, vcycles, vsource),
          "vcycles": vcycles, "ms_per_vcycle": round(c_med * 1e3, 1), "setup_ms": round(t_setup * 1e3, 1),
          "C_ms": round(t_c * 1e3, 1), "timed_s": round(o.timed, 1)}
    return {"metric": metric_name(args), "value": value, "unit": "ms", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": value, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "impl": "reference",
            "data": "synthetic: seeded trig-basis density, reflect6, vol %.2f, rho^3 (SIMP p=3)" % args.vol,
            "config": workload_config(args, o.m.nlevels),
            "cpu_baseline": cb,
            "e2e": {"value": value, "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def mma_problem(n, m, seed=0):
    """a separable design problem of n variables and m linear constraints: objective
    gradient -w / x^2 (compliance-like), constraints A x - 0.3 sum(A) <= 0"""
    import numpy as np
    rng = np.random.default_rng(seed)
    w = rng.uniform(0.2, 1.0, n)
    A = rng.uniform(0.5, 1.5, (m, n)) / n
    return w, A


def mma_arm(args):
    """--workload mma: ms per MMA design update (MMAOptimizer::update,
    mmaOpt.cu:1021-1062) with reso^3 design variables and --mma-m constraints,
    through the library (h3d_mma_update, wall clock with the device synchronised:
    the update runs its Newton steps under host control), beside the FP64 oracle's
    MMA on the host (cpu_baseline, one update)."""
    import numpy as np
    import torch

    import homo3d_b200 as H
    n, m = args.reso ** 3, args.mma_m
    w, A = mma_problem(n, m)
    x0 = np.full(n, 0.3, np.float32)
    df = (-w / 0.3 ** 2).astype(np.float32)
    g = (A @ x0.astype(np.float64) - 0.3 * A.sum(axis=1)).astype(np.float32)
    dev = torch.device("cuda", 0)
    dft, gt = torch.tensor(df, device=dev), torch.tensor(g, device=dev)
    dgt = [torch.tensor(A[i].astype(np.float32), device=dev) for i in range(m)]
    times = []
    for rep in range(args.warmup + args.steps):
        mma = H.MMAOptimizer(m, n)
        mma.setBound(0.001, 1.0)
        x = torch.tensor(x0, device=dev)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        mma.update(0, x, dft, gt, dgt)
        torch.cuda.synchronize()
        if rep >= args.warmup:
            times.append((time.perf_counter() - t0) * 1e3)
        steps = mma.newton_steps
        mma.close()
    ms = statistics.median(times)
    out = {"metric": "ms per MMA design update, %d^3 design variables, %d constraint(s)" % (args.reso, m),
           "value": round(ms, 3), "unit": "ms", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
           "ms_per_step": round(ms, 3), "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
           "dtype": "f64", "data": "synthetic separable problem (objective gradient -w/x^2, linear constraints)",
           "config": {"workload": "MMA update", "n": n, "m": m}, "newton_steps": steps,
           "ms_all": [round(t, 3) for t in times]}
    if not args.no_cpu_baseline:
        from oracle import oracle as O
        ora = O.MMA(m, n)
        ora.set_bound(0.001, 1.0)
        t0 = time.perf_counter()
        ora.update(0, x0.astype(np.float64), df.astype(np.float64), g.astype(np.float64), A)
        cs = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": round(cs * 1e3, 1), "unit": "ms", "cores": 1, "kind": "port",
                               "sample": "FP64 oracle MMA (oracle/mma_oracle.c), one update of the same problem",
                               "newton_steps": int(ora.newton)}
    return out


def batch_arm(args):
    """--workload batch: designs per second for 24 designs of uneven resolution
    (8 x 64^3, 8 x 96^3, 8 x 128^3; seeded trig-basis densities at volumes U(0.1,
    0.5), zero start, six load cases, relthres 1e-3, FP32 V-cycles): one pass = the
    stencils, the six solves and C of every design.  Three arms through the public
    API, each timed as the best of --steps passes after --warmup (host clock with
    the device synchronised, densities resident on the device): the lockstep batch
    (value), per-design streams and one design at a time; C must agree to the last
    bit across the arms."""
    import numpy as np
    import torch

    import homo3d_b200 as H
    from homo3d_b200.batch import make_designs, parse_sizes, run_pass
    sizes = parse_sizes("64x8,96x8,128x8")
    designs = make_designs(sizes)
    homs = [H.Homogenization(n, precision=H.PREC_FP32) for n in sizes]
    rhos = [torch.tensor(r, device="cuda") for _, _, _, r in designs]
    tol = 1e-3
    lock = H.Lockstep(homs)
    res = {}
    for arm, batched, ls in (("lockstep", True, lock), ("streams", True, None), ("sequential", False, None)):
        best, C = None, None
        for rep in range(max(args.warmup, 1) + args.steps):
            dt, _, C, stats = run_pass(torch, homs, rhos, tol, batched, ls)
            if rep >= max(args.warmup, 1):
                best = dt if best is None else min(best, dt)
        res[arm] = (best, C, [s["vcycles"] for s in stats])
    lock.close()
    for hd in homs:
        hd.close()
    same = all(np.array_equal(res["lockstep"][1], res[a][1]) for a in ("streams", "sequential"))
    if not same:
        raise RuntimeError("batched C differs from the one-at-a-time C")
    dps = {a: round(len(sizes) / res[a][0], 2) for a in res}
    return {"metric": "designs per second, 24 designs (8x64^3, 8x96^3, 8x128^3), 6 load cases, relthres 1e-3",
            "value": dps["lockstep"], "unit": "designs/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(res["lockstep"][0] * 1e3, 3), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32",
            "data": "synthetic: seeded trig-basis densities, reflect6, volume U(0.1, 0.5), rho^3",
            "config": {"workload": "batched designs (config 4)", "designs": len(sizes), "relthres": tol,
                       "precision": "FP32 V-cycles"},
            "designs_per_s": dps, "C_identical_across_arms": same, "vcycles": res["lockstep"][2],
            "cpu_baseline": None}


def main():
    args = parse()
    if args.workload == "mma":
        print(json.dumps(mma_arm(args)), flush=True)
        return
    if args.workload == "batch":
        print(json.dumps(batch_arm(args)), flush=True)
        return
    if args.impl == "reference":
        out = reference_arm(args)
    else:
        out = gpu_arm(args)
        if out is not None and not args.no_cpu_baseline and out["n_gpus"] == 1:
            os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count()))
            vcycles, vsource = oracle_vcycles(args)
            out["cpu_baseline"] = cpu_sample(args, vcycles, vsource)
    if out is not None:
        print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
