#!/usr/bin/env python
"""CG2D forward + adjoint throughput on B200 (one JSON line on stdout).

Workload (one step): a batch of 64 LLC90 instances (13 tiles of 90x90, seeded synthetic ensemble members with
per-member depth, operator, cg2dNorm and right-hand side), each solved forward (A x = b) and adjoint (A lam = w,
seeded cotangent w) to a normalised residual of 1e-12 (max 300 iterations each), both right-hand sides of an
instance sharing its operator in ONE persistent mixed-precision launch, followed by the edge-product kernel
(coefficient gradients of J = <w, x>). Unit: forward+adjoint solve pairs per second, whole job.

  python bench.py [--gpus N --steps K --warmup W] [--impl reference]
  python bench.py --mode exact [--batch 16 --checkpoint 30]

--impl reference times the reference's CPU path (the oracle restatement of cg2d_fortran, FP64, forward + tight
adjoint solve + coefficient cotangents) on all host cores, one instance per process.

--mode pressure times SOLVE_FOR_PRESSURE around the solve (update_cg2d, cg2d_rhs, the FP64 solve, the post-solve
exchange; default batch 16, 50 levels), each step with its own device time and bandwidth.

--mode mixed_sizes times one mixed-precision launch over 8 LLC270 and 32 LLC90 instances and reports every
solution's error against the FP64 solve of the same instance.

--mode exact times the exact-mode adjoint instead (cg2d_adjoint_exact: FP64 forward, then reverse mode through
every CG iteration with checkpointed, recomputed segments; default batch 16) and reports adjoint solves/s and the
peak device memory of the step. The reference has no exact mode (it differentiates cg2d implicitly), so
--impl reference --mode exact reports itself unavailable.
"""

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "CG2D fwd+adjoint solves/s, batched/mixed vs plain FP64 on B200 at 1e-12 resid"
UNIT = "solves/s"
N_LLC90 = 13 * 90 * 90


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=("ours", "reference"))
    ap.add_argument("--mode", default="forward_adjoint", choices=("forward_adjoint", "exact", "pressure",
                                                                  "mixed_sizes"))
    ap.add_argument("--batch", type=int, default=None, help="instances per GPU (64; 16 with --mode exact/pressure)")
    ap.add_argument("--nr", type=int, default=50, help="--mode pressure: vertical levels")
    ap.add_argument("--checkpoint", type=int, default=30, help="--mode exact: iterations between checkpoints")
    ap.add_argument("--precision", default="mixed", choices=("mixed", "f64"))
    ap.add_argument("--tol", type=float, default=1e-12)
    ap.add_argument("--maxit", type=int, default=300)
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-tune", action="store_true", help="default launch schedule instead of the autotuner's")
    ap.add_argument("--no-graph", action="store_true", help="eager launches instead of CUDA graph replay")
    ap.add_argument("--phases", action="store_true",
                    help="after the timed region, one more launch with the kernel's phase timers (phases_ms)")
    a = ap.parse_args()
    if a.batch is None:
        a.batch = 16 if a.mode in ("exact", "pressure") else 64
    return a


# ------------------------------------------------------------------------------------------------------------------
# CPU leg: the oracle (FP64 cg2d_fortran restatement) on host cores, one instance per process


def _cpu_worker(args):
    os.environ.setdefault("OMP_NUM_THREADS", "1")
    from mit_jax_b200.topology import LLCTopology
    from oracle import cg2d_oracle as O
    ops, b, w, norm, tol, maxit = args
    topo = LLCTopology(90)
    L, tmap = topo.L, topo.maps["T"]
    t0 = time.perf_counter()
    x, d = O.cg2d_fortran(L, tmap, ops, b, np.zeros_like(b), cg2dNorm=norm, tolerance=tol, max_iters=maxit,
                          sum_order="fortran")
    x = np.where(O.interior_mask(L), x, 0.0)
    lam, da = O.tight_solve(L, tmap, ops, w, cg2dNorm=norm, tolerance=tol, max_iters=maxit, sum_order="tile")
    O.coefficient_cotangents(L, tmap, lam, x, norm)
    return time.perf_counter() - t0, d["numIters"], da["numIters"]


class CpuLeg:
    def __init__(self, inputs, procs):
        import multiprocessing as mp
        self.procs = procs
        self.inputs = inputs
        self.pool = mp.get_context("spawn").Pool(procs)

    def step(self):
        n = self.procs
        args = [self.inputs[i % len(self.inputs)] for i in range(n)]
        t0 = time.perf_counter()
        res = self.pool.map(_cpu_worker, args, chunksize=1)
        wall = time.perf_counter() - t0
        return n / wall, wall, res

    def close(self):
        self.pool.close()
        self.pool.join()


def _cpu_inputs(count, tol, maxit):
    from mit_jax_b200.synthetic import LLCSynthetic
    syn = LLCSynthetic(90)
    out = []
    for m in range(count):
        ops, norm = syn.operator(m)
        out.append((ops, syn.rhs(m), syn.cotangent(m), norm, tol, maxit))
    return out


def arm_config(a, world):
    """The workload both arms report: the batched LLC90 forward + adjoint step of this bench."""
    return {"workload": f"batch {a.batch} LLC90 CG2D forward + adjoint (2 right-hand sides per instance, one "
                        f"persistent launch) + edge products, {a.precision}",
            "batch_per_gpu": a.batch, "tolerance": a.tol, "max_iters": a.maxit,
            "grid": "LLC90 13x90x90, halo 4", "l2": "inputs larger than L2 (no flush)",
            "parallelism": f"instances sharded, {world} GPU(s), no collective in the solve"}


def run_reference(a):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    procs = max(1, min(os.cpu_count() or 1, a.batch))
    leg = CpuLeg(_cpu_inputs(min(procs, a.batch), a.tol, a.maxit), procs)
    for _ in range(a.warmup):
        leg.step()
    rates, walls = [], []
    for _ in range(a.steps):
        r, w, res = leg.step()
        rates.append(r)
        walls.append(w)
    leg.close()
    value = len(rates) * procs / sum(walls)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": a.gpus, "steps": a.steps, "warmup": a.warmup,
        "ms_per_step": 1e3 * statistics.mean(walls), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "impl": "reference",
        "config": arm_config(a, a.gpus),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": procs, "kind": "port",
                         "sample": f"each step: {procs} of the {a.batch} LLC90 instances (one per host process), "
                                   f"FP64 forward (fortran sum order) + adjoint + coefficient cotangents by the "
                                   f"oracle port of cg2d_fortran; {a.steps} steps"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


# ------------------------------------------------------------------------------------------------------------------
# GPU leg


class Clocks:
    """nvidia-smi samples during a timed region (SM clock, max clock, throttle reasons)."""

    FIELDS = ("clocks.sm", "clocks.max.sm", "power.draw", "clocks_event_reasons.active",
              "clocks_event_reasons.hw_slowdown", "clocks_event_reasons.hw_thermal_slowdown",
              "clocks_event_reasons.sw_thermal_slowdown", "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id):
        self.gpu_id = gpu_id
        self.proc = None
        self.f = None

    def __enter__(self):
        try:
            self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={','.join(self.FIELDS)}",
                                          "--format=csv,noheader,nounits", "-lms", "200", "-i", str(self.gpu_id)],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if self.proc is None or self.f is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.f.flush()
        rows = [r.split(",") for r in Path(self.f.name).read_text().splitlines() if r.strip()]
        os.unlink(self.f.name)
        sm, smax, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for r in rows:
            r = [c.strip() for c in r]
            try:
                sm.append(float(r[0]))
                smax.append(float(r[1]))
            except (ValueError, IndexError):
                continue
            for n, v in zip(names, r[4:8]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peak():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
        except Exception:
            pass
    return 6650.0, "fallback"


def algorithmic_bytes(diag_f, diag_a, precision):
    """Per launch: sum over solves of N_pts x iterations x bytes per point-iteration (12 words: 6 coefficients,
    r, s, x read, r, s, x written; MIXED: 10 FP32 words + x in FP64 = 56 B; FP64: 96 B) plus, MIXED, 96 B per point
    per true-residual replacement."""
    per_it = 56 if precision == "mixed" else 96
    tot = 0
    for d in diag_f + diag_a:
        tot += N_LLC90 * (d["numIters"] * per_it + d.get("replacements", 0) * 96)
    return tot


def shared_coefficient_bytes(diag_f, diag_a, precision):
    """The coefficient bytes the 12-word model counts twice: while an instance's forward and adjoint solves both
    iterate, the launch stages that instance's six coefficients once for both (24 B per point in FP32, 48 B in
    FP64), and the model charges them to each solve."""
    coef = 24 if precision == "mixed" else 48
    return sum(N_LLC90 * coef * min(f["numIters"], a["numIters"]) for f, a in zip(diag_f, diag_a))


def error_vs_fp64(cg, G, slots, L, a):
    """Every member's error against FP64: the same group solved once more in FP64 (ROWBLOCK order, which the tests
    tie to the reference's own solution), outside the timed region; per right-hand side the relative max-norm error
    over the interior, max |x - x64| / max |x64|, for every member (forward x and adjoint lam)."""
    (ref,) = cg.solve_groups([G], precision="f64", check_status=False)
    J, I = L.interior
    out = {}
    for name, (got, want) in zip(("x", "lam"), ((slots[0][0], ref[0][0]), (slots[1][0], ref[1][0]))):
        g, r = got[:, :, J, I], want[:, :, J, I]
        err = ((g - r).abs().amax(dim=(1, 2, 3)) / r.abs().amax(dim=(1, 2, 3))).cpu().numpy()
        out[f"{name}_max"] = float(err.max())
        out[f"{name}_per_member"] = [float(f"{e:.2e}") for e in err]
    out["reference"] = "FP64 ROWBLOCK solve of every member, same tolerance (tests tie it to the reference's x)"
    return out


def _gpu_uuid(torch, dev):
    """The device's UUID as nvidia-smi -i accepts it (falls back to the ordinal)."""
    u = getattr(torch.cuda.get_device_properties(dev), "uuid", None)
    if u is None:
        return dev.index
    return str(u) if str(u).startswith("GPU-") else f"GPU-{u}"


def run_gpu(a):
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)

    from mit_jax_b200 import cg2d as cg
    from mit_jax_b200.synthetic import make_batch

    from mit_jax_b200.sharding import estimated_work, max_over_ranks, shard_instances

    # inputs: this rank's own batch of members (weak scaling: world x batch members in all, disjoint per rank)
    members = None
    if world > 1:
        members = shard_instances(estimated_work([N_LLC90] * (world * a.batch)), world, rank)
    syn, B = make_batch(90, a.batch, with_cotangent=True, members=members)
    ex = cg.default_exchanger(syn.L)
    ops = tuple(torch.as_tensor(B[k]).to(dev) for k in cg.OPS)
    b = torch.as_tensor(B["b"]).to(dev)
    mask = cg._interior_mask(syn.L, dev)
    w = torch.where(mask, torch.as_tensor(B["w"]).to(dev), torch.zeros((), dtype=torch.float64, device=dev))
    x0 = torch.zeros_like(b)
    norms = torch.as_tensor(B["cg2dNorm"]).to(dev)
    G = cg.GroupSpec(ex, ops, [b, w], [x0, torch.zeros_like(w)], [a.tol, a.tol], [a.maxit, a.maxit], norms)
    stream = torch.cuda.current_stream(dev)

    # launch schedule from the autotuner (timed on this workload before the timed region), then the solve
    # captured once in a CUDA graph and replayed every step
    from mit_jax_b200 import autotune
    from mit_jax_b200.graph import GraphedSolve
    tune_report = []
    sched = None if a.no_tune else autotune.tune([G], precision=a.precision, report=tune_report)
    if a.no_graph:
        def step():
            (slots,) = cg.solve_groups([G], precision=a.precision, check_status=False, schedule=sched)
            return slots
    else:
        graphed = GraphedSolve([G], precision=a.precision, schedule=sched)

        def step():
            (slots,), _ = graphed.replay()
            return slots

    def barrier():
        torch.cuda.synchronize(dev)
        if world > 1:
            dist.barrier()

    for _ in range(a.warmup):
        slots = step()
        cg.edge_products(ex, slots[1][0], slots[0][0], norms)
    barrier()
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(a.steps)]
    with Clocks(_gpu_uuid(torch, dev)) as clk:
        time.sleep(0.25)
        barrier()
        for s in range(a.steps):
            ev[s][0].record(stream)
            slots = step()
            ev[s][1].record(stream)
            cg.edge_products(ex, slots[1][0], slots[0][0], norms)
            ev[s][2].record(stream)
        barrier()
    clocks = clk.summary()
    total_ms = ev[0][0].elapsed_time(ev[-1][2])
    solver_ms = [e[0].elapsed_time(e[1]) for e in ev]
    edge_ms = [e[1].elapsed_time(e[2]) for e in ev]
    total_ms = max_over_ranks(total_ms, dev)
    ms_per_step = total_ms / a.steps
    value = world * a.batch / (ms_per_step / 1e3)

    diag_f = cg.diag_records(slots[0][2])
    diag_a = cg.diag_records(slots[1][2])
    bad = [d for d in diag_f + diag_a if d["status"] != "ok"]
    err_fp64 = error_vs_fp64(cg, G, slots, syn.L, a) if a.precision == "mixed" else None
    alg = algorithmic_bytes(diag_f, diag_a, a.precision)
    shared = shared_coefficient_bytes(diag_f, diag_a, a.precision)
    peak, peak_kind = measured_peak()
    solver_mean = statistics.mean(solver_ms)
    achieved = alg / (solver_mean / 1e3) / 1e9
    traffic = None
    prof = ROOT / "profiles" / "solver_traffic.json"
    if prof.exists():
        try:
            pj = json.loads(prof.read_text())
            if pj.get("workload") == f"batch{a.batch}_{a.precision}":
                traffic = pj.get("bytes_per_launch")
        except Exception:
            traffic = None

    # ---- the kernel's own phase timers: one more launch, outside the timed region
    phases = None
    if a.phases:
        cg.solve_groups([G], precision=a.precision, schedule=sched, profile=True)
        prof = cg.solve_groups.last_profile.astype(np.float64) / 1e6
        phases = {"per_cta_mean": {n: float(prof[:, i].mean()) for i, n in enumerate(cg.PROF_NAMES)},
                  "ctas": int(prof.shape[0]),
                  "note": "ms per CTA over one launch: bar grid-wide waits, mbar waits for stage data, comp chunk "
                          "compute, fin/direct/drain/other the rest of thread 0's time; issue and pwait the copy "
                          "warp's busy and waiting time"}

    # ---- end to end through the public API from pinned host buffers. Every step uploads its inputs and
    #      downloads its solutions, gradients and diagnostics; the steps are pipelined over three streams (step s+1's
    #      inputs upload and step s-1's results download while step s computes), with two device input buffers.
    e2e = None
    if not a.no_e2e:
        host_in = {k: torch.as_tensor(B[k]).pin_memory() for k in (*cg.OPS, "b", "w", "x0")}
        host_in["norm"] = torch.as_tensor(B["cg2dNorm"]).pin_memory()
        keys = ("x", "lam", "gW", "gS", "gC")
        outs = [{k: torch.empty((a.batch, *syn.L.shape2d), dtype=torch.float64).pin_memory() for k in keys}
                for _ in range(2)]
        dgs = [[torch.empty((a.batch, cg.capi.DIAG_BYTES), dtype=torch.uint8).pin_memory() for _ in range(2)]
               for _ in range(2)]
        h2d = sum(v.numel() * v.element_size() for v in host_in.values())
        d2h = sum(v.numel() * v.element_size() for v in outs[0].values()) + 2 * a.batch * cg.capi.DIAG_BYTES
        dbuf = [{k: torch.empty_like(v, device=dev) for k, v in host_in.items()} for _ in range(2)]
        up, down = torch.cuda.Stream(dev), torch.cuda.Stream(dev)
        ev = {n: [torch.cuda.Event() for _ in range(2)] for n in ("in", "comp")}

        def upload(s):
            i = s % 2
            with torch.cuda.stream(up):
                if s >= 2:
                    up.wait_event(ev["comp"][i])            # step s-2 has finished reading buffer i
                for k, v in host_in.items():
                    dbuf[i][k].copy_(v, non_blocking=True)
                ev["in"][i].record(up)

        def compute_and_download(s):
            i = s % 2
            d = dbuf[i]
            with torch.cuda.stream(stream):
                stream.wait_event(ev["in"][i])
                r = cg.solve_with_adjoint(ex, tuple(d[k] for k in cg.OPS), d["b"], d["w"], d["x0"],
                                          cg2dNorm=d["norm"], tolerance=a.tol, max_iters=a.maxit,
                                          adj_tolerance=a.tol, adj_max_iters=a.maxit, precision=a.precision)
                ev["comp"][i].record(stream)
            with torch.cuda.stream(down):                    # downloads into a host buffer stay in stream order
                down.wait_event(ev["comp"][i])
                for k in keys:
                    r[k].record_stream(down)
                    outs[i][k].copy_(r[k], non_blocking=True)
                for j, name in enumerate(("diag_fwd", "diag_adj")):
                    r[name].record_stream(down)
                    dgs[i][j].copy_(r[name], non_blocking=True)

        def run(n):
            upload(0)
            for s in range(n):
                if s + 1 < n:
                    upload(s + 1)
                compute_and_download(s)

        run(max(2, a.warmup))
        barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(up)
        run(a.steps)
        e1.record(down)
        barrier()
        et = max_over_ranks(e0.elapsed_time(e1), dev)
        last = [cg.diag_records(t) for t in dgs[(a.steps - 1) % 2]]
        e2e = {"value": world * a.batch * a.steps / (et / 1e3), "unit": UNIT,
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
               "pipelined": "uploads of step s+1 and downloads of step s-1 overlap step s (three streams)",
               "not_ok": sum(r["status"] != "ok" for recs in last for r in recs)}

    # ---- the plain FP64 one-solve-per-launch kernel: one instance, forward launch then adjoint launch (and the
    # edge products), each replayed from a CUDA graph like the batched launch, so that host work between the
    # launches stays out of the device time of so short a solve
    plain = None
    if not a.no_plain and rank == 0:
        o1 = tuple(o[:1].contiguous() for o in ops)
        n1 = norms[:1].contiguous()
        Gf = cg.GroupSpec(ex, o1, [b[:1].contiguous()], [x0[:1].contiguous()], [a.tol], [a.maxit], n1)
        Ga = cg.GroupSpec(ex, o1, [w[:1].contiguous()], [torch.zeros_like(w[:1])], [a.tol], [a.maxit], n1)
        gf = GraphedSolve([Gf], precision="f64")
        ga = GraphedSolve([Ga], precision="f64",
                          post=lambda r: cg.edge_products(ex, r[0][0][0], gf.result[0][0][0], n1))
        for _ in range(2):
            gf.replay()
            ga.replay()
        torch.cuda.synchronize(dev)
        p0 = torch.cuda.Event(enable_timing=True)
        p1 = torch.cuda.Event(enable_timing=True)
        reps = 5
        p0.record(stream)
        for _ in range(reps):
            (sf,), _ = gf.replay()
            (sa,), _ = ga.replay()
        p1.record(stream)
        torch.cuda.synchronize(dev)
        pms = p0.elapsed_time(p1) / reps
        df, da = cg.diag_records(sf[0][2])[0], cg.diag_records(sa[0][2])[0]
        plain = {"solves_per_s": 1e3 / pms, "ms_per_pair": pms, "iters_fwd": df["numIters"],
                 "iters_adj": da["numIters"], "launch": "one FP64 launch per solve, each replayed from a CUDA graph"}

    cpu = None
    if not a.no_cpu and rank == 0 and world == 1:
        procs = max(1, min(os.cpu_count() or 1, 16))
        leg = CpuLeg(_cpu_inputs(procs, a.tol, a.maxit), procs)
        rate, wall, _ = leg.step()
        leg.close()
        cpu = {"value": rate, "unit": UNIT, "cores": procs, "kind": "port",
               "sample": f"{procs} LLC90 instances, one per process, FP64 forward + adjoint + cotangents, "
                         f"{wall:.1f} s wall"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32+f64" if a.precision == "mixed" else "f64", "data": "synthetic",
            "config": arm_config(a, world),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                         "kernel": "cg2d_persistent (solver launch incl. FP32 pack)",
                         "kernel_ms": solver_mean, "algorithmic_bytes_per_launch": alg,
                         "coefficients_counted_once": {
                             "algorithmic_bytes_per_launch": alg - shared,
                             "frac": (alg - shared) / (solver_mean / 1e3) / 1e9 / peak,
                             "note": "the 12-word model per solve charges an instance's coefficients to both of its "
                                     "solves; the paired launch reads them once"}},
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": 3 * a.steps,
            "clocks": clocks,
            "iterations": {"fwd_mean": statistics.mean(d["numIters"] for d in diag_f),
                           "adj_mean": statistics.mean(d["numIters"] for d in diag_a),
                           "fwd_min": min(d["numIters"] for d in diag_f), "fwd_max": max(d["numIters"] for d in diag_f),
                           "replacements_mean": statistics.mean(d["replacements"] for d in diag_f + diag_a),
                           "not_ok": len(bad)},
            "err_vs_fp64": err_fp64,
            "edge_products_ms": statistics.mean(edge_ms),
            "phases_ms": phases,
            "schedule": {"chosen": sched or "library default", "launch": "eager" if a.no_graph else "CUDA graph replay",
                         "candidates_ms": [[c, ms] for c, ms in tune_report]},
            "plain_f64_one_solve_per_launch": plain,
            "speedup_vs_plain_f64": (value / world) / plain["solves_per_s"] if plain else None,
        }
        print(json.dumps(line))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


# ------------------------------------------------------------------------------------------------------------------
# exact-mode adjoint

EXACT_METRIC = "CG2D exact-mode adjoint solves/s (FP64 forward + reverse through every iteration) on B200"


def exact_config(a):
    return {"workload": f"batch {a.batch} LLC90 exact-mode adjoint: FP64 ROWBLOCK forward to {a.tol:g} storing r and "
                        f"s_prev every {a.checkpoint} iterations, reverse through every iteration with segments "
                        f"recomputed from the solve's alpha and beta; gradients of <w, x> w.r.t. b and all six "
                        f"coefficient arrays",
            "batch_per_gpu": a.batch, "tolerance": a.tol, "max_iters": a.maxit, "checkpoint_every": a.checkpoint,
            "grid": "LLC90 13x90x90, halo 4", "l2": "inputs larger than L2 (no flush)",
            "parallelism": "1 GPU"}


def exact_algorithmic_bytes(iters, checkpoint):
    """Forward + segment recompute + reverse, counted as 3x the FP64 forward (96 B per point-iteration: six
    coefficients, r, s, x read and r, s, x written), plus the checkpoint stores (r and s_prev, 16 B per point each
    checkpoint)."""
    tot = 0
    for k in iters:
        nck = 1 if checkpoint <= 0 else -(-k // checkpoint)
        tot += N_LLC90 * (3 * 96 * k + 16 * nck)
    return tot


def exact_launches(kmax, checkpoint):
    """Kernels one cg2d_solve_exact call launches for a batch whose largest iteration count is kmax (memsets
    excluded): the coefficient pack and the solve; set-up, neighbour table, r_0 and the scalars from the solve's
    sums; the cotangent scaling; per iteration two recompute kernels (k_fa, k_fb) and four reverse kernels
    (k_rev_alpha, k_rq, k_rev_beta, k_rz); per segment the alphabar row dots and the two edge-product launches; and
    the two closing kernels."""
    C = checkpoint if checkpoint > 0 else max(1, kmax)
    nseg = -(-kmax // C) if kmax else 0
    return 2 + 4 + 1 + 6 * kmax + 3 * nseg + 2


def _cpu_exact(B, syn, member, iters):
    """The autograd oracle through the same iterations, one LLC90 instance, timed on host cores."""
    import torch
    from oracle.cg2d_exact_oracle import cg2d_exact_grad
    ops = tuple(B[k][member] for k in ("aW2d", "aS2d", "aC2d", "pW", "pS", "pC"))
    t0 = time.perf_counter()
    cg2d_exact_grad(syn.L, syn.topo.maps["T"], ops, B["b"][member], np.zeros_like(B["b"][member]),
                    B["w"][member], cg2dNorm=B["cg2dNorm"][member], iters=iters)
    return time.perf_counter() - t0, torch.get_num_threads()


def run_exact(a):
    import torch

    from mit_jax_b200 import capi
    from mit_jax_b200 import cg2d as cg
    from mit_jax_b200.synthetic import make_batch

    if int(os.environ.get("RANK", "0")) != 0:
        return 0
    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", "0")))
    torch.cuda.set_device(dev)
    syn, B = make_batch(90, a.batch, with_cotangent=True)
    ex = cg.default_exchanger(syn.L)
    ops = tuple(torch.as_tensor(B[k]).to(dev) for k in cg.OPS)
    b = torch.as_tensor(B["b"]).to(dev)
    mask = cg._interior_mask(syn.L, dev)
    w = torch.where(mask, torch.as_tensor(B["w"]).to(dev), torch.zeros((), dtype=torch.float64, device=dev))
    x0 = torch.zeros_like(b)
    norms = torch.as_tensor(B["cg2dNorm"]).to(dev)
    kw = dict(tolerance=a.tol, max_iters=a.maxit, checkpoint_every=a.checkpoint)
    stream = torch.cuda.current_stream(dev)

    def step():
        return cg.exact_adjoint(ex, ops, b, x0, w, cg2dNorm=norms, **kw)

    for _ in range(max(3, a.warmup)):
        x, d, g = step()
    torch.cuda.synchronize(dev)
    torch.cuda.reset_peak_memory_stats(dev)
    resident = torch.cuda.memory_allocated(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(_gpu_uuid(torch, dev)) as clk:
        time.sleep(0.25)
        torch.cuda.synchronize(dev)
        e0.record(stream)
        for _ in range(a.steps):
            x, d, g = step()
        e1.record(stream)
        torch.cuda.synchronize(dev)
    clocks = clk.summary()
    ms = e0.elapsed_time(e1) / a.steps
    peak_alloc = torch.cuda.max_memory_allocated(dev)
    ws_bytes = capi.lib().cg2d_solve_exact_workspace_size(ex.handle(dev), a.batch, a.maxit, 8, a.checkpoint)
    iters = [r["numIters"] for r in d]
    bad = [r for r in d if r["status"] != "ok"]
    alg = exact_algorithmic_bytes(iters, a.checkpoint)
    peak, peak_kind = measured_peak()
    achieved = alg / (ms / 1e3) / 1e9

    # the exact derivative of the iteration against the implicit derivative of the converged solution
    imp = cg.solve_with_adjoint(ex, ops, b, w, x0, cg2dNorm=norms, tolerance=a.tol, max_iters=a.maxit,
                                precision="f64")
    from mit_jax_b200.topology import exch_vector_adjoint

    def rel(u, ref):
        u, ref = np.asarray(u).reshape(a.batch, -1), np.asarray(ref).reshape(a.batch, -1)
        return float((np.abs(u - ref).max(1) / np.maximum(np.abs(ref).max(1), 1e-300)).max())

    host = {k: v.cpu().numpy() for k, v in (("b", g["b"]), ("aW2d", g["aW2d"]), ("aS2d", g["aS2d"]),
                                            ("aC2d", g["aC2d"]), ("lam", imp["lam"]), ("gW", imp["gW"]),
                                            ("gS", imp["gS"]), ("gC", imp["gC"]))}
    maps_u, maps_v = syn.topo.maps["UVn_u"], syn.topo.maps["UVn_v"]
    eu, ev = exch_vector_adjoint(host["aW2d"], host["aS2d"], maps_u, maps_v)
    iu, iv = exch_vector_adjoint(host["gW"], host["gS"], maps_u, maps_v)
    gap = {"b": rel(host["b"], host["lam"]), "aC2d": rel(host["aC2d"], host["gC"]),
           "aW2d_per_face": rel(eu, iu), "aS2d_per_face": rel(ev, iv),
           "aW2d_per_entry": rel(host["aW2d"], host["gW"]), "aS2d_per_entry": rel(host["aS2d"], host["gS"]),
           "note": "max over members of max|exact - implicit| / max|implicit|; per face = after the transpose of "
                   "the face exchange (each halo face entry's cotangent added onto the edge entry it copies); per "
                   "entry, the two stored copies of a tile-edge face are moved apart, an unsymmetric direction"}

    # end to end: inputs from pinned host buffers, solution and gradients back to pinned host buffers
    e2e = None
    if not a.no_e2e:
        host_in = {k: torch.as_tensor(B[k]).pin_memory() for k in (*cg.OPS, "b", "w")}
        host_norm = torch.as_tensor(B["cg2dNorm"])
        names = ("x", "b") + cg.OPS
        outs = {k: torch.empty((a.batch, *syn.L.shape2d), dtype=torch.float64).pin_memory() for k in names}
        h2d = sum(v.numel() * v.element_size() for v in host_in.values()) + host_norm.numel() * 8
        d2h = sum(v.numel() * v.element_size() for v in outs.values()) + a.batch * capi.DIAG_BYTES

        def e2e_step():
            din = {k: v.to(dev, non_blocking=True) for k, v in host_in.items()}
            xe, de, ge = cg.exact_adjoint(ex, tuple(din[k] for k in cg.OPS), din["b"], torch.zeros_like(din["b"]),
                                          din["w"], cg2dNorm=host_norm.to(dev, non_blocking=True), **kw)
            outs["x"].copy_(xe, non_blocking=True)
            for k in names[1:]:
                outs[k].copy_(ge[k], non_blocking=True)
            return de

        e2e_step()
        torch.cuda.synchronize(dev)
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        for _ in range(a.steps):
            e2e_step()
        t1.record(stream)
        torch.cuda.synchronize(dev)
        e2e = {"value": a.batch * a.steps / (t0.elapsed_time(t1) / 1e3), "unit": "adjoint solves/s",
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)}

    cpu = None
    if not a.no_cpu:
        secs, threads = _cpu_exact(B, syn, 0, iters[0])
        cpu = {"value": 1.0 / secs, "unit": "adjoint solves/s", "cores": threads, "kind": "port",
               "sample": f"member 0 ({iters[0]} iterations): torch float64 autograd through the oracle's "
                         f"iterations, {secs:.2f} s"}

    line = {
        "metric": EXACT_METRIC, "value": a.batch / (ms / 1e3), "unit": "adjoint solves/s", "n_gpus": 1,
        "steps": a.steps, "warmup": max(3, a.warmup), "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": exact_config(a),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": None, "peak_kind": peak_kind,
                     "kernel": "whole step (forward solve + cg2d_adjoint_exact kernels, host syncs included)",
                     "kernel_ms": ms, "algorithmic_bytes_per_launch": alg},
        "cpu_baseline": cpu,
        "e2e": e2e,
        "gpu_launches": a.steps * exact_launches(max(iters), a.checkpoint),
        "clocks": clocks,
        "memory": {"peak_allocated_bytes": int(peak_alloc), "resident_inputs_bytes": int(resident),
                   "workspace_bytes": int(ws_bytes)},
        "iterations": {"mean": statistics.mean(iters), "min": min(iters), "max": max(iters), "not_ok": len(bad)},
        "exact_vs_implicit_rel": gap,
    }
    print(json.dumps(line))
    return 0


# ------------------------------------------------------------------------------------------------------------------
# SOLVE_FOR_PRESSURE around the solve

PRESSURE_METRIC = "SOLVE_FOR_PRESSURE steps/s (update_cg2d + cg2d_rhs + FP64 CG2D + post) on B200"


def pressure_config(a):
    return {"workload": f"batch {a.batch} LLC90 SOLVE_FOR_PRESSURE with {a.nr} levels: update_cg2d (operator and "
                        f"preconditioner from the level sums), cg2d_rhs (g-hat divergence over the levels, fresh-water "
                        f"and etaH terms), FP64 ROWBLOCK CG2D to {a.tol:g}, exchange and etaN",
            "batch_per_gpu": a.batch, "levels": a.nr, "tolerance": a.tol, "max_iters": a.maxit,
            "grid": "LLC90 13x90x90, halo 4", "l2": "inputs larger than L2 (no flush)", "parallelism": "1 GPU"}


def pressure_bytes(B, Nr, n=90, T=13, npad=98):
    """Algorithmic bytes per launch. update_cg2d: hFacW, hFacS and four face metrics read on the (n+1)^2 faces per
    tile for every level, aW2d and aS2d written on the padded tile, then aW2d, aS2d, recip_Bo, rA read on the interior
    and aC2d, pW, pS, pC written. cg2d_rhs: gU, gV, hFacW, hFacS read per interior point and level, EmPmR, etaN,
    etaH, rA, maskInC, Bo_surf, dyG, dxG read and cg2d_b, cg2d_x written per point. Post: x, cg2d_x, recip_Bo read
    and etaN written per padded point."""
    f1, pts, pe = T * (n + 1) ** 2, T * n * n, T * npad * npad
    upd = B * (8 * f1 * (2 * Nr + 4) + 8 * 2 * pe) + B * (8 * 4 * pts + 8 * pe + 8 * 3 * f1)
    rhs = B * (8 * pts * (4 * Nr + 8) + 8 * 2 * pe)
    post = B * 8 * 4 * pe
    return upd, rhs, post


def _cpu_pressure(syn, f, a):
    """The oracle port on one member, one host thread: update_cg2d, cg2d_rhs, the FP64 solve (ROWBLOCK sums, as
    the GPU arm) and the post-solve step."""
    from oracle import cg2d_oracle as O
    from oracle import pressure_oracle as P
    L, tmap = syn.L, syn.topo.maps["T"]
    t0 = time.perf_counter()
    z = np.zeros(L.shape2d)
    ops = P.update_cg2d(L, tmap, hFacW=f["hFacW"], hFacS=f["hFacS"], pW=z, pS=z, pC=z,
                        **{k: f[k] for k in ("drF", "dyG", "dxG", "recip_dxC", "recip_dyC", "rA", "recip_Bo",
                                             "cg2dNorm", "cg2dpcOffDFac", "implicSurfPress", "implicDiv2DFlow",
                                             "freeSurfFac", "deltaTMom", "deltaTFreeSurf")})
    b, x0 = P.cg2d_rhs(L, **{k: f[k] for k in ("gU", "gV", "hFacW", "hFacS", "EmPmR", "etaN", "etaH", "Bo_surf",
                                               "drF", "dyG", "dxG", "rA", "maskInC", "freeSurfFac", "mass2rUnit",
                                               "implicDiv2DFlow", "deltaTMom", "deltaTFreeSurf",
                                               "useRealFreshWaterFlux")})
    x, d = O.cg2d_fortran(L, tmap, ops, b, x0, cg2dNorm=f["cg2dNorm"], tolerance=a.tol, max_iters=a.maxit,
                          sum_order="rowblock")
    P.solve_for_pressure_post(L, tmap, np.where(O.interior_mask(L), x, 0.0), x0, f["recip_Bo"])
    secs = time.perf_counter() - t0
    return {"value": 1.0 / secs, "unit": "instances/s", "cores": 1, "kind": "port",
            "sample": f"member 0 ({d['numIters']} iterations): the oracle port of update_cg2d, cg2d_rhs, the FP64 "
                      f"ROWBLOCK solve and the post-solve step on one host thread, {secs:.2f} s"}


def run_pressure(a):
    import torch

    from mit_jax_b200 import cg2d as cg
    from mit_jax_b200 import pressure as pr
    from mit_jax_b200.synthetic import LLCSynthetic

    if int(os.environ.get("RANK", "0")) != 0:
        return 0
    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", "0")))
    torch.cuda.set_device(dev)
    syn = LLCSynthetic(90)
    distinct = [syn.model_fields(a.nr, m) for m in range(min(a.batch, 8))]
    fs = [distinct[m % len(distinct)] for m in range(a.batch)]
    f0 = fs[0]
    import types
    g = types.SimpleNamespace(layout=syn.L, **{k: f0[k] for k in ("drF", "dyG", "dxG", "recip_dxC", "recip_dyC",
                                                                   "rA", "maskInC")})
    p = pr.FreeSurfParams(deltaTMom=f0["deltaTMom"], deltaTFreeSurf=f0["deltaTFreeSurf"],
                          freeSurfFac=f0["freeSurfFac"], implicSurfPress=f0["implicSurfPress"],
                          implicDiv2DFlow=f0["implicDiv2DFlow"], mass2rUnit=f0["mass2rUnit"],
                          rUnit2mass=1.0 / f0["mass2rUnit"], facEmP=1.0, hFacInf=0.2, hFacSup=2.0,
                          rStarAreaWeight=True, pfFacMom=1.0, select_rStar=2, nonlinFreeSurf=4,
                          useRealFreshWaterFlux=True, Nr=a.nr)
    st = {k: torch.as_tensor(np.stack([f[k] for f in fs])).to(dev)
          for k in ("hFacW", "hFacS", "gU", "gV", "EmPmR", "etaN", "etaH")}
    cpu = None
    if not a.no_cpu:
        cpu = _cpu_pressure(syn, f0, a)
    del distinct, fs
    norms = torch.full((a.batch,), float(f0["cg2dNorm"]), dtype=torch.float64, device=dev)
    cp = cg.Cg2dParams(cg2dMaxIters=a.maxit, cg2dTolerance=a.tol, cg2dNorm=norms, sum_order="rowblock")
    grid = {k: torch.as_tensor(f0[k]).to(dev) for k in ("recip_Bo", "Bo_surf")}
    g = types.SimpleNamespace(layout=syn.L, **{k: torch.as_tensor(getattr(g, k)).to(dev)
                                               for k in ("drF", "dyG", "dxG", "recip_dxC", "recip_dyC", "rA",
                                                         "maskInC")})
    ex = cg.default_exchanger(syn.L)
    prev = [torch.zeros((a.batch,) + syn.L.shape2d, dtype=torch.float64, device=dev) for _ in range(3)]
    stream = torch.cuda.current_stream(dev)

    def step(ev=None):
        rec = (lambda i: ev[i].record(stream)) if ev else (lambda i: None)
        rec(0)
        ops = pr.update_cg2d(p, cp, g, ex, st["hFacW"], st["hFacS"], grid["recip_Bo"], *prev)
        rec(1)
        b, x0 = pr.cg2d_rhs(p, g, st["gU"], st["gV"], st["hFacW"], st["hFacS"], st["EmPmR"], st["etaN"],
                            st["etaH"], grid["Bo_surf"], ex=ex)
        rec(2)
        G = cg.GroupSpec(ex, ops, [b], [x0], [a.tol], [a.maxit], norms)
        ((x, _, dg),), = cg.solve_groups([G], precision="f64", check_status=False)
        rec(3)
        eta = pr.pressure_post(ex, x, x0, grid["recip_Bo"])
        rec(4)
        return eta, dg

    for _ in range(max(3, a.warmup)):
        step()
    torch.cuda.synchronize(dev)
    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(5)] for _ in range(a.steps)]
    with Clocks(_gpu_uuid(torch, dev)) as clk:
        time.sleep(0.25)
        torch.cuda.synchronize(dev)
        for s in range(a.steps):
            eta, dg = step(evs[s])
        torch.cuda.synchronize(dev)
    clocks = clk.summary()
    parts = [[e[i].elapsed_time(e[i + 1]) for e in evs] for i in range(4)]
    total = evs[0][0].elapsed_time(evs[-1][4]) / a.steps
    recs = cg.diag_records(dg)
    upd_b, rhs_b, post_b = pressure_bytes(a.batch, a.nr)
    peak, peak_kind = measured_peak()
    upd_ms, rhs_ms, solve_ms, post_ms = (statistics.mean(x) for x in parts)
    solve_alg = sum(N_LLC90 * r["numIters"] * 96 for r in recs)

    def gbs(nbytes, ms):
        return nbytes / (ms / 1e3) / 1e9

    line = {
        "metric": PRESSURE_METRIC, "value": a.batch / (total / 1e3), "unit": "instances/s", "n_gpus": 1,
        "steps": a.steps, "warmup": max(3, a.warmup), "ms_per_step": total, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": pressure_config(a),
        "roofline": {"bound": "hbm", "achieved": gbs(rhs_b, rhs_ms), "peak": peak, "unit": "GB/s",
                     "frac": gbs(rhs_b, rhs_ms) / peak, "traffic": None, "peak_kind": peak_kind,
                     "kernel": "k_rhs (cg2d_rhs)", "kernel_ms": rhs_ms, "algorithmic_bytes_per_launch": rhs_b},
        "steps_ms": {"update_cg2d": upd_ms, "cg2d_rhs": rhs_ms, "cg2d_solve": solve_ms, "post": post_ms},
        "steps_gbs": {"update_cg2d": gbs(upd_b, upd_ms), "cg2d_rhs": gbs(rhs_b, rhs_ms),
                      "cg2d_solve": gbs(solve_alg, solve_ms), "post": gbs(post_b, post_ms)},
        "cpu_baseline": cpu, "e2e": None,
        "gpu_launches": a.steps * 6,
        "clocks": clocks,
        "iterations": {"mean": statistics.mean(r["numIters"] for r in recs), "not_ok":
                       sum(r["status"] != "ok" for r in recs)},
    }
    print(json.dumps(line))
    return 0


# ------------------------------------------------------------------------------------------------------------------
# mixed sizes: LLC270 and LLC90 instances in one mixed-precision launch

MIXED_SIZES_METRIC = "CG2D mixed-precision solves/s, 8 LLC270 + 32 LLC90 instances in one launch, on B200"


def run_mixed_sizes(a):
    import torch

    from mit_jax_b200 import autotune
    from mit_jax_b200 import cg2d as cg
    from mit_jax_b200.graph import GraphedSolve
    from mit_jax_b200.synthetic import make_batch

    if int(os.environ.get("RANK", "0")) != 0:
        return 0
    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", "0")))
    torch.cuda.set_device(dev)
    sizes = ((270, 8, 1000), (90, 32, a.maxit))
    groups, npts = [], []
    for N, count, maxit in sizes:
        syn, B = make_batch(N, count)
        ex = cg.default_exchanger(syn.L)
        ops = tuple(torch.as_tensor(B[k]).to(dev) for k in cg.OPS)
        b = torch.as_tensor(B["b"]).to(dev)
        norms = torch.as_tensor(B["cg2dNorm"]).to(dev)
        groups.append(cg.GroupSpec(ex, ops, [b], [torch.zeros_like(b)], [a.tol], [maxit], norms))
        npts.append(13 * N * N)
    stream = torch.cuda.current_stream(dev)
    report = []
    sched = autotune.tune(groups, precision="mixed", report=report)
    graphed = GraphedSolve(groups, precision="mixed", schedule=sched)
    for _ in range(max(3, a.warmup)):
        graphed.replay()
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(_gpu_uuid(torch, dev)) as clk:
        time.sleep(0.25)
        torch.cuda.synchronize(dev)
        e0.record(stream)
        for _ in range(a.steps):
            res, _ = graphed.replay()
        e1.record(stream)
        torch.cuda.synchronize(dev)
    clocks = clk.summary()
    ms = e0.elapsed_time(e1) / a.steps
    nsolve = sum(c for _, c, _ in sizes)
    # every solution against the FP64 solve of the same instance (FP64 ROWBLOCK equals the FP64 oracle bit for bit)
    ref = cg.solve_groups(groups, precision="f64")
    errs, iters, alg, bad = {}, {}, 0, 0
    for (N, _, _), r_m, r_f, n in zip(sizes, res, ref, npts):
        xm, xf = r_m[0][0], r_f[0][0]
        num = (xm - xf).abs().flatten(1).amax(1)
        den = xf.abs().flatten(1).amax(1).clamp_min(1e-300)
        e = (num / den).cpu().numpy()
        recs, recs_f = cg.diag_records(r_m[0][2]), cg.diag_records(r_f[0][2])
        errs[f"llc{N}"] = {"max": float(e.max()), "median": float(np.median(e))}
        iters[f"llc{N}"] = {"mixed_mean": statistics.mean(r["numIters"] for r in recs),
                            "f64_mean": statistics.mean(r["numIters"] for r in recs_f),
                            "mixed_max": max(r["numIters"] for r in recs)}
        bad += sum(r["status"] != "ok" for r in recs)
        alg += sum(n * (r["numIters"] * 56 + r["replacements"] * 96) for r in recs)
    peak, peak_kind = measured_peak()
    achieved = alg / (ms / 1e3) / 1e9
    line = {
        "metric": MIXED_SIZES_METRIC, "value": nsolve / (ms / 1e3), "unit": "solves/s", "n_gpus": 1,
        "steps": a.steps, "warmup": max(3, a.warmup), "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
        "config": {"workload": "8 LLC270 + 32 LLC90 instances (two groups) in one mixed-precision persistent launch, "
                               f"to {a.tol:g} (LLC270 cap 1000 iterations, LLC90 {a.maxit})",
                   "grid": "LLC270 13x270x270 and LLC90 13x90x90, halo 4", "l2": "inputs larger than L2 (no flush)",
                   "parallelism": "1 GPU"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": None, "peak_kind": peak_kind, "kernel": "cg2d_persistent (mixed, two groups)",
                     "kernel_ms": ms, "algorithmic_bytes_per_launch": alg},
        "error_vs_f64": errs, "iterations": iters, "not_ok": bad,
        "cpu_baseline": None, "e2e": None, "gpu_launches": 3 * a.steps, "clocks": clocks,
        "schedule": {"chosen": sched, "launch": "CUDA graph replay"},
    }
    print(json.dumps(line))
    return 0


def main():
    a = parse()
    if a.mode == "mixed_sizes":
        if a.impl == "reference":
            if int(os.environ.get("RANK", "0")) == 0:
                print(json.dumps({"impl": "reference", "unavailable": "--mode mixed_sizes has no CPU reference arm"}))
            return 0
        return run_mixed_sizes(a)
    if a.mode == "pressure":
        if a.impl == "reference":
            if int(os.environ.get("RANK", "0")) == 0:
                print(json.dumps({"impl": "reference", "unavailable": "--mode pressure has no CPU reference arm; its "
                                  "parity is checked against the reference's own outputs in the tests"}))
            return 0
        return run_pressure(a)
    if a.mode == "exact":
        if a.impl == "reference":
            if int(os.environ.get("RANK", "0")) == 0:
                print(json.dumps({"impl": "reference", "unavailable": "the reference has no exact-mode adjoint: "
                                  "it differentiates cg2d implicitly (mitgcm_jax/core/cg2d.py:307-348)"}))
            return 0
        return run_exact(a)
    if a.impl == "reference":
        return run_reference(a)
    return run_gpu(a)


if __name__ == "__main__":
    sys.exit(main())
