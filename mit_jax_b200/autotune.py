"""Launch-schedule autotuner for the persistent CG2D launch (cg2d_solve_groups).

A schedule says where the work runs, not what it computes:
- grid_ctas: how many CTAs the cooperative launch has;
- ctas_per_sm: how many of them share an SM (1, or the occupancy maximum);
- unit_deal: how the work units (instance, tile, row block) are dealt to them, round-robin (0) or in contiguous
  runs (1);
- stages: the depth of each CTA's copy pipeline (2 to 4 stage buffers; deeper takes more shared memory).
No schedule changes a result bit: every sum is formed from per-unit partials in one fixed order, whichever CTA
computed a unit (the GPU tests solve every candidate and compare them bit for bit).

`tune` times every candidate on the caller's own groups with a fixed iteration count (tolerance 0 and `iters`
iterations per right-hand side, so that every candidate does the same work and the per-iteration cost decides),
keeps the fastest, and caches it per workload signature: device name and SM count, precision, sum order,
ROWBLOCK height, residual-replacement settings, and per group (tiles, sNy, sNx, count, right-hand sides). The
cache lives in this process; with MIT_JAX_B200_TUNE_CACHE set to a file path it is also read from and written
to that JSON file.
"""

import json
import os
import threading

import torch

_CACHE = {}
_LOCK = threading.Lock()
_LOADED = set()


def signature(groups, *, precision, sum_order, rows_per_block, replace_every=25, replace_above=100.0,
              device=None):
    """The cache key of a workload (a string)."""
    dev = device if device is not None else groups[0].b[0].device
    props = torch.cuda.get_device_properties(dev)
    shapes = []
    for G in groups:
        L = G.ex.L
        shapes.append([int(L.nTiles), int(L.sNy), int(L.sNx), int(G.b[0].shape[0]), len(G.b)])
    key = {"device": props.name, "sms": int(props.multi_processor_count), "precision": precision,
           "sum_order": sum_order, "rows_per_block": int(rows_per_block), "groups": shapes}
    if precision == "mixed":
        key["replace"] = [int(replace_every), float(replace_above)]
    return json.dumps(key, sort_keys=True)


def candidates(sm_count, max_ctas_per_sm=2):
    """Schedules to try: 1 and up to max_ctas_per_sm CTAs per SM, the full co-resident grid and three quarters
    and half of it, each with both unit deals and a two-stage pipeline; and one CTA per SM on every SM with three
    and four stages. The library clamps ctas_per_sm to the occupancy maximum and the grid to the co-resident CTAs
    and to the work units, so every candidate is a valid launch."""
    out = []
    for cps in range(1, max_ctas_per_sm + 1):
        full = cps * sm_count
        for grid in sorted({full, (3 * full) // 4, full // 2}, reverse=True):
            for deal in (0, 1):
                out.append({"grid_ctas": int(max(1, grid)), "ctas_per_sm": cps, "unit_deal": deal, "stages": 2})
    for ns in (3, 4):
        out.append({"grid_ctas": int(sm_count), "ctas_per_sm": 1, "unit_deal": 0, "stages": ns})
    return out


def _load(path):
    if not path or path in _LOADED:
        return
    _LOADED.add(path)
    try:
        with open(path) as f:
            data = json.load(f)
    except (OSError, ValueError):
        return
    if isinstance(data, dict):
        for k, v in data.items():
            if isinstance(v, dict) and {"grid_ctas", "ctas_per_sm", "unit_deal", "stages"} <= set(v):
                _CACHE.setdefault(k, v)


def _save(path):
    if not path:
        return
    tmp = f"{path}.{os.getpid()}.tmp"
    try:
        with open(tmp, "w") as f:
            json.dump(_CACHE, f, indent=1, sort_keys=True)
        os.replace(tmp, path)
    except OSError:
        pass


def cached(key):
    """The cached schedule of a signature, or None."""
    with _LOCK:
        _load(os.environ.get("MIT_JAX_B200_TUNE_CACHE"))
        v = _CACHE.get(key)
        return dict(v) if v is not None else None


def tune(groups, *, precision="f64", sum_order="rowblock", rows_per_block=8, replace_every=25,
         replace_above=100.0, iters=20, reps=3, force=False, report=None):
    """The fastest schedule for these groups (a dict of grid_ctas, ctas_per_sm, unit_deal, stages), from the cache or by
    timing every candidate. report, if a list, receives one (schedule, milliseconds or None) per candidate."""
    from mit_jax_b200 import capi
    from mit_jax_b200.cg2d import GroupSpec, solve_groups

    dev = groups[0].b[0].device
    key = signature(groups, precision=precision, sum_order=sum_order, rows_per_block=rows_per_block,
                    replace_every=replace_every, replace_above=replace_above, device=dev)
    if not force:
        hit = cached(key)
        if hit is not None:
            return hit
    proxy = [GroupSpec(G.ex, G.ops, G.b, G.x0, [0.0] * len(G.b), [iters] * len(G.b), G.norm) for G in groups]
    kw = dict(precision=precision, sum_order=sum_order, rows_per_block=rows_per_block,
              replace_every=replace_every, replace_above=replace_above, check_status=True)
    stream = torch.cuda.current_stream(dev)
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    best, best_ms = None, None
    for cand in candidates(sms):
        try:
            solve_groups(proxy, **kw, **cand)                      # warm-up, and rejects unsupported launches
            torch.cuda.synchronize(dev)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            times = []
            for _ in range(reps):
                e0.record(stream)
                solve_groups(proxy, **{**kw, "check_status": False}, **cand)
                e1.record(stream)
                e1.synchronize()
                times.append(e0.elapsed_time(e1))
            ms = sorted(times)[len(times) // 2]
        except capi.Cg2dError:
            ms = None
        if report is not None:
            report.append((dict(cand), ms))
        if ms is not None and (best_ms is None or ms < best_ms):
            best, best_ms = cand, ms
    if best is None:
        raise RuntimeError("no candidate schedule ran")
    with _LOCK:
        _CACHE[key] = dict(best)
        _save(os.environ.get("MIT_JAX_B200_TUNE_CACHE"))
    return dict(best)
