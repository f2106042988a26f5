"""A persistent CG2D launch captured once in a CUDA graph and replayed.

`GraphedSolve` records one `solve_groups` call, and optionally work that follows it on the same stream (the edge
products of an adjoint, say), into a torch.cuda.CUDAGraph. A replay re-runs the whole sequence: the workspace
clear, the coefficient packing, the persistent cooperative kernel and the follow-up kernels, with no Python and
no per-launch host work. The groups' tensors are the graph's static inputs: write new values into them in place
(`copy_`) between replays. The outputs are static too: replay() returns the same tensors every time, overwritten.

Capture rules the class takes care of:
- one eager call first, with a status check: it creates the device topology of every exchanger (which allocates
  and copies from the host) and sets the kernel's shared-memory attribute, neither of which may happen inside a
  capture;
- the schedule ("auto" included) is resolved before the capture: tuning runs solves and synchronises;
- the capture itself reads nothing back to the host (no status check); check a replay's per-solve outcome in its
  diag records, and launch errors with `status()`.
cg2dNorm per instance must be a device float64 tensor, so that the capture copies nothing from the host.
"""

import torch

from mit_jax_b200 import capi
from mit_jax_b200.cg2d import solve_groups


class GraphedSolve:
    def __init__(self, groups, *, post=None, schedule=None, **solve_kw):
        """groups: GroupSpec list (device tensors, kept as the static inputs). post: optional callable taking the
        solve's result and returning more outputs, captured after the solve. schedule: None, a dict, or "auto".
        solve_kw: the other keyword arguments of solve_groups (precision, sum_order, ...)."""
        for G in groups:
            if isinstance(G.norm, torch.Tensor) and (G.norm.device != G.b[0].device or G.norm.dtype != torch.float64
                                                     or not G.norm.is_contiguous()):
                raise ValueError("cg2dNorm per instance must be a contiguous float64 tensor on the solve's device")
        for k in ("check_status", "profile"):
            if solve_kw.get(k):
                raise ValueError(f"{k} reads back to the host and cannot be captured")
        solve_kw.pop("check_status", None)
        self.groups = groups
        dev = groups[0].b[0].device
        if schedule == "auto":
            from mit_jax_b200 import autotune
            schedule = autotune.tune(groups, **{k: v for k, v in solve_kw.items() if k in (
                "precision", "sum_order", "rows_per_block", "replace_every", "replace_above")})
        self.schedule = schedule
        self._kw = dict(solve_kw, schedule=schedule)
        with torch.cuda.device(dev):
            eager = solve_groups(groups, check_status=True, **self._kw)     # topology handles, attributes
            if post is not None:
                post(eager)
            torch.cuda.synchronize(dev)
            self.graph = torch.cuda.CUDAGraph()
            with torch.cuda.graph(self.graph):
                self.result = solve_groups(groups, check_status=False, **self._kw)
                self.extra = post(self.result) if post is not None else None
        self.device = dev

    def replay(self):
        """Run the captured sequence on the current stream; returns (result, extra), the static outputs."""
        self.graph.replay()
        return self.result, self.extra

    def status(self):
        """Synchronise and return the launch-level error of the last replay, capi.CG2D_OK when none: a barrier
        timeout or an internal error, which the kernel writes into every solve's diag status."""
        from mit_jax_b200.cg2d import diag_records
        torch.cuda.synchronize(self.device)
        codes = {name: code for code, name in capi.STATUS_NAMES.items()}
        for slots in self.result:
            for _, _, dg in slots:
                for r in diag_records(dg):
                    code = codes.get(r["status"], capi.CG2D_INTERNAL_ERROR)
                    if code in (capi.CG2D_BARRIER_TIMEOUT, capi.CG2D_INTERNAL_ERROR):
                        return code
        return capi.CG2D_OK
