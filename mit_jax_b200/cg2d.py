"""CG2D on the B200: the drop-in for mitgcm_jax's cg2d_fortran / cg2d_solve, batched and mixed-precision solves,
and the differentiable wrapper (torch.autograd.Function).

Reference interface mirrored here (same names, arguments and results):
  Cg2dParams                    mitgcm_jax/core/cg2d.py:49-93
  Exchanger / default_exchanger mitgcm_jax/parallel/exchange.py:146-183, 220-222 (scalar kind "T")
  cg2d_fortran                  mitgcm_jax/core/cg2d.py:205-269 -> (x as CG2D returns it, diag)
  cg2d_solve                    mitgcm_jax/core/cg2d.py:351-375 -> (x interior with 0 halos, diag + x_fortran),
                                differentiable: implicit derivative dx = A^-1 (db - dA x) (cg2d.py:318-348),
                                coefficient gradients stopped when stop_coeff_grad (ECCO "passive" operator)
Every solve runs on the GPU through libcg2d.so; numpy inputs are copied to the current CUDA device and the results
copied back. Errors: unported options raise NotImplementedError at construction (cg2d.py:75-90, 212-213); a solve
that does not converge is not an error (diag numIters == max_iters), as in the reference.
"""

import ctypes
from dataclasses import dataclass, replace

import numpy as np
import torch

from mit_jax_b200 import capi
from mit_jax_b200.layout import Layout
from mit_jax_b200.topology import LLCTopology

OPS = ("aW2d", "aS2d", "aC2d", "pW", "pS", "pC")


@dataclass(frozen=True)
class Cg2dParams:
    """Solver parameters (mitgcm_jax/core/cg2d.py:49-67) plus the B200 solver options.

    sum_order "fortran" is the reference's sequential per-tile sum (bitwise reproducible against it, slow on a GPU);
    "tile" and "rowblock" select the GPU's fixed-order row-block sum (the reference's "tile" is an unspecified XLA
    tree, so no order can reproduce it bit for bit)."""
    cg2dMaxIters: int
    cg2dTolerance: float
    cg2dNorm: float
    cg2dpcOffDFac: float = 0.51
    nIterMin: int = -1
    sum_order: str = "fortran"
    sum_unroll: int = 1
    adj_tolerance: float = 1e-13
    adj_max_iters: int = 2000
    stop_coeff_grad: bool = False
    precision: str = "f64"          # "f64" | "mixed"
    rows_per_block: int = 8
    replace_every: int = 25
    replace_above: float = 100.0
    timeout_s: float = 10.0

    def __post_init__(self):
        if self.nIterMin >= 0:
            raise NotImplementedError("nIterMin >= 0 (min-residual solution, cg2d.F:347-378) is not ported")
        if self.sum_order not in ("fortran", "tile", "rowblock"):
            raise ValueError(self.sum_order)
        if self.precision not in ("f64", "mixed"):
            raise ValueError(self.precision)


def _params_struct(precision="f64", sum_order="rowblock", rows_per_block=8, replace_every=25, replace_above=100.0,
                   timeout_s=10.0, grid_ctas=0, ctas_per_sm=0, test_missing_arrivals=0, profile=False, unit_deal=0,
                   stages=0):
    p = capi.default_params()
    p.precision = capi.PREC_MIXED if precision == "mixed" else capi.PREC_F64
    p.sum_order = capi.SUM_FORTRAN if sum_order == "fortran" else capi.SUM_ROWBLOCK
    p.rows_per_block = rows_per_block
    p.replace_every = replace_every
    p.replace_above = replace_above
    p.timeout_s = timeout_s
    p.grid_ctas = grid_ctas
    p.ctas_per_sm = ctas_per_sm
    p.test_missing_arrivals = test_missing_arrivals
    p.profile = 1 if profile else 0
    p.unit_deal = unit_deal
    p.stages = stages
    return p


# ----------------------------------------------------------------------------------------------------------------
# exchange maps and device topology


class Exchanger:
    """The scalar ("T") exch2 halo map of one layout and its device neighbour tables (one per CUDA device).

    maps: {"T": (src int32[N], comp int8[N], sign[N]), ...} in the reference's ExchangeMaps format
    (exchange.py:73-93); extra kinds (e.g. "UVn_u"/"UVn_v") are kept for callers but unused by the solver."""

    def __init__(self, layout: Layout, maps: dict):
        self.L = layout
        self.maps = maps
        src, comp, sign = maps["T"]
        n = layout.nTiles * layout.ny * layout.nx
        if len(src) != n or len(comp) != n:
            raise ValueError("map length does not match the layout")
        if np.any(np.asarray(sign) != 1):
            raise ValueError("the scalar map has a sign flip")
        self._src = np.ascontiguousarray(src, np.int32)
        self._comp = np.ascontiguousarray(comp, np.int8)
        self._handles = {}

    @classmethod
    def from_npz(cls, path):
        """Load maps saved by the reference's ExchangeMaps.save (exchange.py:77-92)."""
        z = np.load(path)
        sNx, sNy, OLx, OLy, nT, Nr = (int(v) for v in z["layout"])
        L = Layout(sNx, sNy, OLx, OLy, nT, Nr)
        names = sorted({k.rsplit(".", 1)[0] for k in z.files if k != "layout"})
        maps = {n: (z[n + ".src"].astype(np.int32), z[n + ".comp"].astype(np.int8), z[n + ".sign"].astype(np.int8))
                for n in names}
        return cls(L, maps)

    def handle(self, device=None):
        dev = torch.cuda.current_device() if device is None else torch.device(device).index
        if dev not in self._handles:
            with torch.cuda.device(dev):
                out = ctypes.c_void_p()
                L = self.L
                capi.check(capi.lib().cg2d_topology_create(L.sNx, L.sNy, L.OLx, L.OLy, L.nTiles,
                                                           self._src.ctypes.data, self._comp.ctypes.data,
                                                           ctypes.byref(out)), "cg2d_topology_create")
                self._handles[dev] = out.value
        return self._handles[dev]

    def exch_xy(self, a):
        """Exchanger.exch_xy (exchange.py:182-183) for [..., T, ny, nx] on the GPU."""
        a, back = _dev(a)
        lead = a.shape[:-3]
        a = a.reshape((-1,) + tuple(self.L.shape2d)).contiguous()
        out = torch.empty_like(a)
        capi.check(capi.lib().cg2d_exchange_scalar(self.handle(a.device), a.shape[0], a.data_ptr(), out.data_ptr(),
                                                   _stream(a.device)), "cg2d_exchange_scalar")
        return back(out.reshape(lead + tuple(self.L.shape2d)))

    def __del__(self):
        try:
            for h in self._handles.values():
                capi.lib().cg2d_topology_destroy(h)
        except Exception:
            pass


_DEFAULT = {}


def default_exchanger(layout: Layout = None):
    """Generated LLC maps for an LLC layout (13 square tiles of one facet size, or facets split into more tiles)."""
    L = layout or Layout()
    key = (L.sNx, L.sNy, L.OLx, L.OLy, L.nTiles)
    if key not in _DEFAULT:
        if L.sNx != L.sNy or L.OLx != L.OLy:
            raise ValueError("generated LLC maps need square tiles and equal halos")
        tiles_per_facet = {13: 1, 52: 2, 117: 3}.get(L.nTiles)
        if tiles_per_facet is None:
            raise ValueError(f"no LLC tiling with {L.nTiles} tiles")
        topo = LLCTopology(L.sNx * tiles_per_facet, L.sNx, L.OLx)
        _DEFAULT[key] = Exchanger(topo.L, topo.maps)
    return _DEFAULT[key]


# ----------------------------------------------------------------------------------------------------------------
# device helpers


def _stream(device):
    return torch.cuda.current_stream(device).cuda_stream


def _dev(a, device=None):
    """(tensor on the CUDA device as float64 contiguous, function mapping results back to the input's kind)."""
    if isinstance(a, torch.Tensor):
        if not a.is_cuda:
            t = a.to(device or "cuda", torch.float64).contiguous()
            return t, lambda r: r.cpu()
        return a.to(torch.float64).contiguous(), lambda r: r
    t = torch.as_tensor(np.asarray(a, np.float64)).to(device or "cuda").contiguous()
    return t, lambda r: r.cpu().numpy()


def _ptr(t):
    return t.data_ptr() if t is not None else None


class GroupSpec:
    """One uniform batch for `solve_groups`: tensors [count, T, ny, nx] on one device."""

    def __init__(self, ex, ops, b, x0, tolerance, max_iters, cg2dNorm, x_fortran=False):
        self.ex = ex
        self.ops = ops                      # tuple of 6 tensors
        self.b = list(b)                    # 1 or 2 tensors (right-hand-side slots)
        self.x0 = list(x0)
        self.tol = list(tolerance)
        self.max_iters = list(max_iters)
        self.norm = cg2dNorm                # float or tensor [count]
        self.want_fortran = x_fortran


PROF_NAMES = ("bar", "mbar", "issue", "comp", "fin", "direct", "other", "total", "drain", "rwait", "ctrl", "pwait")
PROF_SLOTS = len(PROF_NAMES)


def solve_groups(groups, precision="f64", sum_order="rowblock", rows_per_block=8, replace_every=25,
                 replace_above=100.0, timeout_s=10.0, grid_ctas=0, ctas_per_sm=0, check_status=True,
                 test_missing_arrivals=0, profile=False, unit_deal=0, stages=0, schedule=None):
    """Run every right-hand side of every group in one persistent launch (cg2d_solve_groups).

    Returns per group a list (one entry per slot) of (x_out, x_fortran or None, diag ndarray of cg2d_diag_t).
    profile=True records per-CTA phase times; they are left in `solve_groups.last_profile` as an array
    [ctas, PROF_SLOTS] of nanoseconds, columns PROF_NAMES (include/cg2d.h, cg2d_workspace_profile).
    The launch schedule is grid_ctas, ctas_per_sm, unit_deal and stages, or schedule: a dict of those, or "auto"
    for the autotuner's choice for this workload (mit_jax_b200.autotune; tuned once, then cached). No schedule
    changes a result bit."""
    if not 1 <= len(groups) <= 4:
        raise ValueError("1 to 4 groups")
    dev = groups[0].b[0].device
    if schedule is not None:
        if isinstance(schedule, str):
            if schedule != "auto":
                raise ValueError(f"schedule {schedule!r}: a dict or 'auto'")
            from mit_jax_b200 import autotune
            schedule = autotune.tune(groups, precision=precision, sum_order=sum_order, rows_per_block=rows_per_block,
                                     replace_every=replace_every, replace_above=replace_above)
        grid_ctas = int(schedule.get("grid_ctas", grid_ctas))
        ctas_per_sm = int(schedule.get("ctas_per_sm", ctas_per_sm))
        unit_deal = int(schedule.get("unit_deal", unit_deal))
        stages = int(schedule.get("stages", stages))
    params = _params_struct(precision, sum_order, rows_per_block, replace_every, replace_above, timeout_s,
                            grid_ctas, ctas_per_sm, test_missing_arrivals, profile, unit_deal, stages)
    arr = (capi.Group * len(groups))()
    keep, outs = [], []
    for gi, G in enumerate(groups):
        g = arr[gi]
        count = G.b[0].shape[0]
        g.topo = G.ex.handle(dev)
        g.count = count
        g.nrhs = len(G.b)
        for name, t in zip(OPS, G.ops):
            setattr(g, name, t.data_ptr())
        if isinstance(G.norm, torch.Tensor):
            norm_t = G.norm.to(dev, torch.float64).contiguous()
            keep.append(norm_t)
            g.cg2dNorm = 0.0
            g.cg2dNorm_per_instance = norm_t.data_ptr()
        else:
            g.cg2dNorm = float(G.norm)
            g.cg2dNorm_per_instance = None
        slot_out = []
        for s in range(len(G.b)):
            xo = torch.empty_like(G.b[s])
            xf = torch.empty_like(G.b[s]) if G.want_fortran else None
            dg = torch.zeros((count, capi.DIAG_BYTES), dtype=torch.uint8, device=dev)
            g.b[s], g.x0[s], g.x_out[s], g.x_fortran[s], g.diag[s] = (
                G.b[s].data_ptr(), G.x0[s].data_ptr(), xo.data_ptr(), _ptr(xf), dg.data_ptr())
            g.tolerance[s] = float(G.tol[s])
            g.max_iters[s] = int(G.max_iters[s])
            slot_out.append((xo, xf, dg))
        outs.append(slot_out)
    L = capi.lib()
    nbytes = L.cg2d_workspace_size(arr, len(groups), ctypes.byref(params))
    if nbytes == 0:
        raise capi.Cg2dError(capi.CG2D_BAD_ARG, "cg2d_workspace_size")
    ws = torch.empty(nbytes + 256, dtype=torch.uint8, device=dev)
    base = ws.data_ptr()
    off = (-base) % 256
    capi.check(L.cg2d_solve_groups(arr, len(groups), ctypes.byref(params), base + off, nbytes, _stream(dev)),
               "cg2d_solve_groups")
    result = []
    for slot_out in outs:
        res = []
        for xo, xf, dg in slot_out:
            res.append((xo, xf, dg))
        result.append(res)
    if profile:
        buf = np.zeros(1 + PROF_SLOTS * 1184, np.uint64)
        capi.check(L.cg2d_workspace_profile(base + off, arr, len(groups), ctypes.byref(params), buf.ctypes.data, 1184,
                                            _stream(dev)), "cg2d_workspace_profile")
        solve_groups.last_profile = buf[1:1 + PROF_SLOTS * int(buf[0])].reshape(-1, PROF_SLOTS)
    if check_status:
        st = L.cg2d_workspace_status(base + off, _stream(dev))
        if st != capi.CG2D_OK:
            raise capi.Cg2dError(st, "cg2d solve")
    return result


def diag_records(dg):
    """uint8 [count, 48] device/host buffer -> list of dicts (the reference's diag keys + status)."""
    raw = dg.cpu().numpy() if isinstance(dg, torch.Tensor) else np.asarray(dg)
    dt = np.dtype([("firstResidual", "<f8"), ("lastResidual", "<f8"), ("sumRHS", "<f8"), ("rhsMax", "<f8"),
                   ("numIters", "<i4"), ("status", "<i4"), ("replacements", "<i4"), ("reserved", "<i4")])
    rec = raw.reshape(-1).view(dt)
    return [dict(firstResidual=float(r["firstResidual"]), lastResidual=float(r["lastResidual"]),
                 numIters=int(r["numIters"]), sumRHS=float(r["sumRHS"]), rhsMax=float(r["rhsMax"]),
                 status=capi.STATUS_NAMES.get(int(r["status"]), str(int(r["status"]))),
                 replacements=int(r["replacements"])) for r in rec]


# ----------------------------------------------------------------------------------------------------------------
# reference-shaped entry points


def cg2d_fortran(ex, ops, cg2d_b, cg2d_x, *, cg2dNorm, tolerance, max_iters, sum_order, nIterMin=-1, sum_unroll=1,
                 precision="f64", rows_per_block=8, replace_every=25, replace_above=100.0):
    """cg2d_fortran (cg2d.py:205-269) on the GPU. ops = (aW2d, aS2d, aC2d, pW, pS, pC), cg2d_b, cg2d_x:
    [T, ny, nx] (or [batch, T, ny, nx]). Returns (x, diag): x exactly as CG2D leaves it (interior = solution; halos =
    exchanged normalised first guess) and diag with firstResidual, lastResidual, numIters, sumRHS, rhsMax (a list of
    dicts for a batch). sum_unroll only changes the reference's kernel count, not its values: ignored."""
    if nIterMin >= 0:
        raise NotImplementedError("nIterMin >= 0 (min-residual solution) is not ported")
    x, xf, diags = _solve(ex, ops, cg2d_b, cg2d_x, cg2dNorm, tolerance, max_iters, sum_order, precision,
                          rows_per_block, replace_every, replace_above, want_fortran=True)
    return xf, diags


def _solve(ex, ops, cg2d_b, cg2d_x, cg2dNorm, tolerance, max_iters, sum_order, precision="f64", rows_per_block=8,
           replace_every=25, replace_above=100.0, want_fortran=True):
    b, back = _dev(cg2d_b)
    dev = b.device
    batched = b.dim() == 4
    shp = (-1,) + tuple(ex.L.shape2d)
    ops_t = tuple(_dev(a, dev)[0].reshape(shp).contiguous() for a in ops)
    b = b.reshape(shp).contiguous()
    x0 = _dev(cg2d_x, dev)[0].reshape(shp).contiguous()
    if ops_t[0].shape[0] != b.shape[0]:
        ops_t = tuple(a.expand(b.shape[0], *a.shape[1:]).contiguous() for a in ops_t)
    with torch.cuda.device(dev):
        G = GroupSpec(ex, ops_t, [b], [x0], [tolerance], [max_iters], cg2dNorm, x_fortran=want_fortran)
        (res,), = solve_groups([G], precision=precision, sum_order=sum_order, rows_per_block=rows_per_block,
                               replace_every=replace_every, replace_above=replace_above)
    xo, xf, dg = res
    diags = diag_records(dg)
    out_shape = tuple(ex.L.shape2d) if not batched else (-1,) + tuple(ex.L.shape2d)
    xo = back(xo.reshape(out_shape))
    xf = back(xf.reshape(out_shape)) if xf is not None else None
    return xo, xf, (diags if batched else diags[0])


def matvec(ex, A, cg2dNorm, v):
    """_matvec (cg2d.py:292-298): (A / cg2dNorm) v on the interior, 0 on halos. A = (aW2d, aS2d, aC2d)."""
    v, back = _dev(v)
    lead = v.shape[:-3]
    shp = (-1,) + tuple(ex.L.shape2d)
    vv = v.reshape(shp).contiguous()
    A_t = tuple(_dev(a, v.device)[0].reshape(shp).expand(vv.shape[0], *ex.L.shape2d).contiguous() for a in A)
    out = torch.empty_like(vv)
    capi.check(capi.lib().cg2d_apply_operator(ex.handle(v.device), vv.shape[0], float(cg2dNorm), A_t[0].data_ptr(),
                                              A_t[1].data_ptr(), A_t[2].data_ptr(), vv.data_ptr(), out.data_ptr(),
                                              _stream(v.device)), "cg2d_apply_operator")
    return back(out.reshape(lead + tuple(ex.L.shape2d)))


def edge_products(ex, lam, x, cg2dNorm):
    """Coefficient cotangents (gW, gS, gC) of the implicit derivative for adjoint solution lam and solution x."""
    lam, back = _dev(lam)
    lead = lam.shape[:-3]
    shp = (-1,) + tuple(ex.L.shape2d)
    lt = lam.reshape(shp).contiguous()
    xt = _dev(x, lam.device)[0].reshape(shp).contiguous()
    gW, gS, gC = (torch.empty_like(lt) for _ in range(3))
    norm_arr = None
    if isinstance(cg2dNorm, torch.Tensor):
        norm_arr = cg2dNorm.to(lam.device, torch.float64).contiguous()
        nval = 0.0
    else:
        nval = float(cg2dNorm)
    capi.check(capi.lib().cg2d_edge_products(ex.handle(lam.device), lt.shape[0], nval, _ptr(norm_arr), lt.data_ptr(),
                                             xt.data_ptr(), gW.data_ptr(), gS.data_ptr(), gC.data_ptr(),
                                             _stream(lam.device)), "cg2d_edge_products")
    return tuple(back(g.reshape(lead + tuple(ex.L.shape2d))) for g in (gW, gS, gC))


def exact_adjoint(ex, ops, cg2d_b, cg2d_x, x_bar, *, cg2dNorm, tolerance, max_iters, rows_per_block=8,
                  checkpoint_every=30, x_check=False, one_pass=True):
    """Exact-mode adjoint: solve A x = b in FP64 (ROWBLOCK sums), then reverse through the iterations that solve
    took. Returns (x, diag records, grads) with x the solution (interior, 0 on halos) and grads a dict of the
    cotangents of J = <x_bar, x> with respect to cg2d_b ("b") and to the six coefficient arrays (names of OPS); x0 is
    constant. checkpoint_every: iterations between checkpoints (0 = one segment). Arrays [batch, T, ny, nx] or
    [T, ny, nx]; cg2dNorm a float or a [batch] tensor.

    one_pass (default): the solve itself stores the checkpoints and its sums, and the reverse sweep starts from them
    (cg2d_solve_exact). one_pass=False or x_check=True: the solve, then cg2d_adjoint_exact, whose recording forward
    repeats the iterations; x_check adds that recording forward's solution ("x_check"), equal to x bit for bit. Both
    give the same gradients bit for bit."""
    b, back = _dev(cg2d_b)
    dev = b.device
    lead = b.shape[:-3]
    shp = (-1,) + tuple(ex.L.shape2d)
    b = b.reshape(shp)
    ops_t = tuple(_dev(a, dev)[0].reshape(shp) for a in ops)
    x0 = _dev(cg2d_x, dev)[0].reshape(shp)
    xb = _dev(x_bar, dev)[0].reshape(shp)
    batch = b.shape[0]
    norm = cg2dNorm
    if isinstance(norm, np.ndarray):
        norm = torch.as_tensor(norm)
    norm_arr = norm.to(dev, torch.float64).contiguous() if isinstance(norm, torch.Tensor) else None
    nval = 0.0 if norm_arr is not None else float(norm)
    if one_pass and not x_check:
        with torch.cuda.device(dev):
            L = capi.lib()
            topo = ex.handle(dev)
            nbytes = L.cg2d_solve_exact_workspace_size(topo, batch, int(max_iters), int(rows_per_block),
                                                       int(checkpoint_every))
            if nbytes == 0:
                raise capi.Cg2dError(capi.CG2D_BAD_ARG, "cg2d_solve_exact_workspace_size")
            ws = torch.empty(nbytes + 256, dtype=torch.uint8, device=dev)
            base = ws.data_ptr() + (-ws.data_ptr()) % 256
            x = torch.empty_like(b)
            dg = torch.zeros((batch, capi.DIAG_BYTES), dtype=torch.uint8, device=dev)
            outs = {k: torch.empty_like(b) for k in ("b",) + OPS}
            capi.check(L.cg2d_solve_exact(topo, batch, nval, _ptr(norm_arr), *(t.data_ptr() for t in ops_t),
                                          b.data_ptr(), x0.data_ptr(), float(tolerance), int(max_iters),
                                          xb.data_ptr(), int(rows_per_block), int(checkpoint_every), x.data_ptr(),
                                          dg.data_ptr(), outs["b"].data_ptr(), *(outs[k].data_ptr() for k in OPS),
                                          base, nbytes, _stream(dev)), "cg2d_solve_exact")
        shape = lead + tuple(ex.L.shape2d)
        grads = {k: back(v.reshape(shape)) for k, v in outs.items()}
        recs = diag_records(dg)
        return back(x.reshape(shape)), (recs[0] if not lead else recs), grads
    with torch.cuda.device(dev):
        G = GroupSpec(ex, ops_t, [b], [x0], [tolerance], [max_iters], norm)
        (res,), = solve_groups([G], precision="f64", sum_order="rowblock", rows_per_block=rows_per_block)
        x, _, dg = res
        L = capi.lib()
        topo = ex.handle(dev)
        nbytes = L.cg2d_adjoint_exact_workspace_size(topo, batch, int(max_iters), int(checkpoint_every))
        if nbytes == 0:
            raise capi.Cg2dError(capi.CG2D_BAD_ARG, "cg2d_adjoint_exact_workspace_size")
        ws = torch.empty(nbytes + 256, dtype=torch.uint8, device=dev)
        base = ws.data_ptr() + (-ws.data_ptr()) % 256
        outs = {k: torch.empty_like(b) for k in ("b",) + OPS}
        xc = torch.empty_like(b) if x_check else None
        capi.check(L.cg2d_adjoint_exact(topo, batch, nval, _ptr(norm_arr), *(t.data_ptr() for t in ops_t),
                                        b.data_ptr(), x0.data_ptr(), dg.data_ptr(), xb.data_ptr(), int(max_iters),
                                        int(rows_per_block), int(checkpoint_every), outs["b"].data_ptr(),
                                        *(outs[k].data_ptr() for k in OPS), _ptr(xc), base, nbytes, _stream(dev)),
                   "cg2d_adjoint_exact")
    shape = lead + tuple(ex.L.shape2d)
    grads = {k: back(v.reshape(shape)) for k, v in outs.items()}
    if xc is not None:
        grads["x_check"] = back(xc.reshape(shape))
    recs = diag_records(dg)
    return back(x.reshape(shape)), (recs[0] if not lead else recs), grads


# ----------------------------------------------------------------------------------------------------------------
# differentiable solve


def _interior_mask(L, device):
    m = torch.zeros(L.ny, L.nx, dtype=torch.bool, device=device)
    J, I = L.interior
    m[J, I] = True
    return m


class Cg2dSolve(torch.autograd.Function):
    """x = A^-1 b by the literal CG2D forward; backward is the implicit derivative (cg2d.py:318-348):
    lam = A^-1 xbar by a tight CG from a zero first guess (adj_tolerance, adj_max_iters), g_b = lam, and the
    coefficient cotangents gW, gS, gC = edge products of lam and x (zero under stop_coeff_grad). No derivative
    flows to the preconditioner, the first guess or cg2dNorm."""

    @staticmethod
    def forward(ctx, p, ex, box, aW2d, aS2d, aC2d, pW, pS, pC, cg2d_b, cg2d_x):
        xo, xf, diag = _solve(ex, (aW2d, aS2d, aC2d, pW, pS, pC), cg2d_b, cg2d_x, p.cg2dNorm, p.cg2dTolerance,
                              p.cg2dMaxIters, p.sum_order, p.precision, p.rows_per_block, p.replace_every,
                              p.replace_above, want_fortran=True)
        box["diag"] = diag
        ctx.p, ctx.ex = p, ex
        ctx.save_for_backward(aW2d, aS2d, aC2d, pW, pS, pC, xo)
        ctx.mark_non_differentiable(xf)
        return xo, xf

    @staticmethod
    def backward(ctx, xbar, _xf_bar):
        p, ex = ctx.p, ctx.ex
        aW2d, aS2d, aC2d, pW, pS, pC, x = ctx.saved_tensors
        mask = _interior_mask(ex.L, xbar.device)
        rhs = torch.where(mask, xbar, torch.zeros((), dtype=xbar.dtype, device=xbar.device))
        lam, _, _ = _solve(ex, (aW2d, aS2d, aC2d, pW, pS, pC), rhs, torch.zeros_like(rhs), p.cg2dNorm,
                           p.adj_tolerance, p.adj_max_iters, "rowblock", want_fortran=False)
        lam = torch.where(mask, lam, torch.zeros((), dtype=lam.dtype, device=lam.device))
        gW = gS = gC = None
        if not p.stop_coeff_grad and any(ctx.needs_input_grad[3:6]):
            gW, gS, gC = edge_products(ex, lam, x, p.cg2dNorm)
        return None, None, None, gW, gS, gC, None, None, None, lam, None


def cg2d_solve(p: Cg2dParams, ex: Exchanger, ops, cg2d_b, cg2d_x):
    """cg2d_solve (cg2d.py:351-375): (x, diag) with x the solution on the interior and 0 on halo points; diag holds
    cg2d_fortran's diagnostics and x_fortran. Differentiable in aW2d, aS2d, aC2d (unless p.stop_coeff_grad) and
    cg2d_b when they are torch tensors that require grad; numpy inputs give numpy outputs."""
    numpy_in = not isinstance(cg2d_b, torch.Tensor)
    args = [a if isinstance(a, torch.Tensor) else torch.as_tensor(np.asarray(a, np.float64)).cuda()
            for a in (*ops, cg2d_b, cg2d_x)]
    args[7] = args[7].detach()                       # the first guess carries no derivative (cg2d.py:372)
    if p.stop_coeff_grad:
        args[0:3] = [a.detach() for a in args[0:3]]  # ECCO: operator passive (cg2d.py:370-371)
    box = {}
    x, xf = Cg2dSolve.apply(p, ex, box, *args)
    if numpy_in:
        x, xf = x.detach().cpu().numpy(), xf.detach().cpu().numpy()
    if isinstance(box["diag"], list):   # a batch: one record per instance, each with its own x_fortran
        return x, [dict(d, x_fortran=xf[m]) for m, d in enumerate(box["diag"])]
    return x, dict(box["diag"], x_fortran=xf)


# ----------------------------------------------------------------------------------------------------------------
# forward + adjoint in one launch


def solve_with_adjoint(ex, ops, b, w, x0=None, *, cg2dNorm, tolerance=1e-12, max_iters=300, adj_tolerance=1e-13,
                       adj_max_iters=2000, precision="f64", sum_order="rowblock", coeff_grad="implicit",
                       rows_per_block=8, replace_every=25, replace_above=100.0):
    """Forward solve A x = b and adjoint (transpose) solve A lam = w of every instance of a batch in ONE
    persistent launch -- the two right-hand sides of an instance share its operator and preconditioner -- then the
    gradients of J = <w, x>: g_b = lam and, for coeff_grad="implicit", the coefficient cotangents (gW, gS, gC)
    (cg2d.py:318-348); coeff_grad="passive" is the reference's ECCO mode (stop_coeff_grad: no coefficient
    gradient). ops/b/w/x0: [batch, T, ny, nx] (device tensors, or host arrays/tensors, which are copied).
    cg2dNorm: float or [batch] tensor. Returns a dict with x, lam, gW, gS, gC (None when passive) and the
    forward/adjoint diagnostics (lists of dicts)."""
    if coeff_grad not in ("implicit", "passive"):
        raise ValueError(coeff_grad)
    b_t, back = _dev(b)
    dev = b_t.device
    shp = (-1,) + tuple(ex.L.shape2d)
    b_t = b_t.reshape(shp)
    ops_t = tuple(_dev(a, dev)[0].reshape(shp) for a in ops)
    mask = _interior_mask(ex.L, dev)
    w_t = torch.where(mask, _dev(w, dev)[0].reshape(shp), torch.zeros((), dtype=torch.float64, device=dev))
    x0_t = torch.zeros_like(b_t) if x0 is None else _dev(x0, dev)[0].reshape(shp)
    norm = cg2dNorm
    if isinstance(norm, np.ndarray):
        norm = torch.as_tensor(norm)
    with torch.cuda.device(dev):
        G = GroupSpec(ex, ops_t, [b_t, w_t], [x0_t, torch.zeros_like(w_t)], [tolerance, adj_tolerance],
                      [max_iters, adj_max_iters], norm)
        (slots,) = solve_groups([G], precision=precision, sum_order=sum_order, rows_per_block=rows_per_block,
                                replace_every=replace_every, replace_above=replace_above, check_status=False)
        x, _, dg_f = slots[0]
        lam, _, dg_a = slots[1]
        grads = (None, None, None)
        if coeff_grad == "implicit":
            grads = edge_products(ex, lam, x, norm)
    out = dict(x=back(x), lam=back(lam), gW=None, gS=None, gC=None, diag_fwd=dg_f, diag_adj=dg_a)
    if coeff_grad == "implicit":
        out.update(gW=back(grads[0]), gS=back(grads[1]), gC=back(grads[2]))
    return out
