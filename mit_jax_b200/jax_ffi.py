"""jax.ffi custom calls into libcg2d.so and a jax.custom_vjp cg2d_solve: the drop-in for the reference's JAX
entry points (mitgcm_jax/core/cg2d.py:205 cg2d_fortran and cg2d.py:351-375 cg2d_solve) where jax is installed.

The handlers live in libcg2d_ffi.so (csrc/cg2d_ffi.cc, built by mit_jax_b200._build when jax.ffi.include_dir()
exists): `cg2d_b200_solve` runs the persistent CG kernel, `cg2d_b200_adjoint` the adjoint solve and the edge
products. Arrays keep the reference layout [..., T, ny, nx] float64; leading dimensions are a batch of instances.

Differentiation (jax.custom_vjp, the transpose of _cg2d_implicit_jvp, cg2d.py:318-348): the cotangent x_bar of the
solution gives lam = A^-1 x_bar by a tight CG from zero (adj_tolerance, adj_max_iters), which is the cotangent of
cg2d_b; the coefficient cotangents of aW2d, aS2d, aC2d are the edge products of lam and x (the transpose of
_matvec(dA, x)), or zero under stop_coeff_grad (the reference's ECCO mode, cg2d.py:370-371). The preconditioner,
the first guess (stop_gradient, cg2d.py:372) and cg2dNorm get no derivative, as in the reference.
"""

import ctypes
import dataclasses
from functools import partial
from pathlib import Path

import numpy as np

import jax
import jax.numpy as jnp

from mit_jax_b200 import capi
from mit_jax_b200.cg2d import Cg2dParams
from mit_jax_b200.layout import Layout

HERE = Path(__file__).resolve().parent
FFI_LIB = HERE / "libcg2d_ffi.so"

_registered = False


def register():
    """Load libcg2d_ffi.so and register its two handlers as CUDA custom-call targets (once)."""
    global _registered
    if _registered:
        return
    if not FFI_LIB.exists():
        raise RuntimeError(f"{FFI_LIB.name} is not built (python -m mit_jax_b200._build with jax installed)")
    capi.lib()                                     # libcg2d.so first: the handler library links against it
    so = ctypes.CDLL(str(FFI_LIB))
    for name in ("cg2d_b200_solve", "cg2d_b200_adjoint"):
        jax.ffi.register_ffi_target(name, jax.ffi.pycapsule(getattr(so, name)), platform="CUDA")
    _registered = True


class Topology:
    """The exch2 scalar ("T") halo map of a layout as device neighbour tables (cg2d_topology_create) on the CUDA
    device of the current context: the reference's Exchanger for kind "T" (exchange.py:146-183)."""

    def __init__(self, layout: Layout, t_map):
        src, comp = np.ascontiguousarray(t_map[0], np.int32), np.ascontiguousarray(t_map[1], np.int8)
        self.L = layout
        out = ctypes.c_void_p()
        capi.check(capi.lib().cg2d_topology_create(layout.sNx, layout.sNy, layout.OLx, layout.OLy, layout.nTiles,
                                                   src.ctypes.data, comp.ctypes.data, ctypes.byref(out)),
                   "cg2d_topology_create")
        self.handle = int(out.value)

    @property
    def per_instance(self):
        return self.L.nTiles * self.L.ny * self.L.nx

    def __del__(self):
        try:
            capi.lib().cg2d_topology_destroy(ctypes.c_void_p(self.handle))
        except Exception:
            pass


_DIAG = 48   # bytes of cg2d_diag_t


def _diag_dict(raw):
    """u8[..., 48] (cg2d_diag_t) -> the reference's diag keys (cg2d.py:267-268) plus status and replacements."""
    f = jax.lax.bitcast_convert_type(raw[..., :32].reshape(raw.shape[:-1] + (4, 8)), jnp.float64)
    i = jax.lax.bitcast_convert_type(raw[..., 32:48].reshape(raw.shape[:-1] + (4, 4)), jnp.int32)
    return dict(firstResidual=f[..., 0], lastResidual=f[..., 1], sumRHS=f[..., 2], rhsMax=f[..., 3],
                numIters=i[..., 0], status=i[..., 1], replacements=i[..., 2])


def _norm_vec(cg2dNorm, lead):
    n = int(np.prod(lead)) if lead else 1
    return jnp.broadcast_to(jnp.asarray(cg2dNorm, jnp.float64).reshape(-1), (n,)).reshape(lead or (1,))


def _solve_call(topo, ops, b, x0, cg2dNorm, tolerance, max_iters, precision, sum_order):
    register()
    lead = b.shape[:-3]
    out = (jax.ShapeDtypeStruct(b.shape, jnp.float64), jax.ShapeDtypeStruct(b.shape, jnp.float64),
           jax.ShapeDtypeStruct(lead + (_DIAG,), jnp.uint8))
    call = jax.ffi.ffi_call("cg2d_b200_solve", out, vmap_method="broadcast_all")
    return call(*ops, b, x0, _norm_vec(cg2dNorm, lead), topo=np.int64(topo.handle), tolerance=np.float64(tolerance),
                max_iters=np.int32(max_iters), precision=np.int32({"f64": 0, "mixed": 1}[precision]),
                sum_order=np.int32({"rowblock": 0, "tile": 0, "fortran": 1}[sum_order]),
                per_instance=np.int64(topo.per_instance))


def _adjoint_call(topo, ops, x, xbar, cg2dNorm, adj_tolerance, adj_max_iters, coeff_grad):
    register()
    lead = xbar.shape[:-3]
    f = jax.ShapeDtypeStruct(xbar.shape, jnp.float64)
    out = (f, f, f, f, jax.ShapeDtypeStruct(lead + (_DIAG,), jnp.uint8))
    call = jax.ffi.ffi_call("cg2d_b200_adjoint", out, vmap_method="broadcast_all")
    return call(*ops, x, xbar, _norm_vec(cg2dNorm, lead), topo=np.int64(topo.handle),
                adj_tolerance=np.float64(adj_tolerance), adj_max_iters=np.int32(adj_max_iters),
                coeff_grad=np.int32(1 if coeff_grad else 0), per_instance=np.int64(topo.per_instance))


def cg2d_fortran(topo, ops, cg2d_b, cg2d_x, *, cg2dNorm, tolerance, max_iters, sum_order="rowblock",
                 precision="f64"):
    """cg2d_fortran (cg2d.py:205-269) on the GPU: (x as cg2d_fortran returns it, halos included; diag)."""
    _, xf, d = _solve_call(topo, tuple(ops), cg2d_b, cg2d_x, cg2dNorm, tolerance, max_iters, precision, sum_order)
    return xf, _diag_dict(d)


@partial(jax.custom_vjp, nondiff_argnums=(0, 1))
def _solve(p, topo, ops, b, x0, cg2dNorm):
    x, xf, d = _solve_call(topo, ops, b, x0, cg2dNorm, p.cg2dTolerance, p.cg2dMaxIters, p.precision, p.sum_order)
    return x, (xf, d)


def _solve_fwd(p, topo, ops, b, x0, cg2dNorm):
    x, xf, d = _solve_call(topo, ops, b, x0, cg2dNorm, p.cg2dTolerance, p.cg2dMaxIters, p.precision, p.sum_order)
    return (x, (xf, d)), (ops, x, x0, cg2dNorm)


def _solve_bwd(p, topo, res, ct):
    ops, x, x0, cg2dNorm = res
    xbar, _ = ct
    lam, gW, gS, gC, _ = _adjoint_call(topo, ops, x, xbar, cg2dNorm, p.adj_tolerance, p.adj_max_iters,
                                       not p.stop_coeff_grad)
    z = jnp.zeros_like
    return ((gW, gS, gC, z(ops[3]), z(ops[4]), z(ops[5])), lam, z(x0), z(jnp.asarray(cg2dNorm, jnp.float64)))


_solve.defvjp(_solve_fwd, _solve_bwd)


def cg2d_solve(p: Cg2dParams, topo: Topology, ops, cg2d_b, cg2d_x):
    """cg2d_solve (cg2d.py:351-375): (x, diag), x the solution on the interior and 0 on halo points, diag with
    x_fortran; differentiable in aW2d, aS2d, aC2d (zero cotangents under p.stop_coeff_grad) and cg2d_b."""
    ops = tuple(jnp.asarray(a, jnp.float64) for a in ops)
    if p.stop_coeff_grad:
        ops = tuple(jax.lax.stop_gradient(a) for a in ops[:3]) + ops[3:]
    x0 = jax.lax.stop_gradient(jnp.asarray(cg2d_x, jnp.float64))
    norm = jnp.asarray(p.cg2dNorm, jnp.float64)
    static = dataclasses.replace(p, cg2dNorm=0.0)     # the static part carries no (possibly traced) array
    x, (xf, d) = _solve(static, topo, ops, jnp.asarray(cg2d_b, jnp.float64), x0, norm)
    return x, dict(_diag_dict(d), x_fortran=xf)
