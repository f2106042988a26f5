"""SOLVE_FOR_PRESSURE on the GPU with the reference's call signatures (mitgcm_jax/core/solve_for_pressure.py), and
the operator normalisation it starts from (mitgcm_jax/core/cg2d.py:108-134):

    ini_cg2d_norm(g, hFacW, hFacS, implicSurfPress, implicDiv2DFlow) -> cg2dNorm                          (:108-134)

    update_cg2d(p, cp, g, ex, hFacW, hFacS, recip_Bo, pW, pS, pC) -> (aW2d, aS2d, aC2d, pW, pS, pC)     (:29-65)
    cg2d_rhs(p, g, gU, gV, hFacW, hFacS, EmPmR, etaN, etaH, Bo_surf) -> (cg2d_b, cg2d_x)               (:68-106)
    solve_for_pressure(p, cp, g, ex, ops, gU, gV, hFacW, hFacS, EmPmR, etaN, etaH, Bo_surf, recip_Bo)
        -> (etaN, info)                                                                                   (:109-123)

p is the reference's FreeSurfParams (or this module's copy, or any object with its fields); cp is a Cg2dParams
(mit_jax_b200.cg2d); g is the grid, any object with drF [Nr] and the [T, ny, nx] fields dyG, dxG, recip_dxC,
recip_dyC, rA, maskInC; ex an Exchanger. Per-instance fields may carry a leading batch dimension (3-D fields
[batch, T, Nr, ny, nx], 2-D fields [batch, T, ny, nx]); grid fields, recip_Bo and Bo_surf are shared by the
batch. Inputs are torch tensors (on the GPU or the host) or numpy arrays; numpy in gives numpy out. The work runs
in the library's kernels (cg2d_update_operator, cg2d_pressure_rhs, cg2d_pressure_post) and the persistent CG2D
solve; the results are bit for bit the reference's (with sum_order="fortran" for the solve).
"""

from dataclasses import dataclass

import numpy as np
import torch

from mit_jax_b200 import capi
from mit_jax_b200.cg2d import _dev, _ptr, _stream, cg2d_solve, default_exchanger


@dataclass(frozen=True)
class FreeSurfParams:
    """The reference's FreeSurfParams (mitgcm_jax/core/free_surface.py): the same fields and default."""
    deltaTMom: float
    deltaTFreeSurf: float
    freeSurfFac: float
    implicSurfPress: float
    implicDiv2DFlow: float
    mass2rUnit: float
    rUnit2mass: float
    facEmP: float
    hFacInf: float
    hFacSup: float
    rStarAreaWeight: bool
    pfFacMom: float
    select_rStar: int
    nonlinFreeSurf: int
    useRealFreshWaterFlux: bool
    Nr: int = 50


def _fs(p, Nr):
    f = capi.FreeSurf()
    f.deltaTMom, f.deltaTFreeSurf = float(p.deltaTMom), float(p.deltaTFreeSurf)
    f.freeSurfFac, f.implicSurfPress = float(p.freeSurfFac), float(p.implicSurfPress)
    f.implicDiv2DFlow, f.mass2rUnit = float(p.implicDiv2DFlow), float(p.mass2rUnit)
    f.useRealFreshWaterFlux = 1 if p.useRealFreshWaterFlux else 0
    f.Nr = int(Nr)
    return f


def _batch3(a, dev, shape2d):
    """A 3-D field as [batch, T, Nr, ny, nx] on dev; returns (tensor, lead dims)."""
    t = _dev(a, dev)[0]
    if tuple(t.shape[-2:]) != tuple(shape2d[-2:]) or t.shape[-4] != shape2d[0]:
        raise ValueError(f"3-D field of shape {tuple(t.shape)} for tiles {tuple(shape2d)}")
    return t.reshape((-1,) + tuple(t.shape[-4:])).contiguous(), tuple(t.shape[:-4])


def _batch2(a, dev, shape2d, B):
    t = _dev(a, dev)[0].reshape((-1,) + tuple(shape2d))
    if t.shape[0] != B:
        if t.shape[0] != 1:
            raise ValueError(f"2-D field with {t.shape[0]} instances for a batch of {B}")
        t = t.expand(B, *shape2d)
    return t.contiguous()


def _grid(a, dev, shape2d):
    t = _dev(a, dev)[0]
    if tuple(t.shape) != tuple(shape2d):
        raise ValueError(f"grid field of shape {tuple(t.shape)}, expected {tuple(shape2d)}")
    return t.contiguous()


def _norm(cg2dNorm, dev, B):
    if isinstance(cg2dNorm, (torch.Tensor, np.ndarray)) and np.ndim(cg2dNorm) > 0:
        t = torch.as_tensor(cg2dNorm).to(dev, torch.float64).reshape(-1).contiguous()
        if t.numel() != B:
            raise ValueError("one cg2dNorm per instance")
        return 0.0, t
    return float(cg2dNorm), None


def ini_cg2d_norm(g, hFacW, hFacS, implicSurfPress, implicDiv2DFlow, *, ex=None):
    """ini_cg2d_norm (mitgcm_jax/core/cg2d.py:108-134) on the GPU: cg2dNorm = 1 / max|aW, aS| of the un-normalised
    initial operator (cg2d_ini_norm), bit for bit the reference's. hFacW, hFacS: the initial face fractions
    [T, Nr, ny, nx] (a float is returned, as the reference returns) or [batch, T, Nr, ny, nx] (one value per
    instance: a tensor, or an array for numpy input). The layout comes from g.layout, or from the Exchanger ex."""
    if ex is None:
        ex = default_exchanger(g.layout)
    shape2d = tuple(ex.L.shape2d)
    hW, back = _dev(hFacW)
    dev = hW.device
    single = hW.dim() == 4
    hW, lead = _batch3(hW, dev, shape2d)
    hS, _ = _batch3(hFacS, dev, shape2d)
    B, Nr = hW.shape[0], hW.shape[2]
    drF = _dev(np.asarray(g.drF, np.float64) if not isinstance(g.drF, torch.Tensor) else g.drF, dev)[0]
    if drF.numel() != Nr:
        raise ValueError("drF has one entry per level")
    grid = [_grid(getattr(g, k), dev, shape2d) for k in ("dyG", "dxG", "recip_dxC", "recip_dyC")]
    out = torch.empty(B, dtype=torch.float64, device=dev)
    capi.check(capi.lib().cg2d_ini_norm(ex.handle(dev), B, Nr, float(implicSurfPress), float(implicDiv2DFlow),
                                        hW.data_ptr(), hS.data_ptr(), drF.contiguous().data_ptr(),
                                        *(t.data_ptr() for t in grid), out.data_ptr(), _stream(dev)),
               "cg2d_ini_norm")
    if single:
        return float(out[0].item())
    return back(out.reshape(lead))


def update_cg2d(p, cp, g, ex, hFacW, hFacS, recip_Bo, pW, pS, pC):
    """update_cg2d (solve_for_pressure.py:29-65) on the GPU. pW, pS, pC: the current preconditioner, kept outside
    i, j = 1..sNx+1, 1..sNy+1 (the inputs are not modified). cp.cg2dNorm: a float, or one per instance."""
    shape2d = tuple(ex.L.shape2d)
    hW, back = _dev(hFacW)
    dev = hW.device
    hW, lead = _batch3(hW, dev, shape2d)
    hS, _ = _batch3(hFacS, dev, shape2d)
    B, Nr = hW.shape[0], hW.shape[2]
    drF = _dev(np.asarray(g.drF, np.float64) if not isinstance(g.drF, torch.Tensor) else g.drF, dev)[0]
    if drF.numel() != Nr:
        raise ValueError("drF has one entry per level")
    grid = [_grid(getattr(g, k), dev, shape2d) for k in ("dyG", "dxG", "recip_dxC", "recip_dyC", "rA")]
    rBo = _grid(recip_Bo, dev, shape2d)
    outs = [torch.empty((B,) + shape2d, dtype=torch.float64, device=dev) for _ in range(3)]
    pre = [_batch2(a, dev, shape2d, B).clone() for a in (pW, pS, pC)]
    nval, narr = _norm(cp.cg2dNorm, dev, B)
    capi.check(capi.lib().cg2d_update_operator(
        ex.handle(dev), B, _fs(p, Nr), nval, _ptr(narr), float(cp.cg2dpcOffDFac), hW.data_ptr(), hS.data_ptr(),
        drF.data_ptr(), *(t.data_ptr() for t in grid), rBo.data_ptr(), *(t.data_ptr() for t in outs),
        *(t.data_ptr() for t in pre), _stream(dev)), "cg2d_update_operator")
    return tuple(back(t.reshape(lead + shape2d)) for t in outs + pre)


def cg2d_rhs(p, g, gU, gV, hFacW, hFacS, EmPmR, etaN, etaH, Bo_surf, *, ex=None):
    """cg2d_rhs (solve_for_pressure.py:68-106) on the GPU: (cg2d_b, cg2d_x). The layout comes from g.layout as in
    the reference (generated LLC maps), or from the Exchanger `ex` when given."""
    if ex is None:
        ex = default_exchanger(g.layout)
    shape2d = tuple(ex.L.shape2d)
    u, back = _dev(gU)
    dev = u.device
    u, lead = _batch3(u, dev, shape2d)
    B, Nr = u.shape[0], u.shape[2]
    v, hW, hS = (_batch3(a, dev, shape2d)[0] for a in (gV, hFacW, hFacS))
    em, en, eh = (_batch2(a, dev, shape2d, B) for a in (EmPmR, etaN, etaH))
    drF = _dev(np.asarray(g.drF, np.float64) if not isinstance(g.drF, torch.Tensor) else g.drF, dev)[0]
    grid = [_grid(getattr(g, k), dev, shape2d) for k in ("dyG", "dxG", "rA", "maskInC")]
    bo = _grid(Bo_surf, dev, shape2d)
    b = torch.empty((B,) + shape2d, dtype=torch.float64, device=dev)
    x = torch.empty_like(b)
    capi.check(capi.lib().cg2d_pressure_rhs(
        ex.handle(dev), B, _fs(p, Nr), u.data_ptr(), v.data_ptr(), hW.data_ptr(), hS.data_ptr(), em.data_ptr(),
        en.data_ptr(), eh.data_ptr(), drF.data_ptr(), *(t.data_ptr() for t in grid), bo.data_ptr(), b.data_ptr(),
        x.data_ptr(), _stream(dev)), "cg2d_pressure_rhs")
    return back(b.reshape(lead + shape2d)), back(x.reshape(lead + shape2d))


def pressure_post(ex, x, cg2d_x, recip_Bo):
    """After the solve (solve_for_pressure.py:116-121): etaN = recip_Bo x, with x exchanged (the first guess where
    the exchange writes nothing)."""
    shape2d = tuple(ex.L.shape2d)
    xt, back = _dev(x)
    dev = xt.device
    lead = tuple(xt.shape[:-3])
    xt = xt.reshape((-1,) + shape2d).contiguous()
    B = xt.shape[0]
    x0 = _batch2(cg2d_x, dev, shape2d, B)
    rBo = _grid(recip_Bo, dev, shape2d)
    eta = torch.empty_like(xt)
    capi.check(capi.lib().cg2d_pressure_post(ex.handle(dev), B, xt.data_ptr(), x0.data_ptr(), rBo.data_ptr(),
                                             eta.data_ptr(), _stream(dev)), "cg2d_pressure_post")
    return back(eta.reshape(lead + shape2d))


def solve_for_pressure(p, cp, g, ex, ops, gU, gV, hFacW, hFacS, EmPmR, etaN, etaH, Bo_surf, recip_Bo):
    """solve_for_pressure (solve_for_pressure.py:109-123) on the GPU: the right-hand side and first guess, the CG2D
    solve (cg2d_solve with cp: sum order, precision, tolerance, iteration cap), the exchange of the solution and
    etaN = recip_Bo x. Returns (etaN, info): info holds the CG2D diagnostics, cg2d_b and cg2d_x0 (the first guess)."""
    cg2d_b, cg2d_x = cg2d_rhs(p, g, gU, gV, hFacW, hFacS, EmPmR, etaN, etaH, Bo_surf, ex=ex)
    x, diag = cg2d_solve(cp, ex, ops, cg2d_b, cg2d_x)
    eta = pressure_post(ex, x, cg2d_x, recip_Bo)
    if isinstance(diag, dict):
        info = dict(diag, cg2d_b=cg2d_b, cg2d_x0=cg2d_x)
    else:
        info = dict(records=diag, cg2d_b=cg2d_b, cg2d_x0=cg2d_x)
    return eta, info
