"""Oracle of the exact-mode adjoint -- TEST INFRASTRUCTURE ONLY.

The reference has no adjoint that reverses through the CG iterations: its JAX code cannot reverse a while_loop and
differentiates cg2d implicitly (mitgcm_jax/core/cg2d.py:307-348). The exact mode is therefore checked against
torch autograd (float64, CPU) through a Python loop of the iterations of cg2d_fortran (cg2d.py:205-269, restated
as in cg2d_oracle.cg2d_fortran: the same stencils, exchange and normalisation) with the iteration count fixed to
the forward's. The dot products are torch sums, not the solver's ordered sums: the oracle and the GPU agree to
rounding, not bit for bit. Only tests import this module.
"""

import numpy as np
import torch
import torch.nn.functional as F

from oracle.cg2d_oracle import exch


def _apply_operator(L, aW, aS, aC, x):
    """cg2d.py:181-188 on torch tensors (the five products added left to right)."""
    J, I, Jm, Jp, Im, Ip = L.js(1, L.sNy), L.is_(1, L.sNx), L.js(0, L.sNy - 1), L.js(2, L.sNy + 1), \
        L.is_(0, L.sNx - 1), L.is_(2, L.sNx + 1)
    return (aW[..., J, I] * x[..., J, Im] + aW[..., J, Ip] * x[..., J, Ip] + aS[..., J, I] * x[..., Jm, I]
            + aS[..., Jp, I] * x[..., Jp, I] + aC[..., J, I] * x[..., J, I])


def _apply_preconditioner(L, pW, pS, pC, r):
    """cg2d.py:191-198 on torch tensors."""
    J, I, Jm, Jp, Im, Ip = L.js(1, L.sNy), L.is_(1, L.sNx), L.js(0, L.sNy - 1), L.js(2, L.sNy + 1), \
        L.is_(0, L.sNx - 1), L.is_(2, L.sNx + 1)
    return (pC[..., J, I] * r[..., J, I] + pW[..., J, I] * r[..., J, Im] + pW[..., J, Ip] * r[..., J, Ip]
            + pS[..., J, I] * r[..., Jm, I] + pS[..., Jp, I] * r[..., Jp, I])


def cg2d_exact_grad(L, tmap, ops, cg2d_b, cg2d_x, x_bar, *, cg2dNorm, iters):
    """Cotangents of J = <x_bar, x> for x = the interior of cg2d_fortran after exactly `iters` iterations, with
    respect to cg2d_b and to ops = (aW2d, aS2d, aC2d, pW, pS, pC); cg2d_x (the first guess) is constant
    (cg2d.py:372). Returns (x, dict of numpy arrays [T, ny, nx] keyed "b", "aW2d", ..., "pC")."""
    names = ("aW2d", "aS2d", "aC2d", "pW", "pS", "pC")
    src, comp = np.asarray(tmap[0]), np.asarray(tmap[1])
    dst = torch.as_tensor(np.nonzero(comp == 1)[0])
    srcs = torch.as_tensor(src[comp == 1].astype(np.int64))

    def exch_t(v):
        flat = v.reshape(-1)
        return flat.index_put((dst,), flat[srcs]).reshape(v.shape)

    def ring(v_i):
        return exch_t(F.pad(v_i, (L.OLx, L.OLx, L.OLy, L.OLy)))

    J, I = L.js(1, L.sNy), L.is_(1, L.sNx)
    leaves = {k: torch.tensor(np.asarray(a, np.float64), requires_grad=True) for k, a in zip(names, ops)}
    b = torch.tensor(np.asarray(cg2d_b, np.float64), requires_grad=True)
    aW, aS, aC, pW, pS, pC = (leaves[k] for k in names)
    rhsMax = np.abs(np.asarray(cg2d_b)[:, J, I] * cg2dNorm).max()                # cg2d.py:222-223
    rhsNorm = 1.0 / rhsMax if rhsMax != 0.0 else 1.0                             # cg2d.py:224-225
    x0 = np.asarray(cg2d_x, np.float64).copy()
    x0[:, J, I] = x0[:, J, I] * rhsNorm                                          # cg2d.py:227
    x0 = torch.tensor(exch(x0, tmap))                                            # cg2d.py:228
    bn = b[:, J, I] * cg2dNorm * rhsNorm                                         # cg2d.py:222, 226
    r_i = bn - _apply_operator(L, aW, aS, aC, x0)                                # cg2d.py:232
    r = ring(r_i)
    s_i = torch.zeros_like(r_i)
    x_i = x0[:, J, I]
    eta_prev = torch.tensor(1.0, dtype=torch.float64)
    for _ in range(iters):
        z = _apply_preconditioner(L, pW, pS, pC, r)                              # cg2d.py:245
        eta = (z * r[:, J, I]).sum()                                             # cg2d.py:246
        beta = eta / eta_prev                                                    # cg2d.py:247
        eta_prev = eta
        s_i = z + beta * s_i                                                     # cg2d.py:249
        q = _apply_operator(L, aW, aS, aC, ring(s_i))                            # cg2d.py:251
        alpha = eta / (s_i * q).sum()                                            # cg2d.py:252-253
        x_i = x_i + alpha * s_i                                                  # cg2d.py:254
        r = ring(r[:, J, I] - alpha * q)                                         # cg2d.py:255, 260
    x_out = x_i / rhsNorm                                                        # cg2d.py:266
    xb = torch.tensor(np.asarray(x_bar, np.float64))[:, J, I]
    Jv = (xb * x_out).sum()
    grads = torch.autograd.grad(Jv, [b] + [leaves[k] for k in names], allow_unused=True)
    out = {}
    for k, g in zip(("b",) + names, grads):
        out[k] = np.zeros(np.shape(cg2d_b)) if g is None else g.detach().numpy()
    x = np.zeros(np.shape(cg2d_b))
    x[:, J, I] = x_out.detach().numpy()
    return x, out
