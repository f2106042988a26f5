"""CPU oracle of the CG2D path -- TEST INFRASTRUCTURE ONLY.

This module is the checker the GPU solver is compared against, and the CPU baseline that bench.py times. Only
tests/, __graft_entry__.smoke() and bench.py's CPU legs may import it; the library never does.

It restates, in numpy, with the same floating-point operations in the same order:
  * Exchanger._apply for a scalar kind          mitgcm_jax/parallel/exchange.py:136-142, 182-183
  * apply_operator / apply_preconditioner       mitgcm_jax/core/cg2d.py:181-198
  * tile_sum ("fortran" order) + global_sum     mitgcm_jax/core/cg2d.py:141-169, mitgcm_jax/parallel/global_sum.py:20-26
  * cg2d_fortran (normalisation, stop rule, diag, halo semantics of the returned array)
                                                mitgcm_jax/core/cg2d.py:205-269
  * _matvec and the implicit-derivative adjoint (tight solve, coefficient cotangents)
                                                mitgcm_jax/core/cg2d.py:292-348
plus what the GPU solver adds: the ROWBLOCK global-sum order and the MIXED-precision iteration (FP32 vectors and
stencils, FP64 dot products and x, periodic FP64 true-residual replacement).

Parity pin: cg2d_fortran here with sum_order="fortran" is checked bit for bit against the reference's own
cg2d_fortran, run through a numpy stand-in for JAX, on the committed fixtures in tests/golden
(tests/golden/make_golden.py).
"""

import numpy as np

# ------------------------------------------------------------------------------------------------------------
# exchange and stencils


def exch(a, tmap):
    """Scalar exchange (exchange.py:136-142): out[p] = a[src[p]] where comp[p] == 1, else a[p] (sign +1)."""
    src, comp = tmap[0], tmap[1]
    a = np.asarray(a)
    flat = a.reshape(a.shape[:-3] + (-1,))
    return np.where(comp == 1, flat[..., src], flat).reshape(a.shape)


def _slices(L):
    J, I = L.js(1, L.sNy), L.is_(1, L.sNx)
    return J, I, L.js(0, L.sNy - 1), L.js(2, L.sNy + 1), L.is_(0, L.sNx - 1), L.is_(2, L.sNx + 1)


def apply_operator(L, aW, aS, aC, x):
    """cg2d.py:181-188, the same five products added left to right."""
    J, I, Jm, Jp, Im, Ip = _slices(L)
    return (aW[..., J, I] * x[..., J, Im] + aW[..., J, Ip] * x[..., J, Ip] + aS[..., J, I] * x[..., Jm, I]
            + aS[..., Jp, I] * x[..., Jp, I] + aC[..., J, I] * x[..., J, I])


def apply_preconditioner(L, pW, pS, pC, r):
    """cg2d.py:191-198."""
    J, I, Jm, Jp, Im, Ip = _slices(L)
    return (pC[..., J, I] * r[..., J, I] + pW[..., J, I] * r[..., J, Im] + pW[..., J, Ip] * r[..., J, Ip]
            + pS[..., J, I] * r[..., Jm, I] + pS[..., Jp, I] * r[..., Jp, I])


# ------------------------------------------------------------------------------------------------------------
# sums


def tile_sum_fortran(a):
    """[T, nj, ni] -> [T]: s = 0; DO j; DO i; s = s + a(i,j) (cg2d.py:141-161), strictly sequential."""
    T = a.shape[0]
    flat = np.concatenate([np.zeros((T, 1)), a.reshape(T, -1)], axis=1)
    return np.add.accumulate(flat, axis=1)[:, -1]


def tile_sum_rowblock(a, rows_per_block=8):
    """[T, nj, ni] -> [T], the GPU solver's ROWBLOCK order: per row, lane l sums a[l], a[l+32], ... from 0, then
    an xor butterfly over the 32 lanes (lane l + lane l^m for m = 16, 8, 4, 2, 1); rows of a block added in order
    from 0; blocks of a tile in order from 0."""
    T, nj, ni = a.shape
    nk = -(-ni // 32)
    pad = np.zeros((T, nj, nk * 32))
    pad[..., :ni] = a
    lanes = pad.reshape(T, nj, nk, 32)
    v = np.zeros((T, nj, 32))
    for k in range(nk):
        v = v + lanes[:, :, k, :]
    idx = np.arange(32)
    for m in (16, 8, 4, 2, 1):
        v = v + v[..., idx ^ m]
    rows = v[..., 0]
    tiles = np.zeros(T)
    for j0 in range(0, nj, rows_per_block):
        blk = np.zeros(T)
        for j in range(j0, min(nj, j0 + rows_per_block)):
            blk = blk + rows[:, j]
        tiles = tiles + blk
    return tiles


def global_sum_tile(phi):
    """global_sum.py:20-26: 0 + tile 1 + tile 2 + ... in order."""
    s = 0.0
    for t in range(phi.shape[0]):
        s = s + phi[t]
    return np.float64(s)


def gsum(a, order, rows_per_block=8):
    if order == "fortran":
        return global_sum_tile(tile_sum_fortran(a))
    if order == "rowblock":
        return global_sum_tile(tile_sum_rowblock(a, rows_per_block))
    if order == "tile":
        return global_sum_tile(np.sum(a, axis=(1, 2)))
    raise ValueError(order)


# ------------------------------------------------------------------------------------------------------------
# the solver


def cg2d_fortran(L, tmap, ops, cg2d_b, cg2d_x, *, cg2dNorm, tolerance, max_iters, sum_order="fortran",
                 rows_per_block=8):
    """cg2d_fortran (cg2d.py:205-269). ops = (aW2d, aS2d, aC2d, pW, pS, pC) [T, ny, nx]; returns (x, diag) with x
    as the reference returns it (interior = solution, halos = exchanged normalised first guess) and
    diag = firstResidual, lastResidual, numIters, sumRHS, rhsMax."""
    aW, aS, aC, pW, pS, pC = (np.asarray(a, np.float64) for a in ops)
    cg2d_b, cg2d_x = np.asarray(cg2d_b, np.float64), np.asarray(cg2d_x, np.float64)
    J, I = L.js(1, L.sNy), L.is_(1, L.sNx)

    def S(a):
        return gsum(a, sum_order, rows_per_block)

    tol2 = tolerance * tolerance                                     # cg2d.py:219
    eta_prev = np.float64(1.0)                                       # cg2d.py:220
    b = cg2d_b[:, J, I] * cg2dNorm                                   # cg2d.py:222
    rhsMax = np.abs(b).max()                                         # cg2d.py:223
    rhsNorm = 1.0 / rhsMax if rhsMax != 0.0 else np.float64(1.0)     # cg2d.py:224-225
    b = b * rhsNorm                                                  # cg2d.py:226
    x = cg2d_x.copy()
    x[:, J, I] = cg2d_x[:, J, I] * rhsNorm                           # cg2d.py:227
    x = exch(x, tmap)                                                # cg2d.py:228
    s = np.zeros_like(cg2d_b)                                        # cg2d.py:231
    r_i = b - apply_operator(L, aW, aS, aC, x)                       # cg2d.py:232
    err_sq = S(r_i * r_i)                                            # cg2d.py:233
    sumRHS = S(b)                                                    # cg2d.py:234
    r = np.zeros_like(cg2d_b)
    r[:, J, I] = r_i
    r = exch(r, tmap)                                                # cg2d.py:235
    firstResidual = np.sqrt(err_sq)
    it = 0
    while it < max_iters and not (err_sq < tol2):                    # cg2d.py:238-241
        q = apply_preconditioner(L, pW, pS, pC, r)                   # cg2d.py:245
        eta = S(q * r[:, J, I])                                      # cg2d.py:246
        beta = eta / eta_prev                                        # cg2d.py:247
        eta_prev = eta
        s_i = q + beta * s[:, J, I]                                  # cg2d.py:249
        s[:, J, I] = s_i
        s = exch(s, tmap)                                            # cg2d.py:250
        q = apply_operator(L, aW, aS, aC, s)                         # cg2d.py:251
        alpha = eta / S(s_i * q)                                     # cg2d.py:252-253
        x[:, J, I] = x[:, J, I] + alpha * s_i                        # cg2d.py:254
        r_i = r[:, J, I] - alpha * q                                 # cg2d.py:255
        err_sq = S(r_i * r_i)                                        # cg2d.py:256
        r[:, J, I] = r_i
        r = exch(r, tmap)                                            # cg2d.py:260
        it += 1
    x[:, J, I] = x[:, J, I] / rhsNorm                                # cg2d.py:266
    diag = dict(firstResidual=firstResidual, lastResidual=np.sqrt(err_sq), numIters=it, sumRHS=sumRHS,
                rhsMax=rhsMax)
    return x, diag


def cg2d_mixed(L, tmap, ops, cg2d_b, cg2d_x, *, cg2dNorm, tolerance, max_iters, replace_every=25,
               replace_above=100.0, rows_per_block=8):
    """The GPU solver's MIXED iteration, operation for operation: r, s, z, q and the stencil coefficients in
    float32 (float32 stencil arithmetic and float32 updates s = z + float32(beta) s, r = r - float32(alpha) q), x and
    every dot product in float64 (products of float32 values are exact in float64). At iteration k (0-based) with
    (k+1) % replace_every == 0, while the residual entering the iteration is above replace_above * tolerance, the
    updated r is instead the float64 true residual b - A x (float64 operator), and z = M r, eta follow from it.
    The stop rule is the reference's, on the residual the iteration carries (cg2d.py:238-241).
    Returns (x, diag) like cg2d_fortran plus diag['replacements']."""
    aW, aS, aC, pW, pS, pC = (np.asarray(a, np.float64) for a in ops)
    aW32, aS32, aC32, pW32, pS32, pC32 = (a.astype(np.float32) for a in (aW, aS, aC, pW, pS, pC))
    cg2d_b, cg2d_x = np.asarray(cg2d_b, np.float64), np.asarray(cg2d_x, np.float64)
    J, I = L.js(1, L.sNy), L.is_(1, L.sNx)

    def S(a):
        return gsum(np.asarray(a, np.float64), "rowblock", rows_per_block)

    def ex32(v):
        full = np.zeros(L.shape2d, np.float32)
        full[:, J, I] = v
        return exch(full, tmap)

    tol2 = tolerance * tolerance
    thresh2 = (replace_above * tolerance) * (replace_above * tolerance)
    b = cg2d_b[:, J, I] * cg2dNorm
    rhsMax = np.abs(b).max()
    rhsNorm = 1.0 / rhsMax if rhsMax != 0.0 else np.float64(1.0)
    b = b * rhsNorm
    x_full = cg2d_x.copy()
    x_full[:, J, I] = cg2d_x[:, J, I] * rhsNorm
    x_out_halo = exch(x_full, tmap)
    x = x_full[:, J, I].copy()

    def true_residual(xi):
        xf = cg2d_x.copy()                       # unwritten halo points keep cg2d_x
        xf[:, J, I] = xi
        return (b - apply_operator(L, aW, aS, aC, exch(xf, tmap))).astype(np.float32)

    def precond(r32):
        z = apply_preconditioner(L, pW32, pS32, pC32, ex32(r32))
        return z, S(z.astype(np.float64) * r32.astype(np.float64))

    r = true_residual(x)
    err_sq = S(r.astype(np.float64) ** 2)
    sumRHS = S(b)
    firstResidual = np.sqrt(err_sq)
    z, eta = precond(r)
    s = np.zeros_like(r)
    eta_prev = np.float64(1.0)
    it = 0
    nrep = 0
    while it < max_iters and not (err_sq < tol2):
        beta = eta / eta_prev
        eta_prev = eta
        s = z + np.float32(beta) * s
        q = apply_operator(L, aW32, aS32, aC32, ex32(s))
        alpha = eta / S(s.astype(np.float64) * q.astype(np.float64))
        x = x + alpha * s.astype(np.float64)
        if replace_every > 0 and (it + 1) % replace_every == 0 and err_sq > thresh2:
            r = true_residual(x)
            nrep += 1
        else:
            r = r - np.float32(alpha) * q
        err_sq = S(r.astype(np.float64) ** 2)
        z, eta = precond(r)
        it += 1
    xo = x_out_halo.copy()
    xo[:, J, I] = x / rhsNorm
    diag = dict(firstResidual=firstResidual, lastResidual=np.sqrt(err_sq), numIters=it, sumRHS=sumRHS,
                rhsMax=rhsMax, replacements=nrep)
    return xo, diag


# ------------------------------------------------------------------------------------------------------------
# derivative pieces (cg2d.py:292-348)


def interior_mask(L):
    m = np.zeros((L.ny, L.nx), bool)
    m[L.js(1, L.sNy), L.is_(1, L.sNx)] = True
    return m


def matvec(L, tmap, A, cg2dNorm, v):
    """_matvec (cg2d.py:292-298): (A / cg2dNorm) v on the interior, 0 on halo points."""
    inner = interior_mask(L)
    J, I = L.js(1, L.sNy), L.is_(1, L.sNx)
    xe = exch(np.where(inner, v, 0.0), tmap)
    out = np.zeros_like(np.asarray(v, np.float64))
    out[:, J, I] = apply_operator(L, *A, xe) / cg2dNorm
    return out


def tight_solve(L, tmap, ops, r, *, cg2dNorm, tolerance=1e-13, max_iters=2000, sum_order="rowblock"):
    """tight / tight_transpose (cg2d.py:333-344): the same CG from a zero first guess on the interior of r;
    the result is 0 on halo points."""
    inner = interior_mask(L)
    y, d = cg2d_fortran(L, tmap, ops, np.where(inner, r, 0.0), np.zeros_like(r), cg2dNorm=cg2dNorm,
                        tolerance=tolerance, max_iters=max_iters, sum_order=sum_order)
    return np.where(inner, y, 0.0), d


def coefficient_cotangents(L, tmap, lam, x, cg2dNorm):
    """Cotangents of aW2d, aS2d, aC2d for rhs = db - _matvec(dA, x) (cg2d.py:331): the transpose of the map
    dA -> (dA / cg2dNorm) xe applied to lam, negated. Returns (gW, gS, gC) [T, ny, nx], 0 where the operator
    reads no coefficient."""
    inner = interior_mask(L)
    J, I, Jm, Jp, Im, Ip = _slices(L)
    xe = exch(np.where(inner, x, 0.0), tmap)
    c = np.zeros_like(xe)
    c[:, J, I] = lam[:, J, I] / cg2dNorm
    gW, gS, gC = np.zeros_like(xe), np.zeros_like(xe), np.zeros_like(xe)
    # aW2d(i) multiplies x(i-1) at point i; aW2d(i+1) multiplies x(i+1) at point i
    J1, I1 = L.js(1, L.sNy), L.is_(1, L.sNx + 1)
    t1 = np.zeros_like(xe)
    t1[:, J, I] = c[:, J, I] * xe[:, J, Im]
    t2 = np.zeros_like(xe)
    t2[:, J, Ip] = c[:, J, I] * xe[:, J, Ip]
    gW[:, J1, I1] = -(t1[:, J1, I1] + t2[:, J1, I1])
    J1s, I1s = L.js(1, L.sNy + 1), L.is_(1, L.sNx)
    u1 = np.zeros_like(xe)
    u1[:, J, I] = c[:, J, I] * xe[:, Jm, I]
    u2 = np.zeros_like(xe)
    u2[:, Jp, I] = c[:, J, I] * xe[:, Jp, I]
    gS[:, J1s, I1s] = -(u1[:, J1s, I1s] + u2[:, J1s, I1s])
    gC[:, J, I] = -(c[:, J, I] * xe[:, J, I])
    return gW, gS, gC
