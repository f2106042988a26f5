"""The exact-mode adjoint oracle (torch autograd through the CG2D iterations, oracle/cg2d_exact_oracle.py) pinned
on CPU: its forward equals cg2d_fortran (ROWBLOCK) to rounding, its gradients equal central differences of the
same fixed-iteration map, and converged they equal the implicit derivative per face."""

import numpy as np

from mit_jax_b200.synthetic import LLCSynthetic
from mit_jax_b200.topology import exch_vector_adjoint
from oracle import cg2d_oracle as O
from oracle.cg2d_exact_oracle import cg2d_exact_grad


def test_exact_oracle_forward_and_finite_differences():
    syn = LLCSynthetic(16, 8, 4)
    ops, norm = syn.operator()
    L, tmap = syn.L, syn.topo.maps["T"]
    b, x0 = syn.rhs(), syn.first_guess()
    xf, d = O.cg2d_fortran(L, tmap, ops, b, x0, cg2dNorm=norm, tolerance=1e-12, max_iters=300,
                           sum_order="rowblock")
    K = d["numIters"]
    inner = O.interior_mask(L)
    w = np.random.default_rng(0).standard_normal(L.shape2d) * inner
    x, g = cg2d_exact_grad(L, tmap, ops, b, x0, w, cg2dNorm=norm, iters=K)
    assert np.abs(x[:, inner] - xf[:, inner]).max() <= 1e-13 * np.abs(xf[:, inner]).max()

    # gradients against central differences after 6 iterations, where x still depends strongly on every input
    # (at convergence the preconditioner moves J only through the residual, below what differences resolve)
    K6 = 6
    _, g = cg2d_exact_grad(L, tmap, ops, b, x0, w, cg2dNorm=norm, iters=K6)

    def J(bb, oo):
        xx, _ = cg2d_exact_grad(L, tmap, oo, bb, x0, w, cg2dNorm=norm, iters=K6)
        return float((w * xx).sum())

    rng = np.random.default_rng(1)
    db = rng.standard_normal(L.shape2d) * inner
    h = 1e-6 * np.abs(b).max()
    fd = (J(b + h * db, ops) - J(b - h * db, ops)) / (2 * h)
    ad = float((g["b"] * db).sum())
    assert abs(fd - ad) <= 1e-6 * abs(ad), (fd, ad)
    for k, name in ((0, "aW2d"), (1, "aS2d"), (2, "aC2d"), (3, "pW"), (5, "pC")):
        da = rng.standard_normal(L.shape2d)
        hh = 1e-6 * np.abs(ops[k]).max()
        o1, o2 = list(ops), list(ops)
        o1[k], o2[k] = ops[k] + hh * da, ops[k] - hh * da
        fd = (J(b, o1) - J(b, o2)) / (2 * hh)
        ad = float((g[name] * da).sum())
        assert abs(fd - ad) <= 1e-6 * abs(ad), (name, fd, ad)


def test_exact_oracle_against_implicit_per_face():
    """Converged (tolerance 1e-13), the exact derivative of the iteration and the implicit derivative of the
    solution (cg2d.py:318-348) agree in b, in aC2d and in every face coefficient: per face after the transpose of
    the face exchange adds each halo face entry's cotangent onto the edge entry it copies. Per array entry they
    agree away from tile edges only: moving one of the two stored copies of a tile-edge face alone makes the
    operator unsymmetric, a direction in which the derivative of the CG iterates is not that of A^-1 b."""
    syn = LLCSynthetic(16, 8, 4)
    ops, norm = syn.operator()
    L, tmap = syn.L, syn.topo.maps["T"]
    b, x0 = syn.rhs(), np.zeros(L.shape2d)
    inner = O.interior_mask(L)
    w = np.random.default_rng(2).standard_normal(L.shape2d) * inner
    x, d = O.cg2d_fortran(L, tmap, ops, b, x0, cg2dNorm=norm, tolerance=1e-13, max_iters=1000,
                          sum_order="rowblock")
    _, g = cg2d_exact_grad(L, tmap, ops, b, x0, w, cg2dNorm=norm, iters=d["numIters"])
    lam, _ = O.tight_solve(L, tmap, ops, w, cg2dNorm=norm, tolerance=1e-13, max_iters=1000)
    gW, gS, gC = O.coefficient_cotangents(L, tmap, lam, np.where(inner, x, 0.0), norm)

    def rel(a, ref):
        return np.abs(a - ref).max() / np.abs(ref).max()

    assert rel(g["b"], lam) < 1e-9
    assert rel(g["aC2d"], gC) < 1e-9
    maps_u, maps_v = syn.topo.maps["UVn_u"], syn.topo.maps["UVn_v"]
    eu, ev = exch_vector_adjoint(g["aW2d"], g["aS2d"], maps_u, maps_v)
    iu, iv = exch_vector_adjoint(gW, gS, maps_u, maps_v)
    assert rel(eu, iu) < 1e-9 and rel(ev, iv) < 1e-9, (rel(eu, iu), rel(ev, iv))
    off_edge = np.ones(L.shape2d[-1], bool)
    off_edge[[L.OLx, L.OLx + L.sNx]] = False
    assert rel(g["aW2d"][..., off_edge], gW[..., off_edge]) < 1e-9
