"""The differentiable GPU solve (Cg2dSolve, implicit derivative of cg2d.py:318-348) against finite differences,
the transpose-solve identities and the ECCO passive-operator mode (test designs of test_cg2d.py:214-300)."""

import numpy as np
import pytest
import torch

from golden_cases import load
from oracle import cg2d_oracle as O

pytestmark = pytest.mark.gpu

cg = pytest.importorskip("mit_jax_b200.cg2d")


@pytest.fixture(scope="module")
def prob():
    from mit_jax_b200.synthetic import LLCSynthetic
    syn = LLCSynthetic(32, 16, 4)
    ops, norm = syn.operator()
    ex = cg.Exchanger(syn.L, syn.topo.maps)
    return syn, ex, ops, norm


def _t(a, grad=False):
    t = torch.as_tensor(np.asarray(a, np.float64)).cuda()
    return t.requires_grad_(grad)


def test_transpose_solve_identities(prob):
    """z = dJ/db for J = <w, x(b)> solves A z = w (relative residual < 1e-11), is 0 on halo points, and
    <z, b> = <w, x> with x from a forward solve at 1e-13 (to 1e-9)."""
    syn, ex, ops, norm = prob
    L = syn.L
    inner = O.interior_mask(L)
    w = np.random.default_rng(1).standard_normal(L.shape2d) * inner
    p = cg.Cg2dParams(cg2dMaxIters=300, cg2dTolerance=1e-12, cg2dNorm=norm, sum_order="rowblock")
    b = _t(syn.rhs(), True)
    x, _ = cg.cg2d_solve(p, ex, tuple(_t(a) for a in ops), b, _t(syn.first_guess()))
    (x * _t(w)).sum().backward()
    z = b.grad.cpu().numpy()
    assert np.all(np.isfinite(z)) and np.all(z[:, ~inner] == 0.0)
    res = np.abs(O.matvec(L, syn.topo.maps["T"], ops[:3], norm, z) - w).max() / np.abs(w).max()
    assert res < 1e-11, res
    pt = cg.Cg2dParams(cg2dMaxIters=1000, cg2dTolerance=1e-13, cg2dNorm=norm, sum_order="rowblock")
    xt, _ = cg.cg2d_solve(pt, ex, ops, syn.rhs(), syn.first_guess())
    np.testing.assert_allclose(np.vdot(z, syn.rhs()), np.vdot(w, xt), rtol=1e-9)


def test_gradients_match_central_differences(prob):
    """d/d(aW2d), d/d(aC2d), d/d(cg2d_b) of J = <w, x> against central differences along random directions on a
    3x3 window, h-sweep, tolerances 1e-6 / 1e-5 / 1e-8 (test_cg2d.py:240-277)."""
    syn, ex, ops, norm = prob
    L = syn.L
    rng = np.random.default_rng(2)
    w = rng.standard_normal(L.shape2d) * O.interior_mask(L)
    p = cg.Cg2dParams(cg2dMaxIters=300, cg2dTolerance=1e-12, cg2dNorm=norm, sum_order="rowblock")
    tight = cg.Cg2dParams(cg2dMaxIters=1000, cg2dTolerance=1e-13, cg2dNorm=norm, sum_order="rowblock")
    x0 = syn.first_guess()

    def J(params, aW, aC, b):
        x, _ = cg.cg2d_solve(params, ex, (aW, ops[1], aC, *ops[3:]), b, x0)
        return float(np.vdot(w, x))

    aW_t, aC_t, b_t = _t(ops[0], True), _t(ops[2], True), _t(syn.rhs(), True)
    x, _ = cg.cg2d_solve(p, ex, (aW_t, _t(ops[1]), aC_t, *(_t(a) for a in ops[3:])), b_t, _t(x0))
    (x * _t(w)).sum().backward()
    grads = [aW_t.grad.cpu().numpy(), aC_t.grad.cpu().numpy(), b_t.grad.cpu().numpy()]
    base = [ops[0], ops[2], syn.rhs()]
    # a 3x3 window whose west faces are all wet (first one found scanning tile 4, then the others)
    Jw, Iw = L.interior
    found = None
    for t in (4, 3, 5, 1, 7, 8):
        for j in range(Jw.start, Jw.stop - 2):
            for i in range(Iw.start, Iw.stop - 2):
                if np.all(ops[0][t, j:j + 3, i:i + 3] != 0):
                    found = (t, j, i)
                    break
            if found:
                break
        if found:
            break
    t, j0, i0 = found
    for k, name, hs, tol in ((0, "aW2d", (1e-2, 1e-3, 1e-4, 1e-5), 1e-6), (1, "aC2d", (1e-3, 1e-4, 1e-5), 1e-5),
                             (2, "cg2d_b", (1e-1, 1e-2, 1e-3), 1e-8)):
        win = base[k][t, j0:j0 + 3, i0:i0 + 3]
        d = np.zeros(L.shape2d)
        d[t, j0:j0 + 3, i0:i0 + 3] = rng.standard_normal((3, 3)) * np.abs(win).max()
        gd = float(np.vdot(grads[k], d))
        errs = []
        for h in hs:
            plus = [a + h * d if n == k else a for n, a in enumerate(base)]
            minus = [a - h * d if n == k else a for n, a in enumerate(base)]
            fd = (J(tight, *plus) - J(tight, *minus)) / (2 * h)
            errs.append(abs(fd - gd) / abs(gd))
        assert min(errs) < tol, (name, errs)


def test_ecco_mode_stops_coefficient_gradient(prob):
    """stop_coeff_grad=True: forward bitwise equal to the exact mode, d/d(aC2d) exactly 0 (no gradient), d/d(b)
    unchanged (test_cg2d.py:280-300)."""
    syn, ex, ops, norm = prob
    L = syn.L
    w = _t(np.random.default_rng(4).standard_normal(L.shape2d) * O.interior_mask(L))
    out = {}
    for mode in (False, True):
        p = cg.Cg2dParams(cg2dMaxIters=300, cg2dTolerance=1e-12, cg2dNorm=norm, sum_order="rowblock",
                          stop_coeff_grad=mode)
        aC, b = _t(ops[2], True), _t(syn.rhs(), True)
        x, _ = cg.cg2d_solve(p, ex, (_t(ops[0]), _t(ops[1]), aC, *(_t(a) for a in ops[3:])), b,
                             _t(syn.first_guess()))
        (x * w).sum().backward()
        out[mode] = (x.detach().cpu().numpy(), aC.grad, b.grad.cpu().numpy())
    np.testing.assert_array_equal(out[True][0], out[False][0])
    assert out[False][1] is not None and torch.abs(out[False][1]).max() > 0
    assert out[True][1] is None or torch.all(out[True][1] == 0)
    np.testing.assert_array_equal(out[True][2], out[False][2])


def test_adjoint_coefficient_gradient_equals_oracle():
    """Edge products of the GPU adjoint solution equal the oracle's coefficient cotangents of the same lam, x."""
    c = load("llc16_guess")
    ex = cg.Exchanger(c.L, c.topo.maps)
    x, _ = O.cg2d_fortran(c.L, c.tmap, c.ops, c.b, c.x0, cg2dNorm=c.norm, tolerance=1e-12, max_iters=300,
                          sum_order="rowblock")
    inner = O.interior_mask(c.L)
    x = np.where(inner, x, 0.0)
    w = np.random.default_rng(9).standard_normal(c.L.shape2d) * inner
    lam, _ = O.tight_solve(c.L, c.tmap, c.ops, w, cg2dNorm=c.norm)
    got = cg.edge_products(ex, lam, x, c.norm)
    ref = O.coefficient_cotangents(c.L, c.tmap, lam, x, c.norm)
    for g, r in zip(got, ref):
        np.testing.assert_array_equal(g, r)
