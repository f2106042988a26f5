"""Exact-mode adjoint on the GPU (reverse mode through the CG iterations the forward took: cg2d_solve_exact, and
the two-call cg2d_adjoint_exact): the recording forward equals the FP64 solve bit for bit, and both paths give the
same gradients bit for bit; the gradients equal torch autograd through the same iterations
(oracle/cg2d_exact_oracle.py) to rounding, for single and batched solves, whatever the checkpoint interval, and
central differences; at a tight tolerance they approach the implicit derivative (measured here, not assumed)."""

import numpy as np
import pytest
import torch

from mit_jax_b200.topology import exch_vector_adjoint
from oracle import cg2d_oracle as O
from oracle.cg2d_exact_oracle import cg2d_exact_grad

pytestmark = pytest.mark.gpu

cg = pytest.importorskip("mit_jax_b200.cg2d")
NAMES = ("b",) + cg.OPS


def _np(a):
    return a.detach().cpu().numpy() if isinstance(a, torch.Tensor) else np.asarray(a)


def _rel(a, b):
    a, b = _np(a), _np(b)
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.fixture(scope="module")
def small():
    from mit_jax_b200.synthetic import LLCSynthetic
    syn = LLCSynthetic(16, 8, 4)
    return syn, cg.default_exchanger(syn.L)


def test_exact_adjoint_matches_autograd(small):
    """Six iterations (tolerance 0): every gradient equals autograd's; converged (1e-12): the recording forward is
    the solve bit for bit, and the gradients in b and in the operator equal autograd's. (At convergence the
    preconditioner moves x only through the residual: its gradients are rounding-level there.)"""
    syn, ex = small
    L, tmap = syn.L, syn.topo.maps["T"]
    inner = O.interior_mask(L)
    ops, norm = syn.operator()
    b, x0 = syn.rhs(), syn.first_guess()
    w = np.random.default_rng(3).standard_normal(L.shape2d) * inner
    x, d, g = cg.exact_adjoint(ex, ops, b, x0, w, cg2dNorm=norm, tolerance=0.0, max_iters=6, checkpoint_every=4)
    assert d["numIters"] == 6
    _, go = cg2d_exact_grad(L, tmap, ops, b, x0, w, cg2dNorm=norm, iters=6)
    for k in NAMES:
        assert _rel(g[k], go[k]) < 1e-10, (k, _rel(g[k], go[k]))
    x, d, g = cg.exact_adjoint(ex, ops, b, x0, w, cg2dNorm=norm, tolerance=1e-12, max_iters=300,
                               checkpoint_every=10, x_check=True)
    np.testing.assert_array_equal(_np(g["x_check"])[:, inner], _np(x)[:, inner])
    xo, go = cg2d_exact_grad(L, tmap, ops, b, x0, w, cg2dNorm=norm, iters=d["numIters"])
    assert _rel(_np(x), xo) < 1e-13
    for k in ("b", "aW2d", "aS2d", "aC2d"):
        assert _rel(g[k], go[k]) < 1e-8, (k, _rel(g[k], go[k]))


def test_exact_adjoint_checkpoints_and_batch(small):
    """Three members with their own operators and iteration counts in one call; checkpoint intervals 0 (one
    segment), 4 and 30 give the same gradients bit for bit, each equal to its member's autograd gradient (b and
    the operator)."""
    from mit_jax_b200.synthetic import make_batch
    syn, B = make_batch(16, ts=8, members=[0, 1, 2])
    ex = cg.default_exchanger(syn.L)
    L, tmap = syn.L, syn.topo.maps["T"]
    # right-hand sides whose oracle solves take 37, 39 and 36 iterations at tolerance 1e-12
    B["b"][1] = O.interior_mask(L).astype(np.float64)
    B["b"][2] = B["b"][2] ** 2 * np.sign(B["b"][2])
    rng = np.random.default_rng(4)
    w = rng.standard_normal((3,) + L.shape2d) * O.interior_mask(L)
    ops = tuple(torch.as_tensor(B[k]).cuda() for k in cg.OPS)
    norm = torch.as_tensor(B["cg2dNorm"])
    runs = [cg.exact_adjoint(ex, ops, torch.as_tensor(B["b"]).cuda(), torch.as_tensor(B["x0"]).cuda(),
                             torch.as_tensor(w).cuda(), cg2dNorm=norm, tolerance=1e-12, max_iters=300,
                             checkpoint_every=c) for c in (0, 4, 30)]
    for _, _, g in runs[1:]:
        for k in NAMES:
            torch.testing.assert_close(g[k], runs[0][2][k], rtol=0, atol=0)
    x, d, g = runs[0]
    assert len({r["numIters"] for r in d}) == 3, [r["numIters"] for r in d]
    for m in range(3):
        ops_m = tuple(B[k][m] for k in cg.OPS)
        _, go = cg2d_exact_grad(L, tmap, ops_m, B["b"][m], B["x0"][m], w[m], cg2dNorm=B["cg2dNorm"][m],
                                iters=d[m]["numIters"])
        for k in ("b", "aW2d", "aS2d", "aC2d"):
            assert _rel(g[k][m], go[k]) < 1e-8, (m, k)


def test_exact_adjoint_approaches_implicit(small):
    """At tolerance 1e-13 the exact derivative of the iteration and the implicit derivative of the converged
    solution (cg2d.py:318-348) differ by O(residual): here well below 1e-6 relative in d/db and, per face (after
    the transpose of the face exchange), in d/d(aW2d) and d/d(aS2d)."""
    syn, ex = small
    L = syn.L
    ops, norm = syn.operator()
    b, x0 = syn.rhs(), syn.first_guess()
    w = np.random.default_rng(5).standard_normal(L.shape2d) * O.interior_mask(L)
    _, _, g = cg.exact_adjoint(ex, ops, b, x0, w, cg2dNorm=norm, tolerance=1e-13, max_iters=1000)
    p = cg.Cg2dParams(cg2dMaxIters=1000, cg2dTolerance=1e-13, cg2dNorm=norm, sum_order="rowblock")
    bt = torch.as_tensor(b).cuda().requires_grad_(True)
    opt = [torch.as_tensor(a).cuda().requires_grad_(i < 3) for i, a in enumerate(ops)]
    xi, _ = cg.cg2d_solve(p, ex, tuple(opt), bt, torch.as_tensor(x0).cuda())
    (xi * torch.as_tensor(w).cuda()).sum().backward()
    assert _rel(g["b"], bt.grad) < 1e-6
    maps_u, maps_v = syn.topo.maps["UVn_u"], syn.topo.maps["UVn_v"]
    eu, ev = exch_vector_adjoint(_np(g["aW2d"]), _np(g["aS2d"]), maps_u, maps_v)
    iu, iv = exch_vector_adjoint(_np(opt[0].grad), _np(opt[1].grad), maps_u, maps_v)
    assert _rel(eu, iu) < 1e-6 and _rel(ev, iv) < 1e-6


def test_exact_adjoint_finite_differences(small):
    """The exact derivative of the iteration map: at a fixed iteration count (tolerance 0, 20 iterations) the
    solution is a nonlinear function of b and of the coefficients; the directional derivative <g, d> equals the
    central difference (J(p + h d) - J(p - h d)) / 2h, h = 1e-6 relative, on random directions of b, aW2d and
    aS2d, to 1e-6 relative."""
    syn, ex = small
    L = syn.L
    inner = O.interior_mask(L)
    ops, norm = syn.operator()
    ops = tuple(torch.as_tensor(a).cuda() for a in ops)
    b, x0 = torch.as_tensor(syn.rhs()).cuda(), torch.as_tensor(syn.first_guess()).cuda()
    w = torch.as_tensor(np.random.default_rng(6).standard_normal(L.shape2d) * inner).cuda()
    kw = dict(cg2dNorm=norm, tolerance=0.0, max_iters=20, checkpoint_every=7)

    def J(b_, ops_):
        x, d, _ = cg.exact_adjoint(ex, ops_, b_, x0, w, **kw)
        assert d["numIters"] == 20
        return float((x * w).sum())

    _, _, g = cg.exact_adjoint(ex, ops, b, x0, w, **kw)
    rng = np.random.default_rng(7)
    for name in ("b", "aW2d", "aS2d"):
        base = b if name == "b" else ops[cg.OPS.index(name)]
        for _ in range(3):
            dvec = torch.as_tensor(rng.standard_normal(L.shape2d)).cuda() * (base != 0)
            h = 1e-6 * float(base.abs().max()) / float(dvec.abs().max())

            def moved(sign):
                p = base + sign * h * dvec
                if name == "b":
                    return J(p, ops)
                return J(b, tuple(p if k == name else o for k, o in zip(cg.OPS, ops)))

            fd = (moved(1.0) - moved(-1.0)) / (2 * h)
            an = float((g[name] * dvec).sum())
            assert abs(fd - an) <= 1e-6 * abs(an), (name, fd, an)


def test_exact_adjoint_one_pass_equals_recording_forward():
    """The solve storing its own checkpoints and sums (cg2d_solve_exact) gives the two-call path's solution and
    gradients bit for bit: three members with 37, 39 and 36 iterations, checkpoint intervals 0, 7 and 30, and a run
    stopped by the iteration cap at a multiple of the interval (its last checkpoint lands in the spare slot)."""
    from mit_jax_b200.synthetic import make_batch
    syn, B = make_batch(16, ts=8, members=[0, 1, 2])
    ex = cg.default_exchanger(syn.L)
    B["b"][1] = O.interior_mask(syn.L).astype(np.float64)
    B["b"][2] = B["b"][2] ** 2 * np.sign(B["b"][2])
    w = np.random.default_rng(8).standard_normal((3,) + syn.L.shape2d) * O.interior_mask(syn.L)
    ops = tuple(torch.as_tensor(B[k]).cuda() for k in cg.OPS)
    args = (ex, ops, torch.as_tensor(B["b"]).cuda(), torch.as_tensor(B["x0"]).cuda(), torch.as_tensor(w).cuda())
    norm = torch.as_tensor(B["cg2dNorm"])
    for tol, maxit, c in ((1e-12, 300, 0), (1e-12, 300, 7), (1e-12, 300, 30), (0.0, 28, 7)):
        x1, d1, g1 = cg.exact_adjoint(*args, cg2dNorm=norm, tolerance=tol, max_iters=maxit, checkpoint_every=c)
        x2, d2, g2 = cg.exact_adjoint(*args, cg2dNorm=norm, tolerance=tol, max_iters=maxit, checkpoint_every=c,
                                      one_pass=False)
        assert [r["numIters"] for r in d1] == [r["numIters"] for r in d2]
        if tol == 0.0:
            assert [r["numIters"] for r in d1] == [maxit] * 3
        torch.testing.assert_close(x1, x2, rtol=0, atol=0)
        for k in NAMES:
            torch.testing.assert_close(g1[k], g2[k], rtol=0, atol=0, msg=f"{k} checkpoint {c}")
