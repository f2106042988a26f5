"""The C entry points cg2d_solve_mixed and cg2d_adjoint_ecco, called through ctypes, against the paths they
package: cg2d_solve_mixed equals solve_groups(precision="mixed") bit for bit; cg2d_adjoint_ecco equals the
backward of cg2d_solve (the tight solve of cg2d.py:333-344 and the edge products) bit for bit, with the operator
active (coefficient cotangents) and passive (the reference's ECCO mode: zero coefficient cotangents)."""

import ctypes

import numpy as np
import pytest
import torch

from mit_jax_b200 import capi

pytestmark = pytest.mark.gpu

cg = pytest.importorskip("mit_jax_b200.cg2d")


def _p(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


@pytest.fixture(scope="module")
def problem():
    from mit_jax_b200.synthetic import LLCSynthetic
    syn = LLCSynthetic(90)
    ops1, norm = syn.operator()
    dev = torch.device("cuda")
    ops = tuple(torch.as_tensor(np.stack([a, a])).to(dev) for a in ops1)       # two instances, one operator
    b = torch.as_tensor(np.stack([syn.rhs(), syn.cotangent()])).to(dev)
    w = torch.as_tensor(np.stack([syn.cotangent(), syn.rhs()])).to(dev)
    return syn, cg.default_exchanger(syn.L), ops, float(norm), b, w


def test_solve_mixed_entry_equals_solve_groups(problem):
    syn, ex, ops, norm, b, _ = problem
    x0 = torch.zeros_like(b)
    ((x_ref, xf_ref, d_ref),), = cg.solve_groups([cg.GroupSpec(ex, ops, [b], [x0], [1e-12], [300], norm,
                                                               x_fortran=True)], precision="mixed")
    L = capi.lib()
    params = capi.default_params()
    params.precision = capi.PREC_MIXED
    g = capi.Group()
    g.topo, g.count, g.nrhs = ex.handle(b.device), 2, 1
    g.max_iters[0], g.tolerance[0] = 300, 1e-12
    nbytes = L.cg2d_workspace_size(ctypes.byref(g), 1, ctypes.byref(params))
    ws = torch.empty(nbytes + 256, dtype=torch.uint8, device=b.device)
    base = ws.data_ptr() + (-ws.data_ptr()) % 256
    x, xf = torch.empty_like(b), torch.empty_like(b)
    dg = torch.zeros((2, capi.DIAG_BYTES), dtype=torch.uint8, device=b.device)
    params_f64 = capi.default_params()                  # the entry point selects mixed precision itself
    st = L.cg2d_solve_mixed(ex.handle(b.device), 2, norm, *(_p(t) for t in ops), _p(b), _p(x0), 1e-12, 300, _p(x),
                            _p(xf), _p(dg), ctypes.byref(params_f64), base, nbytes,
                            torch.cuda.current_stream().cuda_stream)
    assert st == capi.CG2D_OK
    torch.cuda.synchronize()
    torch.testing.assert_close(x, x_ref, rtol=0, atol=0)
    torch.testing.assert_close(xf, xf_ref, rtol=0, atol=0)
    assert torch.equal(dg, d_ref)
    assert all(r["status"] == "ok" and r["replacements"] > 0 for r in cg.diag_records(dg))


@pytest.mark.parametrize("coeff_grad", [1, 0])
def test_adjoint_ecco_entry_equals_autograd(problem, coeff_grad):
    syn, ex, ops, norm, b, w = problem
    p = cg.Cg2dParams(cg2dMaxIters=300, cg2dTolerance=1e-12, cg2dNorm=norm, sum_order="rowblock",
                      stop_coeff_grad=not coeff_grad)
    bt = b.clone().requires_grad_(True)
    opt = [a.clone().requires_grad_(i < 3) for i, a in enumerate(ops)]
    x, _ = cg.cg2d_solve(p, ex, tuple(opt), bt, torch.zeros_like(b))
    (x * w).sum().backward()
    L = capi.lib()
    params = capi.default_params()
    nbytes = L.cg2d_adjoint_ecco_workspace_size(ex.handle(b.device), 2, p.adj_max_iters, ctypes.byref(params))
    assert nbytes > 0
    ws = torch.empty(nbytes + 256, dtype=torch.uint8, device=b.device)
    base = ws.data_ptr() + (-ws.data_ptr()) % 256
    xd = x.detach().contiguous()
    lam = torch.empty_like(b)
    gW, gS, gC = (torch.full_like(b, 7.0) for _ in range(3))
    dg = torch.zeros((2, capi.DIAG_BYTES), dtype=torch.uint8, device=b.device)
    stream = torch.cuda.current_stream().cuda_stream
    assert L.cg2d_adjoint_ecco(ex.handle(b.device), 2, norm, None, *(_p(t) for t in ops), _p(xd), _p(w),
                               p.adj_tolerance, p.adj_max_iters, coeff_grad, _p(lam), _p(gW), _p(gS), _p(gC),
                               _p(dg), ctypes.byref(params), base, nbytes - 8, stream) == \
        capi.CG2D_WORKSPACE_TOO_SMALL
    st = L.cg2d_adjoint_ecco(ex.handle(b.device), 2, norm, None, *(_p(t) for t in ops), _p(xd), _p(w),
                             p.adj_tolerance, p.adj_max_iters, coeff_grad, _p(lam), _p(gW), _p(gS), _p(gC), _p(dg),
                             ctypes.byref(params), base, nbytes, stream)
    assert st == capi.CG2D_OK
    torch.cuda.synchronize()
    assert all(r["status"] == "ok" for r in cg.diag_records(dg))
    torch.testing.assert_close(lam, bt.grad, rtol=0, atol=0)
    for g, a in zip((gW, gS, gC), opt[:3]):
        if coeff_grad:
            torch.testing.assert_close(g, a.grad, rtol=0, atol=0)
        else:
            assert a.grad is None and not g.any()
