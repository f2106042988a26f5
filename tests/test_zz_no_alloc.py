"""cg2d_solve_f64_noalloc: the solve for callers that cannot allocate device memory where they solve (a custom
call inside a framework that owns the device pool, code that must not let a cudaMalloc synchronise the device).
It uses a fixed array in the library's device memory as its workspace. Checked against cg2d_solve_f64 with a
caller workspace on the same inputs, on two calls in a row (the second one runs on the array the first one
left behind), and for the size limit. Collected last, so that a stop-at-first-failure run has already run every
other test."""

import ctypes

import numpy as np
import pytest
import torch

from mit_jax_b200 import capi
from mit_jax_b200 import cg2d as cg
from mit_jax_b200.synthetic import make_batch

pytestmark = pytest.mark.gpu


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


def _inputs(batch):
    syn, B = make_batch(90, batch)
    dev = torch.device("cuda")
    ops = [torch.as_tensor(np.ascontiguousarray(B[k])).to(dev) for k in cg.OPS]
    b = torch.as_tensor(np.ascontiguousarray(B["b"])).to(dev)
    x0 = torch.as_tensor(np.ascontiguousarray(B["x0"])).to(dev)
    return syn, B, ops, b, x0


def _solve(L, topo, batch, norm, ops, b, x0, params, stream, workspace=None):
    x_out = torch.empty_like(b)
    x_f = torch.empty_like(b)
    diag = torch.zeros((batch, capi.DIAG_BYTES), dtype=torch.uint8, device=b.device)
    args = [topo, batch, norm, *[_ptr(t) for t in ops], _ptr(b), _ptr(x0), 1e-12, 300, _ptr(x_out), _ptr(x_f),
            _ptr(diag), ctypes.byref(params)]
    if workspace is None:
        st = L.cg2d_solve_f64_noalloc(*args, stream)
    else:
        st = L.cg2d_solve_f64(*args, _ptr(workspace), workspace.numel(), stream)
    return st, x_out, x_f, diag


@pytest.mark.parametrize("batch", [1, 2])
def test_noalloc_matches_workspace_solve_twice(batch):
    L = capi.lib()
    dev = torch.device("cuda")
    stream = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    params = capi.default_params()
    syn, B, ops, b, x0 = _inputs(batch)
    ex = cg.default_exchanger(syn.L)
    topo = ex.handle(dev)
    norm = float(B["cg2dNorm"][0])
    # the reference path: cg2d_solve_f64 with a workspace the caller allocated
    need = L.cg2d_workspace_size(*_group_for_size(topo, ops, b, x0, norm), ctypes.byref(params))
    assert 0 < need <= capi.NOALLOC_SCRATCH_BYTES        # two LLC90 FP64 instances fit the fixed array
    ws = torch.empty(need + 256, dtype=torch.uint8, device=dev)
    ws_aligned = ws[(-ws.data_ptr()) % 256:]
    for call, rhs in enumerate((b, 0.5 * b + 0.25 * x0)):
        rhs = rhs.contiguous()
        st_ref, x_ref, xf_ref, dg_ref = _solve(L, topo, batch, norm, ops, rhs, x0, params, stream, ws_aligned)
        st, x_new, xf_new, dg_new = _solve(L, topo, batch, norm, ops, rhs, x0, params, stream)
        torch.cuda.synchronize()
        assert st_ref == capi.CG2D_OK and st == capi.CG2D_OK, (call, st_ref, st)
        for m in range(batch):
            d_ref, d_new = cg.diag_records(dg_ref)[m], cg.diag_records(dg_new)[m]
            assert d_new["status"] == "ok" and d_ref["status"] == "ok"
            # the same kernel on the same inputs in the same order: equal bit for bit
            assert d_new == d_ref, (call, m, d_new, d_ref)
        torch.testing.assert_close(x_new, x_ref, rtol=0, atol=0)
        torch.testing.assert_close(xf_new, xf_ref, rtol=0, atol=0)


def test_noalloc_second_call_reserves_nothing():
    """The first call on a device loads the library's device module, which reserves the fixed array; a later call
    must leave the device's free memory unchanged."""
    L = capi.lib()
    dev = torch.device("cuda")
    stream = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    params = capi.default_params()
    syn, B, ops, b, x0 = _inputs(1)
    topo = cg.default_exchanger(syn.L).handle(dev)
    norm = float(B["cg2dNorm"][0])
    st, *_ = _solve(L, topo, 1, norm, ops, b, x0, params, stream)      # first call: module loaded here at latest
    torch.cuda.synchronize()
    assert st == capi.CG2D_OK
    outs = [torch.empty_like(b), torch.empty_like(b)]
    diag = torch.zeros((1, capi.DIAG_BYTES), dtype=torch.uint8, device=dev)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info(dev)
    st = L.cg2d_solve_f64_noalloc(topo, 1, norm, *[_ptr(t) for t in ops], _ptr(b), _ptr(x0), 1e-12, 300,
                                  _ptr(outs[0]), _ptr(outs[1]), _ptr(diag), ctypes.byref(params), stream)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info(dev)
    assert st == capi.CG2D_OK
    assert cg.diag_records(diag)[0]["status"] == "ok"
    assert free1 == free0, (free0, free1)


def test_noalloc_argument_statuses():
    """Refusals: a profile request (the profile would land in the hidden array) and, for arguments the solver
    rejects, the status cg2d_solve_f64 gives (here an unsupported batch of 257 right-hand sides; both calls stop at
    the argument checks, before any launch)."""
    L = capi.lib()
    dev = torch.device("cuda")
    stream = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    syn, B, ops, b, x0 = _inputs(1)
    topo = cg.default_exchanger(syn.L).handle(dev)
    norm = float(B["cg2dNorm"][0])
    prof = capi.default_params()
    prof.profile = 1
    st, *_ = _solve(L, topo, 1, norm, ops, b, x0, prof, stream)
    assert st == capi.CG2D_BAD_ARG
    params = capi.default_params()
    x_out = torch.empty_like(b)
    diag = torch.zeros((1, capi.DIAG_BYTES), dtype=torch.uint8, device=dev)
    args = [topo, 257, norm, *[_ptr(t) for t in ops], _ptr(b), _ptr(x0), 1e-12, 300, _ptr(x_out), None,
            _ptr(diag), ctypes.byref(params)]
    st_ref = L.cg2d_solve_f64(*args, _ptr(x_out), x_out.numel() * 8, stream)
    st = L.cg2d_solve_f64_noalloc(*args, stream)
    assert st_ref == capi.CG2D_UNSUPPORTED
    assert st == st_ref


def _group_for_size(topo, ops, b, x0, norm):
    """(groups, ngroups) for cg2d_workspace_size of a one-instance FP64 solve."""
    g = capi.Group()
    g.topo = topo
    g.count = b.shape[0]
    g.nrhs = 1
    for name, t in zip(cg.OPS, ops):
        setattr(g, name, t.data_ptr())
    g.cg2dNorm = norm
    g.b[0], g.x0[0] = b.data_ptr(), x0.data_ptr()
    g.tolerance[0], g.max_iters[0] = 1e-12, 300
    return ctypes.byref(g), 1


def test_noalloc_rejects_oversize_batch():
    L = capi.lib()
    dev = torch.device("cuda")
    stream = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    params = capi.default_params()
    syn, B, ops, b, x0 = _inputs(3)          # three LLC90 instances need more than the fixed array holds
    topo = cg.default_exchanger(syn.L).handle(dev)
    need = L.cg2d_workspace_size(*_group_for_size(topo, ops, b, x0, float(B["cg2dNorm"][0])), ctypes.byref(params))
    assert need > capi.NOALLOC_SCRATCH_BYTES
    st, *_ = _solve(L, topo, 3, float(B["cg2dNorm"][0]), ops, b, x0, params, stream)
    assert st == capi.CG2D_WORKSPACE_TOO_SMALL
