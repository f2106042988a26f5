"""The jax.ffi custom calls and the jax.custom_vjp cg2d_solve (mit_jax_b200.jax_ffi over csrc/cg2d_ffi.cc).

jax is not installed in every environment this package runs in; there every test here is skipped. Where it is, the
GPU tests compare the JAX entry points with the torch/ctypes ones on the same inputs: cg2d_fortran bit for bit, and
the custom_vjp gradients (cg2d_b, aW2d, aS2d, aC2d) with the autograd backward of cg2d.cg2d_solve bit for bit, the
ECCO mode giving zero coefficient cotangents (test_cg2d.py:280-300)."""

import numpy as np
import pytest

jax = pytest.importorskip("jax")
jax.config.update("jax_enable_x64", True)


def test_ffi_library_built_with_jax():
    from mit_jax_b200 import _build
    if _build.jax_ffi_include() is None:
        pytest.skip("this jax has no FFI headers")
    assert _build.build_ffi() is not None and _build.FFI_OUT.exists()


@pytest.mark.gpu
@pytest.mark.parametrize("stop_coeff_grad", [False, True])
def test_jax_cg2d_solve_matches_torch_path(stop_coeff_grad):
    import jax.numpy as jnp
    import torch

    from mit_jax_b200 import cg2d as cg
    from mit_jax_b200 import jax_ffi as jf
    from mit_jax_b200.synthetic import LLCSynthetic
    syn = LLCSynthetic(32, 16, 4)
    L = syn.L
    ops, norm = syn.operator()
    b, x0 = syn.rhs(), syn.first_guess()
    w = syn.cotangent()
    topo = jf.Topology(L, syn.topo.maps["T"])
    p = cg.Cg2dParams(cg2dMaxIters=300, cg2dTolerance=1e-12, cg2dNorm=norm, sum_order="rowblock",
                      stop_coeff_grad=stop_coeff_grad)
    xf, d = jf.cg2d_fortran(topo, ops, b, x0, cg2dNorm=norm, tolerance=1e-12, max_iters=300)
    ex = cg.Exchanger(L, syn.topo.maps)
    xf_t, d_t = cg.cg2d_fortran(ex, ops, b, x0, cg2dNorm=norm, tolerance=1e-12, max_iters=300, sum_order="rowblock")
    np.testing.assert_array_equal(np.asarray(xf), xf_t)
    assert int(d["numIters"]) == d_t["numIters"]

    def J(aW, aS, aC, bb):
        x, _ = jf.cg2d_solve(p, topo, (aW, aS, aC) + tuple(ops[3:]), bb, x0)
        return jnp.vdot(jnp.asarray(w), x)

    g = jax.grad(J, argnums=(0, 1, 2, 3))(*(jnp.asarray(a) for a in (ops[0], ops[1], ops[2], b)))
    tt = [torch.as_tensor(a).cuda().requires_grad_(True) for a in (ops[0], ops[1], ops[2], b)]
    x, _ = cg.cg2d_solve(p, ex, (tt[0], tt[1], tt[2]) + tuple(torch.as_tensor(a).cuda() for a in ops[3:]), tt[3],
                         torch.as_tensor(x0).cuda())
    (x * torch.as_tensor(w).cuda()).sum().backward()
    for k in range(4):
        ref = tt[k].grad.cpu().numpy() if tt[k].grad is not None else np.zeros_like(np.asarray(g[k]))
        np.testing.assert_array_equal(np.asarray(g[k]), ref)
    if stop_coeff_grad:
        assert all(np.all(np.asarray(g[k]) == 0) for k in range(3))
