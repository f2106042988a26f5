"""GPU parity of the persistent CG2D solver (libcg2d.so through the C ABI) against the oracle and the reference's
own outputs (golden fixtures).

Bars: bitwise for the "fortran" sum order (== the reference) and for the ROWBLOCK order (== the oracle's
restatement of the same operations); against the FP64 reference order, solution within 1e-12 relative (FP64) and
iteration count within +-1; the MIXED iteration (fused FP32 arithmetic) within 1e-11 relative of FP64."""

import numpy as np
import pytest
import torch

from golden_cases import CASES, GOLDEN, load
from oracle import cg2d_oracle as O

pytestmark = pytest.mark.gpu

cg = pytest.importorskip("mit_jax_b200.cg2d")


def _ex(c):
    return cg.Exchanger(c.L, c.topo.maps)


def _diag_vec(d):
    return np.array([d["firstResidual"], d["lastResidual"], d["sumRHS"], d["rhsMax"]])


def _rel(a, b, L):
    J, I = L.interior
    return np.abs(a[..., J, I] - b[..., J, I]).max() / max(np.abs(b[..., J, I]).max(), 1e-300)


@pytest.mark.parametrize("name", CASES)
def test_fortran_order_bitwise_equals_reference(name):
    """sum_order="fortran" on the GPU gives the reference's x (halos included), iteration count and diagnostics
    bit for bit."""
    c = load(name)
    x, d = cg.cg2d_fortran(_ex(c), c.ops, c.b, c.x0, cg2dNorm=c.norm, tolerance=c.tol, max_iters=c.maxit,
                           sum_order="fortran")
    assert d["numIters"] == c.numIters
    np.testing.assert_array_equal(x, c.x_fortran)
    np.testing.assert_array_equal(_diag_vec(d), c.diag)
    assert d["status"] == ("not_converged" if name == "llc8_cap" else "ok")


@pytest.mark.parametrize("name", CASES)
def test_rowblock_order_bitwise_equals_oracle(name):
    c = load(name)
    x, d = cg.cg2d_fortran(_ex(c), c.ops, c.b, c.x0, cg2dNorm=c.norm, tolerance=c.tol, max_iters=c.maxit,
                           sum_order="rowblock")
    xo, do = O.cg2d_fortran(c.L, c.tmap, c.ops, c.b, c.x0, cg2dNorm=c.norm, tolerance=c.tol, max_iters=c.maxit,
                            sum_order="rowblock")
    assert d["numIters"] == do["numIters"]
    np.testing.assert_array_equal(x, xo)
    np.testing.assert_array_equal(_diag_vec(d), _diag_vec(do))
    if name not in ("llc8_cap", "llc8_zero_iters", "llc8_onemore"):
        assert abs(d["numIters"] - c.numIters) <= 1
        if name == "llc8_zero_rhs":      # the exact solution is 0: compare absolutely
            J, I = c.L.interior
            assert np.abs(x[:, J, I] - c.x_fortran[:, J, I]).max() < 1e-10
        else:
            assert _rel(x, c.x_fortran, c.L) < 1e-12


@pytest.fixture(scope="module")
def llc90():
    from mit_jax_b200.synthetic import LLCSynthetic
    syn = LLCSynthetic(90)
    m = np.load(GOLDEN / "llc90_T_map.npz")
    ones = np.ones_like(m["comp"])
    ex_ref = cg.Exchanger(syn.L, {"T": (m["src"], m["comp"], ones)})
    return syn, ex_ref, (m["src"], m["comp"])


def test_llc90_reference_map_fortran_order(llc90):
    """LLC90 with the reference's full probed exch2 map: the GPU reproduces the reference's solution (SHA-256 of
    the whole array, halos and corners included) and its diagnostics."""
    import hashlib
    syn, ex_ref, _ = llc90
    z = np.load(GOLDEN / "cg2d_llc90_ref_map.npz")
    ops, norm = syn.operator()
    x, d = cg.cg2d_fortran(ex_ref, ops, syn.rhs(), syn.first_guess(), cg2dNorm=norm, tolerance=1e-12,
                           max_iters=300, sum_order="fortran")
    assert d["numIters"] == int(z["numIters"])
    np.testing.assert_array_equal(x.reshape(-1)[z["sample_idx"]], z["sample"])
    assert hashlib.sha256(np.ascontiguousarray(x).tobytes()).hexdigest() == str(z["x_sha"])


def test_llc90_rowblock_and_guess_halos(llc90):
    """ROWBLOCK order on LLC90 with a non-zero first guess (halos and corners included): bitwise the oracle, whose
    x_fortran halos follow exchange-of-the-normalised-guess semantics with the reference's full map."""
    syn, ex_ref, tmap = llc90
    ops, norm = syn.operator()
    b = syn.rhs()
    x0 = np.random.default_rng(11).standard_normal(syn.L.shape2d) * 1e-4
    x, d = cg.cg2d_fortran(ex_ref, ops, b, x0, cg2dNorm=norm, tolerance=1e-12, max_iters=300, sum_order="rowblock")
    xo, do = O.cg2d_fortran(syn.L, tmap, ops, b, x0, cg2dNorm=norm, tolerance=1e-12, max_iters=300,
                            sum_order="rowblock")
    assert d["numIters"] == do["numIters"]
    np.testing.assert_array_equal(x, xo)


def test_batched_members_one_launch():
    """Four ensemble members (different operators, norms and right-hand sides) in one launch, per-instance
    convergence: each member equals its own oracle solve bit for bit."""
    from mit_jax_b200.synthetic import make_batch
    syn, B = make_batch(90, 4)
    ex = cg.default_exchanger(syn.L)
    dev = torch.device("cuda")
    ops = tuple(torch.as_tensor(B[k]).to(dev) for k in cg.OPS)
    G = cg.GroupSpec(ex, ops, [torch.as_tensor(B["b"]).to(dev)], [torch.as_tensor(B["x0"]).to(dev)], [1e-12],
                     [300], torch.as_tensor(B["cg2dNorm"]), x_fortran=True)
    (res,), = cg.solve_groups([G], sum_order="rowblock")
    xo, xf, dg = res
    diags = cg.diag_records(dg)
    iters = set()
    for m in range(4):
        ops_m = tuple(B[k][m] for k in cg.OPS)
        ref, dref = O.cg2d_fortran(syn.L, syn.topo.maps["T"], ops_m, B["b"][m], B["x0"][m],
                                   cg2dNorm=B["cg2dNorm"][m], tolerance=1e-12, max_iters=300, sum_order="rowblock")
        assert diags[m]["numIters"] == dref["numIters"]
        iters.add(dref["numIters"])
        np.testing.assert_array_equal(xf[m].cpu().numpy(), ref)
        J, I = syn.L.interior
        got = xo[m].cpu().numpy()
        np.testing.assert_array_equal(got[:, J, I], ref[:, J, I])
        assert np.all(got[:, ~O.interior_mask(syn.L)] == 0)
    assert len(iters) >= 2                      # uneven counts exercised the per-instance retirement


@pytest.mark.parametrize("precision", ["f64", "mixed"])
def test_nan_instance_is_reported_and_isolated(precision):
    """A NaN in one instance's right-hand side: that solve runs to its iteration cap and reports status "nan" (the
    reference lets NaNs through silently), the launch itself succeeds, and the other instance of the same launch is
    bit for bit its solo solve."""
    from mit_jax_b200.synthetic import make_batch
    syn, B = make_batch(16, ts=8, members=[0, 1])
    ex = cg.default_exchanger(syn.L)
    dev = torch.device("cuda")
    ops = tuple(torch.as_tensor(B[k]).to(dev) for k in cg.OPS)
    b = torch.as_tensor(B["b"]).to(dev)
    J, I = syn.L.interior
    b_nan = b.clone()
    b_nan[1, 3, J.start + 2, I.start + 5] = float("nan")
    x0 = torch.zeros_like(b)
    G = cg.GroupSpec(ex, ops, [b_nan], [x0], [1e-12], [60], torch.as_tensor(B["cg2dNorm"]))
    ((x, _, dg),), = cg.solve_groups([G], precision=precision)
    d = cg.diag_records(dg)
    assert d[1]["status"] == "nan" and d[1]["numIters"] == 60
    G1 = cg.GroupSpec(ex, tuple(o[:1].contiguous() for o in ops), [b[:1].contiguous()], [x0[:1].contiguous()],
                      [1e-12], [60], torch.as_tensor(B["cg2dNorm"][:1]))
    ((x1, _, dg1),), = cg.solve_groups([G1], precision=precision)
    torch.testing.assert_close(x[0], x1[0], rtol=0, atol=0)
    assert d[0] == cg.diag_records(dg1)[0]


def test_mixed_precision_matches_mixed_oracle_and_fp64(llc90):
    """The mixed iteration (FP32 stencils and updates with fused multiply-adds) against the FP64 oracle: within
    1e-11 relative, converged; its iteration count within 5 of the mixed oracle's (the same iteration with every
    FP32 product and sum rounded separately)."""
    syn, ex_ref, tmap = llc90
    ex = cg.default_exchanger(syn.L)
    T = syn.topo.maps["T"]
    ops, norm = syn.operator()
    b, x0 = syn.rhs(), syn.first_guess()
    x, d = cg.cg2d_fortran(ex, ops, b, x0, cg2dNorm=norm, tolerance=1e-12, max_iters=300, sum_order="rowblock",
                           precision="mixed")
    xm, dm = O.cg2d_mixed(syn.L, T, ops, b, x0, cg2dNorm=norm, tolerance=1e-12, max_iters=300)
    assert d["status"] == "ok" and d["lastResidual"] < 1e-12
    assert abs(d["numIters"] - dm["numIters"]) <= 5, (d["numIters"], dm["numIters"])
    x64, d64 = O.cg2d_fortran(syn.L, T, ops, b, x0, cg2dNorm=norm, tolerance=1e-12, max_iters=300,
                              sum_order="rowblock")
    assert _rel(x, x64, syn.L) < 1e-11
    assert _rel(xm, x64, syn.L) < 1e-11


def test_two_rhs_share_the_operator():
    """Forward and adjoint right-hand sides of one instance in one launch give the same results as two separate
    single-right-hand-side launches."""
    c = load("llc16_guess")
    ex = _ex(c)
    dev = torch.device("cuda")
    t = lambda a: torch.as_tensor(a).to(dev)[None]          # noqa: E731
    ops = tuple(t(a) for a in c.ops)
    w = np.random.default_rng(3).standard_normal(c.L.shape2d)
    G2 = cg.GroupSpec(ex, ops, [t(c.b), t(w)], [t(c.x0), t(np.zeros_like(w))], [1e-12, 1e-13], [300, 2000], c.norm)
    (slots2,) = cg.solve_groups([G2])
    for slot, (b, x0, tol, mi) in enumerate(((c.b, c.x0, 1e-12, 300), (w, np.zeros_like(w), 1e-13, 2000))):
        G1 = cg.GroupSpec(ex, ops, [t(b)], [t(x0)], [tol], [mi], c.norm)
        (slots1,) = cg.solve_groups([G1])
        np.testing.assert_array_equal(slots2[slot][0].cpu().numpy(), slots1[0][0].cpu().numpy())
        assert cg.diag_records(slots2[slot][2]) == cg.diag_records(slots1[0][2])


def test_mixed_size_groups_llc270_and_llc90():
    """LLC270 and LLC90 instances in one MIXED launch (two groups): each converges and lies within 1e-11 of the
    FP64 solve of the same instance (the same two groups in one FP64 launch); the LLC90 iteration counts are within
    5 of the mixed oracle's."""
    from mit_jax_b200.synthetic import LLCSynthetic
    dev = torch.device("cuda")
    groups, refs = [], []
    for N, count in ((270, 1), (90, 2)):
        syn = LLCSynthetic(N)
        ex = cg.default_exchanger(syn.L)
        mats, bs, norms = [], [], []
        for m in range(count):
            ops, norm = syn.operator(m if count > 1 else None)
            mats.append(ops)
            bs.append(syn.rhs(m if count > 1 else None))
            norms.append(norm)
        ops_t = tuple(torch.as_tensor(np.stack([o[k] for o in mats])).to(dev) for k in range(6))
        b_t = torch.as_tensor(np.stack(bs)).to(dev)
        groups.append(cg.GroupSpec(ex, ops_t, [b_t], [torch.zeros_like(b_t)], [1e-12], [1000],
                                   torch.as_tensor(norms)))
        refs.append((syn, mats, bs, norms))
    res = cg.solve_groups(groups, precision="mixed")
    res64 = cg.solve_groups(groups, precision="f64")
    for (syn, mats, bs, norms), (slot0,), (slot64,) in zip(refs, res, res64):
        xo, _, dg = slot0
        diags = cg.diag_records(dg)
        for m in range(len(mats)):
            assert diags[m]["status"] == "ok", diags[m]
            assert _rel(xo[m].cpu().numpy(), slot64[0][m].cpu().numpy(), syn.L) < 1e-11
            if syn.L.sNx == 90:
                xm, dm = O.cg2d_mixed(syn.L, syn.topo.maps["T"], mats[m], bs[m], np.zeros_like(bs[m]),
                                      cg2dNorm=norms[m], tolerance=1e-12, max_iters=1000)
                assert abs(diags[m]["numIters"] - dm["numIters"]) <= 5


def test_matvec_exchange_and_edge_products_equal_oracle():
    c = load("llc16_guess")
    ex = _ex(c)
    rng = np.random.default_rng(5)
    v = rng.standard_normal(c.L.shape2d)
    np.testing.assert_array_equal(cg.matvec(ex, c.ops[:3], c.norm, v), O.matvec(c.L, c.tmap, c.ops[:3], c.norm, v))
    np.testing.assert_array_equal(ex.exch_xy(v), O.exch(v, c.tmap))
    lam = rng.standard_normal(c.L.shape2d) * O.interior_mask(c.L)
    x = rng.standard_normal(c.L.shape2d) * O.interior_mask(c.L)
    got = cg.edge_products(ex, lam, x, c.norm)
    ref = O.coefficient_cotangents(c.L, c.tmap, lam, x, c.norm)
    for g, r in zip(got, ref):
        np.testing.assert_array_equal(g, r)


def test_operator_symmetric():
    """<A u, v> = <u, A v> (test_cg2d.py:214-226) for the synthetic LLC operator on the GPU."""
    from mit_jax_b200.synthetic import LLCSynthetic
    syn = LLCSynthetic(90)
    ex = cg.default_exchanger(syn.L)
    ops, norm = syn.operator()
    inner = O.interior_mask(syn.L)
    rng = np.random.default_rng(1)
    u, v = (rng.standard_normal(syn.L.shape2d) * inner for _ in range(2))
    lhs = np.vdot(cg.matvec(ex, ops[:3], norm, u), v)
    rhs = np.vdot(u, cg.matvec(ex, ops[:3], norm, v))
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs)


def test_barrier_time_limit_reports_status():
    """A grid-wide wait that can never complete (one arrival more than there are CTAs) runs out after the time
    limit; every solve reports barrier_timeout and the context stays usable."""
    c = load("llc8")
    ex = _ex(c)
    dev = torch.device("cuda")
    t = lambda a: torch.as_tensor(a).to(dev)[None]          # noqa: E731
    G = cg.GroupSpec(ex, tuple(t(a) for a in c.ops), [t(c.b)], [t(c.x0)], [c.tol], [c.maxit], c.norm)
    ((xo, xf, dg),), = cg.solve_groups([G], timeout_s=0.2, check_status=False, test_missing_arrivals=1)
    torch.cuda.synchronize()
    assert cg.diag_records(dg)[0]["status"] == "barrier_timeout"
    x, d = cg.cg2d_fortran(ex, c.ops, c.b, c.x0, cg2dNorm=c.norm, tolerance=c.tol, max_iters=c.maxit,
                           sum_order="fortran")
    np.testing.assert_array_equal(x, c.x_fortran)          # the next solve on the same context is fine
