"""Parity on the grid and in the sum order the headline measurement uses: LLC90, ROWBLOCK sums, FP64 and mixed
precision, forward and ECCO (implicit-derivative) adjoint.

* The reference's own LLC90 solution is reproduced in-test by the FORTRAN-order GPU solve on the reference's probed
  exch2 map, which equals the reference's cg2d_fortran bit for bit (SHA-256 of the whole array, pinned by
  tests/golden/cg2d_llc90_ref_map.npz). Against it: ROWBLOCK FP64 within 1e-12 relative with the iteration count
  within +-1, mixed precision within 1e-11 (test_cg2d.py:127-145 for the bar).
* A batch of headline members (forward + adjoint right-hand sides in one launch): mixed within 1e-11 of the FP64
  reference-order solve of the same member, for x and for lam.
* The ECCO adjoint (gradients of J = <w, x> w.r.t. cg2d_b, aW2d and aS2d) against central differences at
  h = 1e-6 relative on 20 seeded random directions, to 1e-6 (test_cg2d.py:240-277 for the design).
* The GPU lam, gW, gS, gC against the reference's implicit derivative (cg2d.py:318-348: the literal forward, the
  tight transpose solve in the "tile" sum order at adj_tolerance 1e-13, the transpose of _matvec), as the oracle
  restates it, to 1e-11 relative.
"""

import hashlib

import numpy as np
import pytest
import torch

from golden_cases import GOLDEN
from oracle import cg2d_oracle as O

pytestmark = pytest.mark.gpu

cg = pytest.importorskip("mit_jax_b200.cg2d")


def _rel(a, b, L):
    """max |a - b| / max |b| over the interior points (all leading dimensions)."""
    J, I = L.interior
    a, b = np.asarray(a), np.asarray(b)
    return float(np.abs(a[..., J, I] - b[..., J, I]).max() / max(np.abs(b[..., J, I]).max(), 1e-300))


@pytest.fixture(scope="module")
def llc90():
    from mit_jax_b200.synthetic import LLCSynthetic
    syn = LLCSynthetic(90)
    m = np.load(GOLDEN / "llc90_T_map.npz")
    ex_ref = cg.Exchanger(syn.L, {"T": (m["src"], m["comp"], np.ones_like(m["comp"]))})
    return syn, ex_ref


@pytest.fixture(scope="module")
def reference_solution(llc90):
    """The reference's LLC90 solution: the FORTRAN-order GPU solve, checked against the pinned SHA-256."""
    syn, ex_ref = llc90
    z = np.load(GOLDEN / "cg2d_llc90_ref_map.npz")
    ops, norm = syn.operator()
    x, d = cg.cg2d_fortran(ex_ref, ops, syn.rhs(), syn.first_guess(), cg2dNorm=norm, tolerance=1e-12,
                           max_iters=300, sum_order="fortran")
    assert hashlib.sha256(np.ascontiguousarray(x).tobytes()).hexdigest() == str(z["x_sha"])
    assert d["numIters"] == int(z["numIters"])
    return x, d


def test_llc90_rowblock_f64_matches_reference_solution(llc90, reference_solution):
    syn, ex_ref = llc90
    x_ref, d_ref = reference_solution
    ops, norm = syn.operator()
    x, d = cg.cg2d_fortran(ex_ref, ops, syn.rhs(), syn.first_guess(), cg2dNorm=norm, tolerance=1e-12,
                           max_iters=300, sum_order="rowblock")
    assert d["status"] == "ok"
    assert abs(d["numIters"] - d_ref["numIters"]) <= 1, (d["numIters"], d_ref["numIters"])
    err = _rel(x, x_ref, syn.L)
    assert err <= 1e-12, err


def test_llc90_mixed_matches_reference_solution(llc90, reference_solution):
    syn, ex_ref = llc90
    x_ref, d_ref = reference_solution
    ops, norm = syn.operator()
    x, d = cg.cg2d_fortran(ex_ref, ops, syn.rhs(), syn.first_guess(), cg2dNorm=norm, tolerance=1e-12,
                           max_iters=300, sum_order="rowblock", precision="mixed")
    assert d["status"] == "ok" and d["lastResidual"] < 1e-12
    err = _rel(x, x_ref, syn.L)
    assert err <= 1e-11, err


def test_llc90_batch_mixed_forward_and_adjoint_vs_fp64_reference_order():
    """Eight headline members, forward and adjoint right-hand sides in one launch (as the bench runs them): each
    mixed solution within 1e-11 of the FP64 FORTRAN-order (reference-order) solve of the same member, and the FP64
    ROWBLOCK batch within 1e-12 of it with iteration counts within +-1."""
    from mit_jax_b200.synthetic import make_batch
    syn, B = make_batch(90, 8, with_cotangent=True)
    ex = cg.default_exchanger(syn.L)
    dev = torch.device("cuda")
    ops = tuple(torch.as_tensor(B[k]).to(dev) for k in cg.OPS)
    mask = cg._interior_mask(syn.L, dev)
    b = torch.as_tensor(B["b"]).to(dev)
    w = torch.where(mask, torch.as_tensor(B["w"]).to(dev), torch.zeros((), dtype=torch.float64, device=dev))
    z = torch.zeros_like(b)
    norms = torch.as_tensor(B["cg2dNorm"])
    out = {}
    for prec, order in (("f64", "fortran"), ("f64", "rowblock"), ("mixed", "rowblock")):
        G = cg.GroupSpec(ex, ops, [b, w], [z, z], [1e-12, 1e-12], [300, 300], norms)
        (slots,) = cg.solve_groups([G], precision=prec, sum_order=order)
        out[prec, order] = [(xo.cpu().numpy(), cg.diag_records(dg)) for xo, _, dg in slots]
    ref = out["f64", "fortran"]
    for key, bar in ((("f64", "rowblock"), 1e-12), (("mixed", "rowblock"), 1e-11)):
        for s in range(2):
            x, diags = out[key][s]
            xr, dr = ref[s]
            for m in range(8):
                assert diags[m]["status"] == "ok", (key, s, m, diags[m])
                err = _rel(x[m], xr[m], syn.L)
                assert err <= bar, (key, s, m, err)
                if key[0] == "f64":
                    assert abs(diags[m]["numIters"] - dr[m]["numIters"]) <= 1, (key, s, m)


def _direction(rng, syn, ops, b):
    """A random direction in (cg2d_b, aW2d, aS2d), each entry scaled by the magnitude of the entry it moves, so
    land faces and land points stay 0 (h = 1e-6 is then a relative perturbation). The face directions are set on
    the interior faces and exchanged into the east / north face halos with the UVn map, as the operator's faces are
    (init.py:345-350): every face moves with its copy, so the perturbed operator stays symmetric."""
    from mit_jax_b200.topology import exch_vector
    L, maps = syn.L, syn.topo.maps
    J, I = L.interior
    inner = O.interior_mask(L)
    db = rng.standard_normal(L.shape2d) * np.abs(b) * inner
    dW = np.zeros(L.shape2d)
    dS = np.zeros(L.shape2d)
    dW[:, J, I] = rng.standard_normal(dW[:, J, I].shape) * np.abs(ops[0][:, J, I])
    dS[:, J, I] = rng.standard_normal(dS[:, J, I].shape) * np.abs(ops[1][:, J, I])
    dW, dS = exch_vector(dW, dS, maps["UVn_u"], maps["UVn_v"])
    return db, dW, dS


@pytest.mark.parametrize("precision", ["f64", "mixed"])
def test_llc90_ecco_adjoint_central_differences_20_directions(precision):
    """Gradients of J = <w, x> from the one-launch forward + adjoint (mixed: the headline's own path) against
    central differences (J(a + h d) - J(a - h d)) / 2h, h = 1e-6 relative, on 20 seeded random directions that move
    cg2d_b, aW2d and aS2d together; relative error below 1e-6 on every direction. The 40 perturbed forward solves
    run as one FP64 batch to a normalised residual of 1e-14, so that solver noise in J stays far below h^2."""
    from mit_jax_b200.synthetic import LLCSynthetic
    syn = LLCSynthetic(90)
    L = syn.L
    ex = cg.default_exchanger(L)
    ops, norm = syn.operator()
    b, w = syn.rhs(), syn.cotangent() * O.interior_mask(L)
    r = cg.solve_with_adjoint(ex, [a[None] for a in ops], b[None], w[None], cg2dNorm=norm, tolerance=1e-12,
                              max_iters=300, adj_tolerance=1e-12 if precision == "mixed" else 1e-13,
                              adj_max_iters=2000, precision=precision)
    for d in cg.diag_records(r["diag_fwd"]) + cg.diag_records(r["diag_adj"]):
        assert d["status"] == "ok", d
    gb, gW, gS = r["lam"][0], r["gW"][0], r["gS"][0]
    rng = np.random.default_rng(4)
    h = 1e-6
    dirs = [_direction(rng, syn, ops, b) for _ in range(20)]
    dev = torch.device("cuda")
    batch = {k: [] for k in cg.OPS + ("b",)}
    for db, dW, dS in dirs:
        for sgn in (1.0, -1.0):
            batch["aW2d"].append(ops[0] + sgn * h * dW)
            batch["aS2d"].append(ops[1] + sgn * h * dS)
            for k, a in zip(cg.OPS[2:], ops[2:]):
                batch[k].append(a)
            batch["b"].append(b + sgn * h * db)
    t = {k: torch.as_tensor(np.stack(v)).to(dev) for k, v in batch.items()}
    n = t["b"].shape[0]
    G = cg.GroupSpec(ex, tuple(t[k] for k in cg.OPS), [t["b"]], [torch.zeros_like(t["b"])], [1e-14], [1000], norm)
    (slots,) = cg.solve_groups([G], precision="f64")
    x, _, dg = slots[0]
    assert all(d["status"] == "ok" for d in cg.diag_records(dg))
    J, I = L.interior
    Jv = (x[:, :, J, I].cpu().numpy() * w[None, :, J, I]).reshape(n, -1).sum(axis=1)
    errs = []
    for q, (db, dW, dS) in enumerate(dirs):
        fd = (Jv[2 * q] - Jv[2 * q + 1]) / (2 * h)
        gd = float(np.vdot(gb, db) + np.vdot(gW, dW) + np.vdot(gS, dS))
        errs.append(abs(fd - gd) / abs(gd))
    assert max(errs) < 1e-6, errs


@pytest.mark.parametrize("precision", ["f64", "mixed"])
def test_llc90_adjoint_matches_reference_implicit_gradient(llc90, precision):
    """lam (= dJ/d cg2d_b) and the coefficient cotangents gW, gS, gC of the one-launch forward + adjoint, on the
    reference's own exch2 map, against the reference's implicit derivative restated by the oracle: x from the
    FORTRAN-order forward, lam from the tight solve in the "tile" sum order at 1e-13 from zero (cg2d.py:333-338),
    the cotangents as the transpose of _matvec(dA, x) (cg2d.py:331); 1e-11 relative on every array."""
    syn, ex_ref = llc90
    L = syn.L
    T = syn.topo.maps["T"]
    ops, norm = syn.operator()
    b, w = syn.rhs(), syn.cotangent() * O.interior_mask(L)
    r = cg.solve_with_adjoint(ex_ref, [a[None] for a in ops], b[None], w[None], cg2dNorm=norm, tolerance=1e-12,
                              max_iters=300, adj_tolerance=1e-12 if precision == "mixed" else 1e-13,
                              adj_max_iters=2000, precision=precision)
    inner = O.interior_mask(L)
    x_ref, _ = O.cg2d_fortran(L, T, ops, b, np.zeros_like(b), cg2dNorm=norm, tolerance=1e-12, max_iters=300,
                              sum_order="fortran")
    lam_ref, _ = O.tight_solve(L, T, ops, w, cg2dNorm=norm, tolerance=1e-13, max_iters=2000, sum_order="tile")
    g_ref = O.coefficient_cotangents(L, T, lam_ref, np.where(inner, x_ref, 0.0), norm)
    assert _rel(r["x"][0], x_ref, L) <= (1e-11 if precision == "mixed" else 1e-12)
    assert _rel(r["lam"][0], lam_ref, L) <= 1e-11
    assert np.all(r["lam"][0][:, ~inner] == 0.0)
    for name, got, ref in zip(("gW", "gS", "gC"), (r["gW"][0], r["gS"][0], r["gC"][0]), g_ref):
        err = float(np.abs(got - ref).max() / np.abs(ref).max())
        assert err <= 1e-11, (name, err)
