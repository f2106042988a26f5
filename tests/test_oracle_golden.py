"""The CPU oracle against the reference's own outputs (golden fixtures made by running mitgcm_jax's cg2d_fortran
through a numpy stand-in for JAX): bitwise, sum_order="fortran"."""

import hashlib

import numpy as np
import pytest

from golden_cases import CASES, GOLDEN, load
from mit_jax_b200.synthetic import LLCSynthetic
from oracle import cg2d_oracle as O


@pytest.mark.parametrize("name", CASES)
def test_oracle_matches_reference_bitwise(name):
    c = load(name)
    x, d = O.cg2d_fortran(c.L, c.tmap, c.ops, c.b, c.x0, cg2dNorm=c.norm, tolerance=c.tol, max_iters=c.maxit,
                          sum_order="fortran")
    assert d["numIters"] == c.numIters
    np.testing.assert_array_equal(x, c.x_fortran)
    got = np.array([d["firstResidual"], d["lastResidual"], d["sumRHS"], d["rhsMax"]])
    np.testing.assert_array_equal(got, c.diag)


def test_stop_rule_one_more_iteration():
    """test_cg2d.py:187-189 transcribed: a tolerance 0.99 x the last residual needs exactly one more iteration."""
    base, more = load("llc8"), load("llc8_onemore")
    assert more.numIters == base.numIters + 1
    assert np.isclose(more.tol, 0.99 * base.diag[1])


def test_negative_controls_fail():
    """A planted cg2dNorm * (1 + 1e-6) and a planted pW * (1 + 1e-6) both change the solution (test_cg2d.py:170-184)."""
    c = load("llc8")
    x, _ = O.cg2d_fortran(c.L, c.tmap, c.ops, c.b, c.x0, cg2dNorm=c.norm * (1 + 1e-6), tolerance=c.tol,
                          max_iters=c.maxit, sum_order="fortran")
    assert not np.array_equal(x, c.x_fortran)
    ops = list(c.ops)
    pW = ops[3].copy()
    J, I = c.L.interior
    t, j, i = np.argwhere(pW[:, J, I] != 0)[len(np.argwhere(pW[:, J, I] != 0)) // 2]
    pW[t, J.start + j, I.start + i] *= 1 + 1e-6          # a wet face in the middle of the domain
    ops[3] = pW
    x, _ = O.cg2d_fortran(c.L, c.tmap, tuple(ops), c.b, c.x0, cg2dNorm=c.norm, tolerance=c.tol, max_iters=c.maxit,
                          sum_order="fortran")
    assert not np.array_equal(x, c.x_fortran)


def test_llc90_reference_map_case():
    """LLC90 with the reference's probed exch2 map: the oracle reproduces the reference's x (SHA-256), iteration
    count and diagnostics bit for bit on the synthetic config-0 problem."""
    z = np.load(GOLDEN / "cg2d_llc90_ref_map.npz")
    m = np.load(GOLDEN / "llc90_T_map.npz")
    syn = LLCSynthetic(90)
    ops, norm = syn.operator()
    b, x0 = syn.rhs(), syn.first_guess()
    h = hashlib.sha256()
    for a in (*ops, b, x0):
        h.update(np.ascontiguousarray(a).tobytes())
    assert h.hexdigest() == str(z["inputs_sha"]), "synthetic generator drifted from the fixture"
    assert norm == float(z["cg2dNorm"])
    tmap = (m["src"], m["comp"])
    x, d = O.cg2d_fortran(syn.L, tmap, ops, b, x0, cg2dNorm=norm, tolerance=1e-12, max_iters=300,
                          sum_order="fortran")
    assert d["numIters"] == int(z["numIters"])
    np.testing.assert_array_equal(x.reshape(-1)[z["sample_idx"]], z["sample"])
    assert hashlib.sha256(np.ascontiguousarray(x).tobytes()).hexdigest() == str(z["x_sha"])
    np.testing.assert_array_equal(np.array([d["firstResidual"], d["lastResidual"], d["sumRHS"], d["rhsMax"]]),
                                  z["diag"])
