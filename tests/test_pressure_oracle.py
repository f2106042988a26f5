"""The CPU oracle of the steps either side of the solve (oracle/pressure_oracle.py) against the reference's own
update_cg2d, cg2d_rhs, solve_for_pressure and ini_cg2d_norm (golden fixtures made by running mitgcm_jax through a
numpy stand-in for JAX): bitwise, including the preconditioner points update_cg2d keeps and both fresh-water-flux
branches."""

import numpy as np
import pytest

from golden_cases import PRESSURE_CASES, load_pressure, pressure_sha
from oracle import cg2d_oracle as O
from oracle import pressure_oracle as P

OPS = ("aW2d", "aS2d", "aC2d", "pW", "pS", "pC")
UPDATE_KEYS = ("drF", "dyG", "dxG", "recip_dxC", "recip_dyC", "rA", "recip_Bo", "cg2dNorm", "cg2dpcOffDFac",
               "implicSurfPress", "implicDiv2DFlow", "freeSurfFac", "deltaTMom", "deltaTFreeSurf")
RHS_KEYS = ("gU", "gV", "hFacW", "hFacS", "EmPmR", "etaN", "etaH", "Bo_surf", "drF", "dyG", "dxG", "rA", "maskInC",
            "freeSurfFac", "mass2rUnit", "implicDiv2DFlow", "deltaTMom", "deltaTFreeSurf", "useRealFreshWaterFlux")


@pytest.mark.parametrize("name", list(PRESSURE_CASES))
def test_pressure_oracle_matches_reference_bitwise(name):
    syn, f, prev, z = load_pressure(name)
    assert pressure_sha(f, prev) == str(z["inputs_sha"]), "the synthetic generator changed: regenerate fixtures"
    L, tmap = syn.L, syn.topo.maps["T"]
    ops = P.update_cg2d(L, tmap, hFacW=f["hFacW"], hFacS=f["hFacS"], pW=prev[0], pS=prev[1], pC=prev[2],
                        **{k: f[k] for k in UPDATE_KEYS})
    for k, a in zip(OPS, ops):
        np.testing.assert_array_equal(a, z[k], err_msg=k)
    b, x0 = P.cg2d_rhs(L, **{k: f[k] for k in RHS_KEYS})
    np.testing.assert_array_equal(b, z["cg2d_b"])
    np.testing.assert_array_equal(x0, z["cg2d_x"])
    x, d = O.cg2d_fortran(L, tmap, ops, b, x0, cg2dNorm=f["cg2dNorm"], tolerance=1e-12, max_iters=300,
                          sum_order="fortran")
    assert d["numIters"] == int(z["numIters"])
    eta = P.solve_for_pressure_post(L, tmap, np.where(O.interior_mask(L), x, 0.0), x0, f["recip_Bo"])
    np.testing.assert_array_equal(eta, z["etaN"])


INI_KEYS = ("hFacW", "hFacS", "drF", "dyG", "dxG", "recip_dxC", "recip_dyC", "implicSurfPress", "implicDiv2DFlow")


@pytest.mark.parametrize("name", list(PRESSURE_CASES))
def test_ini_cg2d_norm_oracle_matches_reference(name):
    """ini_cg2d_norm (cg2d.py:108-134): the oracle's cg2dNorm equals the reference's bit for bit."""
    syn, f, prev, z = load_pressure(name)
    got = P.ini_cg2d_norm(syn.L, **{k: f[k] for k in INI_KEYS})
    assert got == float(z["ini_cg2d_norm"])


def test_update_keeps_preconditioner_outside_its_range():
    """pW, pS, pC are rewritten on j, i = 1..sNy+1, 1..sNx+1 only (solve_for_pressure.py:64-65)."""
    syn, f, prev, z = load_pressure("llc8_nr5")
    L = syn.L
    keep = np.ones(L.shape2d, bool)
    keep[:, L.js(1, L.sNy + 1), L.is_(1, L.sNx + 1)] = False
    for k, p0 in zip(("pW", "pS", "pC"), prev):
        np.testing.assert_array_equal(z[k][keep], p0[keep])
