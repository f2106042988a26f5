"""The steps either side of the solve on the GPU (mit_jax_b200.pressure: update_cg2d, cg2d_rhs, solve_for_pressure
through cg2d_update_operator, cg2d_pressure_rhs, cg2d_pressure_post), bit for bit against the reference's own
outputs (golden fixtures) and, batched on LLC90 with 50 levels and one cg2dNorm per member, against the oracle."""

import types

import numpy as np
import pytest
import torch

from golden_cases import PRESSURE_CASES, load_pressure
from oracle import pressure_oracle as P

pytestmark = pytest.mark.gpu

cg = pytest.importorskip("mit_jax_b200.cg2d")
pr = pytest.importorskip("mit_jax_b200.pressure")
OPS = ("aW2d", "aS2d", "aC2d", "pW", "pS", "pC")


def _params(f):
    return pr.FreeSurfParams(deltaTMom=f["deltaTMom"], deltaTFreeSurf=f["deltaTFreeSurf"], freeSurfFac=f["freeSurfFac"],
                             implicSurfPress=f["implicSurfPress"], implicDiv2DFlow=f["implicDiv2DFlow"],
                             mass2rUnit=f["mass2rUnit"], rUnit2mass=1.0 / f["mass2rUnit"], facEmP=1.0, hFacInf=0.2,
                             hFacSup=2.0, rStarAreaWeight=True, pfFacMom=1.0, select_rStar=2, nonlinFreeSurf=4,
                             useRealFreshWaterFlux=f["useRealFreshWaterFlux"], Nr=f["Nr"])


def _grid(syn, f):
    return types.SimpleNamespace(layout=syn.L, **{k: f[k] for k in ("drF", "dyG", "dxG", "recip_dxC", "recip_dyC",
                                                                     "rA", "maskInC")})


@pytest.mark.parametrize("name", list(PRESSURE_CASES))
def test_pressure_steps_match_reference_bitwise(name):
    syn, f, prev, z = load_pressure(name)
    ex = cg.default_exchanger(syn.L)
    p, g = _params(f), _grid(syn, f)
    cp = cg.Cg2dParams(cg2dMaxIters=300, cg2dTolerance=1e-12, cg2dNorm=f["cg2dNorm"],
                       cg2dpcOffDFac=f["cg2dpcOffDFac"], sum_order="fortran")
    ops = pr.update_cg2d(p, cp, g, ex, f["hFacW"], f["hFacS"], f["recip_Bo"], *prev)
    for k, a in zip(OPS, ops):
        np.testing.assert_array_equal(a, z[k], err_msg=k)
    np.testing.assert_array_equal(prev[0][0, 0], ops[3][0, 0])   # a kept point of the previous preconditioner
    b, x0 = pr.cg2d_rhs(p, g, f["gU"], f["gV"], f["hFacW"], f["hFacS"], f["EmPmR"], f["etaN"], f["etaH"],
                        f["Bo_surf"])
    np.testing.assert_array_equal(b, z["cg2d_b"])
    np.testing.assert_array_equal(x0, z["cg2d_x"])
    eta, info = pr.solve_for_pressure(p, cp, g, ex, ops, f["gU"], f["gV"], f["hFacW"], f["hFacS"], f["EmPmR"],
                                      f["etaN"], f["etaH"], f["Bo_surf"], f["recip_Bo"])
    assert info["numIters"] == int(z["numIters"])
    np.testing.assert_array_equal(np.array([info["firstResidual"], info["lastResidual"], info["sumRHS"],
                                            info["rhsMax"]]), z["diag"])
    np.testing.assert_array_equal(eta, z["etaN"])


INI_KEYS = ("hFacW", "hFacS", "drF", "dyG", "dxG", "recip_dxC", "recip_dyC", "implicSurfPress", "implicDiv2DFlow")


@pytest.mark.parametrize("name", list(PRESSURE_CASES))
def test_ini_cg2d_norm_matches_reference_bitwise(name):
    """ini_cg2d_norm on the GPU (cg2d_ini_norm): the reference's cg2dNorm bit for bit, as a float."""
    syn, f, prev, z = load_pressure(name)
    got = pr.ini_cg2d_norm(_grid(syn, f), f["hFacW"], f["hFacS"], f["implicSurfPress"], f["implicDiv2DFlow"])
    assert isinstance(got, float) and got == float(z["ini_cg2d_norm"])


def test_ini_cg2d_norm_batched_llc90_nr50():
    """Three LLC90 members with 50 levels in one call: each member's cg2dNorm equals the oracle's bit for bit."""
    from mit_jax_b200.synthetic import LLCSynthetic
    syn = LLCSynthetic(90)
    fs = [syn.model_fields(50, m) for m in range(3)]
    g = _grid(syn, fs[0])
    hW = np.stack([f["hFacW"] for f in fs])
    hS = np.stack([f["hFacS"] for f in fs])
    got = pr.ini_cg2d_norm(g, hW, hS, fs[0]["implicSurfPress"], fs[0]["implicDiv2DFlow"])
    assert got.shape == (3,)
    for m, f in enumerate(fs):
        ref = P.ini_cg2d_norm(syn.L, **{k: (f if k.startswith("hFac") else fs[0])[k] for k in INI_KEYS})
        assert got[m] == ref, (m, got[m], ref)


def test_pressure_steps_batched_llc90_nr50():
    """Three LLC90 members with 50 levels in one call of each step, one cg2dNorm per member; every member equals
    its oracle bit for bit; then a batched mixed-precision solve_for_pressure converges for every member."""
    from mit_jax_b200.synthetic import LLCSynthetic
    syn = LLCSynthetic(90)
    fs = [syn.model_fields(50, m) for m in range(3)]
    f0 = fs[0]
    dev = torch.device("cuda")
    ex = cg.default_exchanger(syn.L)
    p, g = _params(f0), _grid(syn, f0)
    stack = {k: torch.as_tensor(np.stack([f[k] for f in fs])).to(dev)
             for k in ("hFacW", "hFacS", "gU", "gV", "EmPmR", "etaN", "etaH")}
    norms = np.array([f["cg2dNorm"] for f in fs])
    rng = np.random.default_rng(5)
    prev = [torch.as_tensor(rng.standard_normal((3,) + syn.L.shape2d)).to(dev) for _ in range(3)]
    cp = cg.Cg2dParams(cg2dMaxIters=300, cg2dTolerance=1e-12, cg2dNorm=torch.as_tensor(norms),
                       cg2dpcOffDFac=f0["cg2dpcOffDFac"], sum_order="rowblock", precision="mixed")
    ops = pr.update_cg2d(p, cp, g, ex, stack["hFacW"], stack["hFacS"], f0["recip_Bo"], *prev)
    b, x0 = pr.cg2d_rhs(p, g, stack["gU"], stack["gV"], stack["hFacW"], stack["hFacS"], stack["EmPmR"],
                        stack["etaN"], stack["etaH"], f0["Bo_surf"])
    L, tmap = syn.L, syn.topo.maps["T"]
    kw = {k: f0[k] for k in ("drF", "dyG", "dxG", "recip_dxC", "recip_dyC", "rA", "recip_Bo", "cg2dpcOffDFac",
                             "implicSurfPress", "implicDiv2DFlow", "freeSurfFac", "deltaTMom", "deltaTFreeSurf")}
    for m, f in enumerate(fs):
        o = P.update_cg2d(L, tmap, hFacW=f["hFacW"], hFacS=f["hFacS"], pW=prev[0][m].cpu().numpy(),
                          pS=prev[1][m].cpu().numpy(), pC=prev[2][m].cpu().numpy(), cg2dNorm=norms[m], **kw)
        for k, a, e in zip(OPS, ops, o):
            np.testing.assert_array_equal(a[m].cpu().numpy(), e, err_msg=f"{k} member {m}")
        ob, ox = P.cg2d_rhs(L, **{k: f[k] for k in ("gU", "gV", "hFacW", "hFacS", "EmPmR", "etaN", "etaH")},
                            **{k: f0[k] for k in ("Bo_surf", "drF", "dyG", "dxG", "rA", "maskInC", "freeSurfFac",
                                                  "mass2rUnit", "implicDiv2DFlow", "deltaTMom", "deltaTFreeSurf",
                                                  "useRealFreshWaterFlux")})
        np.testing.assert_array_equal(b[m].cpu().numpy(), ob)
        np.testing.assert_array_equal(x0[m].cpu().numpy(), ox)
    eta, info = pr.solve_for_pressure(p, cp, g, ex, ops, stack["gU"], stack["gV"], stack["hFacW"], stack["hFacS"],
                                      stack["EmPmR"], stack["etaN"], stack["etaH"], f0["Bo_surf"], f0["recip_Bo"])
    assert [r["status"] for r in info["records"]] == ["ok"] * 3
    assert eta.shape == (3,) + syn.L.shape2d and torch.isfinite(eta).all()
