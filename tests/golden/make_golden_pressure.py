"""Generate the golden fixtures of the steps either side of the solve from the REFERENCE's own code (run once, where
the reference source is available; the fixtures are committed and the tests never read the reference).

    python tests/golden/make_golden_pressure.py [--reference /root/reference]

pressure_<case>.npz: outputs of mitgcm_jax.core.solve_for_pressure.update_cg2d (:29-65), cg2d_rhs (:68-106) and
solve_for_pressure (:109-123, with cg2d_solve in sum_order="fortran"), and of mitgcm_jax.core.cg2d.ini_cg2d_norm
(:108-134) on the same face fractions, executed by the reference module itself
through the numpy stand-in for JAX (jax_standin.py), on seeded synthetic model fields
(mit_jax_b200.synthetic.LLCSynthetic.model_fields) with exchange maps from mit_jax_b200.topology. The inputs are
regenerated by the tests from the stored case parameters; their SHA-256 is stored to catch a changed generator.
The previous preconditioner handed to update_cg2d is seeded noise, so that the points it keeps are checked too.
"""

import argparse
import sys
import types
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]
sys.path.insert(0, str(REPO))
sys.path.insert(0, str(HERE))
sys.path.insert(0, str(REPO / "tests"))

from golden_cases import PRESSURE_CASES as CASES  # noqa: E402
from golden_cases import pressure_inputs as case_inputs  # noqa: E402
from golden_cases import pressure_sha  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default="/root/reference")
    args = ap.parse_args()
    import jax_standin
    jax_standin.install()
    sys.path.insert(0, args.reference)
    from mitgcm_jax.core import cg2d as refcg
    from mitgcm_jax.core import solve_for_pressure as sfp
    from mitgcm_jax.core.free_surface import FreeSurfParams
    from mitgcm_jax.layout import Layout as RefLayout
    from mitgcm_jax.parallel.exchange import ExchangeMaps, Exchanger

    from oracle import cg2d_oracle as O
    from oracle import pressure_oracle as P

    for name, c in CASES.items():
        syn, f, prev = case_inputs(**c)
        L, tmap = syn.L, syn.topo.maps["T"]
        rl = RefLayout(L.sNx, L.sNy, L.OLx, L.OLy, L.nTiles, c["Nr"])
        ex = Exchanger(ExchangeMaps(rl, {"T": (np.asarray(tmap[0], np.int32), np.asarray(tmap[1], np.int8),
                                               np.asarray(tmap[2], np.float64))}))
        g = types.SimpleNamespace(layout=rl, drF=f["drF"], dyG=f["dyG"], dxG=f["dxG"], recip_dxC=f["recip_dxC"],
                                  recip_dyC=f["recip_dyC"], rA=f["rA"], maskInC=f["maskInC"],
                                  maskC=(f["hFacW"] > 0).astype(np.float64))
        p = FreeSurfParams(deltaTMom=f["deltaTMom"], deltaTFreeSurf=f["deltaTFreeSurf"], freeSurfFac=f["freeSurfFac"],
                           implicSurfPress=f["implicSurfPress"], implicDiv2DFlow=f["implicDiv2DFlow"],
                           mass2rUnit=f["mass2rUnit"], rUnit2mass=1.0 / f["mass2rUnit"], facEmP=1.0, hFacInf=0.2,
                           hFacSup=2.0, rStarAreaWeight=True, pfFacMom=1.0, select_rStar=2, nonlinFreeSurf=4,
                           useRealFreshWaterFlux=f["useRealFreshWaterFlux"], Nr=c["Nr"])
        cp = refcg.Cg2dParams(cg2dMaxIters=300, cg2dTolerance=1e-12, cg2dNorm=f["cg2dNorm"],
                              cg2dpcOffDFac=f["cg2dpcOffDFac"], sum_order="fortran")
        ops = tuple(np.asarray(a, np.float64) for a in sfp.update_cg2d(p, cp, g, ex, f["hFacW"], f["hFacS"],
                                                                       f["recip_Bo"], *prev))
        cg2d_b, cg2d_x = (np.asarray(a, np.float64) for a in sfp.cg2d_rhs(
            p, g, f["gU"], f["gV"], f["hFacW"], f["hFacS"], f["EmPmR"], f["etaN"], f["etaH"], f["Bo_surf"]))
        etaN_new, info = sfp.solve_for_pressure(p, cp, g, ex, ops, f["gU"], f["gV"], f["hFacW"], f["hFacS"],
                                                f["EmPmR"], f["etaN"], f["etaH"], f["Bo_surf"], f["recip_Bo"])
        etaN_new = np.asarray(etaN_new, np.float64)
        diag = np.array([float(info["firstResidual"]), float(info["lastResidual"]), float(info["sumRHS"]),
                         float(info["rhsMax"])])
        it = int(info["numIters"])

        # the oracle restatement must reproduce every output bit for bit
        kw = {k: f[k] for k in ("drF", "dyG", "dxG", "recip_dxC", "recip_dyC", "rA", "recip_Bo", "cg2dNorm",
                                "cg2dpcOffDFac", "implicSurfPress", "implicDiv2DFlow", "freeSurfFac", "deltaTMom",
                                "deltaTFreeSurf")}
        o_ops = P.update_cg2d(L, tmap, hFacW=f["hFacW"], hFacS=f["hFacS"], pW=prev[0], pS=prev[1], pC=prev[2], **kw)
        for a, b in zip(o_ops, ops):
            assert np.array_equal(a, b), name
        o_b, o_x = P.cg2d_rhs(L, **{k: f[k] for k in ("gU", "gV", "hFacW", "hFacS", "EmPmR", "etaN", "etaH",
                                                       "Bo_surf", "drF", "dyG", "dxG", "rA", "maskInC",
                                                       "freeSurfFac", "mass2rUnit", "implicDiv2DFlow", "deltaTMom",
                                                       "deltaTFreeSurf", "useRealFreshWaterFlux")})
        assert np.array_equal(o_b, cg2d_b) and np.array_equal(o_x, cg2d_x), name
        xs, ds = O.cg2d_fortran(L, tmap, ops, cg2d_b, cg2d_x, cg2dNorm=f["cg2dNorm"], tolerance=1e-12,
                                max_iters=300, sum_order="fortran")
        x_int = np.where(O.interior_mask(L), xs, 0.0)
        o_eta = P.solve_for_pressure_post(L, tmap, x_int, cg2d_x, f["recip_Bo"])
        assert np.array_equal(o_eta, etaN_new) and ds["numIters"] == it, name
        # ini_cg2d_norm (cg2d.py:108-134) on the same face fractions
        ini = refcg.ini_cg2d_norm(g, f["hFacW"], f["hFacS"], f["implicSurfPress"], f["implicDiv2DFlow"])
        o_ini = P.ini_cg2d_norm(L, **{k: f[k] for k in ("hFacW", "hFacS", "drF", "dyG", "dxG", "recip_dxC",
                                                         "recip_dyC", "implicSurfPress", "implicDiv2DFlow")})
        assert float(o_ini) == float(ini), name

        np.savez_compressed(HERE / f"pressure_{name}.npz", **{k: v for k, v in c.items() if v is not None},
                            inputs_sha=pressure_sha(f, prev),
                            aW2d=ops[0], aS2d=ops[1], aC2d=ops[2], pW=ops[3], pS=ops[4], pC=ops[5],
                            cg2d_b=cg2d_b, cg2d_x=cg2d_x, etaN=etaN_new, diag=diag, numIters=it,
                            ini_cg2d_norm=np.float64(ini))
        print(f"{name}: Nr={c['Nr']} iters={it} last={diag[1]:.3e}")


if __name__ == "__main__":
    main()
