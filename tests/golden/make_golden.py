"""Generate the golden fixtures of tests/golden from the REFERENCE's own code (run once, where the reference source
is available; the fixtures are committed and the tests never read the reference).

    python tests/golden/make_golden.py [--reference /root/reference]

* cg2d_*.npz: inputs and outputs of mitgcm_jax.core.cg2d.cg2d_fortran (mitgcm_jax/core/cg2d.py:205-269) with
  sum_order="fortran", executed by the reference module itself through the numpy stand-in for JAX
  (jax_standin.py), on seeded synthetic LLC problems (mit_jax_b200.synthetic) with exchange maps from
  mit_jax_b200.topology. Cases cover convergence, a non-zero first guess with halo values, the iteration cap,
  the stop rule (tolerance 0.99 x the last residual -> exactly one more iteration, test_cg2d.py:187-189),
  a zero right-hand side and a zero-iteration solve.
* cg2d_llc90_ref_map.npz: the same on LLC90 with the reference's probed exchange map
  (mitgcm_jax/data/exch_maps_13x90x90.npz); inputs are regenerated by the tests (their SHA-256 is stored), the
  output is stored as a SHA-256 plus diagnostics and samples.
* llc90_T_map.npz: the reference's LLC90 scalar map (T.src, T.comp) and the UVn face maps at the face halos, for
  the topology tests and for x_fortran halos with the full map.
"""

import argparse
import hashlib
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]
sys.path.insert(0, str(REPO))
sys.path.insert(0, str(HERE))


def sha(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def run_reference(refcg, Exchanger, ExchangeMaps, RefLayout, L, tmap, ops, b, x0, norm, tol, maxit):
    rl = RefLayout(L.sNx, L.sNy, L.OLx, L.OLy, L.nTiles, 50)
    ex = Exchanger(ExchangeMaps(rl, {"T": (np.asarray(tmap[0], np.int32), np.asarray(tmap[1], np.int8),
                                           np.asarray(tmap[2], np.float64))}))
    x, d = refcg.cg2d_fortran(ex, ops, b, x0, cg2dNorm=norm, tolerance=tol, max_iters=maxit, sum_order="fortran")
    diag = np.array([float(d["firstResidual"]), float(d["lastResidual"]), float(d["sumRHS"]), float(d["rhsMax"])])
    return np.asarray(x, np.float64), diag, int(d["numIters"])


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default="/root/reference")
    args = ap.parse_args()
    import jax_standin
    jax_standin.install()
    sys.path.insert(0, args.reference)
    from mitgcm_jax.core import cg2d as refcg
    from mitgcm_jax.layout import Layout as RefLayout
    from mitgcm_jax.parallel.exchange import ExchangeMaps, Exchanger

    from mit_jax_b200.synthetic import LLCSynthetic
    from oracle import cg2d_oracle as O

    def case(name, N, ts, OL, tol=1e-12, maxit=300, x0_kind="zero", b_kind="rhs", member=None):
        syn = LLCSynthetic(N, ts, OL)
        L, tmap = syn.L, syn.topo.maps["T"]
        ops, norm = syn.operator(member)
        b = syn.rhs(member) if b_kind == "rhs" else np.zeros(L.shape2d)
        if x0_kind == "zero":
            x0 = syn.first_guess()
        else:
            x0 = np.random.default_rng(7).standard_normal(L.shape2d) * 1e-3   # halos included
        x, diag, it = run_reference(refcg, Exchanger, ExchangeMaps, RefLayout, L, tmap, ops, b, x0, norm, tol, maxit)
        xo, do = O.cg2d_fortran(L, tmap, ops, b, x0, cg2dNorm=norm, tolerance=tol, max_iters=maxit,
                                sum_order="fortran")
        assert np.array_equal(xo, x) and do["numIters"] == it, name
        np.savez_compressed(HERE / f"cg2d_{name}.npz", N=N, ts=ts, OL=OL, tol=tol, maxit=maxit, cg2dNorm=norm,
                            aW2d=ops[0], aS2d=ops[1], aC2d=ops[2], pW=ops[3], pS=ops[4], pC=ops[5], b=b, x0=x0,
                            x_fortran=x, diag=diag, numIters=it)
        print(f"{name}: N={N} ts={ts} OL={OL} iters={it} last={diag[1]:.3e}")
        return it, diag

    it, diag = case("llc8", 8, 8, 4)
    case("llc16_guess", 16, 8, 2, x0_kind="random")
    case("llc8_cap", 8, 8, 4, maxit=5)
    case("llc8_onemore", 8, 8, 4, tol=0.99 * diag[1])
    case("llc8_zero_rhs", 8, 8, 4, b_kind="zero", x0_kind="random")
    case("llc8_zero_iters", 8, 8, 4, tol=1e3)

    # LLC90 with the reference's probed map
    zmap = np.load(Path(args.reference) / "mitgcm_jax" / "data" / "exch_maps_13x90x90.npz")
    tmap = (zmap["T.src"].astype(np.int32), zmap["T.comp"].astype(np.int8), zmap["T.sign"].astype(np.int8))
    syn = LLCSynthetic(90)
    L = syn.L
    ops, norm = syn.operator()
    b, x0 = syn.rhs(), syn.first_guess()
    x, diag, it = run_reference(refcg, Exchanger, ExchangeMaps, RefLayout, L, tmap, ops, b, x0, norm, 1e-12, 300)
    xo, do = O.cg2d_fortran(L, tmap, ops, b, x0, cg2dNorm=norm, tolerance=1e-12, max_iters=300, sum_order="fortran")
    assert np.array_equal(xo, x) and do["numIters"] == it
    np.savez_compressed(HERE / "cg2d_llc90_ref_map.npz", inputs_sha=sha(*ops, b, x0), cg2dNorm=norm,
                        x_sha=sha(x), diag=diag, numIters=it, sample_idx=np.arange(0, x.size, 997),
                        sample=x.reshape(-1)[::997])
    print(f"llc90_ref_map: iters={it} last={diag[1]:.3e}")

    pts_u = np.array([(t * 98 + (j + 4)) * 98 + 94 for t in range(13) for j in range(90)])
    pts_v = np.array([(t * 98 + 94) * 98 + (i + 4) for t in range(13) for i in range(90)])
    np.savez_compressed(HERE / "llc90_T_map.npz", src=tmap[0], comp=tmap[1],
                        uvn_u_pts=pts_u, uvn_u_src=zmap["UVn_u.src"][pts_u], uvn_u_comp=zmap["UVn_u.comp"][pts_u],
                        uvn_v_pts=pts_v, uvn_v_src=zmap["UVn_v.src"][pts_v], uvn_v_comp=zmap["UVn_v.comp"][pts_v])


if __name__ == "__main__":
    main()
