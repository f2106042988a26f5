"""Loading of the committed golden fixtures: tests/golden/cg2d_*.npz (made by tests/golden/make_golden.py) and
tests/golden/pressure_*.npz (made by tests/golden/make_golden_pressure.py)."""

from pathlib import Path

import numpy as np

from mit_jax_b200.topology import LLCTopology

GOLDEN = Path(__file__).resolve().parent / "golden"
CASES = ("llc8", "llc16_guess", "llc8_cap", "llc8_onemore", "llc8_zero_rhs", "llc8_zero_iters")
OPS = ("aW2d", "aS2d", "aC2d", "pW", "pS", "pC")


class Case:
    def __init__(self, name):
        z = np.load(GOLDEN / f"cg2d_{name}.npz")
        self.name = name
        self.N, self.ts, self.OL = int(z["N"]), int(z["ts"]), int(z["OL"])
        self.tol, self.maxit, self.norm = float(z["tol"]), int(z["maxit"]), float(z["cg2dNorm"])
        self.ops = tuple(z[k] for k in OPS)
        self.b, self.x0 = z["b"], z["x0"]
        self.x_fortran, self.diag, self.numIters = z["x_fortran"], z["diag"], int(z["numIters"])
        self.topo = LLCTopology(self.N, self.ts, self.OL)
        self.L = self.topo.L
        self.tmap = self.topo.maps["T"]


def load(name):
    return Case(name)


# ---- the steps either side of the solve (update_cg2d, cg2d_rhs, solve_for_pressure)

PRESSURE_CASES = {
    "llc8_nr5": dict(N=8, ts=8, OL=4, Nr=5, member=None, fresh_water=True),
    "llc8_nr3_m1_nofw": dict(N=8, ts=8, OL=4, Nr=3, member=1, fresh_water=False),
}
PRESSURE_INPUT_KEYS = ("drF", "hFacW", "hFacS", "dyG", "dxG", "recip_dxC", "recip_dyC", "rA", "maskInC", "Bo_surf",
                       "recip_Bo", "gU", "gV", "EmPmR", "etaN", "etaH")


def pressure_inputs(N, ts, OL, Nr, member, fresh_water):
    """(syn, fields, previous preconditioner (pW, pS, pC)) of a case: seeded synthetic model fields."""
    from mit_jax_b200.synthetic import LLCSynthetic
    syn = LLCSynthetic(N, ts, OL)
    f = syn.model_fields(Nr, member)
    f["useRealFreshWaterFlux"] = fresh_water
    rng = np.random.default_rng(11)
    prev = tuple(rng.standard_normal(syn.L.shape2d) for _ in range(3))
    return syn, f, prev


def pressure_sha(f, prev):
    import hashlib
    h = hashlib.sha256()
    for a in [f[k] for k in PRESSURE_INPUT_KEYS] + list(prev):
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def load_pressure(name):
    """(syn, fields, prev, expected outputs dict) of a pressure case."""
    syn, f, prev = pressure_inputs(**PRESSURE_CASES[name])
    z = dict(np.load(GOLDEN / f"pressure_{name}.npz"))
    return syn, f, prev, z
