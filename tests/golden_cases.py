"""Loading of the committed golden fixtures (tests/golden/cg2d_*.npz, made by tests/golden/make_golden.py)."""

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
