"""Array layout of the CG2D fields: `[tile, j, i]` float64 with OLx/OLy halo points on every side.

Mirrors mitgcm_jax/layout.py:16-54 (the reference's `Layout`): tile t (0-based) is exch2 tile t+1, a Fortran index
i (1-based; halo points <= 0 or > sNx) sits at array index i - 1 + OLx. A batch of instances adds a leading axis:
`[batch, tile, j, i]`.
"""

from dataclasses import dataclass


@dataclass(frozen=True)
class Layout:
    sNx: int = 90
    sNy: int = 90
    OLx: int = 4
    OLy: int = 4
    nTiles: int = 13
    Nr: int = 50

    @property
    def nx(self):
        return self.sNx + 2 * self.OLx

    @property
    def ny(self):
        return self.sNy + 2 * self.OLy

    def is_(self, lo, hi):
        """Array slice of the Fortran i-range lo..hi (inclusive)."""
        return slice(lo - 1 + self.OLx, hi + self.OLx)

    def js(self, lo, hi):
        """Array slice of the Fortran j-range lo..hi (inclusive)."""
        return slice(lo - 1 + self.OLy, hi + self.OLy)

    def ii(self, i):
        return i - 1 + self.OLx

    def jj(self, j):
        return j - 1 + self.OLy

    @property
    def shape2d(self):
        return (self.nTiles, self.ny, self.nx)

    @property
    def interior(self):
        """(j-slice, i-slice) of the interior points i = 1..sNx, j = 1..sNy."""
        return self.js(1, self.sNy), self.is_(1, self.sNx)

    @property
    def n_points(self):
        return self.nTiles * self.sNx * self.sNy


LLC90 = Layout()
LLC270 = Layout(sNx=270, sNy=270)
