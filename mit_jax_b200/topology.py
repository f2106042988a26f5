"""LLC exch2 connectivity: the 5-facet lat-lon-cap topology generated from its facet edge links.

The reference ships the connectivity only for LLC90, as exchange maps probed from the Fortran exch2 routines
(mitgcm_jax/data/exch_maps_13x90x90.npz, built by mitgcm_jax/parallel/exchange.py:95-122). This module generates the
same maps for any facet size N and square tile size from the facet topology itself:

* facet shapes (nx, ny): (N, 3N), (N, 3N), (N, N), (3N, N), (3N, N) -- `dimsFacets` of the reference's
  data.exch2_13x90x90:24 (reference/data.exch2_13x90x90), facets split into tiles of ts x ts numbered facet by facet,
  x fastest (mitgcm_jax/grid/load.py:233-249, w2_set_map_tiles.F);
* facet edge links (`facetEdgeLink` of data.exch2_13x90x90:25-29): facet f's edge e touches facet f2's edge e2.
  Along an edge the position runs with i for N/S edges and with j for E/W edges; it is kept when the two edges are
  of the same kind (N-S or E-W) and reversed when one is N/S and the other E/W (the rotated facets 4-5 and the
  cap).

Only the points the 5-point stencil and the face-coefficient exchange need are generated: the first halo row and
column of every tile, corners excluded. Output uses the reference's ExchangeMaps format (exchange.py:73-93):
per padded point a source index `src` into the flat [T, ny, nx] array, `comp` (0 = point keeps its value,
1 = u-like/scalar source, 2 = v-like source) and `sign`. Kinds generated: "T" (scalar, EXCH_XY_RL) and
"UVn_u"/"UVn_v" (EXCH_UV_XY_RL(u, v, .FALSE.)) at the east face column i = sNx+1 of u and the north face row
j = sNy+1 of v, which is what INI_CG2D's face exchange fills for the operator (init.py:350).
"""

from dataclasses import dataclass

import numpy as np

from mit_jax_b200.layout import Layout

# facetEdgeLink of the LLC 5-facet topology (edges N, S, E, W); None = open edge
FACET_LINKS = {
    1: {"N": (3, "W"), "S": None, "E": (2, "W"), "W": (5, "N")},
    2: {"N": (3, "S"), "S": None, "E": (4, "S"), "W": (1, "E")},
    3: {"N": (5, "W"), "S": (2, "N"), "E": (4, "W"), "W": (1, "N")},
    4: {"N": (5, "S"), "S": (2, "E"), "E": None, "W": (3, "E")},
    5: {"N": (1, "W"), "S": (4, "N"), "E": None, "W": (3, "N")},
}


def facet_dims(N):
    """{facet: (nx, ny)} of the LLC-N grid."""
    return {1: (N, 3 * N), 2: (N, 3 * N), 3: (N, N), 4: (3 * N, N), 5: (3 * N, N)}


@dataclass(frozen=True)
class LLCGrid:
    N: int          # facet size (90 for LLC90)
    ts: int         # tile size

    @property
    def dims(self):
        return facet_dims(self.N)

    def tiles(self):
        """[(facet, I0, J0)] for tile ids 0.. (facet by facet, x fastest)."""
        out = []
        for f in range(1, 6):
            fx, fy = self.dims[f]
            if fx % self.ts or fy % self.ts:
                raise ValueError(f"facet {f} ({fx}x{fy}) is not a multiple of the tile size {self.ts}")
            for ty in range(fy // self.ts):
                for tx in range(fx // self.ts):
                    out.append((f, tx * self.ts, ty * self.ts))
        return out

    @property
    def nTiles(self):
        return len(self.tiles())

    def layout(self, OL=4):
        return Layout(sNx=self.ts, sNy=self.ts, OLx=OL, OLy=OL, nTiles=self.nTiles)


def _cross(dims, f, e, pos):
    """Facet point just across edge e of facet f at edge position pos, as (f2, I, J, e2); None if open."""
    link = FACET_LINKS[f][e]
    if link is None:
        return None
    f2, e2 = link
    nx, ny = dims[f]
    nx2, ny2 = dims[f2]
    length = nx if e in "NS" else ny
    length2 = nx2 if e2 in "NS" else ny2
    if length != length2:
        raise ValueError(f"edge {f}{e} ({length}) does not match {f2}{e2} ({length2})")
    same_kind = (e in "NS") == (e2 in "NS")
    p2 = pos if same_kind else length - 1 - pos
    if e2 == "N":
        return f2, p2, ny2 - 1, e2
    if e2 == "S":
        return f2, p2, 0, e2
    if e2 == "E":
        return f2, nx2 - 1, p2, e2
    return f2, 0, p2, e2


def facet_neighbour(dims, f, I, J, d):
    """Facet point next to (f, I, J) in direction d (N, S, E, W) as (f2, I2, J2, e2), e2 = the edge of f2 that was
    crossed (None inside a facet); None across an open edge."""
    nx, ny = dims[f]
    I2, J2 = I + {"E": 1, "W": -1}.get(d, 0), J + {"N": 1, "S": -1}.get(d, 0)
    if 0 <= I2 < nx and 0 <= J2 < ny:
        return f, I2, J2, None
    return _cross(dims, f, d, I if d in "NS" else J)


class LLCTopology:
    """Generated exchange maps of one LLC layout (facet size N, tile size ts, halo OL)."""

    def __init__(self, N=90, ts=None, OL=4):
        ts = N if ts is None else ts
        self.grid = LLCGrid(N, ts)
        self.L = self.grid.layout(OL)
        self._tiles = self.grid.tiles()
        self._index = {(f, I0, J0): t for t, (f, I0, J0) in enumerate(self._tiles)}
        self._build()

    def _tile_of(self, f, I, J):
        ts = self.grid.ts
        t = self._index[(f, (I // ts) * ts, (J // ts) * ts)]
        return t, J % ts, I % ts

    def _pad(self, t, j, i):
        L = self.L
        return (t * L.ny + (j + L.OLy)) * L.nx + (i + L.OLx)

    def _build(self):
        L, dims, ts = self.L, self.grid.dims, self.grid.ts
        npad = L.nTiles * L.ny * L.nx
        own = np.arange(npad, dtype=np.int32)
        T_src, T_comp = own.copy(), np.zeros(npad, np.int8)
        Uu_src, Uu_comp = own.copy(), np.zeros(npad, np.int8)
        Uv_src, Uv_comp = own.copy(), np.zeros(npad, np.int8)
        for t, (f, I0, J0) in enumerate(self._tiles):
            for k in range(ts):
                # (halo position in this tile (j, i), facet point on the tile edge, direction)
                for (hj, hi), (I, J), d in (((k, -1), (I0, J0 + k), "W"), ((k, ts), (I0 + ts - 1, J0 + k), "E"),
                                            ((-1, k), (I0 + k, J0), "S"), ((ts, k), (I0 + k, J0 + ts - 1), "N")):
                    nb = facet_neighbour(dims, f, I, J, d)
                    p = self._pad(t, hj, hi)
                    if nb is None:
                        continue
                    f2, I2, J2, e2 = nb
                    t2, j2, i2 = self._tile_of(f2, I2, J2)
                    T_src[p], T_comp[p] = self._pad(t2, j2, i2), 1
                    # faces: u at the east face column (i = ts, the face between the edge point and its east
                    # neighbour), v at the north face row; the neighbour's face toward this tile is its W face
                    # (u, same point) when entered through its W edge or inside a facet, its S face (v) through
                    # its S edge
                    if d in ("E", "N"):
                        kind = e2 if e2 is not None else ("W" if d == "E" else "S")
                        if kind == "W":
                            comp, src = 1, self._pad(t2, j2, i2)
                        elif kind == "S":
                            comp, src = 2, self._pad(t2, j2, i2)
                        else:
                            raise ValueError(f"face across {f}{d} lands on edge {e2}: not an LLC topology")
                        if d == "E":
                            Uu_src[p], Uu_comp[p] = src, comp
                        else:
                            Uv_src[p], Uv_comp[p] = src, comp
        ones = np.ones(npad, np.int8)
        self.maps = {"T": (T_src, T_comp, ones), "UVn_u": (Uu_src, Uu_comp, ones), "UVn_v": (Uv_src, Uv_comp, ones)}

    # -------------------------------------------------------------------------------------------------------
    def stencil_points(self):
        """Flat padded indices of the first halo row/column (corners excluded), in tile, side (W, E, S, N), k order."""
        L, ts = self.L, self.grid.ts
        pts = []
        for t in range(L.nTiles):
            for hj, hi in ([(k, -1) for k in range(ts)] + [(k, ts) for k in range(ts)]
                           + [(-1, k) for k in range(ts)] + [(ts, k) for k in range(ts)]):
                pts.append(self._pad(t, hj, hi))
        return np.asarray(pts, np.int64)


def exch_scalar(a, src, comp):
    """Exchanger._apply for a scalar kind (exchange.py:136-142) on [..., T, ny, nx]: comp==1 -> a[src], else a."""
    a = np.asarray(a, np.float64)
    lead = a.shape[:-3]
    flat = a.reshape(lead + (-1,))
    out = np.where(comp == 1, flat[..., src], flat)
    return out.reshape(a.shape)


def exch_vector(u, v, maps_u, maps_v):
    """Exchanger.vector (exchange.py:174-179) for the generated face kinds (sign +1)."""
    u = np.asarray(u, np.float64)
    v = np.asarray(v, np.float64)
    lead = u.shape[:-3]
    fu, fv = u.reshape(lead + (-1,)), v.reshape(lead + (-1,))

    def apply(m, own):
        src, comp, sign = m
        out = np.where(comp == 1, fu[..., src], own)
        out = np.where(comp == 2, fv[..., src], out)
        return out * sign

    return apply(maps_u, fu).reshape(u.shape), apply(maps_v, fv).reshape(v.shape)


def exch_vector_adjoint(gu, gv, maps_u, maps_v):
    """The transpose of exch_vector: cotangents of the (u, v) that exch_vector reads, given cotangents (gu, gv) of
    the pair it returns. An entry that exch_vector copies from another adds its cotangent onto that source and
    keeps none; an entry it keeps passes its own through.

    Applied to coefficient cotangents of a solve (aW2d, aS2d), which are per array entry, it gives the cotangents
    of the physical faces: a face on a tile edge is stored twice, as the tile's edge entry and as the
    neighbour's halo entry filled by this exchange (mitgcm_jax/init.py:345-350), and moving the face moves both.
    Per entry, the two copies may be moved apart, which makes the operator unsymmetric."""
    gu = np.asarray(gu, np.float64)
    gv = np.asarray(gv, np.float64)
    shape = gu.shape
    fu, fv = gu.reshape(-1, int(np.prod(shape[-3:]))), gv.reshape(-1, int(np.prod(shape[-3:])))
    ou, ov = np.zeros_like(fu), np.zeros_like(fv)
    for (src, comp, sign), g, own in ((maps_u, fu, ou), (maps_v, fv, ov)):
        src, comp = np.asarray(src).astype(np.int64), np.asarray(comp)
        sg = g * np.asarray(sign, np.float64)
        keep = comp == 0
        own[:, keep] += sg[:, keep]
        for c, tgt in ((1, ou), (2, ov)):
            sel = comp == c
            np.add.at(tgt, (slice(None), src[sel]), sg[:, sel])
    return ou.reshape(shape), ov.reshape(shape)
