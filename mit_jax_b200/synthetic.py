"""Seeded synthetic CG2D inputs on an LLC grid (no ECCO data is available): land mask, depth, grid spacing, the
operator aW2d/aS2d/aC2d, the preconditioner pW/pS/pC, right-hand sides and adjoint cotangents.

Construction (all fields per facet, then cut into tiles as the layout does):
* land: standard-normal noise smoothed with a Gaussian of sigma = 5 N/90 cells, thresholded at its 30th percentile
  (about 30 % land); seed 0.
* depth H ~ U(500, 6000) m on ocean cells, 0 on land; seed 1. Ensemble member m multiplies it by
  1 + 0.1 e_m, e_m smooth noise scaled to [-1, 1], seed 1000 + m.
* spacing: a latitude-like coordinate per facet (facets 1-2 south to north along j, the cap from its centre,
  facets 4-5 along -i); dx = 20 km + 90 km cos(lat) (zonal), dy = 20 km + 90 km (0.5 + 0.5 cos(lat)), both scaled
  by 90/N; rA = dx dy.
* faces (interior, Fortran i, j = 1..N): aW = H_w dy/dx, aS = H_s dx/dy, H_w = min(H, H of the west neighbour)
  (0 across land or an open edge); cg2dNorm = 1/max|aW, aS| (ini_cg2d_norm, mitgcm_jax/core/cg2d.py:108-134);
  aW2d = aW cg2dNorm, aS2d = aS cg2dNorm; the east/north face halos come from the neighbour tiles through the
  UVn face exchange, as INI_CG2D does (mitgcm_jax/init.py:345-350).
* aC2d = -(aW2d(i) + aW2d(i+1) + aS2d(j) + aS2d(j+1) + cg2dNorm recip_Bo rA / dt / dt), recip_Bo = 1/g, g = 9.81,
  dt = 3600 s, exchanged (UPDATE_CG2D, mitgcm_jax/core/solve_for_pressure.py:49-53).
* pW, pS, pC from aW2d, aS2d, aC2d on i, j = 1..N+1 with cg2dpcOffDFac = 0.51 (solve_for_pressure.py:55-63).
* right-hand side: smoothed noise (same sigma), 0 on land, ocean mean removed; seed 2 (member m: 2000 + m).
  Adjoint cotangent: the same with seed 3 (member m: 3000 + m). First guess 0.
"""

import numpy as np
from scipy.ndimage import gaussian_filter

from mit_jax_b200.topology import LLCTopology, exch_scalar, exch_vector

GRAVITY = 9.81
DELTA_T = 3600.0
PC_OFFDIAG_FAC = 0.51


def _facet_noise(grid, seed, sigma):
    rng = np.random.default_rng(seed)
    out = {}
    for f in range(1, 6):
        nx, ny = grid.dims[f]
        out[f] = gaussian_filter(rng.standard_normal((ny, nx)), sigma=sigma, mode="nearest")
    return out


def _to_tiles(topo, fac, fill=0.0):
    """{facet: [ny, nx]} -> padded [T, ny, nx] (halos = fill)."""
    L, ts = topo.L, topo.grid.ts
    a = np.full(L.shape2d, fill, np.float64)
    J, I = L.interior
    for t, (f, I0, J0) in enumerate(topo.grid.tiles()):
        a[t, J, I] = fac[f][J0:J0 + ts, I0:I0 + ts]
    return a


def _latitude(grid):
    """A smooth latitude-like coordinate (radians) per facet."""
    N = grid.N
    lat = {}
    for f in (1, 2):
        nx, ny = grid.dims[f]
        jj = (np.arange(ny) + 0.5) / ny
        lat[f] = np.repeat((-75.0 + 140.0 * jj)[:, None], nx, axis=1)
    jj, ii = np.meshgrid((np.arange(N) + 0.5) / N - 0.5, (np.arange(N) + 0.5) / N - 0.5, indexing="ij")
    lat[3] = 90.0 - 50.0 * np.sqrt(jj ** 2 + ii ** 2)
    for f in (4, 5):
        nx, ny = grid.dims[f]
        ii = (np.arange(nx) + 0.5) / nx
        lat[f] = np.repeat((65.0 - 140.0 * ii)[None, :], ny, axis=0)
    return {f: np.deg2rad(v) for f, v in lat.items()}


class LLCSynthetic:
    """Grid-level fields (land, depth, spacing) of one LLC layout; operators and right-hand sides per member."""

    def __init__(self, N=90, ts=None, OL=4, land_fraction=0.30):
        self.topo = LLCTopology(N, ts, OL)
        self.L = self.topo.L
        grid = self.topo.grid
        self.sigma = 5.0 * N / 90.0
        noise = _facet_noise(grid, 0, self.sigma)
        thr = np.quantile(np.concatenate([v.ravel() for v in noise.values()]), land_fraction)
        ocean = {f: (v >= thr).astype(np.float64) for f, v in noise.items()}
        self.ocean = _to_tiles(self.topo, ocean)
        rng = np.random.default_rng(1)
        depth = {}
        for f in range(1, 6):
            nx, ny = grid.dims[f]
            depth[f] = rng.uniform(500.0, 6000.0, size=(ny, nx)) * ocean[f]
        self.depth = _to_tiles(self.topo, depth)
        lat = _latitude(grid)
        scale = 90.0 / N
        dx = {f: (20e3 + 90e3 * np.cos(v)) * scale for f, v in lat.items()}
        dy = {f: (20e3 + 90e3 * (0.5 + 0.5 * np.cos(v))) * scale for f, v in lat.items()}
        self.dx = _to_tiles(self.topo, dx, 1.0)
        self.dy = _to_tiles(self.topo, dy, 1.0)
        self.rA = self.dx * self.dy

    # ---------------------------------------------------------------------------------------------------------
    def member_depth(self, member=None):
        if member is None:
            return self.depth
        e = _to_tiles(self.topo, _facet_noise(self.topo.grid, 1000 + member, self.sigma))
        J, I = self.L.interior
        e = e / np.abs(e[:, J, I]).max()
        return self.depth * (1.0 + 0.1 * e)

    def operator(self, member=None):
        """(ops, cg2dNorm): ops = (aW2d, aS2d, aC2d, pW, pS, pC), each padded [T, ny, nx] float64."""
        L, maps = self.L, self.topo.maps
        J, I = L.interior
        H = self.member_depth(member)
        He = exch_scalar(H, *maps["T"][:2])
        Im, Jm = L.is_(0, L.sNx - 1), L.js(0, L.sNy - 1)
        Hw = np.minimum(He[:, J, I], He[:, J, Im])
        Hs = np.minimum(He[:, J, I], He[:, Jm, I])
        dx, dy = self.dx[:, J, I], self.dy[:, J, I]
        aW = Hw * dy / dx
        aS = Hs * dx / dy
        myNorm = max(np.abs(aW).max(), np.abs(aS).max())                  # cg2d.py:132-134
        cg2dNorm = 1.0 / myNorm if myNorm != 0.0 else 1.0
        z = np.zeros(L.shape2d)
        aW2d, aS2d = z.copy(), z.copy()
        aW2d[:, J, I] = aW * cg2dNorm
        aS2d[:, J, I] = aS * cg2dNorm
        aW2d, aS2d = exch_vector(aW2d, aS2d, maps["UVn_u"], maps["UVn_v"])
        Ip, Jp = L.is_(2, L.sNx + 1), L.js(2, L.sNy + 1)
        recip_Bo = 1.0 / GRAVITY
        aC = -(aW2d[:, J, I] + aW2d[:, J, Ip] + aS2d[:, J, I] + aS2d[:, Jp, I]
               + 1.0 * cg2dNorm * recip_Bo * self.rA[:, J, I] / DELTA_T / DELTA_T)
        aC2d = z.copy()
        aC2d[:, J, I] = aC
        aC2d = exch_scalar(aC2d, *maps["T"][:2])
        # preconditioner on j = 1..sNy+1, i = 1..sNx+1 (solve_for_pressure.py:55-63)
        J1, I1 = L.js(1, L.sNy + 1), L.is_(1, L.sNx + 1)
        Im1, Jm1 = L.is_(0, L.sNx), L.js(0, L.sNy)
        a = aC2d[:, J1, I1]
        pC, pW, pS = z.copy(), z.copy(), z.copy()
        with np.errstate(divide="ignore", invalid="ignore"):
            pC[:, J1, I1] = np.where(a == 0.0, 1.0, 1.0 / np.where(a == 0.0, 1.0, a))
            tw = a + aC2d[:, J1, Im1]
            pW[:, J1, I1] = np.where(tw == 0.0, 0.0,
                                     -aW2d[:, J1, I1] / (PC_OFFDIAG_FAC * np.where(tw == 0.0, 1.0, tw)) ** 2)
            tsum = a + aC2d[:, Jm1, I1]
            pS[:, J1, I1] = np.where(tsum == 0.0, 0.0,
                                     -aS2d[:, J1, I1] / (PC_OFFDIAG_FAC * np.where(tsum == 0.0, 1.0, tsum)) ** 2)
        return (aW2d, aS2d, aC2d, pW, pS, pC), cg2dNorm

    def _smooth_rhs(self, seed):
        J, I = self.L.interior
        f = _to_tiles(self.topo, _facet_noise(self.topo.grid, seed, self.sigma))[:, J, I]
        m = self.ocean[:, J, I].astype(bool)
        out = np.zeros(self.L.shape2d)
        out[:, J, I] = np.where(m, f - f[m].mean(), 0.0)
        return out

    def rhs(self, member=None):
        return self._smooth_rhs(2 if member is None else 2000 + member)

    def cotangent(self, member=None):
        return self._smooth_rhs(3 if member is None else 3000 + member)

    def first_guess(self):
        return np.zeros(self.L.shape2d)

    # ---------------------------------------------------------------------------------------------------------
    def model_fields(self, Nr=50, member=None):
        """Inputs of UPDATE_CG2D and SOLVE_FOR_PRESSURE (mitgcm_jax/core/solve_for_pressure.py:29-123) for one member:
        a dict of float64 arrays, 3-D fields [T, Nr, ny, nx], 2-D fields [T, ny, nx], plus the scalars of the
        free-surface and CG2D parameters (V4r4 values: dt = 3600 s, freeSurfFac = implicSurfPress =
        implicDiv2DFlow = 1, rhoConst = 1029, cg2dpcOffDFac = 0.51).

        * drF: layer thicknesses growing geometrically from 10 m, scaled to 6000 m in all;
        * hFacC(k): wet fraction of level k above the member's depth (0 below it and on land); hFacW, hFacS:
          min of the two cells of a face on the interior faces (Fortran i, j = 1..N), the east / north face halos
          through the UVn exchange (EXCH_UV_XYZ), so that the operator built from them is symmetric;
        * face metrics dyG, recip_dxC (u faces) and dxG, recip_dyC (v faces) from the spacing, exchanged as pairs;
          rA through the scalar exchange; maskInC = ocean;
        * Bo_surf = g (1 + 0.01 e), recip_Bo = 1 / Bo_surf; gU, gV: smooth noise of 1e-5 m/s^2 on wet faces;
          EmPmR: smooth noise of 1e-5 on ocean; etaN, etaH: smooth noise of 0.5 m on ocean (scalar exchange);
        * cg2dNorm: 1 / max|aW, aS| of the level-summed faces (ini_cg2d.F as in mitgcm_jax/init.py:325-345)."""
        L, maps = self.L, self.topo.maps
        J, I = L.interior
        T, ny, nx = L.shape2d
        tsrc, tcomp = maps["T"][:2]
        seed = 0 if member is None else 100 + member
        g = np.geomspace(10.0, 460.0, Nr)
        drF = g * (6000.0 / g.sum())
        zF = np.concatenate([[0.0], np.cumsum(drF)])
        He = exch_scalar(self.member_depth(member), tsrc, tcomp)
        hFacC = np.clip((He[:, None] - zF[None, :-1, None, None]) / drF[None, :, None, None], 0.0, 1.0)
        Im, Jm = L.is_(0, L.sNx - 1), L.js(0, L.sNy - 1)
        hW = np.zeros((T, Nr, ny, nx))
        hS = np.zeros((T, Nr, ny, nx))
        hW[:, :, J, I] = np.minimum(hFacC[:, :, J, I], hFacC[:, :, J, Im])
        hS[:, :, J, I] = np.minimum(hFacC[:, :, J, I], hFacC[:, :, Jm, I])
        hW, hS = (np.moveaxis(a, 1, 0) for a in exch_vector(np.moveaxis(hW, 1, 0), np.moveaxis(hS, 1, 0),
                                                             maps["UVn_u"], maps["UVn_v"]))
        z = np.zeros(L.shape2d)

        def inner(a):
            out = z.copy()
            out[:, J, I] = a[:, J, I]
            return out

        dyG, dxG = exch_vector(inner(self.dy), inner(self.dx), maps["UVn_u"], maps["UVn_v"])
        rdxC, rdyC = exch_vector(inner(1.0 / self.dx), inner(1.0 / self.dy), maps["UVn_u"], maps["UVn_v"])
        rA = exch_scalar(inner(self.rA), tsrc, tcomp)
        grid = self.topo.grid

        def noise(k, scale, mask):
            f = _to_tiles(self.topo, _facet_noise(grid, 5000 + 10 * seed + k, self.sigma))
            f = f / max(np.abs(f).max(), 1e-300)
            return exch_scalar(inner(scale * f * mask), tsrc, tcomp)

        ocean = self.ocean
        Bo = exch_scalar(inner(GRAVITY * (1.0 + 0.01 * noise(0, 1.0, np.ones(L.shape2d)))), tsrc, tcomp)
        Bo = np.where(Bo == 0.0, GRAVITY, Bo)                            # unwritten halo points: plain g
        recip_Bo = 1.0 / Bo
        rng = np.random.default_rng(6000 + seed)
        gU = np.zeros((T, Nr, ny, nx))
        gV = np.zeros((T, Nr, ny, nx))
        gU[:, :, J, I] = 1e-5 * rng.standard_normal((T, Nr, L.sNy, L.sNx)) * (hW[:, :, J, I] > 0)
        gV[:, :, J, I] = 1e-5 * rng.standard_normal((T, Nr, L.sNy, L.sNx)) * (hS[:, :, J, I] > 0)
        gU, gV = (np.moveaxis(a, 1, 0) for a in exch_vector(np.moveaxis(gU, 1, 0), np.moveaxis(gV, 1, 0),
                                                             maps["UVn_u"], maps["UVn_v"]))
        aW = np.zeros((T, L.sNy, L.sNx))
        aS = np.zeros((T, L.sNy, L.sNx))
        for k in range(Nr):
            aW = aW + (dyG[:, J, I] * drF[k] * hW[:, k][:, J, I]) * rdxC[:, J, I]
            aS = aS + (dxG[:, J, I] * drF[k] * hS[:, k][:, J, I]) * rdyC[:, J, I]
        my = max(np.abs(aW).max(), np.abs(aS).max())
        hW, hS, gU, gV = (np.ascontiguousarray(a) for a in (hW, hS, gU, gV))   # [T, Nr, ny, nx] in C order
        return dict(
            Nr=Nr, drF=drF, hFacW=hW, hFacS=hS, dyG=dyG, dxG=dxG, recip_dxC=rdxC, recip_dyC=rdyC, rA=rA,
            maskInC=inner(ocean), Bo_surf=Bo, recip_Bo=recip_Bo, gU=gU, gV=gV,
            EmPmR=noise(1, 1e-5, ocean), etaN=noise(2, 0.5, ocean), etaH=noise(3, 0.5, ocean),
            cg2dNorm=(1.0 / my) if my != 0.0 else 1.0, cg2dpcOffDFac=PC_OFFDIAG_FAC,
            deltaTMom=DELTA_T, deltaTFreeSurf=DELTA_T, freeSurfFac=1.0, implicSurfPress=1.0, implicDiv2DFlow=1.0,
            mass2rUnit=1.0 / 1029.0, useRealFreshWaterFlux=True)


def make_batch(N=90, count=1, ts=None, with_cotangent=False, members=None):
    """Stacked inputs of `count` members (or of the listed ensemble members): dict of [count, T, ny, nx] arrays plus
    cg2dNorm [count]. A single member without a list is the unperturbed configuration."""
    syn = LLCSynthetic(N, ts)
    out = {k: [] for k in ("aW2d", "aS2d", "aC2d", "pW", "pS", "pC", "b", "x0", "w")}
    norms = []
    if members is None:
        members = [None] if count == 1 else list(range(count))
    for member in members:
        ops, norm = syn.operator(member)
        for k, a in zip(("aW2d", "aS2d", "aC2d", "pW", "pS", "pC"), ops):
            out[k].append(a)
        out["b"].append(syn.rhs(member))
        out["x0"].append(syn.first_guess())
        if with_cotangent:
            out["w"].append(syn.cotangent(member))
        norms.append(norm)
    res = {k: np.stack(v) for k, v in out.items() if v}
    res["cg2dNorm"] = np.asarray(norms)
    return syn, res
