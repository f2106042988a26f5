"""Generated LLC exch2 connectivity against the reference's probed LLC90 maps (tests/golden/llc90_T_map.npz, from
mitgcm_jax/data/exch_maps_13x90x90.npz), and structural properties at other sizes (LLC270 has no reference map)."""

import numpy as np
import pytest

from golden_cases import GOLDEN
from mit_jax_b200.topology import LLCTopology, exch_scalar, exch_vector, exch_vector_adjoint


@pytest.fixture(scope="module")
def ref():
    return np.load(GOLDEN / "llc90_T_map.npz")


def test_llc90_scalar_map_matches_reference_at_stencil_points(ref):
    tp = LLCTopology(90)
    src, comp, _ = tp.maps["T"]
    pts = tp.stencil_points()
    np.testing.assert_array_equal(comp[pts], ref["comp"][pts])
    w = ref["comp"][pts] == 1
    np.testing.assert_array_equal(src[pts][w], ref["src"][pts][w])
    assert w.sum() == 4320 and (~w).sum() == 360          # 4 open tile edges x 90 points


def test_llc90_face_map_matches_reference(ref):
    tp = LLCTopology(90)
    for kind, key in (("UVn_u", "uvn_u"), ("UVn_v", "uvn_v")):
        src, comp, _ = tp.maps[kind]
        p = ref[key + "_pts"]
        np.testing.assert_array_equal(comp[p], ref[key + "_comp"])
        w = ref[key + "_comp"] > 0
        np.testing.assert_array_equal(src[p][w], ref[key + "_src"][w])


def test_reference_full_map_unwritten_count(ref):
    """exchange.py test design (test_exchange.py:71-72): 4 x 90 x OL halo points of the C grid are unwritten."""
    comp = ref["comp"].reshape(13, 98, 98)
    halo = np.ones((13, 98, 98), bool)
    halo[:, 4:94, 4:94] = False
    assert ((comp == 0) & halo).sum() == 4 * 90 * 4


@pytest.mark.parametrize("N,ts", [(90, 90), (270, 270), (16, 8), (90, 30)])
def test_neighbour_relation_is_symmetric(N, ts):
    """Every written stencil halo point p of tile t (the neighbour q of edge point e) has e among q's own stencil
    neighbours: the connectivity is a symmetric graph, as an exactly symmetric operator needs."""
    tp = LLCTopology(N, ts, 1)
    L = tp.L
    src, comp, _ = tp.maps["T"]
    T, ny, nx = L.shape2d

    def neighbours(p):
        t, rem = divmod(p, ny * nx)
        j, i = divmod(rem, nx)
        out = []
        for dj, di in ((0, -1), (0, 1), (-1, 0), (1, 0)):
            h = (t * ny + j + dj) * nx + i + di
            if 1 <= j + dj <= L.sNy and 1 <= i + di <= L.sNx:
                out.append(h)
            elif comp[h] == 1:
                out.append(int(src[h]))
        return out

    n_open = 0
    for p in tp.stencil_points():
        t, rem = divmod(int(p), ny * nx)
        j, i = divmod(rem, nx)
        e = (t * ny + min(max(j, 1), L.sNy)) * nx + min(max(i, 1), L.sNx)   # the edge point this halo belongs to
        if comp[p] == 0:
            n_open += 1
            continue
        assert e in neighbours(int(src[p])), (N, ts, p)
    assert n_open == 4 * N                                   # facets 1, 2 south and 4, 5 east edges are open


def test_exchange_adjoint_identity():
    """<E x, y> == <x, E^T y> (test_exchange.py:106-118): the gather's transpose is the scatter-add."""
    tp = LLCTopology(16, 8, 2)
    src, comp, _ = tp.maps["T"]
    rng = np.random.default_rng(0)
    x = rng.standard_normal(tp.L.shape2d)
    y = rng.standard_normal(tp.L.shape2d)
    ex = exch_scalar(x, src, comp)
    yf = y.reshape(-1)
    et = np.where(comp == 1, 0.0, yf)
    np.add.at(et, src[comp == 1], yf[comp == 1])
    np.testing.assert_allclose(np.vdot(ex, y), np.vdot(x.reshape(-1), et), rtol=1e-13)


def test_face_exchange_adjoint_identity():
    """<E (u, v), (a, b)> == <(u, v), E^T (a, b)> for the UVn face exchange and its transpose, batched."""
    tp = LLCTopology(16, 8, 2)
    rng = np.random.default_rng(1)
    u, v, a, b = (rng.standard_normal((2,) + tp.L.shape2d) for _ in range(4))
    eu, ev = exch_vector(u, v, tp.maps["UVn_u"], tp.maps["UVn_v"])
    ta, tb = exch_vector_adjoint(a, b, tp.maps["UVn_u"], tp.maps["UVn_v"])
    for m in range(2):
        lhs = np.vdot(eu[m], a[m]) + np.vdot(ev[m], b[m])
        rhs = np.vdot(u[m], ta[m]) + np.vdot(v[m], tb[m])
        np.testing.assert_allclose(lhs, rhs, rtol=1e-13)
