"""CPU oracle of the steps either side of the CG2D solve -- TEST INFRASTRUCTURE ONLY (tests/, smoke() and bench.py's
CPU legs import it; the library never does).

Numpy restatements, operation for operation, of mitgcm_jax/core/cg2d.py:108-134 (ini_cg2d_norm, the operator
normalisation set up once) and of mitgcm_jax/core/solve_for_pressure.py:
* update_cg2d (:29-65): the operator aW2d, aS2d, aC2d and the preconditioner pW, pS, pC from the level-summed
  face areas;
* cg2d_rhs (:68-106): the right-hand side cg2d_b (fresh-water flux, the divergence of the g-hat transports summed
  from level Nr up to 1, the exactConserv etaH term) and the first guess cg2d_x = Bo_surf etaN;
* solve_for_pressure_post (:109-123, after the solve): the exchange of the solution and etaN = recip_Bo x.
The vertical factors deepFacC, rhoFacC and deepFac2F are all 1 in the reference (free_surface.py:121-125); the
products with them are exact and are left out. Pinned bit for bit to the reference's own functions
(tests/golden/make_golden_pressure.py, tests/test_pressure_oracle.py).
"""

import numpy as np

from oracle.cg2d_oracle import exch


def _ksum(terms):
    """0 + terms[0] + terms[1] + ... in order (solve_for_pressure.py:23-26)."""
    out = np.zeros_like(terms[0])
    for t in terms:
        out = out + t
    return out


def ini_cg2d_norm(L, *, hFacW, hFacS, drF, dyG, dxG, recip_dxC, recip_dyC, implicSurfPress, implicDiv2DFlow):
    """ini_cg2d_norm (mitgcm_jax/core/cg2d.py:108-134, ini_cg2d.F:90-135) for one instance: cg2dNorm =
    1 / max|aW, aS| over the interior faces, aW = sum over k = 1..Nr in order of
    (fac ((dyG drF(k)) hFacW(k))) recip_dxC with fac = implicSurfPress implicDiv2DFlow, aS likewise (1 where the
    maximum is 0). hFacW/S [T, Nr, ny, nx]; 2-D fields [T, ny, nx]."""
    J, I = L.js(1, L.sNy), L.is_(1, L.sNx)
    fac = implicSurfPress * implicDiv2DFlow
    tW = [fac * (dyG[:, J, I] * drF[k] * hFacW[:, k, J, I]) * recip_dxC[:, J, I] for k in range(len(drF))]
    tS = [fac * (dxG[:, J, I] * drF[k] * hFacS[:, k, J, I]) * recip_dyC[:, J, I] for k in range(len(drF))]
    aW, aS = _ksum(tW), _ksum(tS)
    my = max(np.abs(aW).max(), np.abs(aS).max())
    return 1.0 / my if my != 0.0 else 1.0


def update_cg2d(L, tmap, *, hFacW, hFacS, drF, dyG, dxG, recip_dxC, recip_dyC, rA, recip_Bo, pW, pS, pC,
                cg2dNorm, cg2dpcOffDFac, implicSurfPress, implicDiv2DFlow, freeSurfFac, deltaTMom, deltaTFreeSurf):
    """update_cg2d (solve_for_pressure.py:29-65) for one instance. hFacW/S [T, Nr, ny, nx]; 2-D fields [T, ny, nx].
    Returns (aW2d, aS2d, aC2d, pW, pS, pC); pW, pS, pC keep their input values outside j, i = 1..sNy+1, 1..sNx+1."""
    Nr = len(drF)
    J1, I1 = L.js(1, L.sNy + 1), L.is_(1, L.sNx + 1)
    z2 = np.zeros(L.shape2d)
    tW = [dyG[:, J1, I1] * drF[k] * hFacW[:, k, J1, I1] * recip_dxC[:, J1, I1] for k in range(Nr)]   # :41-43
    tS = [dxG[:, J1, I1] * drF[k] * hFacS[:, k, J1, I1] * recip_dyC[:, J1, I1] for k in range(Nr)]
    aW, aS = _ksum(tW), _ksum(tS)
    aW = aW * cg2dNorm * implicSurfPress * implicDiv2DFlow                                          # :44-47
    aS = aS * cg2dNorm * implicSurfPress * implicDiv2DFlow
    aW2d, aS2d = z2.copy(), z2.copy()
    aW2d[:, J1, I1] = aW
    aS2d[:, J1, I1] = aS
    J, I, Jp, Ip = L.js(1, L.sNy), L.is_(1, L.sNx), L.js(2, L.sNy + 1), L.is_(2, L.sNx + 1)         # :49-52
    aC = -(aW2d[:, J, I] + aW2d[:, J, Ip] + aS2d[:, J, I] + aS2d[:, Jp, I]
           + freeSurfFac * cg2dNorm * recip_Bo[:, J, I] * rA[:, J, I] / deltaTMom / deltaTFreeSurf)
    aC2d = z2.copy()
    aC2d[:, J, I] = aC
    aC2d = exch(aC2d, tmap)                                                                         # :53
    Im, Jm = L.is_(0, L.sNx), L.js(0, L.sNy)                                                        # :55-65
    a = aC2d[:, J1, I1]
    with np.errstate(divide="ignore", invalid="ignore"):
        pC_n = np.where(a == 0.0, 1.0, 1.0 / np.where(a == 0.0, 1.0, a))
        tw = a + aC2d[:, J1, Im]
        pW_n = np.where(tw == 0.0, 0.0, -aW2d[:, J1, I1] / (cg2dpcOffDFac * np.where(tw == 0.0, 1.0, tw)) ** 2)
        ts = a + aC2d[:, Jm, I1]
        pS_n = np.where(ts == 0.0, 0.0, -aS2d[:, J1, I1] / (cg2dpcOffDFac * np.where(ts == 0.0, 1.0, ts)) ** 2)
    pW, pS, pC = (np.array(v, np.float64, copy=True) for v in (pW, pS, pC))
    pW[:, J1, I1] = pW_n
    pS[:, J1, I1] = pS_n
    pC[:, J1, I1] = pC_n
    return aW2d, aS2d, aC2d, pW, pS, pC


def cg2d_rhs(L, *, gU, gV, hFacW, hFacS, EmPmR, etaN, etaH, Bo_surf, drF, dyG, dxG, rA, maskInC, freeSurfFac,
             mass2rUnit, implicDiv2DFlow, deltaTMom, deltaTFreeSurf, useRealFreshWaterFlux):
    """cg2d_rhs (solve_for_pressure.py:68-106) for one instance. Returns (cg2d_b, cg2d_x): cg2d_b on the interior
    (0 on halos), cg2d_x = Bo_surf etaN on the full array."""
    Nr = len(drF)
    J, I = L.js(1, L.sNy), L.is_(1, L.sNx)
    cg2d_x = Bo_surf * etaN                                                                         # :76
    cg2d_b = np.zeros(L.shape2d)                                                                    # :77
    if useRealFreshWaterFlux:                                                                       # :78-80
        tmpFac = freeSurfFac * mass2rUnit * implicDiv2DFlow
        cg2d_b[:, J, I] = tmpFac * rA[:, J, I] * EmPmR[:, J, I] / deltaTMom * maskInC[:, J, I]
    b = cg2d_b[:, J, I]
    J1, I1 = L.js(1, L.sNy + 1), L.is_(1, L.sNx + 1)
    Ju, Iu = L.js(1, L.sNy), L.is_(1, L.sNx + 1)
    Jv, Iv = L.js(1, L.sNy + 1), L.is_(1, L.sNx)
    for k in range(Nr - 1, -1, -1):                                                                 # :95-101
        xA = dyG[:, J1, I1] * drF[k] * hFacW[:, k, J1, I1]                                          # :90-91
        yA = dxG[:, J1, I1] * drF[k] * hFacS[:, k, J1, I1]
        pu = xA[:, :-1, :] * gU[:, k, Ju, Iu] / deltaTMom                                           # :92
        pv = yA[:, :, :-1] * gV[:, k, Jv, Iv] / deltaTMom                                           # :93
        b = b + pu[:, :, 1:] - pu[:, :, :-1]                                                        # :97-98
        b = b + pv[:, 1:, :] - pv[:, :-1, :]
    b = b - (freeSurfFac * rA[:, J, I] / deltaTMom / deltaTFreeSurf * etaH[:, J, I])                # :103-105
    cg2d_b[:, J, I] = b
    return cg2d_b, cg2d_x


def solve_for_pressure_post(L, tmap, x, cg2d_x, recip_Bo):
    """After the solve (solve_for_pressure.py:116-121): x (interior = solution) with every halo point taking its
    exchanged value, or the first guess where no exchange writes; etaN = recip_Bo x on the full array."""
    inner = np.zeros(L.shape2d, bool)
    inner[:, L.js(1, L.sNy), L.is_(1, L.sNx)] = True
    xf = exch(np.where(inner, x, cg2d_x), tmap)
    return recip_Bo * xf
