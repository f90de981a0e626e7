"""Seeded stand-ins for the inputs of the momentum biharmonic friction
(lt_hdiffu_del4): the del4 stencil coefficients restated from init_del4u
(hmix_del4.F90:88-288) on a synthetic domain's grid metrics, and smooth seeded
velocities at U points.  The momentum equations that produce the velocities
are not on this path, so tests and the benchmark use these.

In the reference the coefficients are built with Fortran arrays (i, j) and
``eoshift`` along dim=1 (i) and dim=2 (j); here the arrays are [j][i] (i
fastest), so dim=1 is axis 1 and dim=2 is axis 0.
"""
import numpy as np


def _eoshift(a, shift, axis):
    """Fortran eoshift with zero fill: shift=1 gives b(i) = a(i+1)."""
    b = np.zeros_like(a)
    if axis == 1:
        if shift == 1:
            b[:, :-1] = a[:, 1:]
        else:
            b[:, 1:] = a[:, :-1]
    else:
        if shift == 1:
            b[:-1] = a[1:]
        else:
            b[1:] = a[:-1]
    return b


def coefficients(f):
    """DUC .. DMW, AMF, UAREA_R, DXUR, DYUR from the grid fields HUN, HUE, HTW,
    HTS, DXU, DYU, TAREA_R of a synthetic domain (dict of arrays)."""
    hun, hue, htw, hts = f["HUN"], f["HUE"], f["HTW"], f["HTS"]
    dxu, dyu, tarea_r = f["DXU"], f["DYU"], f["TAREA_R"]
    with np.errstate(divide="ignore", invalid="ignore"):
        uarea = dxu * dyu
        uarea_r = np.where(uarea > 0, 1.0 / uarea, 0.0)
        dxur = np.where(dxu > 0, 1.0 / dxu, 0.0)
        dyur = np.where(dyu > 0, 1.0 / dyu, 0.0)
        w1 = np.where(htw != 0, hun / htw, 0.0)
        dun = w1 * uarea_r
        dus = _eoshift(w1, 1, 0) * uarea_r
        w1 = np.where(hts != 0, hue / hts, 0.0)
        due = w1 * uarea_r
        duw = _eoshift(w1, -1, 1) * uarea_r
        kxu = (hue - _eoshift(hue, -1, 1)) * uarea_r
        kyu = (_eoshift(hun, 1, 0) - hun) * uarea_r
        w1 = (_eoshift(htw, 1, 1) - htw) * tarea_r
        w2 = 0.5 * (w1 + _eoshift(w1, 1, 0))
        dxkx = (w2 - _eoshift(w2, -1, 1)) * dxur
        w2 = 0.5 * (w1 + _eoshift(w1, -1, 1))
        dykx = (_eoshift(w2, 1, 0) - w2) * dyur
        w1 = (hts - _eoshift(hts, -1, 0)) * tarea_r
        w2 = 0.5 * (w1 + _eoshift(w1, -1, 1))
        dyky = (_eoshift(w2, 1, 0) - w2) * dyur
        w2 = 0.5 * (w1 + _eoshift(w1, 1, 0))
        dxky = (w2 - _eoshift(w2, -1, 1)) * dxur
        dum = -(dxkx + dyky + 2.0 * (kxu ** 2 + kyu ** 2))
        dmc = dxky - dykx
        s = hts + _eoshift(hts, -1, 1)
        dme = np.where(s != 0, 2.0 * kyu / s, 0.0)
        s = htw + _eoshift(htw, 1, 0)
        dms = np.where(s != 0, -2.0 * kxu / s, 0.0)
    duc = -(dun + dus + due + duw)
    dmw = -dme
    dmn = -dms
    umean = uarea[uarea > 0].mean()
    amf = (np.abs(uarea) / umean) ** 1.5
    c = np.ascontiguousarray
    return dict(DUC=c(duc), DUM=c(dum), DUN=c(dun), DUS=c(dus), DUE=c(due), DUW=c(duw), DMC=c(dmc), DMN=c(dmn),
                DMS=c(dms), DME=c(dme), DMW=c(dmw), AMF=c(amf), UAREA_R=c(uarea_r), DXUR=c(dxur), DYUR=c(dyur))


def velocities(kmu, km, seed=1, umax=0.5):
    """UP, VP [km][jmt][imt]: large-scale gyres plus seeded small-scale noise,
    zero below the U-point bottom; DLU, DLV start as seeded tendencies."""
    rng = np.random.default_rng(seed)
    jmt, imt = kmu.shape
    jj, ii = np.mgrid[0:jmt, 0:imt]
    k = np.arange(km)[:, None, None]
    wet = k < kmu[None]
    decay = np.exp(-k / max(km / 3.0, 1.0))
    up = umax * decay * np.sin(2 * np.pi * jj / jmt)[None] * np.cos(4 * np.pi * ii / imt)[None]
    vp = umax * decay * np.cos(2 * np.pi * jj / jmt)[None] * np.sin(2 * np.pi * ii / imt)[None]
    up = (up + 0.05 * umax * rng.standard_normal((km, jmt, imt))) * wet
    vp = (vp + 0.05 * umax * rng.standard_normal((km, jmt, imt))) * wet
    dlu = 1e-6 * rng.standard_normal((km, jmt, imt)) * wet
    dlv = 1e-6 * rng.standard_normal((km, jmt, imt)) * wet
    c = np.ascontiguousarray
    return dict(UP=c(up), VP=c(vp), DLU=c(dlu), DLV=c(dlv))
