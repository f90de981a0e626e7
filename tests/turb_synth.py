"""Seeded stand-ins for the inputs of the Canuto turbulence closure (lt_turb).

The reference fills its closure tables in canuto_ini_2002.F90 (Fortran, run
at model start) and produces the closure's per-level inputs in other parts of
the model (readyc1_2 for the shear and Richardson numbers, the equation of
state for the density, the forcing for the buoyancy fluxes and the tidal
dissipation).  None of that is on this path, so tests and the benchmark use
these stand-ins:

* ``tables()``: the table grids exactly as canuto_ini_2002.F90:416-470 builds
  them (Ri step 0.01 up to |i| = mt0, geometric beyond with the ratio of the
  last two linear entries; the same grid for N_d^2/N^2; angle step pi/300),
  B_1 = 16.6 (canuto_2002.F90:2138), and smooth positive stability functions
  on those grids in place of the solutions of the Canuto 2002 model;
* ``inputs(at, kmt, dzp, seed)``: density from a linear equation of state of the
  domain's T and S, N^2 from its vertical differences, shear from a seeded
  log-normal field, Ri = N^2 / S^2 (as readyc1_2), Ri_d a seeded fraction of
  Ri, buoyancy fluxes, Coriolis parameter and tidal dissipation of the right
  sizes.  A few columns are made strongly unstable with weak shear (the
  zero-shear branch) and a few levels statically unstable; the top level
  stays stable (the reference leaves the buoyancy frequency unset when
  N^2 < 0 there).
"""
import math

import numpy as np

MT, MT0, NTH = 1462, 400, 75
N1, NB = 2 * MT + 1, 4 * NTH + 1


def _grid(step):
    """Linear for |i| <= MT0, geometric beyond (canuto_ini_2002.F90:420-464)."""
    i = np.arange(-MT, MT + 1)
    g = i * step
    r = (MT0 * step) / ((MT0 - 1) * step)
    big = np.abs(i) > MT0
    g[big] = np.sign(i[big]) * (MT0 * step) * r ** (np.abs(i[big]) - MT0)
    return g, r


def tables():
    """Dict of numpy arrays and scalars with the lt_turb_tables layout."""
    dri = 4.0 / MT0                       # -ri0 / mt0, ri0 = -4 (canuto_mod.h)
    rib, rri = _grid(dri)
    and2on2a1, rnd2on2 = _grid(dri)
    # realizability limit in Ri for each Ri_d
    rimax = 0.2 + 0.1 * np.tanh(0.5 * rib)
    irimax = np.searchsorted(rib, rimax, side="right") - 1 - MT
    irimax = np.clip(irimax, -MT, MT).astype(np.int32)
    ri = rib[None, :]            # columns: Ri
    rid = rib[:, None]           # rows: Ri_d
    pos = np.maximum(ri, 0.0)
    neg = np.sqrt(np.maximum(-ri, 0.0))
    slq2b = 0.01 * np.sqrt(np.maximum(1.0 - pos / (rimax[:, None] + 1e-3), 0.0)) + 1e-4 + 0.01 * neg / (1.0 + 0.1 * neg)
    smb = 0.10 / (1.0 + 8.0 * pos) * (1.0 + 0.1 * np.tanh(rid)) * (1.0 + 0.5 * neg / (1.0 + neg))
    shb = 0.12 / (1.0 + 12.0 * pos) * (1.0 + 0.2 * np.tanh(rid)) * (1.0 + 0.6 * neg / (1.0 + neg))
    ssb = 0.11 / (1.0 + 10.0 * pos) * (1.0 - 0.1 * np.tanh(rid)) * (1.0 + 0.6 * neg / (1.0 + neg))
    x = and2on2a1
    amtaun2a1 = 0.5 + 0.1 * np.tanh(x)
    sma1 = 0.08 + 0.01 * np.tanh(x)
    sha1 = 0.10 + 0.02 * np.tanh(x)
    ssa1 = 0.09 - 0.01 * np.tanh(x)
    dth = (math.pi / 4.0) / NTH
    th = np.arange(-NTH, 3 * NTH + 1) * dth
    back_ra_r = 0.3 + 0.1 * np.cos(2.0 * th)
    sm_r1 = 0.05 + 0.01 * np.sin(th)
    sh_r1 = 0.06 + 0.01 * np.cos(th)
    ss_r1 = 0.055 + 0.01 * np.sin(2.0 * th)
    slq2_r1 = 0.005 + 0.001 * np.cos(th)
    rrcrp = -0.5                           # critical R_r; its reciprocal is the other root
    theta_rcrp = math.atan(rrcrp)
    theta_rcrn = math.atan(1.0 / rrcrp)
    if theta_rcrn < -math.pi / 4:
        theta_rcrn += math.pi
    if theta_rcrp < -math.pi / 4:
        theta_rcrp += math.pi
    c = np.ascontiguousarray
    return dict(rib=c(rib), irimax=c(irimax), slq2b=c(slq2b), smb=c(smb), shb=c(shb), ssb=c(ssb),
                and2on2a1=c(and2on2a1), amtaun2a1=c(amtaun2a1), sma1=c(sma1), sha1=c(sha1), ssa1=c(ssa1),
                back_ra_r=c(back_ra_r), sm_r1=c(sm_r1), sh_r1=c(sh_r1), ss_r1=c(ss_r1), slq2_r1=c(slq2_r1),
                rri=float(rri), rnd2on2=float(rnd2on2), dri=float(dri), deltheta_r=float(dth), b1=16.6,
                theta_rcrp=float(theta_rcrp), theta_rcrn=float(theta_rcrn), dand2on2=float(dri))


def inputs(at, kmt, dzp, seed=1, lat_s=-78.0, lat_n=88.0):
    """Closure inputs for a domain with state ``at`` [2][km][jmt][imt], masks
    ``kmt`` and layer thicknesses ``dzp`` (m): dict of field name -> array."""
    rng = np.random.default_rng(seed)
    _, km, jmt, imt = at.shape
    zkp = np.zeros(km + 1)
    zkp[1:] = -np.cumsum(dzp)
    t = at[0]
    s = at[1] * 1000.0 + 35.0
    depth = -0.5 * (zkp[:-1] + zkp[1:])
    pd = np.empty((km + 1, jmt, imt))
    pd[:km] = 1025.0 + 0.78 * (s - 35.0) - 0.17 * (t - 10.0) + 0.0006 * depth[:, None, None]
    pd[km] = pd[km - 1]
    dzi = 0.5 * (dzp[:-1] + dzp[1:])
    n2 = 9.806 / 1025.0 * (pd[1:km] - pd[:km - 1]) / dzi[:, None, None]
    n2 += rng.normal(0.0, 2e-6, size=n2.shape)
    n2[0] = np.abs(n2[0]) + 1e-7                     # top interface stable
    s2 = np.exp(rng.normal(math.log(5e-5), 1.5, size=n2.shape))
    # a few strongly unstable, weakly sheared interfaces (zero-shear branch)
    weak = rng.uniform(size=n2.shape) < 0.01
    weak[0] = False
    n2[weak] = -np.abs(n2[weak]) - 1e-5
    s2[weak] = 1e-9
    rit = n2 / (s2 + 1e-25)
    ricdttms = rit * rng.uniform(-1.5, 1.5, size=rit.shape)
    jj = np.arange(jmt)
    lat = lat_n + (lat_s - lat_n) * (jj - 2) / max(jmt - 5, 1)   # j = 0 the northern edge
    fcort = np.repeat((2.0 * 7.292e-5 * np.sin(np.radians(lat)))[:, None], imt, axis=1)
    hcol = np.where(kmt > 0, -zkp[np.clip(kmt, 0, km)], 1.0)
    zc = -0.5 * (zkp[:-1] + zkp[1:])
    fz = np.exp((zc[:, None, None] - hcol[None]) / 500.0)
    fz /= np.maximum(fz.sum(axis=0, keepdims=True), 1e-30)
    c = np.ascontiguousarray
    return dict(ZKP=c(zkp), PDENSITY=c(pd), RICT=c(n2), S2T=c(s2), RIT=c(rit), RICDTTMS=c(ricdttms),
                FCORT=c(fcort), FZ_TIDE=c(fz),
                BUOYTUR=c(rng.normal(0.0, 1e-8, size=(jmt, imt))),
                BUOYSOL=c(np.abs(rng.normal(0.0, 3e-9, size=(jmt, imt)))),
                WAVE_DIS=c(np.exp(rng.normal(math.log(3e-3), 1.0, size=(jmt, imt)))))
