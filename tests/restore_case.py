"""Seeded cases for the restoring branch of the tracer step (tracer_7 with
boundary_restore == 1, tracer.cpp:1571-1627): every level below the surface
is relaxed toward RESTORE with a 15-day time scale.

The synthetic generator's RESTORE is the initial state itself, which the
relaxation would leave untouched at the first step, so these cases build a
target that differs from the state by a deterministic pattern of integer
multiples (exact arithmetic, the same bits on every machine): up to
+-0.25 K for T and +-0.25e-3 psu for S.
"""
import numpy as np

# (forced, steps, seed)
RESTORE_CASES = [(1, 4, 31), (0, 3, 5)]


def restore_target(at):
    n, km, jmt, imt = at.shape
    k, j, i = np.meshgrid(np.arange(km), np.arange(jmt), np.arange(imt), indexing="ij")
    m = ((7 * i + 13 * j + 3 * k) % 11 - 5).astype(np.float64)      # -5 .. 5
    out = np.empty_like(at)
    out[0] = at[0] + 0.25 * m / 5.0
    out[1] = at[1] + 0.25e-6 * m / 5.0
    return out


def case(lt, forced, seed, nx=36, ny=40, km=55, **kw):
    """A domain of the reference's block size (or the given size) with the
    restoring branch switched on: (synth, params, fields)."""
    if (nx, ny, km) == (36, 40, 55):
        kw = dict(dict(cap_north=0, cap_south=3, dz_top=5.0, dz_bot=300.0), **kw)
    syn = lt.Synth(nx, ny, km, forced=forced, seed=seed, **kw)
    p = syn.params
    p.boundary_restore = 1
    f = syn.all_fields()
    f["RESTORE"] = restore_target(f["AT"])
    return syn, p, f
