"""Seeded cases of the turbulence closure for the tests: a synthetic domain,
its closure inputs and the stand-in closure tables (tests/turb_synth.py), at
the reference's built-in block size by default."""
import functools

import numpy as np

NCC = 4              # pconst_mod ncc of the cases
DFRICMX = 0.1        # pconst_mod dfricmx (m^2/s)
# (seed, forced) of the pinned cases
TURB_CASES = [(3, 1), (8, 0), (21, 1)]


@functools.lru_cache(maxsize=1)
def tables(lt):
    import turb_synth
    return turb_synth.tables()


def case(lt, seed, forced=1, nx=36, ny=40, km=55, **kw):
    """(synth, fields) with the closure inputs added to the synth's fields."""
    import turb_synth
    opts = dict(cap_north=0, cap_south=3, dz_top=5.0, dz_bot=300.0)
    opts.update(kw)
    syn = lt.Synth(nx, ny, km, seed=seed, forced=forced, **opts)
    f = syn.all_fields()
    f.update(turb_synth.inputs(f["AT"], f["KMT"], f["DZP"], seed=seed))
    # AKT starts as the synth's field: the closure leaves the columns it does
    # not compute (and the bottom level) as they are
    return syn, f
