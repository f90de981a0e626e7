"""tracer_7 alone (tracer.cpp:1571-1626): its nudging branch (simple_assm,
levels k < ktv) and its restoring branch (boundary_restore), on seeded
arrays of the reference's block size.  The reference's tracer_ always passes
simple_assm = 0, so the nudging branch is pinned through the kernel itself:
the reference's tracer_7 against the oracle's restatement, on the same
arrays, and against the golden digests of tests/golden/make_golden.py."""
import numpy as np

# (boundary_restore, simple_assm, ktv, seed); ktv above 45 reaches the
# weaker rate of the deep levels
ASSM_CASES = [(0, 1, 55, 3), (1, 1, 50, 4), (0, 1, 20, 5), (1, 0, 0, 6)]


def arrays(nx, ny, km, seed):
    """tf, vit [km][jmt][imt]; atb [2][km+1][jmt][imt]; restore, restore_at
    [2][km][jmt][imt]; a column depth per cell with land and full columns."""
    imt, jmt = nx + 4, ny + 4
    rng = np.random.default_rng(seed)
    kmt = rng.integers(0, km + 1, size=(jmt, imt))
    vit = (np.arange(km)[:, None, None] < kmt[None]).astype(np.float64)
    tf = rng.normal(0.0, 1.0e-6, size=(km, jmt, imt))
    atb = rng.normal(10.0, 5.0, size=(2, km + 1, jmt, imt))
    restore = atb[:, 1:] + rng.normal(0.0, 0.5, size=(2, km, jmt, imt))
    restore_at = atb[:, 1:] + rng.normal(0.0, 0.5, size=(2, km, jmt, imt))
    return tf, vit, atb, restore, restore_at


def key(boundary_restore, simple_assm, ktv, seed):
    return "tracer7_restore%d_assm%d_ktv%d_seed%d" % (boundary_restore, simple_assm, ktv, seed)
