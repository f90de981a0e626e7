"""Seeded cases for the centred and flux advection schemes of the tracer step
(pconst_mod adv_tracer "centered" / "flux", matched at tracer.cpp:1712-1714;
the Str 0 / 1 branches of advection_tracer_1_0 and advection_tracer_1,
tracer.cpp:83-289).

The reference writes the top- and bottom-level statements of the centred
scheme (tracer.cpp:132-160, 208-256) without a level guard, so every thread
of the launch's level dimension (km rounded up to the block's 4 levels)
repeats them.  adv_tt gets the same value from every repetition, but the
diagnostic accumulations ax, ay, az of levels 0 and km-1 race on a GPU; the
CPU emulation of the reference adds them once per repetition.  This build
accumulates each level once, so comparisons of AX, AY, AZ with the
reference leave those two levels out in the centred scheme.
"""

# (scheme, forced, steps, seed)
SCHEME_CASES = [("centered", 1, 3, 41), ("centered", 0, 2, 8), ("flux", 1, 3, 43), ("flux", 0, 2, 9)]
RACY_DIAG = ("AX", "AY", "AZ")


def case(lt, scheme, forced, seed, nx=36, ny=40, km=55, **kw):
    """A domain of the reference's block size (or the given size) with the
    advection scheme set: (synth, params, fields)."""
    if (nx, ny, km) == (36, 40, 55):
        kw = dict(dict(cap_north=0, cap_south=3, dz_top=5.0, dz_bot=300.0), **kw)
    syn = lt.Synth(nx, ny, km, forced=forced, seed=seed, **kw)
    p = syn.params
    p.adv_tracer = lt.ADV_SCHEMES[scheme]
    return syn, p, syn.all_fields()


def comparable(scheme, name, a):
    """The part of field `name` ([n][k][j][i] for the diagnostics) that the
    reference computes without a race in this scheme."""
    if scheme == "centered" and name in RACY_DIAG:
        return a[:, 1:-1]
    return a
