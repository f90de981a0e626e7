"""Seeded cases of the momentum biharmonic friction for the tests: a synthetic
domain with the del4 stencil coefficients and velocities of
tests/del4u_synth.py, at the reference's block size by default."""
DEL4U_CASES = [(4, 0), (9, 1), (17, 0)]   # (seed, cap_north)
C0F = 2.6e-3


def case(lt, seed, cap_north=0, nx=36, ny=40, km=55, **kw):
    import del4u_synth
    opts = dict(cap_south=3, dz_top=5.0, dz_bot=300.0)
    opts.update(kw)
    syn = lt.Synth(nx, ny, km, seed=seed, cap_north=cap_north, **opts)
    f = syn.all_fields()
    f.update(del4u_synth.coefficients(f))
    f.update(del4u_synth.velocities(f["KMU"], km, seed=seed))
    am = 4.0 * syn.params.ah
    return syn, f, am
