"""Batched stepping (include/licom_batch.h): several domains advanced by one
batch step must give, member by member, exactly what stepping each domain
alone gives, for every launch shape the autotuner may pick, with graphs and
without; the ensemble configuration (perturbed members of the 1-degree grid,
mixed precision) stays within the mixed-precision bounds of each member's
FP64 run."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SIZES = [(64, 40, 20), (96, 60, 30), (48, 32, 20)]   # uneven members (nx + 4 a multiple of 4)


def members(lt, precision, seed0=11, hypsometry=0):
    syns = [lt.Synth(nx, ny, km, seed=seed0 + i, forced=1, hypsometry=hypsometry)
            for i, (nx, ny, km) in enumerate(SIZES)]
    return syns, [s.domain(precision=precision) for s in syns]


def assert_same(doms_a, doms_b):
    for a, b in zip(doms_a, doms_b):
        for f in ("AT", "ATB", "WS", "NET"):
            np.testing.assert_array_equal(a.get(f), b.get(f), err_msg=f)


@pytest.mark.parametrize("hypsometry", [0, 1])
@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_batch_equals_members_stepped_alone(lt, precision, hypsometry):
    """hypsometry 1: most tiles march from a wet bottom level."""
    prec = lt.PREC_MIXED if precision == "mixed" else lt.PREC_FP64
    syns, doms = members(lt, prec, hypsometry=hypsometry)
    alone = [s.domain(precision=prec) for s in syns]
    for d in alone:
        d.step(5)
        d.sync()
    b = lt.Batch(doms)
    b.step(5)
    b.sync()
    assert_same(doms, alone)
    b.close()


@pytest.mark.parametrize("ctas,tile_y,graph", [(2, 8, 1), (2, 4, 1), (1, 16, 1), (2, 16, 0), (1, 8, 0)])
def test_every_launch_shape_gives_the_same_bits(lt, ctas, tile_y, graph):
    syns, doms = members(lt, lt.PREC_MIXED, seed0=5)
    ref = [s.domain(precision=lt.PREC_MIXED) for s in syns]
    for d in ref:
        d.step(3)
        d.sync()
    b = lt.Batch(doms)
    b.set_config(column_ctas_per_sm=ctas, continuity_tile_y=tile_y, use_graph=graph)
    b.step(3)
    b.sync()
    assert_same(doms, ref)
    b.close()


def test_batch_with_members_of_any_row_pitch(lt):
    """Members whose row pitch TMA cannot take (nx + 4 odd or not a multiple
    of 4) step in the same batch as the others, each exactly as alone."""
    sizes = [(49, 30, 12), (64, 40, 20), (50, 34, 30)]
    kw = dict(forced=1, ew_cyclic=0, tripole=0)
    syns = [lt.Synth(nx, ny, km, seed=40 + i, **kw) for i, (nx, ny, km) in enumerate(sizes)]
    doms = [lt.TracerDomain(s.nx, s.ny, s.km, s.params, precision=lt.PREC_MIXED, ew_cyclic=False, tripole=False)
            for s in syns]
    alone = [lt.TracerDomain(s.nx, s.ny, s.km, s.params, precision=lt.PREC_MIXED, ew_cyclic=False, tripole=False)
             for s in syns]
    for s, d, e in zip(syns, doms, alone):
        s.upload(d)
        s.upload(e)
        e.step(4)
        e.sync()
    b = lt.Batch(doms)
    b.step(4)
    b.sync()
    assert_same(doms, alone)
    b.close()


def test_batch_steps_mix_with_single_steps(lt):
    """A member stepped on its own between batch steps is picked up correctly."""
    syns, doms = members(lt, lt.PREC_MIXED, seed0=21)
    ref = [s.domain(precision=lt.PREC_MIXED) for s in syns]
    for d in ref:
        d.step(4)
        d.sync()
    b = lt.Batch(doms)
    b.step(1)
    b.sync()
    for d in doms:
        d.step(1)
        d.sync()
    b.step(2)
    b.sync()
    assert_same(doms, ref)
    b.close()


def test_autotune_keeps_the_state(lt):
    syns, doms = members(lt, lt.PREC_MIXED, seed0=31)
    ref = [s.domain(precision=lt.PREC_MIXED) for s in syns]
    for d in ref:
        d.step(2)
        d.sync()
    b = lt.Batch(doms)
    cfg = b.autotune(trial_steps=1)
    assert cfg == b.config()
    assert cfg["column_ctas_per_sm"] in (1, 2) and cfg["continuity_tile_y"] in (4, 8, 16)
    b.step(2)
    b.sync()
    assert_same(doms, ref)
    b.close()


def test_ensemble_members_within_mixed_bounds(lt):
    """Four members of the 1-degree grid, T perturbed by N(0, 0.01 K) per
    member, 100 steps as one mixed-precision batch, each against the FP64 run
    of the same member: |dT| <= 1e-4 K, |dS| <= 1e-5 psu."""
    nmem = 4
    syns = [lt.Synth(360, 218, 30, member=m + 1, tpert=0.01, forced=1, cap_north=0) for m in range(nmem)]
    mix = [s.domain(precision=lt.PREC_MIXED) for s in syns]
    b = lt.Batch(mix)
    b.step(100)
    b.sync()
    t0 = []
    for s, d in zip(syns, mix):
        ref = s.domain(precision=lt.PREC_FP64)
        ref.step(100)
        ref.sync()
        kmt = s.field("KMT")
        wet = (np.arange(30)[:, None, None] < kmt[None])[:, 2:-2, 2:-2]
        a, g = ref.get("AT")[:, :, 2:-2, 2:-2], d.get("AT")[:, :, 2:-2, 2:-2]
        dt = np.abs(a[0] - g[0])[wet].max()
        ds = np.abs(a[1] - g[1])[wet].max() * 1e3
        print("member: max |dT| %.3e K, |dS| %.3e psu" % (dt, ds))
        assert dt <= 1e-4 and ds <= 1e-5
        t0.append(g[0][wet])
    # the perturbations make the members differ
    assert np.abs(t0[0] - t0[1]).max() > 1e-3
    b.close()
