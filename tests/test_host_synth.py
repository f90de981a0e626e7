"""The host build of the input generator (oracle/liblicom_synth_host.so, used
by the CPU baseline) gives the same inputs as the product library's
generator, bit for bit, for the whole domain and for a northern band; its
ctypes structures match the product's."""
import ctypes as C

import numpy as np

import pyoracle


def test_struct_layouts_match(lt):
    for a, b in ((pyoracle.Params, lt.Params), (pyoracle.SynthConfig, lt.SynthConfig)):
        assert C.sizeof(a) == C.sizeof(b)
        assert [(n, t, getattr(a, n).offset) for n, t in a._fields_] == \
               [(n, t, getattr(b, n).offset) for n, t in b._fields_]


def test_host_generator_matches_product_generator(lt):
    kw = dict(forced=1, cap_north=0, umax=0.3, dz_top=5.0, dz_bot=300.0, seed=77)
    hs = pyoracle.HostSynth(64, 40, 20, **kw)
    syn = lt.Synth(64, 40, 20, **kw)
    assert bytes(hs.params) == bytes(syn.params)
    o = pyoracle.Oracle(64, 40, 20, hs.params)
    hs.fill(o)
    for n in pyoracle.INPUTS:
        a, b = o.get(n), syn.field(n)
        assert np.array_equal(a.view(np.uint8), b.view(np.uint8)), n
    # the northern band: the same cells, its own ghost rows at the cut
    ob = pyoracle.Oracle(64, 12, 20, hs.params)
    hs.fill(ob, rows=16)
    for n in ("UTF", "VTL", "AKT", "KMT", "TAREA"):
        a, b = ob.get(n), syn.field(n)
        assert np.array_equal(a, b[..., :16, :]), n
    a, b = ob.get("AT"), syn.field("AT")
    assert np.array_equal(a[:, :, :14], b[:, :, :14])


def test_hypsometry_keeps_the_land_and_deepens_the_ocean(lt):
    """hypsometry 1 keeps the land mask of the linear depth map and places
    the ocean's depths on the global area-depth curve: shallow next to the
    coast (the lowest land-field values), most of the ocean abyssal; the
    host build agrees bit for bit."""
    kw = dict(forced=1, cap_north=0)
    lin = lt.Synth(120, 80, 30, **kw).field("KMT")[2:-2, 2:-2]
    syn = lt.Synth(120, 80, 30, hypsometry=1, **kw)
    hyp = syn.field("KMT")[2:-2, 2:-2]
    assert np.array_equal(lin == 0, hyp == 0)
    ocean = hyp[hyp > 0]
    assert hyp[1:][hyp[1:] > 0].min() >= 3 and ocean.max() == 30   # (row 0 mirrors the fold)
    zkp = np.concatenate([[0.0], np.cumsum(syn.field("DZP"))])
    depth = 0.5 * (zkp[ocean - 1] + zkp[ocean])            # centre depth of the bottom level
    assert 3000.0 < depth.mean() < 4300.0, depth.mean()
    assert 0.15 < (depth < 2000.0).mean() < 0.25
    assert (hyp[hyp > 0].mean()) > 2.0 * lin[lin > 0].mean()
    hs = pyoracle.HostSynth(120, 80, 30, hypsometry=1, **kw)
    o = pyoracle.Oracle(120, 80, 30, hs.params)
    hs.fill(o)
    assert np.array_equal(o.get("KMT"), syn.field("KMT"))
