"""A domain's state through the reference's restart file: saved from one
domain and loaded into another, T and S come back bit for bit with the
domain's halo and fold, ATB = AT as NEXTSTEP sets it, h0 as the reference's
reader leaves it (the file's interior after its halo update), and the fields
the reference's writer masks over land are zero there."""
import numpy as np
import pytest

import pyoracle

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_save_load_round_trip(lt, tmp_path, precision):
    prec = lt.PREC_FP64 if precision == "fp64" else lt.PREC_MIXED
    syn = lt.Synth(64, 40, 12, seed=3, forced=1, cap_north=0)
    src = syn.domain(precision=prec)
    src.step(3)
    src.sync()
    nx, ny, km = syn.nx, syn.ny, syn.km
    rng = np.random.default_rng(0)
    u = rng.standard_normal((km, ny, nx))
    v = rng.standard_normal((km, ny, nx))
    su = rng.standard_normal((ny, nx))
    p = str(tmp_path / "fort.22.0001-02-03")
    src.save_restart(p, extra={"u": u, "v": v, "su": su}, month=14, day=3)
    dst = lt.Synth(64, 40, 12, seed=9, forced=1, cap_north=0).domain(precision=prec)
    u2, v2, month, day = dst.load_restart(p)
    assert (month, day) == (14, 3)
    assert np.array_equal(u2, u) and np.array_equal(v2, v)
    at = src.get("AT")
    assert np.array_equal(dst.get("AT"), at)
    atb = dst.get("ATB")
    assert np.array_equal(atb[:, 1:], at)
    # h0: the file holds the interior; loading applies the halo update the
    # reference applies after reading (POP_HaloUpdate, fill 0), which on a
    # tripole grid also averages the top row with its mirror
    arr, _, _ = lt.restart_read(p, nx, ny, km)
    h0 = src.get("H0F")
    assert np.array_equal(arr["h0"], h0[2:-2, 2:-2])
    want = np.zeros_like(h0)
    want[2:-2, 2:-2] = arr["h0"]
    o = pyoracle.Oracle(nx, ny, km, syn.params)
    want = o.halo(want, ew_cyclic=syn.cfg.ew_cyclic, tripole=syn.cfg.tripole)
    assert np.array_equal(dst.get("H0F"), want)
    # what the file holds: the masks of the reference's writer
    kmu = syn.field("KMU")[2:-2, 2:-2]
    kmt = syn.field("KMT")[2:-2, 2:-2]
    assert not arr["su"][kmu < 1].any() and np.array_equal(arr["su"][kmu >= 1], su[kmu >= 1])
    assert not arr["swv"][kmt < 1].any()
    np.testing.assert_array_equal(arr["ws"], src.get("WS")[:km, 2:-2, 2:-2])
    # the loaded domain steps
    dst.step(1)
    dst.sync()
    assert dst.check_numeric() == 0
