"""GPU parity of the sea-ice adjustment (icesnow.cpp:15-85) against the CPU
oracle, bit for bit (the kernel keeps the reference's operation order and is
compiled with -fmad=false): alone on cold states in both precisions and both
QICE modes, in the stepon.cpp:69-77 order tracer_ -> icesnow_ -> convadj_,
through the reference-named shim, and on a 1-degree tripole grid.  The
oracle itself is pinned to the reference's icesnow.cpp (test_icesnow_pin)."""
import hashlib
import json
import os

import numpy as np
import pytest
from conftest import REPO
from icesnow_state import TBICE, cold_state

import pyoracle

pytestmark = pytest.mark.gpu


def bits_equal(a, b):
    return np.array_equal(np.ascontiguousarray(a).view(np.uint64), np.ascontiguousarray(b).view(np.uint64))


def mismatch(a, b):
    d = np.abs(a - b)
    idx = np.unravel_index(np.argmax(d), d.shape)
    return "max diff %.3e at %s (gpu %r oracle %r), %d cells differ" % (d[idx], idx, a[idx], b[idx],
                                                                         int(np.sum(a != b)))


def setup(lt, seed, precision, nx=36, ny=40, km=55, **kw):
    opts = dict(forced=1, cap_north=0, cap_south=3, dz_top=5.0, dz_bot=300.0)
    opts.update(kw)
    syn = lt.Synth(nx, ny, km, seed=seed, **opts)
    inp = syn.all_fields()
    inp["AT"], inp["QICE"] = cold_state(inp, seed)
    dom = lt.TracerDomain(nx, ny, km, syn.params, precision=precision,
                          ew_cyclic=bool(syn.cfg.ew_cyclic), tripole=bool(syn.cfg.tripole))
    for n in lt.INPUT_FIELDS:
        dom.set(n, inp[n])
    o = pyoracle.Oracle(nx, ny, km, syn.params, ew_cyclic=syn.cfg.ew_cyclic, tripole=syn.cfg.tripole)
    o.load(inp)
    o.sum_order(1)
    return syn, inp, dom, o


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("frc_core", [1, 0])
def test_icesnow_alone_bitexact(lt, precision, frc_core):
    prec = lt.PREC_FP64 if precision == "fp64" else lt.PREC_MIXED
    syn, inp, dom, o = setup(lt, 5 + frc_core, prec)
    p = lt.IcesnowParams(reset_qice=frc_core)
    dom.icesnow(p)
    o.icesnow(p)
    for n in ("AT", "QICE"):
        g, r = dom.get(n), o.get(n)
        assert bits_equal(g, r), n + ": " + mismatch(g, r)
    assert np.any(o.get("QICE") > 0.0) and np.all(dom.get("AT")[0] >= TBICE)


def test_icesnow_in_the_step_sequence_bitexact(lt):
    """Three steps of tracer -> icesnow (convadj after the first), as the
    reference's stepon orders them, FP64 domain against the oracle."""
    syn, inp, dom, o = setup(lt, 7, lt.PREC_FP64)
    p = lt.IcesnowParams()
    for s in range(3):
        dom.step(1)
        dom.icesnow(p)
        o.step(1)
        o.icesnow(p)
        if s == 0:
            dom.convadj()
            o.convadj()
    for n in ("AT", "ATB", "QICE", "DT_CONV"):
        g, r = dom.get(n), o.get(n)
        assert bits_equal(g, r), n + ": " + mismatch(g, r)


def test_icesnow_shim_matches_golden(lt):
    """icesnow_ on a bound domain: the reference's parameters and FRC_CORE
    reset, compared with the digests of the reference's own icesnow.cpp."""
    syn, inp, dom, o = setup(lt, 5, lt.PREC_FP64)
    dom.bind_shim()
    assert lt.icesnow_() == ""
    gold = json.load(open(os.path.join(REPO, "tests", "golden", "reference_digests.json")))["icesnow_frc1_steps0_seed5"]
    for n in ("AT", "QICE"):
        assert hashlib.sha256(dom.get(n).tobytes()).hexdigest() == gold["outputs"][n], n


def test_icesnow_one_degree_tripole(lt):
    syn, inp, dom, o = setup(lt, 11, lt.PREC_FP64, nx=360, ny=218, km=30, cap_south=3, dz_top=10.0, dz_bot=250.0)
    p = lt.IcesnowParams(reset_qice=0)
    for _ in range(2):
        dom.icesnow(p)
        o.icesnow(p)
    for n in ("AT", "QICE"):
        g, r = dom.get(n), o.get(n)
        assert bits_equal(g, r), n + ": " + mismatch(g, r)
