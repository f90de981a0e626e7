"""GPU parity of the centred and flux advection schemes (pconst_mod
adv_tracer "centered" / "flux", selected at tracer.cpp:1712-1714; the Str 0
and Str 1 branches of advection_tracer_1_0 / advection_tracer_1,
tracer.cpp:83-289).

The FP64 column kernel with either scheme's advective tendency (and the flux
scheme's dx/dy-weighted face transports in the continuity march) against the
CPU oracle, bit for bit: on the reference's block size with the fold, on
grids of several tiles whose row pitch does and does not allow TMA boxes
(the schemes run in the plain-load kernel either way), with and without the
diagnostics, through the tracer_ shim, and with the scheme switched between
steps by lt_set_params.  The oracle itself is pinned to the reference's own
code for these schemes in tests/test_oracle_pin.py.
"""
import numpy as np
import pytest

import pyoracle
import scheme_case

pytestmark = pytest.mark.gpu

STATE = ["AT", "ATB", "WS", "NET", "AKT", "UTF_OUT", "VTF_OUT", "H0F_OUT"]
DIAG = ["AX", "AY", "AZ", "DZ", "PENETRATE", "TEND", "DT_DIFF"]


def bits_equal(a, b):
    return np.array_equal(np.ascontiguousarray(a).view(np.uint64), np.ascontiguousarray(b).view(np.uint64))


def mismatch(a, b):
    d = np.abs(a - b)
    idx = np.unravel_index(np.argmax(d), d.shape)
    return "max diff %.3e at %s (gpu %r oracle %r), %d cells differ" % (d[idx], idx, a[idx], b[idx],
                                                                         int(np.sum(a != b)))


def run_pair(lt, syn, p, f, nsteps, diagnostics):
    dom = lt.TracerDomain(syn.nx, syn.ny, syn.km, p, diagnostics=diagnostics,
                          ew_cyclic=bool(syn.cfg.ew_cyclic), tripole=bool(syn.cfg.tripole))
    for n in lt.INPUT_FIELDS:
        dom.set(n, f[n])
    dom.step(nsteps)
    o = pyoracle.Oracle(syn.nx, syn.ny, syn.km, p, ew_cyclic=syn.cfg.ew_cyclic, tripole=syn.cfg.tripole)
    o.load(f)
    o.sum_order(1)
    o.step(nsteps)
    return dom, o


def check(dom, o, names):
    for n in names:
        g, r = dom.get(n), o.get(n)
        assert bits_equal(g, r), n + ": " + mismatch(g, r)
    assert dom.fw_norm2() == o.fw_norm2()


# scheme, (nx, ny, km), synth keywords, steps, diagnostics
CASES = [
    ("centered", (36, 40, 55), dict(forced=1, cap_north=0), 3, True),
    ("flux", (36, 40, 55), dict(forced=1, cap_north=0), 3, True),
    ("centered", (120, 80, 30), dict(forced=0, cap_north=3), 4, False),
    ("flux", (124, 72, 30), dict(forced=1, cap_north=0), 4, False),
    ("centered", (49, 33, 20), dict(forced=1, cap_north=0, ew_cyclic=0, tripole=0), 2, True),
    ("flux", (50, 35, 24), dict(forced=0, cap_north=0), 3, True),
]


@pytest.mark.parametrize("scheme,size,kw,nsteps,diagnostics", CASES)
def test_scheme_step_bitexact(lt, scheme, size, kw, nsteps, diagnostics):
    syn, p, f = scheme_case.case(lt, scheme, seed=11 + nsteps, nx=size[0], ny=size[1], km=size[2],
                                 **dict(dict(forced=1), **kw))
    dom, o = run_pair(lt, syn, p, f, nsteps, diagnostics)
    check(dom, o, STATE + (DIAG if diagnostics else []))
    # the centred scheme accumulated its diagnostics; the flux scheme left them alone
    if diagnostics:
        ax = dom.get("AX")
        assert (np.abs(ax).max() > 0) == (scheme == "centered")
    dom.close()


@pytest.mark.parametrize("scheme", ["centered", "flux"])
def test_scheme_through_shim(lt, scheme):
    """tracer_ (the reference-named shim) on a domain with the scheme set:
    utf/vtf scaled in place and vtl left holding S, as the oracle's literal
    tracer_ sequence does."""
    syn, p, f = scheme_case.case(lt, scheme, forced=1, seed=5)
    dom = lt.TracerDomain(syn.nx, syn.ny, syn.km, p, diagnostics=True)
    for n in lt.INPUT_FIELDS:
        dom.set(n, f[n])
    dom.bind_shim()
    for s in range(2):
        assert lt.tracer_(s) == ""
    o = pyoracle.Oracle(syn.nx, syn.ny, syn.km, p)
    o.load(f)
    o.sum_order(1)
    for _ in range(2):
        o.tracer_call()
    for n in ("AT", "ATB", "UTF", "VTF", "VTL", "AX", "AY", "AZ"):
        g, r = dom.get(n), o.get(n)
        assert bits_equal(g, r), n + ": " + mismatch(g, r)
    dom.close()


def test_scheme_switched_between_steps(lt):
    """tspas, then centred, then flux steps on one domain (lt_set_params
    between them), as the oracle run with the same switches."""
    syn, p, f = scheme_case.case(lt, "centered", forced=1, seed=3, nx=72, ny=40, km=16, cap_north=0)
    dom = lt.TracerDomain(syn.nx, syn.ny, syn.km, p)
    for n in lt.INPUT_FIELDS:
        dom.set(n, f[n])
    o = pyoracle.Oracle(syn.nx, syn.ny, syn.km, p)
    o.load(f)
    o.sum_order(1)
    for scheme in ("tspas", "centered", "flux"):
        q = type(p).from_buffer_copy(p)
        q.adv_tracer = lt.ADV_SCHEMES[scheme]
        dom.set_params(q)
        o.set_params(q)
        dom.step(2)
        o.step(2)
    check(dom, o, STATE)
    dom.close()


def test_mixed_refuses_scheme(lt):
    syn, p, _ = scheme_case.case(lt, "flux", forced=0, seed=1, nx=40, ny=24, km=10)
    with pytest.raises(lt.LtError) as e:
        lt.TracerDomain(syn.nx, syn.ny, syn.km, p, precision=lt.PREC_MIXED)
    assert e.value.code == lt.LT_E_INVALID
    q = type(p).from_buffer_copy(p)
    q.adv_tracer = lt.ADV_TSPAS
    dom = lt.TracerDomain(syn.nx, syn.ny, syn.km, q, precision=lt.PREC_MIXED)
    with pytest.raises(lt.LtError) as e:
        dom.set_params(p)
    assert e.value.code == lt.LT_E_INVALID
    dom.close()
