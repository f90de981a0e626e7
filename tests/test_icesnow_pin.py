"""Sea-ice adjustment (icesnow.cpp:15-85) on the CPU: the oracle restatement
pinned bit for bit

1. against the reference's own icesnow.cpp compiled for the CPU, as it is
   configured (FRC_CORE: licomqice zeroed before each call) and compiled
   without FRC_CORE (licomqice carried over), alone and in the stepon.cpp:69-77
   order tracer_ -> icesnow_ -> convadj_ (where the reference tree is present);
2. against the committed digests of those reference runs
   (tests/golden/reference_digests.json, made by tests/golden/make_golden.py);

and the properties the adjustment must have whatever the order of operations:
no water below the freezing point afterwards, ice only where ocean water was
below it, the brine term on S, a second call changing nothing when QICE
carries over.
"""
import hashlib
import json
import os

import numpy as np
import pytest
from conftest import REPO
from icesnow_state import ICE_CASES, TBICE, cold_state

import pyoracle

GOLDEN = os.path.join(REPO, "tests", "golden", "reference_digests.json")
ICE_OUT = ["AT", "ATB", "QICE", "TEND", "DT_CONV", "WS", "NET"]


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def ref_syn(lt, seed):
    return lt.Synth(36, 40, 55, forced=1, cap_north=0, cap_south=3, dz_top=5.0, dz_bot=300.0, seed=seed)


def ice_inputs(lt, seed):
    syn = ref_syn(lt, seed)
    inp = syn.all_fields()
    inp["AT"], inp["QICE"] = cold_state(inp, seed)
    return syn, inp


def run_oracle(lt, syn, inp, frc_core, nsteps):
    o = pyoracle.Oracle(syn.nx, syn.ny, syn.km, syn.params)
    o.load(inp)
    p = lt.IcesnowParams(reset_qice=frc_core)
    if nsteps == 0:
        o.icesnow(p)
    for s in range(nsteps):
        o.tracer_call()
        o.icesnow(p)
        if s == 0:
            o.convadj()
    return o


@pytest.mark.skipif(not pyoracle.reference_available(), reason="reference tree not built here")
@pytest.mark.parametrize("frc_core,nsteps,seed", ICE_CASES)
def test_icesnow_oracle_bitexact_vs_reference(lt, frc_core, nsteps, seed):
    syn, inp = ice_inputs(lt, seed)
    ref = pyoracle.Reference(syn.params)
    ref.load(inp)
    if nsteps == 0:
        ref.icesnow(frc_core=frc_core)
    for s in range(nsteps):
        ref.tracer_call(s)
        ref.icesnow(frc_core=frc_core)
        if s == 0:
            ref.convadj()
    o = run_oracle(lt, syn, inp, frc_core, nsteps)
    for name in ICE_OUT:
        a, b = o.get(name), ref.get(name)
        assert np.array_equal(a.view(np.uint64), b.view(np.uint64)), name


@pytest.mark.parametrize("frc_core,nsteps,seed", ICE_CASES)
def test_icesnow_oracle_matches_golden_digests(lt, frc_core, nsteps, seed):
    gold = json.load(open(GOLDEN))
    key = "icesnow_frc%d_steps%d_seed%d" % (frc_core, nsteps, seed)
    assert key in gold, "regenerate tests/golden with make_golden.py"
    syn, inp = ice_inputs(lt, seed)
    assert digest(inp["AT"]) == gold[key]["inputs"]["AT"]
    assert digest(inp["QICE"]) == gold[key]["inputs"]["QICE"]
    o = run_oracle(lt, syn, inp, frc_core, nsteps)
    for name in ICE_OUT:
        assert digest(o.get(name)) == gold[key]["outputs"][name], name


def test_icesnow_properties(lt):
    syn, inp = ice_inputs(lt, 3)
    at0, kmt = inp["AT"], inp["KMT"]
    o = run_oracle(lt, syn, inp, 1, 0)
    at1, q = o.get("AT"), o.get("QICE")
    assert np.all(at1[0] >= TBICE)
    # T raised exactly to the freezing point where it was below, else untouched
    below = at0[0] < TBICE
    assert np.all(at1[0][below] == TBICE)
    assert np.array_equal(at1[0][~below], at0[0][~below])
    # S changes only at level 0 of ocean columns that froze
    froze = below[0] & (kmt > 0)
    assert np.array_equal(at1[1, 1:], at0[1, 1:])
    assert np.array_equal(at1[1, 0][~froze], at0[1, 0][~froze])
    # ice = the deficit, the brine term on S
    np.testing.assert_allclose(q[froze], TBICE - at0[0, 0][froze], rtol=1e-15, atol=0)
    assert np.all(q[~froze] == 0.0)
    brine = q * (34.7 - 4.0) * 3996.0 / 3.337e5 * 1e-3
    np.testing.assert_allclose(at1[1, 0][froze] - at0[1, 0][froze], brine[froze], rtol=1e-9, atol=1e-18)


def test_icesnow_melts_carried_ice_and_is_idempotent(lt):
    syn, inp = ice_inputs(lt, 4)
    at0, q0, kmt = inp["AT"], inp["QICE"], inp["KMT"]
    o = run_oracle(lt, syn, inp, 0, 0)
    at1, q1 = o.get("AT"), o.get("QICE")
    warm = (at0[0, 0] > TBICE) & (q0 > 0)
    assert warm.sum() > 50
    melt = np.minimum(at0[0, 0] - TBICE, q0)
    np.testing.assert_allclose(q1[warm], q0[warm] - melt[warm], rtol=0, atol=1e-15)
    np.testing.assert_allclose(at1[0, 0][warm], at0[0, 0][warm] - melt[warm], rtol=0, atol=1e-14)
    assert np.all(q1 >= 0.0) and np.all(at1[0] >= TBICE)
    o.icesnow(lt.IcesnowParams(reset_qice=0))
    assert np.array_equal(o.get("AT"), at1)
    assert np.array_equal(o.get("QICE"), q1)
