"""Momentum biharmonic friction (readyc.cpp:343-577, the BIHAR sequence of
readyc_ at readyc.cpp:1754-1775) on the CPU: the oracle restatement pinned
bit for bit against the reference's own readyc.cpp compiled for the CPU
(where the reference tree is present) and against the committed digests of
those runs; plus properties: the friction vanishes for a uniform flow away
from boundaries and where the reference does not apply it, and the drag
speed is c0f*|u|."""
import hashlib
import json
import os

import numpy as np
import pytest
from conftest import REPO
from del4u_case import C0F, DEL4U_CASES, case

import pyoracle

GOLDEN = os.path.join(REPO, "tests", "golden", "reference_digests.json")
DEL4U_OUT = ["DLU", "DLV", "WKA_DRAG"]


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def run_oracle(syn, f, am):
    o = pyoracle.Oracle(syn.nx, syn.ny, syn.km, syn.params)
    o.load(f)
    o.hdiffu_del4(am, C0F)
    return o


@pytest.mark.skipif(not pyoracle.reference_readyc_available(), reason="reference tree not built here")
@pytest.mark.parametrize("seed,cap_north", DEL4U_CASES)
def test_del4u_oracle_bitexact_vs_reference(lt, seed, cap_north):
    syn, f, am = case(lt, seed, cap_north)
    ref = pyoracle.ReferenceReadyc()
    ref.load(f)
    ref.del4u(am, C0F)
    o = run_oracle(syn, f, am)
    for name in DEL4U_OUT:
        a, b = o.get(name), ref.get(name)
        assert np.array_equal(a.view(np.uint64), b.view(np.uint64)), name


@pytest.mark.parametrize("seed,cap_north", DEL4U_CASES)
def test_del4u_oracle_matches_golden_digests(lt, seed, cap_north):
    gold = json.load(open(GOLDEN))
    key = "del4u_seed%d_cap%d" % (seed, cap_north)
    assert key in gold, "regenerate tests/golden with make_golden.py"
    syn, f, am = case(lt, seed, cap_north)
    for n in ("UP", "DUC", "DMS"):
        assert digest(f[n]) == gold[key]["inputs"][n], n
    o = run_oracle(syn, f, am)
    for name in DEL4U_OUT:
        assert digest(o.get(name)) == gold[key]["outputs"][name], name


def test_del4u_properties(lt):
    syn, f, am = case(lt, 4, 0)
    o = run_oracle(syn, f, am)
    dlu, dlv = o.get("DLU"), o.get("DLV")
    du, dv = dlu - f["DLU"], dlv - f["DLV"]
    km = syn.km
    # nothing outside the interior ring the reference updates, nor below kmu
    assert np.all(du[:, 0] == 0) and np.all(du[:, -1] == 0) and np.all(du[:, :, 0] == 0) and np.all(du[:, :, -1] == 0)
    below = np.arange(km)[:, None, None] >= f["KMU"][None]
    assert np.all(du[below] == 0) and np.all(dv[below] == 0)
    # the friction acts
    assert np.abs(du).max() > 0 and np.abs(dv).max() > 0
    # drag speed
    np.testing.assert_array_equal(o.get("WKA_DRAG"), C0F * np.sqrt(f["UP"] ** 2 + f["VP"] ** 2))
    # linear in the velocity where the flow-dependent factor sits at its floor:
    # scaling up and vp by 2 scales the friction by 2 wherever am_f stays 1
    f2 = dict(f)
    f2["UP"] = 2.0 * f["UP"]
    f2["VP"] = 2.0 * f["VP"]
    f2["DLU"] = np.zeros_like(f["DLU"])
    f2["DLV"] = np.zeros_like(f["DLV"])
    f0 = dict(f)
    f0["DLU"] = np.zeros_like(f["DLU"])
    f0["DLV"] = np.zeros_like(f["DLV"])
    a1 = run_oracle(syn, f0, am).get("DLU")
    a2 = run_oracle(syn, f2, am).get("DLU")
    ratio = np.abs(a2) / np.maximum(np.abs(a1), 1e-300)
    sel = np.abs(a1) > 1e-20
    assert np.median(ratio[sel]) >= 2.0 - 1e-9      # am_f grows with the flow, never shrinks
