"""Canuto turbulence closure (turb_cu, readyc.cpp:880-1612) on the CPU: the
oracle restatement pinned bit for bit

1. against the reference's own readyc.cpp compiled for the CPU (where the
   reference tree is present), on seeded synthetic inputs with the stand-in
   tables at the reference's block size;
2. against the committed digests of those reference runs
   (tests/golden/reference_digests.json, made by tests/golden/make_golden.py);

and properties the closure must have: diffusivities within [0, dfricmx]
apart from the tidal part, the wind-mixing floor at the surface, the tidal
mixing non-decreasing downward, zero output where no column is computed.
"""
import hashlib
import json
import os

import numpy as np
import pytest
from conftest import REPO
from turb_case import DFRICMX, NCC, TURB_CASES, case, tables

import pyoracle

GOLDEN = os.path.join(REPO, "tests", "golden", "reference_digests.json")
TURB_OUT = ["AKT", "AKMT", "AK_TIDE", "AMLD", "RICHARDSON", "FZTIDAL", "WP3_TIDAL"]


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def run_oracle(lt, syn, f):
    o = pyoracle.Oracle(syn.nx, syn.ny, syn.km, syn.params)
    o.load(f)
    st = lt.turb_tables_struct(tables(lt))
    o.turb(st, NCC, DFRICMX)
    return o


@pytest.mark.skipif(not pyoracle.reference_readyc_available(), reason="reference tree not built here")
@pytest.mark.parametrize("seed,forced", TURB_CASES)
def test_turb_oracle_bitexact_vs_reference(lt, seed, forced):
    syn, f = case(lt, seed, forced)
    ref = pyoracle.ReferenceReadyc()
    ref.load(f)
    ref.set_tables(lt.turb_tables_struct(tables(lt)))
    ref.call(NCC, DFRICMX, syn.params.dwndmix)
    o = run_oracle(lt, syn, f)
    for name in TURB_OUT:
        a, b = o.get(name), ref.get(name)
        assert np.array_equal(a.view(np.uint64), b.view(np.uint64)), name


@pytest.mark.parametrize("seed,forced", TURB_CASES)
def test_turb_oracle_matches_golden_digests(lt, seed, forced):
    gold = json.load(open(GOLDEN))
    key = "turb_seed%d_forced%d" % (seed, forced)
    assert key in gold, "regenerate tests/golden with make_golden.py"
    syn, f = case(lt, seed, forced)
    for n in ("RIT", "PDENSITY", "AT"):
        assert digest(f[n]) == gold[key]["inputs"][n], n
    o = run_oracle(lt, syn, f)
    for name in TURB_OUT:
        assert digest(o.get(name)) == gold[key]["outputs"][name], name


def test_turb_properties(lt):
    syn, f = case(lt, 5, 1)
    o = run_oracle(lt, syn, f)
    kmt = f["KMT"]
    km = syn.km
    akt, akmt, tide, amld = o.get("AKT"), o.get("AKMT"), o.get("AK_TIDE"), o.get("AMLD")
    inner = np.zeros_like(kmt, dtype=bool)
    inner[1:-1, 1:-1] = True
    col = inner & (kmt > 0)
    # no column: the memsets' zeros; AKT untouched
    assert np.all(akmt[:, ~col] == 0.0) and np.all(tide[:, ~col] == 0.0) and np.all(amld[~col] == 0.0)
    assert np.array_equal(akt[:, :, ~col], f["AKT"][:, :, ~col])
    assert np.array_equal(akt[:, km - 1], f["AKT"][:, km - 1])
    # tidal mixing within its bounds and non-decreasing downward over the wet interfaces
    kk = np.arange(km)[:, None, None]
    wet = (kk < (kmt - 1)[None]) & col[None]
    assert np.all(tide[wet] >= 1e-6 - 1e-18) and np.all(tide[wet] <= 1e-2)
    pair = wet[:-1] & wet[1:]
    assert np.all(tide[1:][pair] >= tide[:-1][pair])
    # turbulent part of AKT within [0, dfricmx] / ncc, the surface at least dwndmix / ncc
    turb_t = akt[0, :km - 1] * NCC - tide[:km - 1]
    w = wet[:km - 1]
    assert np.all(turb_t[w] >= -1e-15) and np.all(turb_t[w] <= DFRICMX + 1e-12)
    top = col & (kmt > 1)
    assert np.all(turb_t[0][top] >= syn.params.dwndmix - 1e-15)
    # the mixed layer lies within the water column
    h = -f["ZKP"][np.clip(kmt, 0, km)]
    assert np.all(amld[top] >= 0.0) and np.all(amld[top] <= h[top] + 1e-9)
    # the closure produced a spread of values, not one branch
    assert np.unique(np.round(np.log10(turb_t[w] + 1e-30), 1)).size > 10
