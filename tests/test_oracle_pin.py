"""Pins the CPU oracle (oracle/licom_oracle.cpp) on CPU.

1. Against the reference's own tracer.cpp / convadj.cpp compiled for the CPU
   (oracle/_ref, built from the reference tree by oracle/Makefile), at the
   reference's built-in block size 36 x 40 x 55: every output field bit-exact.
2. Against the committed golden digests of those reference runs
   (tests/golden/reference_digests.json, made by tests/golden/make_golden.py),
   so the pin holds where the reference tree is absent.
3. Against independent properties: halo/fold against the POP semantics,
   the implicit vertical solve against a dense solve, conservation.
"""
import hashlib
import json
import os

import numpy as np
import pytest
from conftest import REPO

import pyoracle
import assm_case
import restore_case
import scheme_case

GOLDEN = os.path.join(REPO, "tests", "golden", "reference_digests.json")
OUT_FIELDS = ["AT", "ATB", "WS", "NET", "UTF", "VTF", "VTL", "H0F", "AKT", "AX", "AY", "AZ", "DZ", "TEND",
              "DT_DIFF", "DT_CONV", "PENETRATE"]


def ref_config(lt, forced, seed=20240611, cap_north=0):
    return lt.Synth(36, 40, 55, forced=forced, cap_north=cap_north, cap_south=3, dz_top=5.0, dz_bot=300.0,
                    seed=seed)


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def run_oracle_literal(lt, syn, nsteps, convadj=True):
    o = pyoracle.Oracle(syn.nx, syn.ny, syn.km, syn.params)
    o.load(syn.all_fields())
    for _ in range(nsteps):
        o.tracer_call()
    if convadj:
        o.convadj()
    return o


CASES = [(1, 5, 20240611), (0, 3, 7), (1, 2, 99)]


@pytest.mark.skipif(not pyoracle.reference_available(), reason="reference tree not built here")
@pytest.mark.parametrize("forced,nsteps,seed", CASES)
def test_oracle_bitexact_vs_reference(lt, forced, nsteps, seed):
    syn = ref_config(lt, forced, seed)
    ref = pyoracle.Reference(syn.params)
    ref.load(syn.all_fields())
    for s in range(nsteps):
        ref.tracer_call(s)
    ref.convadj()
    o = run_oracle_literal(lt, syn, nsteps)
    assert o.fw_norm2() == ref.fw_norm2()
    for name in OUT_FIELDS:
        a, b = o.get(name), ref.get(name)
        assert np.array_equal(a.view(np.uint64), b.view(np.uint64)), name


@pytest.mark.parametrize("forced,nsteps,seed", CASES)
def test_oracle_matches_golden_digests(lt, forced, nsteps, seed):
    gold = json.load(open(GOLDEN))
    key = "forced%d_steps%d_seed%d" % (forced, nsteps, seed)
    assert key in gold, "regenerate tests/golden with make_golden.py"
    syn = ref_config(lt, forced, seed)
    # the inputs themselves are pinned too: a change of the generator would
    # silently change what the golden digests mean
    assert digest(syn.field("AT")) == gold[key]["inputs"]["AT"]
    assert digest(syn.field("UTF")) == gold[key]["inputs"]["UTF"]
    o = run_oracle_literal(lt, syn, nsteps)
    for name in OUT_FIELDS:
        assert digest(o.get(name)) == gold[key]["outputs"][name], name
    assert o.fw_norm2() == gold[key]["fw_norm2"]


def run_restore_oracle(lt, forced, nsteps, seed):
    syn, p, f = restore_case.case(lt, forced, seed)
    o = pyoracle.Oracle(syn.nx, syn.ny, syn.km, p)
    o.load(f)
    for _ in range(nsteps):
        o.tracer_call()
    o.convadj()
    return syn, p, f, o


@pytest.mark.skipif(not pyoracle.reference_available(), reason="reference tree not built here")
@pytest.mark.parametrize("forced,nsteps,seed", restore_case.RESTORE_CASES)
def test_oracle_restoring_bitexact_vs_reference(lt, forced, nsteps, seed):
    """boundary_restore = 1 (tracer_7's 15-day relaxation below the surface)
    against the reference's own tracer.cpp, bit for bit."""
    syn, p, f, o = run_restore_oracle(lt, forced, nsteps, seed)
    ref = pyoracle.Reference(p)
    ref.load(f)
    for s in range(nsteps):
        ref.tracer_call(s)
    ref.convadj()
    assert o.fw_norm2() == ref.fw_norm2()
    for name in OUT_FIELDS:
        a, b = o.get(name), ref.get(name)
        assert np.array_equal(a.view(np.uint64), b.view(np.uint64)), name


@pytest.mark.parametrize("forced,nsteps,seed", restore_case.RESTORE_CASES)
def test_oracle_restoring_matches_golden_digests(lt, forced, nsteps, seed):
    gold = json.load(open(GOLDEN))
    key = "restore_forced%d_steps%d_seed%d" % (forced, nsteps, seed)
    assert key in gold, "regenerate tests/golden with make_golden.py"
    syn, p, f, o = run_restore_oracle(lt, forced, nsteps, seed)
    assert digest(f["RESTORE"]) == gold[key]["inputs"]["RESTORE"]
    assert digest(f["AT"]) == gold[key]["inputs"]["AT"]
    for name in OUT_FIELDS:
        assert digest(o.get(name)) == gold[key]["outputs"][name], name
    assert o.fw_norm2() == gold[key]["fw_norm2"]
    # the relaxation moved the state: the same run without it differs below the surface
    off = type(p).from_buffer_copy(p)
    off.boundary_restore = 0
    q = pyoracle.Oracle(syn.nx, syn.ny, syn.km, off)
    q.load(f)
    for _ in range(nsteps):
        q.tracer_call()
    q.convadj()
    d = np.abs(o.get("AT") - q.get("AT"))
    assert d[0, 1:].max() > 1e-4 and d[0, 0].max() < d[0, 1:].max()


def run_scheme_oracle(lt, scheme, forced, nsteps, seed):
    syn, p, f = scheme_case.case(lt, scheme, forced, seed)
    o = pyoracle.Oracle(syn.nx, syn.ny, syn.km, p)
    o.load(f)
    for _ in range(nsteps):
        o.tracer_call()
    o.convadj()
    return syn, p, f, o


@pytest.mark.skipif(not pyoracle.reference_available(), reason="reference tree not built here")
@pytest.mark.parametrize("scheme,forced,nsteps,seed", scheme_case.SCHEME_CASES)
def test_oracle_scheme_bitexact_vs_reference(lt, scheme, forced, nsteps, seed):
    """The centred and flux advection schemes against the reference's own
    tracer.cpp, bit for bit (the centred scheme's racy diagnostic levels left
    out; their emulated value is the once-per-level one times the number of
    level threads of the launch)."""
    syn, p, f, o = run_scheme_oracle(lt, scheme, forced, nsteps, seed)
    ref = pyoracle.Reference(p)
    ref.load(f)
    for s in range(nsteps):
        ref.tracer_call(s)
    ref.convadj()
    assert o.fw_norm2() == ref.fw_norm2()
    for name in OUT_FIELDS:
        a = scheme_case.comparable(scheme, name, o.get(name))
        b = scheme_case.comparable(scheme, name, ref.get(name))
        assert np.array_equal(a.view(np.uint64), b.view(np.uint64)), name
    if scheme == "centered":
        repeats = -(-syn.km // 4) * 4     # the launch's level threads (blocks of 4 levels)
        for name in scheme_case.RACY_DIAG:
            a, b = o.get(name), ref.get(name)
            assert np.abs(a[:, 0]).max() > 0
            for k in (0, syn.km - 1):
                assert np.allclose(b[:, k], repeats * a[:, k], rtol=1e-9, atol=0), (name, k)
    else:
        assert not np.any(o.get("AX"))   # the flux scheme writes no diagnostics
    # the scheme matters: the tspas run of the same inputs differs
    tspas = type(p).from_buffer_copy(p)
    tspas.adv_tracer = lt.ADV_TSPAS
    q = pyoracle.Oracle(syn.nx, syn.ny, syn.km, tspas)
    q.load(f)
    for _ in range(nsteps):
        q.tracer_call()
    q.convadj()
    assert np.abs(o.get("AT") - q.get("AT")).max() > 1e-6


@pytest.mark.parametrize("scheme,forced,nsteps,seed", scheme_case.SCHEME_CASES)
def test_oracle_scheme_matches_golden_digests(lt, scheme, forced, nsteps, seed):
    gold = json.load(open(GOLDEN))
    key = "scheme_%s_forced%d_steps%d_seed%d" % (scheme, forced, nsteps, seed)
    assert key in gold, "regenerate tests/golden with make_golden.py"
    syn, p, f, o = run_scheme_oracle(lt, scheme, forced, nsteps, seed)
    assert digest(f["AT"]) == gold[key]["inputs"]["AT"]
    for name in OUT_FIELDS:
        assert digest(scheme_case.comparable(scheme, name, o.get(name))) == gold[key]["outputs"][name], name
    assert o.fw_norm2() == gold[key]["fw_norm2"]


def test_halo_restatement_matches_generator_halo(lt):
    """The oracle's POP halo restatement and the builder's halo agree (they are
    written independently) on a field f(i,j) = i + 1000 j plus noise."""
    nx, ny = 36, 40
    imt, jmt = nx + 4, ny + 4
    rng = np.random.default_rng(3)
    j, i = np.mgrid[0:jmt, 0:imt]
    f = (i + 1000.0 * j + rng.normal(size=(jmt, imt))).astype(np.float64)
    syn = lt.Synth(nx, ny, 5)
    o = pyoracle.Oracle(nx, ny, 5, syn.params)
    g = o.halo(f)
    # east-west cyclic on physical rows below the fold
    assert np.array_equal(g[3:jmt - 2, 0], f[3:jmt - 2, nx])
    assert np.array_equal(g[3:jmt - 2, 1], f[3:jmt - 2, nx + 1])
    assert np.array_equal(g[3:jmt - 2, nx + 2], f[3:jmt - 2, 2])
    assert np.array_equal(g[3:jmt - 2, nx + 3], f[3:jmt - 2, 3])
    # closed south: untouched
    assert np.array_equal(g[jmt - 2:], f[jmt - 2:])
    # fold: ghost rows mirror physical rows 4 and 3 about global i <-> nx - i
    for gcol in range(1, nx + 1):
        src = nx - gcol if gcol != nx else nx
        assert g[0, gcol + 1] == f[4, src + 1]
        assert g[1, gcol + 1] == f[3, src + 1]
    # top physical row: symmetric average with the mirror point
    for gcol in range(1, nx // 2):
        avg = 0.5 * (f[2, gcol + 1] + f[2, nx - gcol + 1])
        assert g[2, gcol + 1] == avg and g[2, nx - gcol + 1] == avg
    assert g[2, nx // 2 + 1] == f[2, nx // 2 + 1] and g[2, nx + 1] == f[2, nx + 1]
    # idempotent
    assert np.array_equal(o.halo(g), g)


def test_vertical_solve_matches_dense(lt):
    """With advection, del4 and forcing switched off the step is the implicit
    half of the vertical diffusion on top of the explicit half; rebuild the
    tridiagonal system from AKT and check the oracle's Thomas sweep against a
    dense solve."""
    nx, ny, km = 16, 12, 20
    syn = lt.Synth(nx, ny, km, umax=0.0, forced=0, cap_north=2, cap_south=2)
    p = syn.params
    p.ah = 0.0
    inp = syn.all_fields()
    o = pyoracle.Oracle(nx, ny, km, p)
    o.load(inp)
    o.tracer_call()
    at1 = o.get("AT")
    akt = o.get("AKT")   # after the surface floor applied by the step
    atb = inp["ATB"]
    at0 = inp["AT"]
    kmt = inp["KMT"]
    dzp, odzp, odzt = inp["DZP"], inp["ODZP"], inp["ODZT"]
    dts = p.dts
    checked = 0
    for (j, i) in [(5, 5), (6, 9), (8, 3), (4, 12)]:
        kz = kmt[j, i]
        if kz < 3:
            continue
        for n in range(2):
            wkc = akt[n, :, j, i]
            b = atb[n, :, j, i]
            # explicit half (tracer_5) plus the forcing-free surface terms
            tf = np.zeros(km)
            for k in range(1, km - 1):
                w1 = wkc[k - 1] * (b[k] - b[k + 1]) * odzt[k] * (k < kz)
                w2 = wkc[k] * (b[k + 1] - b[k + 2]) * odzt[k + 1] * (k + 1 < kz)
                tf[k] += odzp[k] * (w1 - w2) * 0.5
            tf[0] -= odzp[0] * wkc[0] * (b[1] - b[2]) * odzt[1] * (1 < kz) * 0.5
            tf[km - 1] += odzp[km - 1] * wkc[km - 2] * (b[km - 1] - b[km]) * odzt[km - 1] * (km - 1 < kz) * 0.5
            d = at0[n, :, j, i] + dts * tf
            M = np.zeros((kz, kz))
            for k in range(kz):
                a8 = wkc[k - 1] * odzt[k] * odzp[k] * dts * 0.5 if k >= 1 else odzp[0] * dts * 0.5
                c8 = wkc[k] * odzt[k + 1] * odzp[k] * dts * 0.5 if k < kz - 1 else 0.0
                M[k, k] = 1.0 + (a8 if k >= 1 else 0.0) + c8
                if k >= 1:
                    M[k, k - 1] = -a8
                if k < kz - 1:
                    M[k, k + 1] = -c8
            x = np.linalg.solve(M, d[:kz])
            np.testing.assert_allclose(at1[n, :kz, j, i], x, rtol=1e-12, atol=1e-15)
            checked += 1
    assert checked >= 4


def test_oracle_conserves_tracer_content(lt):
    """Zero surface fluxes, land-capped north and south rows, non-divergent
    flow: the global tracer integrals are conserved to round-off."""
    syn = lt.Synth(72, 40, 15, forced=0, cap_north=3, cap_south=3)
    o = pyoracle.Oracle(72, 40, 15, syn.params)
    o.load(syn.all_fields())
    c0 = np.array(o.tracer_content())
    o.step(10)
    c1 = np.array(o.tracer_content())
    rel = np.abs(c1 - c0) / np.abs(c0)
    assert rel[0] < 1e-13, rel
    assert rel[1] < 1e-12, rel


def test_tree_order_only_moves_the_sss_sum(lt):
    """The device's tree-ordered SSS sum differs from the sequential one by
    round-off only."""
    syn = ref_config(lt, 1)
    a = pyoracle.Oracle(syn.nx, syn.ny, syn.km, syn.params)
    b = pyoracle.Oracle(syn.nx, syn.ny, syn.km, syn.params)
    b.sum_order(1)
    inp = syn.all_fields()
    a.load(inp)
    b.load(inp)
    a.step(3)
    b.step(3)
    assert abs(a.fw_norm2() - b.fw_norm2()) <= 1e-14 * abs(a.fw_norm2())
    ta, tb = a.get("AT"), b.get("AT")
    assert np.max(np.abs(ta - tb)) <= 1e-12 * np.max(np.abs(ta))


@pytest.mark.parametrize("forced,nsteps,seed", CASES)
def test_tree_order_reproduces_reference_temperature(lt, forced, nsteps, seed):
    """In the device's fixed-tree SSS-norm order the oracle still gives the
    reference's temperature digests exactly: the sum feeds salinity only."""
    gold = json.load(open(GOLDEN))["forced%d_steps%d_seed%d" % (forced, nsteps, seed)]
    syn = ref_config(lt, forced, seed)
    o = pyoracle.Oracle(syn.nx, syn.ny, syn.km, syn.params)
    o.load(syn.all_fields())
    o.sum_order(1)
    for _ in range(nsteps):
        o.tracer_call()
    o.convadj()
    for n in ("AT", "ATB"):
        assert digest(o.get(n)[0]) == gold["outputs_T"][n], n


def _tracer7_oracle(params, br, sa, ktv, tf, vit, atb, restore, restore_at):
    p = type(params).from_buffer_copy(params)
    p.boundary_restore, p.simple_assm, p.ktv = br, sa, ktv
    out = {}
    for n in (0, 1):
        t, d = tf.copy(), np.zeros_like(restore)
        pyoracle.oracle_tracer7(p, n, t, vit, atb, restore, restore_at, d)
        out[n] = (t, d)
    return out


@pytest.mark.skipif(not pyoracle.reference_available(), reason="reference tree not built here")
@pytest.mark.parametrize("br,sa,ktv,seed", assm_case.ASSM_CASES)
def test_oracle_tracer7_bitexact_vs_reference(lt, br, sa, ktv, seed):
    """tracer_7 with its nudging branch (simple_assm), which the reference's
    tracer_ never runs: the reference's own kernel against the oracle."""
    syn = lt.Synth(36, 40, 55)
    ref = pyoracle.Reference(syn.params)
    tf, vit, atb, restore, restore_at = assm_case.arrays(ref.nx, ref.ny, ref.km, seed)
    mine = _tracer7_oracle(syn.params, br, sa, ktv, tf, vit, atb, restore, restore_at)
    for n in (0, 1):
        t, d = tf.copy(), np.zeros_like(restore)
        ref.tracer7(n, t, vit, atb, restore, restore_at, d, br, sa, ktv)
        assert np.array_equal(t.view(np.uint64), mine[n][0].view(np.uint64)), n
        assert np.array_equal(d.view(np.uint64), mine[n][1].view(np.uint64)), n
        if sa and n == 0:
            assert np.count_nonzero(d[0, :min(ktv, ref.km)]) > 0 and not d[0, ktv:].any()


@pytest.mark.parametrize("br,sa,ktv,seed", assm_case.ASSM_CASES)
def test_oracle_tracer7_matches_golden_digests(lt, br, sa, ktv, seed):
    gold = json.load(open(os.path.join(REPO, "tests", "golden", "reference_digests.json")))[
        assm_case.key(br, sa, ktv, seed)]
    syn = lt.Synth(36, 40, 55)
    tf, vit, atb, restore, restore_at = assm_case.arrays(36, 40, 55, seed)
    assert hashlib.sha256(atb.tobytes()).hexdigest() == gold["inputs"]["ATB"]
    mine = _tracer7_oracle(syn.params, br, sa, ktv, tf, vit, atb, restore, restore_at)
    for n in (0, 1):
        assert hashlib.sha256(mine[n][0].tobytes()).hexdigest() == gold["outputs"]["TF%d" % n]
        assert hashlib.sha256(mine[n][1].tobytes()).hexdigest() == gold["outputs"]["DT_RESTORE%d" % n]
