"""GPU parity: the sm_100a FP64 tracer step against the CPU oracle.

The FP64 kernels keep the reference's operation order and are compiled with
-fmad=false, so the comparison is bit-for-bit.  The one reduction on the path
(the SSS-normalisation sum, tracer.cpp:1849-1868) runs on the device in a
fixed tree order; the oracle is switched to the same order for the bit-exact
checks, and compared in the reference's sequential order with a 1e-13
relative tolerance.
"""
import json
import os

import numpy as np
import pytest
from conftest import REPO

import pyoracle

pytestmark = pytest.mark.gpu

STATE = ["AT", "ATB", "WS", "NET", "AKT", "UTF_OUT", "VTF_OUT", "H0F_OUT"]
DIAG = ["AX", "AY", "AZ", "DZ", "PENETRATE"]


def bits_equal(a, b):
    return np.array_equal(np.ascontiguousarray(a).view(np.uint64 if a.dtype == np.float64 else np.uint32),
                          np.ascontiguousarray(b).view(np.uint64 if b.dtype == np.float64 else np.uint32))


def mismatch(a, b):
    d = np.abs(a.astype(np.float64) - b.astype(np.float64))
    idx = np.unravel_index(np.argmax(d), d.shape)
    return "max diff %.3e at %s (gpu %r oracle %r), %d cells differ" % (d[idx], idx, a[idx], b[idx],
                                                                         int(np.sum(a != b)))


def make(lt, nx, ny, km, **kw):
    syn = lt.Synth(nx, ny, km, **kw)
    return syn, syn.all_fields()


def gpu_domain(lt, syn, fields, diagnostics=False, device_fill=False):
    dom = lt.TracerDomain(syn.nx, syn.ny, syn.km, syn.params, diagnostics=diagnostics,
                          ew_cyclic=bool(syn.cfg.ew_cyclic), tripole=bool(syn.cfg.tripole))
    if device_fill:
        syn.upload(dom)
    else:
        for n in lt.INPUT_FIELDS:
            dom.set(n, fields[n])
    return dom


def oracle_for(syn, fields, tree=True):
    o = pyoracle.Oracle(syn.nx, syn.ny, syn.km, syn.params, ew_cyclic=syn.cfg.ew_cyclic, tripole=syn.cfg.tripole)
    o.load(fields)
    o.sum_order(1 if tree else 0)
    return o


def test_device_generation_matches_host(lt):
    syn, f = make(lt, 64, 40, 12, forced=1, cap_north=0)
    dom = gpu_domain(lt, syn, f, device_fill=True)
    for n in ("AT", "ATB", "UTF", "VTF", "UTL", "VTL", "AKT", "KMT", "TAREA", "DZP"):
        g = dom.get(n)
        assert bits_equal(g, f[n]), n + ": " + mismatch(g, f[n])


@pytest.mark.parametrize("forced,cap_north,nsteps", [(1, 0, 5), (0, 3, 3)])
def test_step_bitexact_reference_size(lt, forced, cap_north, nsteps):
    """36 x 40 x 55, the reference's own block size; fold active when
    cap_north == 0."""
    syn, f = make(lt, 36, 40, 55, forced=forced, cap_north=cap_north, cap_south=3, dz_top=5.0, dz_bot=300.0)
    dom = gpu_domain(lt, syn, f)
    dom.step(nsteps)
    o = oracle_for(syn, f)
    o.step(nsteps)
    for n in STATE:
        g, r = dom.get(n), o.get(n)
        assert bits_equal(g, r), n + ": " + mismatch(g, r)
    assert dom.fw_norm2() == o.fw_norm2()


def test_step_close_to_sequential_sum_order(lt):
    syn, f = make(lt, 36, 40, 55, forced=1, cap_north=0, cap_south=3, dz_top=5.0, dz_bot=300.0)
    dom = gpu_domain(lt, syn, f)
    dom.step(5)
    o = oracle_for(syn, f, tree=False)
    o.step(5)
    for n in ("AT", "ATB"):
        g, r = dom.get(n), o.get(n)
        scale = np.abs(r).max(axis=(1, 2, 3), keepdims=True)
        assert np.all(np.abs(g - r) <= 1e-13 * scale), n + ": " + mismatch(g, r)
    assert abs(dom.fw_norm2() - o.fw_norm2()) <= 1e-13 * abs(o.fw_norm2())


def test_diagnostics_bitexact(lt):
    syn, f = make(lt, 36, 40, 55, forced=1, cap_north=0, cap_south=3, dz_top=5.0, dz_bot=300.0)
    dom = gpu_domain(lt, syn, f, diagnostics=True)
    dom.step(2)
    o = oracle_for(syn, f)
    o.step(2)
    for n in DIAG:
        g, r = dom.get(n), o.get(n)
        assert bits_equal(g, r), n + ": " + mismatch(g, r)
    for n in ("TEND", "DT_DIFF"):
        g, r = dom.get(n), o.get(n)
        assert bits_equal(g, r), n + ": " + mismatch(g, r)


def test_multistep_medium_grid(lt):
    """20 steps (the configuration-0 step count) on a 1-degree-like patch."""
    syn, f = make(lt, 120, 80, 30, forced=1, cap_north=0)
    dom = gpu_domain(lt, syn, f)
    dom.step(20)
    o = oracle_for(syn, f)
    o.step(20)
    for n in ("AT", "ATB", "WS", "NET"):
        g, r = dom.get(n), o.get(n)
        assert bits_equal(g, r), n + ": " + mismatch(g, r)


@pytest.mark.parametrize("diagnostics", [False, True])
def test_deep_ocean_bitexact(lt, diagnostics):
    """Depths from the global ocean's area-depth curve: the column march
    starts at the bottom level in most tiles and the deep-level paths (copies
    below the tile's bottom, the diagnostics' deep kernel) see few levels."""
    syn, f = make(lt, 120, 80, 30, forced=1, cap_north=0, hypsometry=1)
    dom = gpu_domain(lt, syn, f, diagnostics=diagnostics)
    dom.step(10)
    o = oracle_for(syn, f)
    o.step(10)
    for n in ("AT", "ATB", "WS") + (("AX", "AY", "AZ", "DZ", "TEND", "DT_DIFF") if diagnostics else ()):
        g, r = dom.get(n), o.get(n)
        assert bits_equal(g, r), n + ": " + mismatch(g, r)


@pytest.mark.parametrize("tma", [True, False])
def test_both_column_kernels(lt, tma):
    """The column kernel's level slots filled by TMA boxes or by per-thread
    asynchronous copies: the same bits as the oracle either way."""
    syn, f = make(lt, 100, 60, 20, forced=1, cap_north=0)
    dom = gpu_domain(lt, syn, f, diagnostics=True)
    dom.use_tma(tma)
    dom.step(3)
    o = oracle_for(syn, f)
    o.step(3)
    for n in ("AT", "ATB", "AX", "AZ", "DZ", "TEND", "DT_DIFF"):
        g, r = dom.get(n), o.get(n)
        assert bits_equal(g, r), n + ": " + mismatch(g, r)


@pytest.mark.parametrize("diagnostics", [False, True])
def test_odd_row_pitch_copy_fill(lt, diagnostics):
    """nx = 49 (closed domain): the row pitch is not a multiple of 16 bytes,
    TMA boxes are refused, and the column kernel's slots filled by per-thread
    copies still match the oracle bit for bit (with the diagnostics, also
    below the tile's march)."""
    syn, f = make(lt, 49, 30, 10, forced=1, cap_north=2, ew_cyclic=0, tripole=0)
    dom = gpu_domain(lt, syn, f, diagnostics=diagnostics)
    with pytest.raises(lt.LtError):
        dom.use_tma(True)
    dom.step(3)
    o = oracle_for(syn, f)
    o.step(3)
    names = ["AT", "ATB", "WS"] + (["AX", "AY", "AZ", "DZ", "PENETRATE", "TEND", "DT_DIFF"] if diagnostics else [])
    for n in names:
        g, r = dom.get(n), o.get(n)
        assert bits_equal(g, r), n + ": " + mismatch(g, r)


def test_closed_boundaries(lt):
    syn, f = make(lt, 50, 30, 12, forced=1, cap_north=2, ew_cyclic=0, tripole=0)
    dom = gpu_domain(lt, syn, f)
    dom.step(4)
    o = oracle_for(syn, f)
    o.step(4)
    for n in ("AT", "ATB", "NET"):
        g, r = dom.get(n), o.get(n)
        assert bits_equal(g, r), n + ": " + mismatch(g, r)


def test_convadj_bitexact(lt):
    syn, f = make(lt, 36, 40, 55, forced=1, cap_north=0, cap_south=3, dz_top=5.0, dz_bot=300.0)
    dom = gpu_domain(lt, syn, f, diagnostics=True)
    dom.step(1)
    dom.convadj()
    o = oracle_for(syn, f)
    o.step(1)
    o.convadj()
    for n in ("AT", "ATB", "DT_CONV", "TEND"):
        g, r = dom.get(n), o.get(n)
        assert bits_equal(g, r), n + ": " + mismatch(g, r)
    assert np.any(o.get("DT_CONV") != 0.0)  # adjustment did something


def test_reference_shims_match_golden(lt):
    """tracer_/convadj_ on a bound domain reproduce the reference's literal
    call sequence (utf scaled in place, vtl left holding S), compared with
    the oracle in the device's sum order and with the golden digests of the
    reference's own code."""
    import hashlib
    syn, f = make(lt, 36, 40, 55, forced=1, cap_north=0, cap_south=3, dz_top=5.0, dz_bot=300.0, seed=20240611)
    dom = gpu_domain(lt, syn, f, diagnostics=True)
    dom.bind_shim()
    for s in range(5):
        lt.tracer_(s)
    lt.convadj_()
    o = oracle_for(syn, f)
    for _ in range(5):
        o.tracer_call()
    o.convadj()
    for n in ("AT", "ATB", "UTF", "VTF", "VTL", "H0F", "NET"):
        g, r = dom.get(n), o.get(n)
        assert bits_equal(g, r), n + ": " + mismatch(g, r)
    gold = json.load(open(os.path.join(REPO, "tests", "golden", "reference_digests.json")))["forced1_steps5_seed20240611"]
    # temperature: the reference's own digests, bit for bit (the SSS-norm sum
    # order touches salinity only)
    for n in ("AT", "ATB"):
        assert hashlib.sha256(np.ascontiguousarray(dom.get(n)[0]).tobytes()).hexdigest() == gold["outputs_T"][n], n
    t_ref = np.array(gold["surface_T_sample"])
    assert np.array_equal(dom.get("AT")[0, 0, 20, 5:15], t_ref)
    # salinity: the oracle in the reference's sequential sum order reproduces
    # the reference's digests, and the device (fixed-tree order) is within
    # 1e-13 of it relative to max |S|
    q = oracle_for(syn, f, tree=False)
    for _ in range(5):
        q.tracer_call()
    q.convadj()
    for n in ("AT", "ATB", "VTL"):
        assert hashlib.sha256(q.get(n).tobytes()).hexdigest() == gold["outputs"][n], n
    for n in ("AT", "ATB"):
        g, r = dom.get(n)[1], q.get(n)[1]
        assert np.abs(g - r).max() <= 1e-13 * np.abs(r).max(), n + " S: " + mismatch(g, r)
    g, r = dom.get("VTL"), q.get("VTL")
    assert np.abs(g - r).max() <= 1e-13 * np.abs(r).max(), "VTL: " + mismatch(g, r)


def test_derive_masks(lt):
    syn, f = make(lt, 64, 40, 20, forced=0, cap_north=0)
    dom = gpu_domain(lt, syn, f)
    for n in ("KMU", "KMTN", "KMTS", "KMTE", "KMTW"):
        dom.set(n, np.zeros_like(f[n]))
    dom.set("OHBT", np.zeros_like(f["OHBT"]))
    dom.set("OHBU", np.zeros_like(f["OHBU"]))
    dom.set("ODZP", np.zeros_like(f["ODZP"]))
    dom.derive_masks()
    for n in ("KMU", "KMTN", "KMTS", "KMTE", "KMTW", "OHBT", "OHBU", "ODZP"):
        g = dom.get(n)
        assert bits_equal(g, f[n]), n + ": " + mismatch(g, f[n])


def test_conservation_on_device(lt):
    syn, f = make(lt, 144, 72, 30, forced=0, cap_north=3, cap_south=3)
    dom = gpu_domain(lt, syn, f)
    c0 = np.array(dom.tracer_content())
    dom.step(20)
    c1 = np.array(dom.tracer_content())
    rel = np.abs(c1 - c0) / np.abs(c0)
    assert rel[0] < 1e-13 and rel[1] < 1e-13, rel


def test_step_host_reports_scalars(lt):
    syn, f = make(lt, 64, 40, 12, forced=1, cap_north=0)
    dom = gpu_domain(lt, syn, f)
    forcing = {n: f[n] for n in ("SWV", "NSWV", "SST", "SSS", "FRESH", "SEAICE")}
    fw, ct, cs = dom.step_host(forcing)
    assert fw == dom.fw_norm2()
    t2 = dom.tracer_content()
    assert (ct, cs) == t2
    o = oracle_for(syn, f)
    o.step(1)
    assert bits_equal(dom.get("AT"), o.get("AT"))


def test_step_host_new_forcing_every_step(lt):
    """lt_step_host uploads each step's forcing on a copy stream while the
    step's continuity runs: several steps, each with its own forcing, match
    the oracle given the same forcing before each of its steps, bit for bit
    (mixed-precision domains take the same path)."""
    syn, f = make(lt, 96, 56, 16, forced=1, cap_north=0)
    dom = gpu_domain(lt, syn, f)
    o = oracle_for(syn, f)
    rng = np.random.default_rng(5)
    names = ("SWV", "NSWV", "SST", "SSS", "FRESH", "SEAICE")
    for step in range(4):
        forcing = {}
        for n in names:
            a = f[n] * (1.0 + 0.05 * rng.standard_normal(f[n].shape))
            if n == "SEAICE":
                a = np.clip(a, 0.0, 1.0)
            forcing[n] = np.ascontiguousarray(a)
            o.set(n, forcing[n])
        fw, _, _ = dom.step_host(forcing)
        o.step(1)
        assert fw == o.fw_norm2(), step
        for name in ("AT", "NET", "AKT"):
            g, r = dom.get(name), o.get(name)
            assert bits_equal(g, r), "step %d %s: %s" % (step, name, mismatch(g, r))


def test_step_host_async_double_buffered_forcing(lt):
    """lt_step_host_async: each step's forcing goes into the other of two
    device sets while the previous step runs.  A run of asynchronous steps
    (some keeping a field from the step before), then a synchronous one and a
    device step, match the oracle given the same forcing, bit for bit, with
    every step's fw_norm2 delivered to pinned host memory."""
    import torch
    syn, f = make(lt, 96, 56, 16, forced=1, cap_north=0)
    dom = gpu_domain(lt, syn, f)
    o = oracle_for(syn, f)
    rng = np.random.default_rng(9)
    names = ("SWV", "NSWV", "SST", "SSS", "FRESH", "SEAICE")
    A = f["SST"].size
    nsteps = 6
    keep = {2: ("SST",), 4: names}          # step -> fields left NULL (kept)
    host = torch.empty((nsteps, 6, A), dtype=torch.float64, pin_memory=True)
    fw = torch.zeros(nsteps, dtype=torch.float64, pin_memory=True)
    fw_ref = []
    for step in range(nsteps):
        ptrs = [0] * 6
        for m, n in enumerate(names):
            if n in keep.get(step, ()):
                continue
            a = f[n] * (1.0 + 0.05 * rng.standard_normal(f[n].shape))
            if n == "SEAICE":
                a = np.clip(a, 0.0, 1.0)
            host[step, m] = torch.from_numpy(np.ascontiguousarray(a).ravel())
            ptrs[m] = host[step, m].data_ptr()
            o.set(n, a)
        dom.step_host_async_ptrs(ptrs, fw.data_ptr() + 8 * step)
        o.step(1)
        fw_ref.append(o.fw_norm2())
    dom.sync()
    assert fw.tolist() == fw_ref
    for name in ("AT", "NET", "AKT", "SST", "SWV"):
        g, r = dom.get(name), o.get(name)
        assert bits_equal(g, r), "%s: %s" % (name, mismatch(g, r))
    # a synchronous step and a device step go on from the set last filled
    forcing = {"SSS": np.ascontiguousarray(f["SSS"] * 1.01)}
    o.set("SSS", forcing["SSS"])
    fw1, _, _ = dom.step_host(forcing)
    dom.step(1)
    o.step(2)
    assert bits_equal(dom.get("AT"), o.get("AT"))


def test_numeric_scan_flags_injected_nan(lt):
    """Failure detection without a GPU fault: a NaN planted in the state on
    the host is reported as a count and a status, the context stays usable."""
    syn, f = make(lt, 40, 24, 8)
    dom = gpu_domain(lt, syn, f)
    assert dom.check_numeric() == 0
    at = f["AT"].copy()
    at[0, 1, 10, 10] = np.nan
    at[1, 2, 11, 12] = np.inf
    dom.set("AT", at)
    assert dom.check_numeric() == 2
    dom.set("AT", f["AT"])
    dom.step(1)
    assert dom.check_numeric() == 0
