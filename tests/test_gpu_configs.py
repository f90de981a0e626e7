"""The device step against the CPU oracle on the stated configurations.

Configuration 0: 360 x 196 x 30 (1 degree, tripole fold, periodic east-west),
20 steps, the FP64 drop-in bit for bit against the oracle (which is itself
bit-exact with the reference's tracer.cpp, tests/test_oracle_pin.py).

Configuration 1: 360 x 218 x 30, 100 steps: the FP64 drop-in bit for bit,
and the mixed-precision form (f32 flux, stencil and diffusion arithmetic, f64
state) within 1e-4 K and 1e-5 psu of the oracle.  The oracle's 100 steps run
once per module.

The restoring branch (tracer_7 with boundary_restore = 1) on the reference's
block size and on a 1-degree grid: FP64 bit for bit with both column kernels,
mixed within the same bounds.
"""
import numpy as np
import pytest

import pyoracle
import restore_case

pytestmark = pytest.mark.gpu

T_TOL_K = 1.0e-4
S_TOL_PSU = 1.0e-5


def bits_equal(a, b):
    return np.array_equal(np.ascontiguousarray(a).view(np.uint64), np.ascontiguousarray(b).view(np.uint64))


def mismatch(a, b):
    d = np.abs(a - b)
    idx = np.unravel_index(np.argmax(d), d.shape)
    return "max diff %.3e at %s, %d cells differ" % (d[idx], idx, int(np.sum(a != b)))


def oracle_run(syn, params, fields, nsteps):
    o = pyoracle.Oracle(syn.nx, syn.ny, syn.km, params, ew_cyclic=syn.cfg.ew_cyclic, tripole=syn.cfg.tripole)
    o.load(fields)
    o.sum_order(1)                  # the device's fixed-tree SSS-norm sum
    o.step(nsteps)
    return o


def device_run(lt, syn, params, fields, nsteps, precision, tma=None):
    dom = lt.TracerDomain(syn.nx, syn.ny, syn.km, params, precision=precision,
                          ew_cyclic=bool(syn.cfg.ew_cyclic), tripole=bool(syn.cfg.tripole))
    for n in lt.INPUT_FIELDS:
        dom.set(n, fields[n])
    if params.boundary_restore == 1:
        dom.set("RESTORE", fields["RESTORE"])
    if tma is not None:
        dom.use_tma(tma)
    dom.step(nsteps)
    return dom


def ocean_errors(fields, km, a_ref, a_dev):
    """max |dT| in K and max |dS| in psu over wet interior cells."""
    kmt = fields["KMT"]
    wet = (np.arange(km)[:, None, None] < kmt[None])[:, 2:-2, 2:-2]
    a, b = a_ref[:, :, 2:-2, 2:-2], a_dev[:, :, 2:-2, 2:-2]
    return np.abs(a[0] - b[0])[wet].max(), np.abs(a[1] - b[1])[wet].max() * 1.0e3


@pytest.mark.parametrize("forced", [0, 1])
def test_config0_fp64_bitexact_20_steps(lt, forced):
    syn = lt.Synth(360, 196, 30, forced=forced)
    f = syn.all_fields()
    o = oracle_run(syn, syn.params, f, 20)
    dom = device_run(lt, syn, syn.params, f, 20, lt.PREC_FP64)
    for n in ("AT", "ATB", "WS", "NET", "UTF_OUT", "VTF_OUT"):
        g, r = dom.get(n), o.get(n)
        assert bits_equal(g, r), n + ": " + mismatch(g, r)
    assert dom.fw_norm2() == o.fw_norm2()


@pytest.fixture(scope="module")
def config1(lt):
    syn = lt.Synth(360, 218, 30, forced=1)
    f = syn.all_fields()
    o = oracle_run(syn, syn.params, f, 100)
    return syn, f, {n: o.get(n) for n in ("AT", "ATB", "WS", "NET")}, o.fw_norm2()


def test_config1_fp64_bitexact_100_steps(lt, config1):
    syn, f, ref, fw = config1
    dom = device_run(lt, syn, syn.params, f, 100, lt.PREC_FP64)
    for n, r in ref.items():
        g = dom.get(n)
        assert bits_equal(g, r), n + ": " + mismatch(g, r)
    assert dom.fw_norm2() == fw


def test_config1_mixed_vs_oracle_100_steps(lt, config1):
    syn, f, ref, fw = config1
    dom = device_run(lt, syn, syn.params, f, 100, lt.PREC_MIXED)
    dt, ds = ocean_errors(f, syn.km, ref["AT"], dom.get("AT"))
    print("config 1 mixed vs oracle after 100 steps: max |dT| %.3e K, max |dS| %.3e psu (ah %.3e)"
          % (dt, ds, syn.params.ah))
    assert dt <= T_TOL_K, dt
    assert ds <= S_TOL_PSU, ds
    assert dom.check_numeric() == 0


@pytest.mark.parametrize("forced,nsteps,seed", restore_case.RESTORE_CASES)
@pytest.mark.parametrize("tma", [True, False])
def test_restoring_fp64_bitexact(lt, forced, nsteps, seed, tma):
    syn, p, f = restore_case.case(lt, forced, seed)
    o = oracle_run(syn, p, f, nsteps)
    dom = device_run(lt, syn, p, f, nsteps, lt.PREC_FP64, tma=tma)
    for n in ("AT", "ATB", "WS", "NET"):
        g, r = dom.get(n), o.get(n)
        assert bits_equal(g, r), n + ": " + mismatch(g, r)


def test_restoring_one_degree(lt):
    """Restoring on a 1-degree 360 x 196 x 30 grid, 10 steps: FP64 bit for
    bit, mixed within 1e-5 K / 1e-6 psu of the oracle."""
    syn, p, f = restore_case.case(lt, 1, 11, nx=360, ny=196, km=30)
    o = oracle_run(syn, p, f, 10)
    r = o.get("AT")
    dom = device_run(lt, syn, p, f, 10, lt.PREC_FP64)
    assert bits_equal(dom.get("AT"), r), mismatch(dom.get("AT"), r)
    mix = device_run(lt, syn, p, f, 10, lt.PREC_MIXED)
    dt, ds = ocean_errors(f, syn.km, r, mix.get("AT"))
    print("restoring, mixed vs oracle after 10 steps: %.3e K, %.3e psu" % (dt, ds))
    assert dt <= 1e-5 and ds <= 1e-6, (dt, ds)


@pytest.mark.parametrize("diagnostics,tma,scheme", [(False, True, 0), (True, True, 0), (False, False, 0),
                                                    (True, None, 1)])
def test_nudging_fp64_bitexact(lt, diagnostics, tma, scheme):
    """tracer_7's nudging toward RESTORE_AT (simple_assm) in the levels
    k < ktv = 50 (the deep ones at the weaker rate), with the 15-day
    restoring on as well: the FP64 step and DT_RESTORE bit for bit against
    the oracle, whose tracer_7 is pinned to the reference's own kernel.
    Both column kernels (TMA boxes, copy fill) and the centred scheme's."""
    syn, p, f = restore_case.case(lt, 1, 23)
    p.simple_assm, p.ktv, p.adv_tracer = 1, 50, scheme
    f["RESTORE_AT"] = 2.0 * f["AT"] - restore_case.restore_target(f["AT"])
    o = pyoracle.Oracle(syn.nx, syn.ny, syn.km, p, ew_cyclic=syn.cfg.ew_cyclic, tripole=syn.cfg.tripole)
    o.load(f)
    o.sum_order(1)
    o.step(3)
    dom = lt.TracerDomain(syn.nx, syn.ny, syn.km, p, precision=lt.PREC_FP64, diagnostics=diagnostics,
                          ew_cyclic=bool(syn.cfg.ew_cyclic), tripole=bool(syn.cfg.tripole))
    for n in lt.INPUT_FIELDS + ["RESTORE", "RESTORE_AT"]:
        dom.set(n, f[n])
    if tma is not None:
        dom.use_tma(tma)
    dom.step(3)
    names = ["AT", "ATB", "WS", "DT_RESTORE"] + (["TEND", "DT_DIFF"] if diagnostics else [])
    for n in names:
        g, r = dom.get(n), o.get(n)
        assert bits_equal(g, r), n + ": " + mismatch(g, r)
    assert np.count_nonzero(dom.get("DT_RESTORE")[0, 45:50]) > 0
