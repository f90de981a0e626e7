"""Mixed precision (f32 flux/stencil/diffusion arithmetic, f64 state and
sweep) against the FP64 form, which is bit-exact with the oracle.

Bounds are the configuration targets: after 100 steps on the 1-degree
360 x 218 x 30 grid the temperature error stays within 1e-4 K and the
salinity error within 1e-5 psu (1e-8 in model units, S stored as
(S_psu - 35)/1000).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

T_TOL_K = 1.0e-4
S_TOL_PSU = 1.0e-5


def run_pair(lt, nx, ny, km, steps, **kw):
    syn = lt.Synth(nx, ny, km, **kw)
    ref = syn.domain(precision=lt.PREC_FP64)
    mix = syn.domain(precision=lt.PREC_MIXED)
    ref.step(steps)
    mix.step(steps)
    return syn, ref, mix


def ocean_errors(syn, ref, mix):
    kmt = syn.field("KMT")
    km = syn.km
    wet = (np.arange(km)[:, None, None] < kmt[None])[:, 2:-2, 2:-2]
    a, b = ref.get("AT")[:, :, 2:-2, 2:-2], mix.get("AT")[:, :, 2:-2, 2:-2]
    dt = np.abs(a[0] - b[0])[wet].max()
    ds = np.abs(a[1] - b[1])[wet].max() * 1.0e3
    return dt, ds


def test_mixed_error_bounds_100_steps(lt):
    syn, ref, mix = run_pair(lt, 360, 218, 30, 100, forced=1, cap_north=0)
    dt, ds = ocean_errors(syn, ref, mix)
    print("mixed vs fp64 after 100 steps: max |dT| = %.3e K, max |dS| = %.3e psu" % (dt, ds))
    assert dt <= T_TOL_K, dt
    assert ds <= S_TOL_PSU, ds
    assert mix.check_numeric() == 0


def test_mixed_error_bounds_deep_ocean(lt):
    """The same bounds on the 1-degree grid with the global ocean's
    area-depth curve: most columns wet through most of the 30 levels."""
    syn, ref, mix = run_pair(lt, 360, 218, 30, 100, forced=1, cap_north=0, hypsometry=1)
    dt, ds = ocean_errors(syn, ref, mix)
    print("deep ocean, mixed vs fp64 after 100 steps: max |dT| = %.3e K, max |dS| = %.3e psu" % (dt, ds))
    assert dt <= T_TOL_K, dt
    assert ds <= S_TOL_PSU, ds
    assert mix.check_numeric() == 0


def test_mixed_deterministic_deep_ocean(lt):
    """Three domains from the same inputs give the same bits.  Deep-ocean
    tiles start their march at a wet bottom level; a missing barrier between
    the first level's predictor and the next level's faces once made the
    limiter flags there, and so the results, differ from run to run."""
    syn = lt.Synth(720, 460, 55, forced=1, cap_north=0, umax=0.3, dz_top=5.0, dz_bot=300.0, hypsometry=1)
    states = []
    for _ in range(3):
        d = syn.domain(precision=lt.PREC_MIXED)
        d.step(2)
        states.append(d.get("AT").view(np.uint64).copy())
        d.close()
    for s in states[1:]:
        assert np.array_equal(states[0], s), int(np.sum(states[0] != s))


def test_mixed_small_grid_close(lt):
    syn, ref, mix = run_pair(lt, 64, 40, 20, 10, forced=1, cap_north=0)
    dt, ds = ocean_errors(syn, ref, mix)
    assert dt <= 1e-5 and ds <= 1e-6, (dt, ds)
    # WS is the small residual of nearly cancelling f32 divergence terms, so
    # its error is f32 rounding of the terms, not of WS itself: bound it by
    # 2^-20 of the vertically summed horizontal transport divergence scale.
    wr, wm = ref.get("WS"), mix.get("WS")
    utf = np.abs(syn.field("UTF")).max()
    dxu = syn.field("DXU")[2:-2, 2:-2].min()
    depth = syn.field("DZP").sum()
    scale = utf / dxu * depth
    err = np.abs(wr - wm).max()
    print("WS: max err %.3e, max |ws| %.3e, divergence scale %.3e" % (err, np.abs(wr).max(), scale))
    assert err <= 2.0 ** -20 * scale, (err, scale)
    # the freshwater norm is f64 surface arithmetic on a surface salinity that
    # differs between the forms by the state error (about 1e-9 psu here)
    assert abs(ref.fw_norm2() - mix.fw_norm2()) <= 1e-8 * abs(ref.fw_norm2()) + 1e-30


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_conservation_100_steps(lt, precision):
    """Zero surface flux on the 1-degree grid: the global tracer integrals
    (f64, fixed-order tree) drift by at most 1e-13 relative over 100 steps."""
    syn = lt.Synth(360, 218, 30, forced=0, cap_north=3, cap_south=3)
    dom = syn.domain(precision=lt.PREC_MIXED if precision == "mixed" else lt.PREC_FP64)
    c0 = np.array(dom.tracer_content())
    dom.step(100)
    c1 = np.array(dom.tracer_content())
    rel = np.abs(c1 - c0) / np.abs(c0)
    print("%s conservation drift after 100 steps: T %.3e, S %.3e" % (precision, rel[0], rel[1]))
    assert rel[0] < 1e-13 and rel[1] < 1e-13, rel


@pytest.mark.parametrize("nx", [49, 50, 51])
def test_mixed_any_row_pitch_vs_oracle(lt, nx):
    """Grids whose row pitch TMA cannot take (imt = nx + 4 not a multiple of
    4 floats) run the mixed step with per-thread copies of the same level
    boxes: within the bounds of the oracle after 20 steps."""
    import pyoracle
    syn = lt.Synth(nx, 30, 12, forced=1, cap_north=2, ew_cyclic=0, tripole=0)
    f = syn.all_fields()
    dom = lt.TracerDomain(nx, 30, 12, syn.params, precision=lt.PREC_MIXED, ew_cyclic=False, tripole=False)
    for n in lt.INPUT_FIELDS:
        dom.set(n, f[n])
    dom.step(20)
    o = pyoracle.Oracle(nx, 30, 12, syn.params, ew_cyclic=0, tripole=0)
    o.load(f)
    o.sum_order(1)
    o.step(20)
    kmt = f["KMT"]
    wet = (np.arange(12)[:, None, None] < kmt[None])[:, 2:-2, 2:-2]
    a, b = o.get("AT")[:, :, 2:-2, 2:-2], dom.get("AT")[:, :, 2:-2, 2:-2]
    dt = np.abs(a[0] - b[0])[wet].max()
    ds = np.abs(a[1] - b[1])[wet].max() * 1e3
    print("nx=%d mixed vs oracle after 20 steps: %.3e K, %.3e psu" % (nx, dt, ds))
    assert dt <= 1e-5 and ds <= 1e-6, (dt, ds)
    assert dom.check_numeric() == 0


def test_mixed_copy_path_equals_tma_path(lt):
    """On a grid TMA can take, the per-thread copy path fills the same level
    slots: both give the same bits."""
    syn = lt.Synth(124, 60, 24, forced=1, cap_north=0)
    a = syn.domain(precision=lt.PREC_MIXED)
    b = syn.domain(precision=lt.PREC_MIXED)
    b.use_tma(False)
    a.step(6)
    b.step(6)
    for n in ("AT", "ATB", "WS", "NET"):
        np.testing.assert_array_equal(a.get(n), b.get(n), err_msg=n)


def test_mixed_refuses_diagnostics(lt):
    """The diagnostic fields are the FP64 form's: a mixed domain asking for
    them is refused, not silently left without them."""
    syn = lt.Synth(64, 40, 12)
    with pytest.raises(lt.LtError):
        lt.TracerDomain(64, 40, 12, syn.params, precision=lt.PREC_MIXED, diagnostics=True)
