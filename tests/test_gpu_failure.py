"""Failure detection on the device without a fault.

The TMA-fed column kernels bound every wait for their level data.  Setting
the bound to zero polls makes every wait give up at once: each CTA records
the timeout, drains the boxes it already issued and returns.  The host must
see LT_E_TIMEOUT at the next synchronising call, and the context must stay
usable: a fresh domain then steps exactly like an untouched twin.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_wait_timeout_is_reported_and_context_survives(lt, precision):
    prec = lt.PREC_MIXED if precision == "mixed" else lt.PREC_FP64
    syn = lt.Synth(64, 40, 20)
    bad = syn.domain(precision=prec)
    bad.set_wait_limit(0)
    bad.step(1)
    with pytest.raises(lt.LtError) as err:
        bad.sync()
    assert err.value.code == lt.LT_E_TIMEOUT
    # reported once: the next synchronising call is clean
    bad.sync()

    a = syn.domain(precision=prec)
    b = syn.domain(precision=prec)
    a.step(2)
    b.step(2)
    a.sync()
    b.sync()
    np.testing.assert_array_equal(a.get("AT"), b.get("AT"))
    assert a.check_numeric() == 0

    # the domain that timed out steps normally again once the bound is restored
    bad.set_wait_limit(1 << 24)
    bad.step(1)
    bad.sync()
