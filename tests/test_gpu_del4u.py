"""GPU parity of the momentum biharmonic friction (lt_hdiffu_del4, one fused
kernel for readyc_'s six-kernel BIHAR sequence) against the CPU oracle, which
test_del4u_pin pins bit for bit to the reference's readyc.cpp.  FP64 with the
reference's operation order and only sqrt among the functions: bit for bit."""
import numpy as np
import pytest
from del4u_case import C0F, case

import pyoracle

pytestmark = pytest.mark.gpu

OUT = ["DLU", "DLV", "WKA_DRAG"]


def check(lt, syn, f, am, precision=None):
    prec = lt.PREC_FP64 if precision is None else precision
    dom = lt.TracerDomain(syn.nx, syn.ny, syn.km, syn.params, precision=prec,
                          ew_cyclic=bool(syn.cfg.ew_cyclic), tripole=bool(syn.cfg.tripole))
    for n in lt.INPUT_FIELDS + lt.MOM_FIELDS:
        dom.set(n, f[n])
    dom.hdiffu_del4(am, C0F)
    dom.sync()
    o = pyoracle.Oracle(syn.nx, syn.ny, syn.km, syn.params, ew_cyclic=syn.cfg.ew_cyclic, tripole=syn.cfg.tripole)
    o.load(f)
    o.hdiffu_del4(am, C0F)
    for n in OUT:
        g, r = dom.get(n), o.get(n)
        bad = np.argwhere(g.view(np.uint64) != r.view(np.uint64))
        assert bad.size == 0, "%s: %d cells differ, first %s (gpu %r oracle %r)" % (
            n, len(bad), bad[0], g[tuple(bad[0])], r[tuple(bad[0])])
    assert np.abs(dom.get("DLU") - f["DLU"]).max() > 0


@pytest.mark.parametrize("seed,cap_north", [(4, 0), (9, 1), (17, 0)])
def test_del4u_bitexact_reference_size(lt, seed, cap_north):
    check(lt, *case(lt, seed, cap_north))


def test_del4u_ragged_tiles_mixed_domain(lt):
    """Sizes that are not multiples of the 32x8 tile; the friction does not
    depend on the domain's precision form."""
    check(lt, *case(lt, 5, 0, nx=52, ny=27, km=13), precision=lt.PREC_MIXED)


def test_del4u_one_degree(lt):
    check(lt, *case(lt, 6, 0, nx=360, ny=218, km=30, dz_top=10.0, dz_bot=250.0))
