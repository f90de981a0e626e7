"""C ABI checks that need no GPU: the library loads, exports every entry
point the public headers declare, reports field metadata consistent with the
oracle, and refuses device work cleanly when no device is visible."""
import ctypes as C
import os
import re

import numpy as np
from conftest import REPO

import pyoracle


def declared_functions():
    names = set()
    for h in sorted(f for f in os.listdir(os.path.join(REPO, "include")) if f.endswith(".h")):
        text = open(os.path.join(REPO, "include", h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_]*\s*\*?\s*([A-Za-z_][A-Za-z0-9_]*)\s*\(", text,
                             flags=re.M):
            names.add(m.group(1))
    return names


def test_library_exports_every_declared_symbol(lt):
    names = declared_functions()
    assert {"tracer_", "convadj_", "lt_create", "lt_step", "lt_synth_build"} <= names
    missing = [n for n in sorted(names) if not hasattr(lt.lib, n)]
    assert not missing, missing


def test_field_metadata_matches_oracle(lt):
    assert lt.FIELDS == pyoracle.FIELDS
    nx, ny, km = 20, 12, 7
    for name in lt.FIELDS:
        assert lt.field_shape(name, nx, ny, km) == pyoracle.shape_of(name, nx, ny, km), name
    assert lt.INT_FIELDS == pyoracle.INT


def test_synthetic_domain_is_deterministic(lt):
    a = lt.Synth(40, 24, 10, seed=5)
    b = lt.Synth(40, 24, 10, seed=5)
    c = lt.Synth(40, 24, 10, seed=6)
    for name in ("AT", "UTF", "AKT", "KMT", "TAREA"):
        assert np.array_equal(a.field(name), b.field(name)), name
    assert not np.array_equal(a.field("AT"), c.field("AT"))


def test_synthetic_domain_is_sane(lt):
    s = lt.Synth(72, 40, 15)
    kmt = s.field("KMT")[2:-2, 2:-2]
    land = (kmt == 0).mean()
    assert 0.2 < land < 0.5
    assert kmt.max() <= 15 and kmt[kmt > 0].min() >= 3
    at = s.field("AT")
    t = at[0][:, 2:-2, 2:-2][np.broadcast_to(np.arange(15)[:, None, None] < kmt[None], (15,) + kmt.shape)]
    assert 1.0 < t.min() and t.max() < 29.0
    dzp = lt.Synth(40, 24, 30).field("DZP")   # 30 levels stretched 10 m .. 250 m to 5000 m
    assert abs(dzp.sum() - 5000.0) < 1e-6 and abs(dzp[0] - 10.0) < 1e-9 and abs(dzp[-1] - 250.0) < 1e-9
    u = s.field("UTL")
    assert 0.05 < np.abs(u).max() < 0.2


def test_no_device_is_a_status_not_a_crash(lt):
    if lt.device_count() > 0:
        return
    g = lt.Grid(16, 12, 5, 0, 0, 1, 1)
    p = lt.Synth(16, 12, 5).params
    h = C.c_void_p()
    rc = lt.lib.lt_create(C.byref(g), C.byref(p), C.byref(h))
    assert rc == lt.LT_E_NODEVICE
    assert b"device" in lt.lib.lt_last_error()


def test_domain_bytes_admission(lt):
    g = lt.Grid(3600, 2302, 55, 0, 0, 1, 1)
    nbytes = lt.lib.lt_domain_bytes(C.byref(g))
    fld = 3604 * 2306 * 55 * 8
    # FP64 working set of the 0.1-degree grid: ~24 3-D fields, under 180 GB
    assert 18 * fld < nbytes < 30 * fld
    assert nbytes < 180e9
    bad = lt.Grid(3601, 2302, 55, 0, 0, 1, 1)  # tripole needs even nx
    assert lt.lib.lt_domain_bytes(C.byref(bad)) == 0


def test_advection_scheme_checked_before_device_work(lt):
    """The scheme is validated on the host (no device needed): an unknown
    scheme, and the centred / flux schemes in mixed precision, are
    LT_E_INVALID with a message."""
    syn = lt.Synth(16, 12, 5)
    h = C.c_void_p()
    for prec, adv, ok in ((lt.PREC_MIXED, lt.ADV_CENTERED, False), (lt.PREC_MIXED, lt.ADV_FLUX, False),
                          (lt.PREC_FP64, 3, False), (lt.PREC_FP64, -1, False)):
        p = type(syn.params).from_buffer_copy(syn.params)
        p.adv_tracer = adv
        g = lt.Grid(16, 12, 5, prec, 0, 1, 1)
        rc = lt.lib.lt_create(C.byref(g), C.byref(p), C.byref(h))
        assert rc == lt.LT_E_INVALID, (prec, adv)
        assert b"adv" in lt.lib.lt_last_error() or b"FP64 form only" in lt.lib.lt_last_error()


def test_nudging_checked_before_device_work(lt):
    """tracer_7's nudging (simple_assm) runs in the FP64 form only, with a
    flag of 0 or 1 and ktv >= 0: anything else is LT_E_INVALID from
    lt_create, before any device work."""
    syn = lt.Synth(16, 12, 5)
    h = C.c_void_p()
    for prec, sa, ktv in ((lt.PREC_MIXED, 1, 5), (lt.PREC_FP64, 2, 5), (lt.PREC_FP64, 1, -1)):
        p = type(syn.params).from_buffer_copy(syn.params)
        p.simple_assm, p.ktv = sa, ktv
        g = lt.Grid(16, 12, 5, prec, 0, 1, 1)
        rc = lt.lib.lt_create(C.byref(g), C.byref(p), C.byref(h))
        assert rc == lt.LT_E_INVALID, (prec, sa, ktv)
        assert b"simple_assm" in lt.lib.lt_last_error() or b"ktv" in lt.lib.lt_last_error()
