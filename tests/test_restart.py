"""The reference's restart file (include/licom_restart.h; written by
ssave-cdf-instant.F90:93-761, read by inirun.F90:598-679): Fortran
unformatted sequential records of global f64 fields.  The library's writer
is checked byte by byte against an independent numpy reading of the format,
its reader against an independent numpy writer, and both against each other;
malformed files are refused with a status, not a crash."""
import os

import numpy as np
import pytest

NX, NY, KM = 24, 16, 5


def fields(seed=0):
    rng = np.random.default_rng(seed)
    a = {n: rng.standard_normal((NY, NX)) for n in ("h0", "su", "sv", "swv", "sshf", "lthf", "fresh")}
    a.update({n: rng.standard_normal((KM, NY, NX)) for n in ("u", "v", "t", "s", "ws")})
    return a


ORDER = [("h0", None)] + [(n, k) for n in ("u", "v", "t", "s", "ws") for k in range(KM)] + \
        [(n, None) for n in ("su", "sv", "swv", "sshf", "lthf", "fresh")]


def numpy_records(path):
    raw = open(path, "rb").read()
    out, p = [], 0
    while p < len(raw):
        n = int(np.frombuffer(raw, "<i4", 1, p)[0])
        out.append(raw[p + 4:p + 4 + n])
        assert int(np.frombuffer(raw, "<i4", 1, p + 4 + n)[0]) == n
        p += 8 + n
    return out


def numpy_write(path, a, month, day):
    with open(path, "wb") as f:
        def rec(b):
            f.write(np.int32(len(b)).tobytes())
            f.write(b)
            f.write(np.int32(len(b)).tobytes())
        for n, k in ORDER:
            rec(np.ascontiguousarray(a[n] if k is None else a[n][k]).tobytes())
        rec(np.array([month, day], dtype="<i4").tobytes())


def test_writer_layout(lt, tmp_path):
    a = fields(1)
    p = str(tmp_path / "fort.22.0001-01-01")
    lt.restart_write(p, NX, NY, KM, a, month=7, day=15)
    recs = numpy_records(p)
    assert len(recs) == len(ORDER) + 1
    for (n, k), r in zip(ORDER, recs):
        want = a[n] if k is None else a[n][k]
        assert r == np.ascontiguousarray(want).tobytes(), (n, k)
    assert np.frombuffer(recs[-1], "<i4").tolist() == [7, 15]


def test_reader_takes_an_independent_file(lt, tmp_path):
    a = fields(2)
    p = str(tmp_path / "restart")
    numpy_write(p, a, 123, 4)
    b, month, day = lt.restart_read(p, NX, NY, KM)
    assert (month, day) == (123, 4)
    for n in a:
        assert np.array_equal(a[n], b[n]), n


def test_missing_fields_are_zeros(lt, tmp_path):
    a = fields(3)
    part = {n: a[n] for n in ("h0", "t", "s")}
    p = str(tmp_path / "partial")
    lt.restart_write(p, NX, NY, KM, part)
    b, _, _ = lt.restart_read(p, NX, NY, KM)
    for n in ("h0", "t", "s"):
        assert np.array_equal(b[n], a[n])
    for n in ("u", "v", "ws", "su", "sv", "swv", "sshf", "lthf", "fresh"):
        assert not b[n].any(), n


def test_malformed_files_are_refused(lt, tmp_path):
    a = fields(4)
    p = str(tmp_path / "r")
    lt.restart_write(p, NX, NY, KM, a)
    with pytest.raises(lt.LtError) as e:
        lt.restart_read(p, NX + 1, NY, KM)          # other grid
    assert e.value.code == lt.LT_E_INVALID
    raw = open(p, "rb").read()
    q = str(tmp_path / "cut")
    open(q, "wb").write(raw[:len(raw) // 2])
    with pytest.raises(lt.LtError) as e:
        lt.restart_read(q, NX, NY, KM)              # truncated
    assert e.value.code == lt.LT_E_STATE
    with pytest.raises(lt.LtError):
        lt.restart_read(str(tmp_path / "absent"), NX, NY, KM)
