"""lt_tracer_content_noalloc, the content sum for callers that may not let a
library allocate device memory (a host model that owns all of HBM through its
own pool or OpenACC/OpenMP data regions), keeps its partial sums in a fixed
2 MiB array inside the library.  Checked here against lt_tracer_content on the
same state: both use the same fixed-order tree, so they must agree bit for
bit, on two calls in a row that see different states (the second call reuses
the array the first one left behind).  This file is collected last."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _bind(lib):
    f = lib.lt_tracer_content_noalloc
    f.argtypes = [C.c_void_p] * 4 + [C.c_int] * 3 + [C.c_void_p, C.c_void_p]
    f.restype = C.c_int
    return f


def _device_copy(torch, lt, dom, name, dtype):
    buf = torch.empty(tuple(dom.shape(name)), dtype=dtype, device="cuda")
    nbytes = buf.numel() * buf.element_size()
    rc = lt.lib.lt_get_field_device(dom.h, lt.FIELD_ID[name], C.c_void_p(buf.data_ptr()), nbytes)
    assert rc == 0, lt.lib.lt_last_error()
    return buf


def test_noalloc_content_matches_existing_entry_point(lt):
    torch = pytest.importorskip("torch")
    fn = _bind(lt.lib)
    nx, ny, km = 96, 64, 24
    syn = lt.Synth(nx, ny, km, forced=1)
    dom = syn.domain()
    tarea = _device_copy(torch, lt, dom, "TAREA", torch.float64)
    dzp = _device_copy(torch, lt, dom, "DZP", torch.float64)
    kmt = _device_copy(torch, lt, dom, "KMT", torch.int32)
    out = torch.full((2,), float("nan"), dtype=torch.float64, device="cuda")

    for call, steps in enumerate((3, 2)):
        dom.step(steps)
        want = np.array(dom.tracer_content())
        at = _device_copy(torch, lt, dom, "AT", torch.float64)
        dom.sync()
        rc = fn(C.c_void_p(at.data_ptr()), C.c_void_p(tarea.data_ptr()), C.c_void_p(dzp.data_ptr()),
                C.c_void_p(kmt.data_ptr()), nx, ny, km, C.c_void_p(out.data_ptr()), None)
        assert rc == 0, lt.lib.lt_last_error()
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        print("call %d: noalloc %r, lt_tracer_content %r" % (call + 1, got.tolist(), want.tolist()))
        assert np.all(np.isfinite(got))
        np.testing.assert_array_equal(got, want)


def test_noalloc_three_tree_levels(lt):
    """256 x 192 x 96 cells: 2304 first-pass blocks, so the partial sums go
    through two more tree passes; still bit for bit lt_tracer_content's."""
    torch = pytest.importorskip("torch")
    fn = _bind(lt.lib)
    nx, ny, km = 256, 192, 96
    syn = lt.Synth(nx, ny, km, forced=1)
    dom = syn.domain()
    dom.step(1)
    want = np.array(dom.tracer_content())
    bufs = {n: _device_copy(torch, lt, dom, n, t) for n, t in
            (("AT", torch.float64), ("TAREA", torch.float64), ("DZP", torch.float64), ("KMT", torch.int32))}
    out = torch.full((2,), float("nan"), dtype=torch.float64, device="cuda")
    dom.sync()
    rc = fn(*[C.c_void_p(bufs[n].data_ptr()) for n in ("AT", "TAREA", "DZP", "KMT")], nx, ny, km,
            C.c_void_p(out.data_ptr()), None)
    assert rc == 0, lt.lib.lt_last_error()
    torch.cuda.synchronize()
    np.testing.assert_array_equal(out.cpu().numpy(), want)


# 2048 x 262011 cells need exactly 2^18 partial sums (262011 first-pass blocks,
# 128 and 1 in the next passes, 4 spare): the largest grid the scratch takes
AT_CAPACITY = (2048, 262011, 1)


def test_noalloc_rejects_sizes_beyond_scratch(lt):
    torch = pytest.importorskip("torch")
    fn = _bind(lt.lib)
    tiny = torch.zeros(16, dtype=torch.float64, device="cuda")
    p = C.c_void_p(tiny.data_ptr())
    # one cell more than the capacity: 262012 first-pass blocks, 2^18 + 1
    # values.  The size check comes before any device work.
    rc = fn(p, p, p, p, 2048 * 262011 + 1, 1, 1, p, None)
    assert rc == lt.LT_E_INVALID
    msg = lt.lib.lt_last_error().decode()
    assert "scratch" in msg, msg
    rc = fn(p, p, p, p, 20000, 20000, 10, p, None)
    assert rc == lt.LT_E_INVALID


def test_noalloc_at_capacity(lt):
    """Exactly at the capacity the sum runs: T = S = 1, tarea = 1, one level
    of thickness 2, every column wet, so each tracer's content is
    2 * nx * ny, exact in f64 whatever the order of the sum."""
    torch = pytest.importorskip("torch")
    fn = _bind(lt.lib)
    nx, ny, km = AT_CAPACITY
    imt, jmt = nx + 4, ny + 4
    at = torch.ones(2 * km * jmt * imt, dtype=torch.float64, device="cuda")
    tarea = torch.ones(jmt * imt, dtype=torch.float64, device="cuda")
    dzp = torch.full((km,), 2.0, dtype=torch.float64, device="cuda")
    kmt = torch.ones(jmt * imt, dtype=torch.int32, device="cuda")
    out = torch.full((2,), float("nan"), dtype=torch.float64, device="cuda")
    for _ in range(2):
        rc = fn(C.c_void_p(at.data_ptr()), C.c_void_p(tarea.data_ptr()), C.c_void_p(dzp.data_ptr()),
                C.c_void_p(kmt.data_ptr()), nx, ny, km, C.c_void_p(out.data_ptr()), None)
        assert rc == 0, lt.lib.lt_last_error()
        torch.cuda.synchronize()
        assert out.cpu().numpy().tolist() == [2.0 * nx * ny] * 2
        out.fill_(float("nan"))
    del at, tarea, kmt
    torch.cuda.empty_cache()
