"""Request server (include/licom_serve.h): requests of different sizes and
step counts arrive over time, are admitted by free HBM, run resident and
batched together, and leave when done.  Each result must be the same as the
same request run alone (stated tolerance: bit for bit, since the batched
kernels compute every member exactly as a lone domain)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CLOSED = dict(ew_cyclic=0, tripole=0, forced=1)
REQS = [  # nx, ny, km, steps, arrival (s), seed
    (64, 48, 30, 7, 0.00, 1),
    (128, 96, 30, 13, 0.00, 2),
    (96, 64, 30, 4, 0.02, 3),
    (160, 128, 55, 9, 0.05, 4),
    (72, 52, 30, 11, 0.10, 5),
    (200, 120, 30, 6, 0.10, 6),
]


def run_alone(lt, nx, ny, km, steps, seed):
    syn = lt.Synth(nx, ny, km, seed=seed, **CLOSED)
    d = syn.domain(precision=lt.PREC_MIXED)
    d.step(steps)
    d.sync()
    return d.get("AT"), d.tracer_content()


def test_results_same_alone_and_in_the_mix(lt):
    srv = lt.Server(precision=lt.PREC_MIXED, chunk_steps=3)
    t0 = srv.clock()
    ids = [srv.submit(nx, ny, km, steps, arrival=t0 + arr, keep_state=True, seed=seed, **CLOSED)
           for nx, ny, km, steps, arr, seed in REQS]
    srv.drain()
    st = srv.stats()
    print("serving stats:", st)
    assert st["requests_done"] == len(REQS) and st["requests_refused"] == 0
    assert st["max_resident"] >= 2          # work overlapped on the device
    for rid, (nx, ny, km, steps, arr, seed) in zip(ids, REQS):
        s = srv.status(rid)
        assert s["state"] == "done" and s["steps_done"] == steps
        assert s["finished"] >= s["admitted"] >= s["arrival"] >= t0 + arr - 1e-9
        at_alone, content_alone = run_alone(lt, nx, ny, km, steps, seed)
        np.testing.assert_array_equal(srv.state(rid), at_alone)
        assert tuple(s["content"]) == tuple(content_alone)
    srv.close()


def test_unrounded_sizes_same_alone_and_in_the_mix(lt):
    """Requests of any size (row pitches TMA cannot take among them) are
    served and give the same result as alone."""
    reqs = [(101, 77, 30, 5, 0.0, 31), (64, 48, 30, 6, 0.0, 32), (150, 90, 55, 4, 0.01, 33), (57, 61, 30, 7, 0.0, 34)]
    srv = lt.Server(precision=lt.PREC_MIXED, chunk_steps=3)
    t0 = srv.clock()
    ids = [srv.submit(nx, ny, km, steps, arrival=t0 + arr, keep_state=True, seed=seed, **CLOSED)
           for nx, ny, km, steps, arr, seed in reqs]
    srv.drain()
    assert srv.stats()["requests_done"] == len(reqs)
    for rid, (nx, ny, km, steps, arr, seed) in zip(ids, reqs):
        at_alone, content_alone = run_alone(lt, nx, ny, km, steps, seed)
        np.testing.assert_array_equal(srv.state(rid), at_alone)
        assert tuple(srv.status(rid)["content"]) == tuple(content_alone)
    srv.close()


def test_admission_waits_for_memory(lt):
    """A budget that holds two of these requests at a time: never more than
    two resident, and every request still finishes."""
    import ctypes
    g = lt.Grid(128, 96, 30, lt.PREC_MIXED, 0, 0, 0)
    one = lt.lib.lt_domain_bytes(ctypes.byref(g))
    srv = lt.Server(precision=lt.PREC_MIXED, hbm_budget=int(2.5 * one), chunk_steps=4)
    ids = [srv.submit(128, 96, 30, 5 + i, seed=10 + i, **CLOSED) for i in range(5)]
    srv.drain()
    st = srv.stats()
    assert st["requests_done"] == 5
    assert st["max_resident"] == 2
    assert st["peak_bytes"] <= int(2.5 * one)
    adm = sorted(srv.status(r)["admitted"] for r in ids)
    assert adm[2] > adm[1]                   # the third waited for memory
    srv.close()


def test_oversized_request_is_refused(lt):
    import ctypes
    g = lt.Grid(96, 64, 30, lt.PREC_MIXED, 0, 0, 0)
    one = lt.lib.lt_domain_bytes(ctypes.byref(g))
    srv = lt.Server(precision=lt.PREC_MIXED, hbm_budget=one + 1024)
    small = srv.submit(96, 64, 30, 3, seed=1, **CLOSED)
    big = srv.submit(400, 300, 55, 3, seed=2, **CLOSED)
    srv.drain()
    assert srv.status(small)["state"] == "done"
    assert srv.status(big)["state"] == "refused"
    assert srv.stats()["requests_refused"] == 1
    srv.close()
