"""Failure detection without a GPU fault: host deadlines that run out on
legitimate work, and served requests dropped before admission.

The reference waits for the device with a 60 s poll deadline
(src/gpu.rs:484-490) and fails the call past it. Here the deadline is an
option (bt_options.wait_seconds); the tests make it expire on ordinary
iterations, never by a kernel that hangs, and check that the context stays
usable: a later wait with the default deadline completes the queued work,
whose results equal an undisturbed run.
"""
import numpy as np
import pytest

import bundling_thingy_b200 as bt
from bundling_thingy_b200 import synthetic

pytestmark = pytest.mark.gpu

TIMEOUT = 6
CANCELLED = 9


def options(w, **kw):
    o = bt.Options(width=w.width, height=w.height, neighbor_radius=w.radius, sample_spacing=w.spacing,
                   blur_sigma=w.sigma, blur_shrink=w.shrink)
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def test_expired_deadline_returns_timeout_and_the_context_recovers():
    w = synthetic.mid()
    ref = bt.Gpu(options(w))
    ref.upload((w.xy, w.starts))
    ref.iterate(30)
    want_xy, want_ids = ref.read_points()
    ref.close()

    g = bt.Gpu(options(w))
    g.upload((w.xy, w.starts))
    # Thirty iterations take milliseconds; a one-microsecond deadline runs
    # out while they are queued.
    g.set_wait_seconds(1e-6)
    with pytest.raises(bt.BtError) as err:
        g.iterate(30)
    assert err.value.status == TIMEOUT
    assert "device wait exceeded" in err.value.message
    # Back to the reference's deadline: the queued work completes and the
    # context is usable again.
    g.set_wait_seconds(0.0)
    g.synchronize()
    assert g.info().iterations == 30
    xy, ids = g.read_points()
    np.testing.assert_array_equal(ids, want_ids)
    np.testing.assert_array_equal(xy, want_xy)
    g.iterate(1)
    g.close()


def test_deadline_option_applies_from_creation():
    w = synthetic.small()
    g = bt.Gpu(options(w, wait_seconds=30.0))
    assert g.upload((w.xy, w.starts)) > 0
    g.iterate(2)
    g.close()
    with pytest.raises(bt.BtError) as err:
        bt.Gpu(options(w, wait_seconds=float("nan")))
    assert err.value.status == 3


def test_cancelled_queued_request_finishes_without_running():
    w = synthetic.small()
    server = bt.Server(0, max_active=4, budget_bytes=8 << 30)
    try:
        # Arrives ten seconds from now: still queued when it is cancelled.
        late = server.submit(options(w), w.xy, w.starts, 5, arrival_s=server.clock() + 10.0)
        now = server.submit(options(w), w.xy, w.starts, 2)
        server.cancel(late)
        got = {}
        for _ in range(2):
            r = server.next(30.0)
            got[r.id] = r
        assert got[late].status == CANCELLED, got[late].message
        assert got[late].device_bytes == 0 and got[late].iterations == 0
        assert got[now].status == 0, got[now].message
        with pytest.raises(bt.BtError):
            server.cancel(late)           # finished: nothing left to cancel
        server.release(late)
        server.release(now)
        assert server.stats()["failed"] == 1
    finally:
        server.close()


def test_request_past_the_admission_deadline_times_out():
    # One request at a time: the first holds the only slot for a few hundred
    # milliseconds, so the second waits in the queue past its deadline.
    mid, small = synthetic.mid(), synthetic.small()
    server = bt.Server(0, max_active=1, budget_bytes=8 << 30, queue_timeout_ms=40)
    try:
        first = server.submit(options(mid), mid.xy, mid.starts, 600)
        second = server.submit(options(small), small.xy, small.starts, 2)
        got = {}
        for _ in range(2):
            r = server.next(60.0)
            got[r.id] = r
        assert got[first].status == 0, got[first].message
        assert got[first].iterations == 600
        assert got[second].status == TIMEOUT
        assert "not admitted within 40 ms" in got[second].message
        assert got[second].finished_s - got[second].arrival_s >= 0.04
        for rid in got:
            server.release(rid)
    finally:
        server.close()
