"""Serving: requests arriving over time, admitted by a memory budget and
advanced together in one batch, give the same results as each graph run
alone, bit for bit.
"""
import numpy as np
import pytest

import bundling_thingy_b200 as bt
from bundling_thingy_b200 import synthetic

from conftest import oracle_config

pytestmark = pytest.mark.gpu


def options(w, **kw):
    o = bt.Options(width=w.width, height=w.height, neighbor_radius=w.radius, sample_spacing=w.spacing,
                   blur_sigma=w.sigma, blur_shrink=w.shrink)
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def standalone(w, o, iterations):
    g = bt.Gpu(o)
    g.upload((w.xy, w.starts))
    if iterations:
        g.iterate(iterations)
    xy, ids = g.read_points()
    dens = g.read_density() if o.color_by == bt.COLOR_BY_DENSITY else None
    bytes_ = g.info().device_bytes
    g.close()
    return xy, ids, dens, bytes_


def mixed_requests():
    small, mid = synthetic.small(), synthetic.mid()
    small2 = synthetic.small(seed_offset=11)
    return [
        (small, options(small), 5),                                          # shrinking sigma
        (mid, options(mid), 3),
        (small2, bt.Options(neighbor_radius=4), 4),                         # reference settings, 1600^2
        (small2, options(small2, color_by=bt.COLOR_BY_EDGE_ID), 2),          # no density passes
        (small, options(small, width=512, height=512, neighbor_radius=1, blur_sigma=3.0, blur_shrink=1.0), 6),
        (mid, options(mid), 0),                                              # upload only
    ]


def drain(server, n, expected, timeout=60.0):
    """Collect n results, check each against its standalone run, release."""
    seen = {}
    for _ in range(n):
        r = server.next(timeout)
        assert r.status == 0, r.message
        w, o, iters = expected[r.id]
        assert r.iterations == iters
        xy, ids = server.read_points(r.id, r.samples)
        sxy, sids, sdens, _ = standalone(w, o, iters)
        np.testing.assert_array_equal(ids, sids)
        np.testing.assert_array_equal(xy, sxy)
        if sdens is not None:
            np.testing.assert_array_equal(server.result(r.id).read_density(), sdens)
        assert r.finished_s >= r.admitted_s >= r.arrival_s
        server.release(r.id)
        seen[r.id] = r
    return seen


@pytest.mark.parametrize("solo_samples", [0, 1, 2**32 - 1])
def test_requests_in_the_mix_match_standalone_runs(solo_samples):
    # Default threshold (the larger requests iterate on their own contexts),
    # every request on its own, every request in the batch.
    server = bt.Server(max_active=8, solo_samples=solo_samples)
    t0 = server.clock() + 0.01
    expected = {}
    for i, (w, o, iters) in enumerate(mixed_requests()):
        # Four arrive together, two join while the first ones iterate.
        rid = server.submit(o, w.xy, w.starts, iters, arrival_s=t0 + 0.003 * max(0, i - 3))
        expected[rid] = (w, o, iters)
    seen = drain(server, len(expected), expected)
    assert set(seen) == set(expected)
    st = server.stats()
    assert st["finished"] == len(expected) and st["failed"] == 0
    assert st["peak_active"] >= 4          # graphs overlapped on the device
    # A second wave reuses the idle contexts of the first.
    expected2 = {}
    for w, o, iters in mixed_requests()[:3]:
        expected2[server.submit(o, w.xy, w.starts, iters)] = (w, o, iters)
    drain(server, len(expected2), expected2)
    server.close()


@pytest.mark.parametrize("solo_samples", [1, 2**32 - 1])
def test_served_results_match_oracle(oracle, solo_samples):
    # Every request of the mix against the oracle's own run of its graph, with
    # all requests on their own contexts (1) or all in the batch (2^32 - 1).
    server = bt.Server(max_active=8, solo_samples=solo_samples)
    expected = {}
    for w, o, iters in mixed_requests()[:5]:
        expected[server.submit(o, w.xy, w.starts, iters)] = (w, o, iters)
    for _ in range(len(expected)):
        r = server.next(60.0)
        assert r.status == 0, r.message
        w, o, iters = expected[r.id]
        ora = oracle.Pipeline(oracle_config(oracle, o))
        assert ora.upload(w.xy, w.starts) == r.samples
        if iters:
            ora.iterate(iters)
        xy, ids = server.read_points(r.id, r.samples)
        oxy, oids = ora.points()
        np.testing.assert_array_equal(ids, oids)
        np.testing.assert_array_equal(xy, oxy)
        if o.color_by == bt.COLOR_BY_DENSITY:
            np.testing.assert_array_equal(server.result(r.id).read_density(), ora.normalized())
        server.release(r.id)
    server.close()


def test_budget_defers_admission_and_results_stay_exact():
    mid = synthetic.mid()
    o = options(mid)
    one = standalone(mid, o, 0)[3] + 12 * bt_samples(mid, o) + (1 << 20)
    budget = int(one * 1.5)               # room for one such graph at a time
    server = bt.Server(max_active=8, budget_bytes=budget)
    expected = {}
    t0 = server.clock() + 0.05              # all three become ready together
    for iters in (3, 2, 4):
        expected[server.submit(o, mid.xy, mid.starts, iters, arrival_s=t0)] = (mid, o, iters)
    drain(server, len(expected), expected)
    st = server.stats()
    assert st["peak_device_bytes"] <= budget
    assert st["budget_waits"] > 0
    server.close()


def bt_samples(w, o):
    g = bt.Gpu(o)
    n = g.upload((w.xy, w.starts))
    g.close()
    return n


def test_request_larger_than_the_budget_fails_alone():
    small = synthetic.small()
    server = bt.Server(budget_bytes=32 << 20)   # a 2048^2 map alone needs 80 MB
    big = server.submit(options(small, width=2048, height=2048), small.xy, small.starts, 2)
    r = server.next(30.0)
    assert r.id == big and r.status == 5, r.message
    server.release(big)
    ok = server.submit(options(small, width=256, height=256, neighbor_radius=2, blur_sigma=2.0, blur_shrink=1.0),
                       small.xy, small.starts, 2)
    r = server.next(30.0)
    assert r.id == ok and r.status == 0, r.message
    server.release(ok)
    server.close()


def test_invalid_request_fails_without_stopping_the_server():
    small = synthetic.small()
    bad = small.starts.copy()
    bad[-1] = small.xy.shape[0] + 3
    server = bt.Server()
    o = options(small)
    b = server.submit(o, small.xy, bad, 2)
    g = server.submit(o, small.xy, small.starts, 2)
    results = {r.id: r for r in (server.next(30.0), server.next(30.0))}
    assert results[b].status == 3
    assert results[g].status == 0
    sxy, sids, _, _ = standalone(small, o, 2)
    xy, ids = server.read_points(g, results[g].samples)
    np.testing.assert_array_equal(xy, sxy)
    for rid in results:
        server.release(rid)
    with pytest.raises(bt.BtError):
        server.release(g)                  # already released
    with pytest.raises(bt.BtError):
        server.next(0.05)                  # nothing left
    server.close()


def test_served_result_renders_like_a_standalone_run():
    # A finished request's context can be drawn (bt_render) before release.
    w = synthetic.small()
    o = options(w, endpoint_dots=True, palette=2)
    server = bt.Server(max_active=4)
    rid = server.submit(o, w.xy, w.starts, 3)
    r = server.next(60.0)
    assert r.status == 0 and r.id == rid, r.message
    frame = server.result(rid).render()
    g = bt.Gpu(o)
    g.upload((w.xy, w.starts))
    g.iterate(3)
    ref = g.render()
    g.close()
    assert frame.colored_pixels == ref.colored_pixels > 0
    np.testing.assert_array_equal(frame.rgba, ref.rgba)
    server.release(rid)
    server.close()
