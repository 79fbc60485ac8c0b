"""Checkpoint and resume: the 12-byte records read after k iterations,
restored into a fresh upload of the same graph, continue exactly as an
uninterrupted run (positions, neighbour counts and density), for the
neighbour mean with and without a shrinking sigma and for the advection mode.
"""
import numpy as np
import pytest

import bundling_thingy_b200 as bt
from bundling_thingy_b200 import synthetic

pytestmark = pytest.mark.gpu


def options(w, **kw):
    o = bt.Options(width=w.width, height=w.height, neighbor_radius=w.radius, sample_spacing=w.spacing,
                   blur_sigma=w.sigma, blur_shrink=w.shrink, record_neighbors=True)
    for k, v in kw.items():
        setattr(o, k, v)
    return o


CASES = [
    ("small, shrinking sigma", synthetic.small, {}),
    ("mid", synthetic.mid, {}),
    ("small, edge-id colouring", synthetic.small, {"color_by": bt.COLOR_BY_EDGE_ID}),
    ("small, advection", synthetic.small, {"neighbor_radius": None, "advect_step": 1.0, "advect_smooth": 0.5,
                                           "record_neighbors": False}),
]


@pytest.mark.parametrize("name,make,kw", CASES, ids=[c[0] for c in CASES])
def test_resume_from_a_checkpoint_matches_an_uninterrupted_run(name, make, kw):
    w = make()
    o = options(w, **kw)
    straight = bt.Gpu(o)
    straight.upload((w.xy, w.starts))
    straight.iterate(4)
    checkpoint = straight.read_records().copy()
    straight.iterate(3)
    want_xy, want_ids = straight.read_points()
    want_density = straight.read_density() if o.color_by == bt.COLOR_BY_DENSITY else None
    want_nb = straight.read_neighbors() if o.record_neighbors else None

    resumed = bt.Gpu(o)
    resumed.upload((w.xy, w.starts))
    resumed.restore_points(checkpoint, 4)
    assert resumed.info().iterations == 4
    xy, _ = resumed.read_points()
    np.testing.assert_array_equal(xy, checkpoint.view(np.uint32).reshape(-1, 3)[:, :2].copy().view(np.float32))
    resumed.iterate(3)
    got_xy, got_ids = resumed.read_points()
    np.testing.assert_array_equal(got_ids, want_ids)
    np.testing.assert_array_equal(got_xy, want_xy)
    if want_density is not None:
        np.testing.assert_array_equal(resumed.read_density(), want_density)
    if want_nb is not None:
        np.testing.assert_array_equal(resumed.read_neighbors(), want_nb)
    assert resumed.info().iterations == 7


def test_checkpoint_of_another_graph_is_refused():
    a, b = synthetic.small(), synthetic.small(seed_offset=3)
    g = bt.Gpu(options(a))
    n = g.upload((a.xy, a.starts))
    rec = g.read_records().copy()
    ids = rec.view(np.uint32).reshape(-1, 3)
    ids[n // 2, 2] += 1                       # an edge id that is not this graph's
    with pytest.raises(bt.BtError) as e:
        g.restore_points(rec, 1)
    assert e.value.status == 3 and "does not match" in e.value.message
    with pytest.raises(bt.BtError) as e:
        g.restore_points(rec[:-12], 1)        # wrong size
    assert e.value.status == 3
    g.iterate(1)                              # the context stays usable
    other = bt.Gpu(options(b))
    other.upload((b.xy, b.starts))
    with pytest.raises(bt.BtError):
        other.restore_points(g.read_records(), 1)
