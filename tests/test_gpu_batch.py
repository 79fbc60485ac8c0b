"""Batches: every slot's results equal a standalone run of the same graph.

The batch advances all of its graphs with persistent launches over a
graph x tile work queue; a graph's results must not depend on what else is
in the batch (alone vs in the mix), bit for bit.
"""
import numpy as np
import pytest

import bundling_thingy_b200 as bt
from bundling_thingy_b200 import synthetic

from conftest import oracle_config

pytestmark = pytest.mark.gpu


def workload_options(w, **kw):
    o = bt.Options(width=w.width, height=w.height, neighbor_radius=w.radius, sample_spacing=w.spacing,
                   blur_sigma=w.sigma, blur_shrink=w.shrink)
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def mixed_jobs():
    small, mid = synthetic.small(), synthetic.mid()
    small2 = synthetic.small(seed_offset=11)
    return [
        (small, workload_options(small)),                                   # shrinking sigma
        (mid, workload_options(mid)),
        (small2, bt.Options(neighbor_radius=4)),                            # reference settings, 1600^2
        (small2, workload_options(small2, color_by=bt.COLOR_BY_EDGE_ID)),   # no density passes
        (small, workload_options(small, width=512, height=512, neighbor_radius=1, blur_sigma=3.0,
                                 blur_shrink=1.0, search_mode=1)),
        # 8M flat search cells: the per-slot scan of the cell-table tile sums
        # runs over more than one tile.
        (small2, workload_options(small2, width=2048, height=2048, neighbor_radius=4, blur_sigma=4.0,
                                  blur_shrink=1.0, fine_cells=4, fine_cells_x=8)),
    ]


# Every slot in the persistent step (the default, the engine under test), or
# every slot on its own context.
PERSISTENT = 2**32 - 1
POLICIES = [PERSISTENT, 1]


def standalone(w, o, iterations):
    g = bt.Gpu(o)
    g.upload((w.xy, w.starts))
    if iterations:
        g.iterate(iterations)
    xy, ids = g.read_points()
    dens = g.read_density() if o.color_by == bt.COLOR_BY_DENSITY else None
    g.close()
    return xy, ids, dens


def check_slot(batch, slot, expected):
    view = batch.slot(slot)
    xy, ids = view.read_points()
    np.testing.assert_array_equal(ids, expected[1])
    np.testing.assert_array_equal(xy, expected[0])
    if expected[2] is not None:
        np.testing.assert_array_equal(view.read_density(), expected[2])


@pytest.mark.parametrize("solo_samples", POLICIES)
def test_mixed_batch_matches_standalone_runs(solo_samples):
    jobs = mixed_jobs()
    batch = bt.Batch(solo_samples=solo_samples)
    slots = [batch.add(o, w.xy, w.starts)[0] for w, o in jobs]
    assert batch.active() == len(jobs)
    batch.iterate(3)
    for (w, o), slot in zip(jobs, slots):
        check_slot(batch, slot, standalone(w, o, 3))
    batch.iterate(2)
    for (w, o), slot in zip(jobs, slots):
        check_slot(batch, slot, standalone(w, o, 5))
    info = batch.slot(slots[0]).info()
    assert info.iterations == 5


def test_first_slot_matches_oracle(oracle):
    w = synthetic.small()
    o = workload_options(w)
    batch = bt.Batch(solo_samples=PERSISTENT)
    slot, n = batch.add(o, w.xy, w.starts)
    batch.add(*(lambda m: (workload_options(m), m.xy, m.starts))(synthetic.mid()))
    batch.iterate(4)
    ora = oracle.Pipeline(oracle_config(oracle, o))
    assert ora.upload(w.xy, w.starts) == n
    ora.iterate(4)
    xy, ids = batch.slot(slot).read_points()
    oxy, oids = ora.points()
    np.testing.assert_array_equal(ids, oids)
    np.testing.assert_array_equal(xy, oxy)
    np.testing.assert_array_equal(batch.slot(slot).read_density(), ora.normalized())


def test_every_mixed_slot_matches_oracle(oracle):
    # Each slot of the mixed batch in the persistent step against the oracle's
    # own run of its graph: maps of 512^2 to 2048^2, radii 1 to 8, both search
    # modes, density on and off, shrinking and constant sigma.
    jobs = mixed_jobs()
    batch = bt.Batch(solo_samples=PERSISTENT)
    slots = [batch.add(o, w.xy, w.starts) for w, o in jobs]
    batch.iterate(3)
    for (w, o), (slot, n) in zip(jobs, slots):
        ora = oracle.Pipeline(oracle_config(oracle, o))
        assert ora.upload(w.xy, w.starts) == n
        ora.iterate(3)
        xy, ids = batch.slot(slot).read_points()
        oxy, oids = ora.points()
        np.testing.assert_array_equal(ids, oids)
        np.testing.assert_array_equal(xy, oxy)
        if o.color_by == bt.COLOR_BY_DENSITY:
            np.testing.assert_array_equal(batch.slot(slot).read_density(), ora.normalized())


@pytest.mark.parametrize("solo_samples", POLICIES + [200000])
def test_slots_join_and_leave_between_iterations(solo_samples):
    # 200000: the small graphs in the persistent step, the mid one on its own.
    jobs = mixed_jobs()
    batch = bt.Batch(solo_samples=solo_samples)
    a = batch.add(jobs[0][1], jobs[0][0].xy, jobs[0][0].starts)[0]
    b = batch.add(jobs[1][1], jobs[1][0].xy, jobs[1][0].starts)[0]
    batch.iterate(1)                       # a, b at parity 1
    c = batch.add(jobs[2][1], jobs[2][0].xy, jobs[2][0].starts)[0]
    batch.iterate(2)                       # a, b: 3 iterations; c: 2
    batch.remove(a)
    d = batch.add(jobs[4][1], jobs[4][0].xy, jobs[4][0].starts)[0]
    assert d == a                          # the freed slot is reused
    batch.iterate(1)                       # b: 4, c: 3, d: 1
    check_slot(batch, b, standalone(*jobs[1], 4))
    check_slot(batch, c, standalone(*jobs[2], 3))
    check_slot(batch, d, standalone(*jobs[4], 1))


def test_long_shrinking_sigma_run_extends_taps():
    w = synthetic.small()
    o = workload_options(w)
    batch = bt.Batch(solo_samples=PERSISTENT)
    slot = batch.add(o, w.xy, w.starts)[0]
    batch.iterate(70)                      # beyond the precomputed taps horizon
    check_slot(batch, slot, standalone(w, o, 70))


def test_batch_errors():
    batch = bt.Batch()
    w = synthetic.small()
    with pytest.raises(bt.BtError) as e:
        batch.add(bt.Options(width=256, height=256), w.xy, w.starts)
    assert e.value.status == 8
    with pytest.raises(bt.BtError):
        batch.remove(3)
    batch.iterate(2)                       # an empty batch is a no-op
    assert batch.active() == 0


def test_add_many_uploads_concurrently_and_matches_standalone():
    jobs = mixed_jobs()
    batch = bt.Batch(solo_samples=PERSISTENT)
    added = batch.add_many([(o, w.xy, w.starts) for w, o in jobs])
    assert [s for s, _ in added] == list(range(len(jobs)))
    for (w, o), (slot, n) in zip(jobs, added):
        assert batch.slot(slot).info().samples == n
    batch.iterate(3)
    for (w, o), (slot, _) in zip(jobs, added):
        check_slot(batch, slot, standalone(w, o, 3))


def test_add_many_is_all_or_nothing():
    w = synthetic.small()
    o = workload_options(w)
    bad = w.starts.copy()
    bad[-1] = w.xy.shape[0] + 5            # last start past the point count
    batch = bt.Batch(solo_samples=PERSISTENT)
    batch.add(o, w.xy, w.starts)
    with pytest.raises(bt.BtError) as e:
        batch.add_many([(o, w.xy, w.starts), (o, w.xy, bad)])
    assert e.value.status == 3
    assert batch.active() == 1
    batch.iterate(1)
    check_slot(batch, 0, standalone(w, o, 1))


def test_slots_change_lanes_between_iterations():
    # The same graphs moved between the persistent step and their own
    # contexts mid-run: results still equal standalone runs.
    jobs = mixed_jobs()[:3]
    batch = bt.Batch(solo_samples=PERSISTENT)
    slots = [batch.add(o, w.xy, w.starts)[0] for w, o in jobs]
    batch.iterate(2)
    batch.set_solo_samples(1)
    batch.iterate(2)
    batch.set_solo_samples(PERSISTENT)
    batch.iterate(1)
    for (w, o), slot in zip(jobs, slots):
        check_slot(batch, slot, standalone(w, o, 5))


@pytest.mark.parametrize("mean_tile,ctas", [(64, 0), (128, 6), (256, 0), (256, 3)])
def test_batch_shapes_do_not_change_results(mean_tile, ctas):
    # The mean tile (= CTA size) and the resident CTAs per SM change only how
    # the work is cut and scheduled, never a slot's results.
    jobs = mixed_jobs()
    batch = bt.Batch()
    batch.set_shape(mean_tile, ctas)
    assert batch.shape() == {"mean_tile": mean_tile, "mean_ctas_per_sm": ctas}
    slots = [batch.add(o, w.xy, w.starts)[0] for w, o in jobs]
    batch.iterate(2)
    for (w, o), slot in zip(jobs, slots):
        check_slot(batch, slot, standalone(w, o, 2))
    # A change of shape between steps keeps the results too.
    batch.set_shape(128, 0)
    batch.iterate(1)
    for (w, o), slot in zip(jobs, slots):
        check_slot(batch, slot, standalone(w, o, 3))
    batch.close()


def test_autotuned_batch_matches_standalone_runs():
    jobs = mixed_jobs()
    shape, ms = bt.Batch.autotune([(o, w.xy, w.starts) for w, o in jobs], iterations=2)
    assert ms > 0 and shape["mean_tile"] in (64, 128, 256)
    batch = bt.Batch()
    batch.set_shape(**shape)
    slots = [batch.add(o, w.xy, w.starts)[0] for w, o in jobs]
    batch.iterate(3)
    for (w, o), slot in zip(jobs, slots):
        check_slot(batch, slot, standalone(w, o, 3))
    batch.close()
    with pytest.raises(bt.BtError) as e:
        bt.Batch().set_shape(96, 0)
    assert e.value.status == 3
