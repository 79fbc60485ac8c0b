"""Search-shape checks during a job (options.shape_checks; bt_iterate,
bt_iterate_timed).

With the option, after 5, 10, 20, ... iterations of an upload the
synchronous calls sample the neighbour search's rows and boundary samples and
may re-bin the graph under another search-cell shape; the asynchronous call
never checks. Every shape gives the same neighbour sets and exact sums, so a
job through the checks must equal the same job without them bit for bit
(positions, neighbour counts, density), whatever the checks decide. On the large workload the checks
re-bin after iteration 10, from 2 x 0.25-texel cells to 4 x 0.5.
"""
import numpy as np
import pytest

import bundling_thingy_b200 as bt
from bundling_thingy_b200 import synthetic

pytestmark = pytest.mark.gpu


def opts_for(w: synthetic.Workload, **kw) -> bt.Options:
    return bt.Options(width=w.width, height=w.height, neighbor_radius=w.radius, sample_spacing=w.spacing,
                      blur_sigma=w.sigma, blur_shrink=w.shrink, record_neighbors=True, **kw)


def outputs(g: bt.Gpu):
    xy, ids = g.read_points()
    return xy, ids, g.read_neighbors(), g.read_density()


def test_large_job_through_checks_equals_job_without():
    w = synthetic.large()
    checked = bt.Gpu(opts_for(w, shape_checks=True))
    plain = bt.Gpu(opts_for(w))
    checked.upload((w.xy, w.starts))
    plain.upload((w.xy, w.starts))
    first = (checked.info().fine_cells, checked.info().fine_cells_x)
    assert first == (plain.info().fine_cells, plain.info().fine_cells_x)
    checked.iterate(30)
    plain.iterate(30)
    assert checked.info().iterations == plain.info().iterations == 30
    last = (checked.info().fine_cells, checked.info().fine_cells_x)
    # The checks moved the large workload to taller rows; without the option
    # the upload's shape stays.
    assert last[0] < first[0], (first, last)
    assert (plain.info().fine_cells, plain.info().fine_cells_x) == first
    for a, b in zip(outputs(checked), outputs(plain)):
        np.testing.assert_array_equal(a, b)
    checked.close()
    plain.close()


def test_fixed_shape_is_never_changed():
    # A shape fixed by the options is the caller's choice: no check applies.
    w = synthetic.mid()
    g = bt.Gpu(opts_for(w, fine_cells=4, fine_cells_x=8, shape_checks=True))
    g.upload((w.xy, w.starts))
    g.iterate(25)
    info = g.info()
    assert (info.fine_cells, info.fine_cells_x) == (4, 8)
    g.close()


def test_timed_iterations_run_the_checks_and_match():
    w = synthetic.mid()
    timed = bt.Gpu(opts_for(w, shape_checks=True))
    plain = bt.Gpu(opts_for(w))
    timed.upload((w.xy, w.starts))
    plain.upload((w.xy, w.starts))
    ms = timed.iterate_timed(w.iterations)
    plain.iterate(w.iterations)
    assert ms > 0.0
    for a, b in zip(outputs(timed), outputs(plain)):
        np.testing.assert_array_equal(a, b)
    timed.close()
    plain.close()


def test_async_iterations_make_no_checks():
    # bt_iterate_async never waits on the host, so it never checks.
    w = synthetic.large()
    g = bt.Gpu(opts_for(w, shape_checks=True))
    g.upload((w.xy, w.starts))
    first = (g.info().fine_cells, g.info().fine_cells_x)
    g.iterate_async(30)
    g.synchronize()
    assert (g.info().fine_cells, g.info().fine_cells_x) == first
    g.close()
