"""GPU parity of the density-gradient advection mode (advect.cu), an
iteration mode beyond the reference, against the oracle's step (or_advect)
composed with its splat, blur and normalisation. Positions and density must
match bit for bit after every iteration."""
import numpy as np
import pytest

import bundling_thingy_b200 as bt
from bundling_thingy_b200 import synthetic

from conftest import oracle_config

pytestmark = pytest.mark.gpu


def run_pair(oracle, w, iterations, step, smooth, color_by=bt.COLOR_BY_DENSITY, **kw):
    o = bt.Options(width=w.width, height=w.height, sample_spacing=w.spacing, blur_sigma=w.sigma,
                   blur_shrink=w.shrink, advect_step=step, advect_smooth=smooth, color_by=color_by, **kw)
    gpu = bt.Gpu(o)
    n = gpu.upload((w.xy, w.starts))
    cfg = oracle_config(oracle, o)
    cfg.accumulate_density = True            # the advection mode always accumulates the density
    ora = oracle.Pipeline(cfg)
    assert ora.upload(w.xy, w.starts) == n
    xy, ids = ora.points()
    norm = ora.normalized()
    gxy, gid = gpu.read_points()
    np.testing.assert_array_equal(gid, ids)
    np.testing.assert_array_equal(gxy, xy)
    np.testing.assert_array_equal(gpu.read_density(), norm)
    sigma = float(np.float32(w.sigma))
    shrink = float(np.float32(w.shrink)) if w.shrink else 1.0
    for k in range(1, iterations + 1):
        xy = oracle.advect(xy, ids, norm, w.width, w.height, step, smooth)
        s = sigma
        for _ in range(k):
            s *= shrink
        counts = oracle.splat(xy, w.width, w.height)
        _, vt, peak = oracle.blur(counts, w.width, w.height, oracle.blur_weights(s))
        norm = oracle.normalize(vt, peak)
        gpu.iterate(1)
        gxy, _ = gpu.read_points()
        assert np.abs(gxy - xy).max() <= 2e-4          # the stated position tolerance
        np.testing.assert_array_equal(gxy, xy)
        np.testing.assert_array_equal(gpu.read_density(), norm)
    return gpu, xy, ids


@pytest.mark.parametrize("step,smooth", [(1.0, 0.0), (2.0, 0.5), (0.5, 1.0)])
def test_small_workload_matches_oracle(oracle, step, smooth):
    w = synthetic.small()
    gpu, xy, _ = run_pair(oracle, w, 6, step, smooth)
    assert gpu.info().iterations == 6


def test_mid_workload_edge_colouring(oracle):
    # Edge-id colouring still accumulates the density the step climbs.
    w = synthetic.mid()
    run_pair(oracle, w, 3, 1.5, 0.25, color_by=bt.COLOR_BY_EDGE_ID)


def test_advection_bundles_and_keeps_endpoints(oracle):
    w = synthetic.small()
    gpu, xy, ids = run_pair(oracle, w, 10, 1.0, 0.5)
    paths = gpu.read_paths()
    first = paths[:, 0][paths[:, 2] >= 2]
    last = (paths[:, 0] + paths[:, 2] - 1)[paths[:, 2] >= 2]
    g0 = bt.Gpu(bt.Options(width=w.width, height=w.height, sample_spacing=w.spacing))
    g0.upload((w.xy, w.starts))
    xy0, _ = g0.read_points()
    np.testing.assert_array_equal(xy[first], xy0[first])
    np.testing.assert_array_equal(xy[last], xy0[last])
    # Samples gather: the occupied texels of the splat shrink.
    occupied0 = np.count_nonzero(oracle.splat(xy0, w.width, w.height))
    occupied = np.count_nonzero(oracle.splat(xy, w.width, w.height))
    assert occupied < occupied0


def test_render_and_distortion_after_advection(oracle):
    w = synthetic.small()
    o = bt.Options(width=w.width, height=w.height, sample_spacing=w.spacing, blur_sigma=w.sigma,
                   advect_step=1.0, advect_smooth=0.5, evaluate_distortion=True)
    gpu = bt.Gpu(o)
    gpu.upload((w.xy, w.starts))
    xy0, ids = gpu.read_points()
    gpu.iterate(4)
    xy, _ = gpu.read_points()
    frame = gpu.render()
    img, colored = oracle.render(xy, ids, gpu.read_segments(), gpu.info().paths, gpu.read_density(), w.width,
                                 w.height)
    assert frame.colored_pixels == colored
    np.testing.assert_array_equal(frame.rgba, img)
    m = gpu.distortion(bt.SIZE)
    d, px = oracle.distortion(gpu.read_paths(), xy0, xy, bt.SIZE)
    assert abs(m.distortion - d) <= 1e-12 * max(d, 1e-30)


def test_options_are_checked():
    w = synthetic.small()
    with pytest.raises(bt.BtError):
        bt.Gpu(bt.Options(neighbor_radius=2, advect_step=1.0))
    with pytest.raises(bt.BtError):
        bt.Gpu(bt.Options(advect_step=-1.0))
    with pytest.raises(bt.BtError):
        bt.Gpu(bt.Options(advect_step=1.0, advect_smooth=1.5))
    g = bt.Gpu(bt.Options(width=w.width, height=w.height))
    g.upload((w.xy, w.starts))
    with pytest.raises(bt.BtError):
        g.iterate(1)          # neither a radius nor an advection step
