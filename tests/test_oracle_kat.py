"""Known-answer tests pinning the CPU oracle.

The reference ships no golden vectors, so each expected value here is derived
by hand from the reference's rules (file:line in each test).
"""
import numpy as np
import pytest


def _pipe(O, w, h, radius=0, sigma=0.0, shrink=1.0, scale=None, capacity=1 << 31):
    return O.Pipeline(O.Config(w, h, radius=radius, sigma=sigma, shrink=shrink, resample_scale=scale,
                               capacity=capacity))


def test_normalization_fits_95_percent(oracle):
    # graph.rs:79-91: span 2 -> scale 0.475, translation (1 - scale*range)/2.
    out = oracle.normalization((0.0, 0.0), (2.0, 1.0))
    f = np.float32
    scale = f(0.95) / f(2.0)
    tx = (f(1.0) - scale * f(2.0)) / f(2.0)   # f32 arithmetic, as glam Vec2
    ty = (f(1.0) - scale * f(1.0)) / f(2.0)
    np.testing.assert_array_equal(out, np.float32([0.0, 0.0, scale, tx, ty]))
    assert abs(tx - 0.025) < 1e-7 and abs(ty - 0.2625) < 1e-7


def test_normalization_rejects_degenerate_extent(oracle):
    with pytest.raises(oracle.OracleError):
        oracle.normalization((1.0, 1.0), (1.0, 1.0))


def test_straight_segment_sample_count(oracle):
    # resampling.wgsl:95-123: a segment of non-integer length L texels yields
    # the first point, samples at 1..floor(L) texels and the endpoint.
    # Map 100 wide -> texel_scale 49.5; the fitted segment spans clip
    # [-0.95, 0.95] = 1.9 clip units = 94.05 texels.
    p = _pipe(oracle, 100, 100)
    n = p.upload(np.float32([[0, 0], [10, 0]]), np.uint32([0, 2]))
    assert n == 94 + 2
    xy, ids = p.points()
    assert (ids == 0).all()
    np.testing.assert_allclose(xy[0], [-0.95, 0.0], atol=1e-7)
    np.testing.assert_allclose(xy[-1], [0.95, 0.0], atol=1e-7)
    k = np.arange(1, 95)
    np.testing.assert_allclose(xy[1:-1, 0], -0.95 + k / 49.5, atol=2e-6)
    assert (xy[:, 1] == 0).all()
    np.testing.assert_array_equal(p.paths(), [[0, 0, 96]])
    np.testing.assert_array_equal(p.segments(), np.arange(95))


def test_consecutive_samples_are_distinct_and_end_at_endpoint(oracle):
    # push_sample drops exact repeats (resampling.wgsl:51-53); the path always
    # ends at its last control point (resampling.wgsl:123).
    p = _pipe(oracle, 201, 201)
    p.upload(np.float32([[0, 0], [3, 1], [5, 5], [9, 2]]), np.uint32([0, 4]))
    xy, _ = p.points()
    assert not (np.all(xy[1:] == xy[:-1], axis=1)).any()
    edges = p.edges()
    np.testing.assert_array_equal(xy[-1], edges[0, 2:])
    np.testing.assert_array_equal(xy[0], edges[0, :2])


def test_short_closed_path_keeps_excursion(oracle):
    # resampling.wgsl:124-134: a closed path A -> B -> A shorter than half a
    # texel resamples to exactly [A, B, A]. The second edge sets the extent.
    cp = np.float32([[50, 0.1], [50.2, 0.1], [50, 0.1], [0, 0], [100, 0]])
    p = _pipe(oracle, 101, 101)
    p.upload(cp, np.uint32([0, 3, 5]))
    paths = p.paths()
    assert paths[0, 2] == 3
    xy, ids = p.points()
    a, b = xy[paths[0, 0]], xy[paths[0, 0] + 1]
    np.testing.assert_array_equal(xy[paths[0, 0] + 2], a)
    assert not np.array_equal(a, b)


def test_single_count_blurs_to_weight_outer_product(oracle):
    # blur.wgsl:42-60: one count at (x, y) gives horizontal = w[|dx|] and
    # vertical = f32(w[|dx|] * w[|dy|]).
    w = oracle.blur_weights(0.0)
    W = H = 64
    counts = np.zeros(W * H, np.uint32)
    counts[30 * W + 20] = 1
    hz, vt, peak = oracle.blur(counts, W, H, w)
    R = len(w) - 1
    ys, xs = np.mgrid[0:H, 0:W]
    dx, dy = np.abs(xs - 20), np.abs(ys - 30)
    wx = np.where(dx <= R, w[np.minimum(dx, R)], 0).astype(np.float32)
    wy = np.where(dy <= R, w[np.minimum(dy, R)], 0).astype(np.float32)
    np.testing.assert_array_equal(hz.reshape(H, W)[30], wx[30])
    np.testing.assert_array_equal(vt.reshape(H, W), (wx * wy).astype(np.float32))
    assert peak == np.float32(w[0] * w[0])


def test_reference_taps_and_general_sigma(oracle):
    # blur.wgsl:42-60 literal table; other sigma: normalised exp(-k^2/2s^2), R = ceil(3s).
    w = oracle.blur_weights(0.0)
    assert len(w) == 19 and w[0] == np.float32(0.0666251319)
    g = oracle.blur_weights(8.0)
    assert len(g) == 25
    k = np.arange(-24, 25)
    ref = np.exp(-k ** 2 / 128.0)
    ref /= ref.sum()
    np.testing.assert_array_equal(g, ref[24:].astype(np.float32))


def test_normalize_clamps_and_handles_zero_peak(oracle):
    v = np.float32([0, 1, 2, 4])
    np.testing.assert_array_equal(oracle.normalize(v, 4.0), [0, 0.25, 0.5, 1.0])
    np.testing.assert_array_equal(oracle.normalize(v, 0.0), [0, 0, 0, 0])


def test_grid_cells_of_corners(oracle):
    # spatial_grid.wgsl:59-70 with ceil(101/10) = 11 cells per side.
    xy = np.float32([[-1, -1], [1, 1], [0, 0], [-1, 1]])
    np.testing.assert_array_equal(oracle.cells(xy, 101, 101, 10), [0, 120, 5 * 11 + 5, 10 * 11])


def test_two_sample_path_does_not_move(oracle):
    # neighbor_mean.wgsl:61-64: a path's first and last samples are fixed.
    cp = np.float32([[0, 0], [0.001, 0], [0, 1], [1, 1]])
    p = _pipe(oracle, 101, 101, radius=3)
    p.upload(cp, np.uint32([0, 2, 4]))
    paths = p.paths()
    assert paths[0, 2] == 2
    before, _ = p.points()
    p.iterate(3)
    after, _ = p.points()
    off = paths[0, 0]
    np.testing.assert_array_equal(after[off:off + 2], before[off:off + 2])


def test_symmetric_neighbours_keep_the_centre(oracle):
    xy = np.float32([[-0.01, 0], [0, 0], [0.01, 0]])
    out, nb = oracle.neighbor_mean(xy, [0, 1, 0], 101, 101, 2)
    np.testing.assert_array_equal(out[1], [0, 0])
    assert nb[1] == 3


def test_mean_of_three_collinear_points(oracle):
    xy = np.float32([[0.001, 0], [0, 0], [0.003, 0]])
    out, nb = oracle.neighbor_mean(xy, [0, 1, 0], 101, 101, 2)
    assert nb[1] == 3
    assert abs(out[1, 0] - 0.004 / 3) < 2e-9 and out[1, 1] == 0


def test_radius_is_inclusive(oracle):
    # neighbor_mean.wgsl:195: dot(d*ts, d*ts) <= r*r. ts = 50, r = 2: a
    # neighbour 0.04 clip away lies exactly on the circle; 0.0401 is outside.
    xy = np.float32([[0.0, 0.0], [0.04, 0.0], [0.0, 0.0401]])
    out, nb = oracle.neighbor_mean(xy, [1, 0, 0], 101, 101, 2)
    assert nb[0] == 2
    assert abs(out[0, 0] - 0.02) < 1e-8 and out[0, 1] == 0


def test_fixed_point_mean_matches_f32_running_sum(oracle):
    # The canonical exact accumulation differs from the reference's f32
    # running sum only by rounding (tolerance 1e-4 of the canvas = 2e-4 clip).
    from bundling_thingy_b200 import synthetic

    w = synthetic.small()
    s = 0.5 / float(np.float32(w.spacing))
    p = _pipe(oracle, w.width, w.height, radius=w.radius, sigma=8.0, scale=(s, s))
    p.upload(w.xy, w.starts)
    xy, _ = p.points()
    mv = np.ones(len(xy), np.uint8)
    paths = p.paths()
    mv[paths[:, 0]] = 0
    mv[paths[:, 0] + paths[:, 2] - 1] = 0
    a, na = oracle.neighbor_mean(xy, mv, w.width, w.height, w.radius, mode=0)
    b, nb = oracle.neighbor_mean(xy, mv, w.width, w.height, w.radius, mode=1)
    np.testing.assert_array_equal(na, nb)
    assert np.abs(a - b).max() < 1e-6


def test_capacity_overflow(oracle):
    # count_paths overflow 1 (resampling.wgsl:151-156).
    p = _pipe(oracle, 100, 100, capacity=50)
    with pytest.raises(oracle.OracleError) as e:
        p.upload(np.float32([[0, 0], [10, 0]]), np.uint32([0, 2]))
    assert e.value.status == 1


def test_distortion_of_a_shift(oracle):
    # distortion.rs:137-168: a rigid shift by d has integral d^2.
    a = np.float32([[0, 0], [0.5, 0], [1, 0]])
    b = a + np.float32([0, 0.25])
    assert abs(oracle.squared_integral(a, b) - 0.0625) < 1e-15
    assert oracle.squared_integral(a, a) == 0.0
    # Equal-edge aggregate of shifts 0.25 and 0.5 (distortion.rs:201-215).
    orig = np.concatenate([a, a])
    cur = np.concatenate([a + np.float32([0, 0.25]), a + np.float32([0, 0.5])])
    paths = np.uint32([[0, 0, 3], [3, 2, 3]])
    d, px = oracle.distortion(paths, orig, cur, 1600)
    rms = np.sqrt((0.0625 + 0.25) / 2)
    assert abs(d - rms / (2 * np.sqrt(2))) < 1e-12
    assert abs(px - rms * 800) < 1e-9


def test_distortion_reparameterisation_invariance(oracle):
    # Correspondence is by normalised arc length: resampling the same line
    # gives zero displacement.
    a = np.float32([[0, 0], [1, 0]])
    b = np.float32([[0, 0], [0.25, 0], [1, 0]])
    assert oracle.squared_integral(a, b) < 1e-30
