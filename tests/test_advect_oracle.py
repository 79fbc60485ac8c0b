"""Known answers for the oracle's density-gradient advection step
(oracle.cpp or_advect), an iteration mode beyond the reference."""
import numpy as np

f = np.float32


def test_flat_density_leaves_a_straight_path_in_place(oracle):
    # No gradient: no advection; the middle sample of an evenly spaced
    # straight path already sits at the mean of its neighbours.
    xy = np.float32([[-0.5, 0.25], [0.0, 0.25], [0.5, 0.25]])
    out = oracle.advect(xy, [0, 0, 0], np.zeros(64 * 64, np.float32), 64, 64, step=1.5, smooth=0.5)
    np.testing.assert_array_equal(out, xy)


def test_relaxation_moves_towards_the_neighbour_mean(oracle):
    xy = np.float32([[-0.5, 0.0], [0.0, 0.1], [0.5, 0.0]])
    out = oracle.advect(xy, [0, 0, 0], np.zeros(64 * 64, np.float32), 64, 64, step=1.0, smooth=0.5)
    # a + 0.5 * ((p + q) / 2 - a) with a = p_mid (no gradient)
    want = f(0.1) + f(0.5) * ((f(0.0) + f(0.0)) * f(0.5) - f(0.1))
    np.testing.assert_array_equal(out[1], [0.0, want])
    np.testing.assert_array_equal(out[[0, 2]], xy[[0, 2]])


def test_sample_climbs_one_step_towards_a_peak(oracle):
    # A ramp rising to the left along x (row direction): the unit gradient is
    # (-1, 0) in map texels, so the sample moves `step` texels left and not
    # vertically, with its neighbours far away (smooth = 0).
    w = h = 65
    u = np.arange(w, dtype=np.float32)
    density = np.tile(f(1.0) - u / f(w), (h, 1)).astype(np.float32)
    xy = np.float32([[-0.9, 0.0], [0.25, 0.0], [0.9, 0.0]])
    out = oracle.advect(xy, [3, 3, 3], density, w, h, step=2.0, smooth=0.0)
    x = f(0.25)
    want = x + (f(2.0) * (f(-1.0))) * (f(2.0) / f(w - 1))
    assert out[1, 1] == 0.0
    np.testing.assert_allclose(out[1, 0], want, rtol=0, atol=2e-7)
    assert out[1, 0] < x


def test_path_ends_stay_fixed(oracle):
    # Two paths back to back (edge ids 0 and 1): each one's first and last
    # samples keep their positions whatever the density.
    rng = np.random.default_rng(5)
    density = rng.random(32 * 32).astype(np.float32)
    xy = rng.uniform(-0.8, 0.8, (7, 2)).astype(np.float32)
    ids = [0, 0, 0, 0, 1, 1, 1]
    out = oracle.advect(xy, ids, density, 32, 32, step=1.0, smooth=0.3)
    for i in (0, 3, 4, 6):
        np.testing.assert_array_equal(out[i], xy[i])
    assert not np.array_equal(out[[1, 2, 5]], xy[[1, 2, 5]])
