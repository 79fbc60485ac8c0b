"""Known-answer tests pinning the oracle's rasteriser (oracle/render.cpp).

The reference renders with a hardware rasteriser, so there are no golden
images to match bit for bit; each expected value here follows from the
render rules (src/shaders/render_paths.wgsl:35-101, src/gpu.rs:572-620) by
hand, with the f32 arithmetic repeated in numpy.
"""
import numpy as np
import pytest

f = np.float32
VIRIDIS = np.float32([[0.267004, 0.004874, 0.329415], [0.282656, 0.100196, 0.422160], [0.277134, 0.185228, 0.489898],
                      [0.253935, 0.265254, 0.529983], [0.221989, 0.339161, 0.548752], [0.190631, 0.407061, 0.556089],
                      [0.163625, 0.471133, 0.558148], [0.139147, 0.533812, 0.555298], [0.120565, 0.596422, 0.543611]])


def u8(r):
    return int(np.clip(np.rint(f(r) * f(255.0)), 0, 255))


BG = np.array([u8(0.025), u8(0.025), u8(0.035)])


def blend_once(col):
    """One alpha-0.1 blend of col over the clear colour (gpu.rs ALPHA_BLENDING)."""
    keep = f(1.0) - f(0.1)
    return np.array([u8(f(c) * f(0.1) + (f(b) / f(255.0)) * keep) for c, b in zip(col, BG)])


def test_half_round_matches_ieee_binary16(oracle):
    rng = np.random.default_rng(7)
    v = np.concatenate([rng.standard_normal(4000).astype(np.float32) * f(10.0) ** rng.integers(-9, 5, 4000),
                        np.float32([0.0, -0.0, 1e-8, 6e-8, 5.96e-8, 65504.0, 65519.0, 65520.0, 1e9, -1e9])])
    got = np.array([oracle.half_round(float(x)) for x in v], np.float32)
    with np.errstate(over="ignore"):
        want = v.astype(np.float16).astype(np.float32)
    np.testing.assert_array_equal(got, want)
    assert np.isnan(oracle.half_round(float("nan")))


def test_blank_frame_is_the_clear_colour(oracle):
    # gpu.rs:580-590: Clear(0.025, 0.025, 0.035) stored as RGBA8 unorm.
    img, colored = oracle.render(np.zeros((0, 2)), np.zeros(0), np.zeros(0), 0, None, 64, 48)
    assert colored == 0 and img.shape == (48, 64, 4)
    assert (img[..., :3] == BG).all() and (img[..., 3] == 255).all()
    assert tuple(BG) == (6, 6, 9)


def test_horizontal_band_covers_two_rows(oracle):
    # A segment across the canvas at Y = 0 on a 2000 x 2000 frame: the quad's
    # half-width 0.001 clip is 1 pixel, so rows 999 and 1000 are covered at
    # every sample and nothing else is (render_paths.wgsl:44-50).
    xy = np.float32([[-1.0, 0.0], [1.0, 0.0]])
    img, colored = oracle.render(xy, [0, 0], [0], 1, None, 2000, 2000, color_by_edge=True)
    assert colored == 4000
    # edge value 0 / (max(1, 2) - 1) -> palette stop 0, one blend per sample.
    want = blend_once(VIRIDIS[0])
    assert (img[999:1001, :, :3] == want).all()
    assert (img[:999, :, :3] == BG).all() and (img[1001:, :, :3] == BG).all()


def test_density_colour_is_sampled_from_the_f16_texture(oracle):
    # fs_main: value 0.5 -> stop 7.5 -> mix(palette[7], palette[8], 0.5).
    xy = np.float32([[-1.0, 0.0], [1.0, 0.0]])
    density = np.full(2000 * 2000, 0.5, np.float32)
    img, colored = oracle.render(xy, [0, 0], [0], 1, density, 2000, 2000)
    col = VIRIDIS[7] * (f(1.0) - f(0.5)) + VIRIDIS[8] * f(0.5)
    assert colored == 4000
    assert (img[999:1001, :, :3] == blend_once(col)).all()


def test_shared_quad_edge_through_sample_centres_is_drawn_once(oracle):
    # Two collinear segments meeting at x = 1000.5 px: with one sample per
    # pixel, the centres of pixel 1000 in rows 999 and 1000 lie exactly on
    # the shared vertical edge; the top-left rule gives them to one quad, so
    # every covered pixel is blended exactly once.
    xy = np.float32([[-1.0, 0.0], [0.0005, 0.0], [1.0, 0.0]])
    img, colored = oracle.render(xy, [0, 0, 0], [0, 1], 1, None, 2000, 2000, color_by_edge=True, msaa=1)
    assert colored == 4000
    assert (img[999:1001, :, :3] == blend_once(VIRIDIS[0])).all()


def test_collapsed_segment_draws_nothing(oracle):
    # render_paths.wgsl:42-43: both ends at one position -> zero-area quad.
    xy = np.float32([[0.1, 0.2], [0.1, 0.2]])
    img, colored = oracle.render(xy, [0, 0], [0], 1, None, 256, 256, color_by_edge=True)
    assert colored == 0


def test_later_segments_blend_over_earlier_ones(oracle):
    # Two identical segments: the second blends over the first (draw order).
    xy = np.float32([[-1.0, 0.0], [1.0, 0.0], [-1.0, 0.0], [1.0, 0.0]])
    img, colored = oracle.render(xy, [0, 0, 1, 1], [0, 2], 2, None, 2000, 2000, color_by_edge=True)
    first = blend_once(VIRIDIS[0])
    keep = f(1.0) - f(0.1)
    last = VIRIDIS[8] * f(0) + np.float32([0.993248, 0.906157, 0.143936])   # edge 1 / (2 - 1) = 1 -> stop 15
    second = np.array([u8(f(c) * f(0.1) + (f(b) / f(255.0)) * keep) for c, b in zip(last, first)])
    assert colored == 4000
    assert (img[999:1001, :, :3] == second).all()


def test_endpoint_dots_cover_the_endpoints(oracle):
    # vs_endpoint + fs_endpoint: the centre pixel of an endpoint takes the
    # palette's endpoint colour (viridis: 1.0, 0.4, 0.7); the ring between 2
    # and 3 pixels holds the outline colour palette[0] * 0.1.
    xy = np.float32([[-0.5, 0.0], [0.5, 0.0]])
    paths = np.uint32([[0, 0, 2]])
    img, _ = oracle.render(xy, [0, 0], [0], 1, None, 2000, 2000, color_by_edge=True, paths=paths,
                           endpoint_dots=True)
    centre = np.array([u8(1.0), u8(0.4), u8(0.7)])
    # clip -0.5 -> x = 500 px, clip 0 -> y = 1000 px: pixels 499..500 x 999..1000
    for y in (999, 1000):
        for x in (499, 500, 1499, 1500):
            assert (img[y, x, :3] == centre).all(), (x, y)
    outline = np.array([u8(f(c) * f(0.1)) for c in VIRIDIS[0]])
    assert (img[..., :3] == outline).all(axis=-1).sum() > 0
    img2, _ = oracle.render(xy, [0, 0], [0], 1, None, 2000, 2000, color_by_edge=True, paths=paths,
                            endpoint_dots=False)
    assert not (img2[..., :3] == centre).all(axis=-1).any()


def test_render_rejects_bad_arguments(oracle):
    with pytest.raises(oracle.OracleError):
        oracle.render(np.zeros((0, 2)), [], [], 0, None, 16, 16, msaa=3)
    with pytest.raises(oracle.OracleError):
        oracle.render(np.zeros((0, 2)), [], [], 0, None, 16, 16, palette=4)
