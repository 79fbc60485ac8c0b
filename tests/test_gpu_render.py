"""GPU parity of the renderer (bt_render) against the oracle's rasteriser.

Both sides follow the same rules (csrc/render.cu, oracle/render.cpp): quads
snapped to 1/256 pixel, 64-bit edge functions, f16 density texels, 8-bit
blends in draw order. The frame (RGBA8) and its coloured-pixel count must
match bit for bit, for every palette, colouring, sample count and tile size,
before and after iterations.
"""
import json

import numpy as np
import pytest

import bundling_thingy_b200 as bt
from bundling_thingy_b200 import synthetic

pytestmark = pytest.mark.gpu


def oracle_frame(oracle, gpu, opts):
    xy, ids = gpu.read_points()
    density = gpu.read_density() if opts.color_by == bt.COLOR_BY_DENSITY else None
    return oracle.render(xy, ids, gpu.read_segments(), gpu.info().paths, density, opts.width, opts.height,
                         color_by_edge=opts.color_by == bt.COLOR_BY_EDGE_ID, palette=opts.palette, msaa=opts.msaa,
                         paths=gpu.read_paths(), endpoint_dots=opts.endpoint_dots)


def check(oracle, gpu, opts):
    frame = gpu.render()
    want, colored = oracle_frame(oracle, gpu, opts)
    assert frame.colored_pixels == colored
    mism = np.argwhere((frame.rgba != want).any(axis=-1))
    assert mism.size == 0, f"{len(mism)} pixels differ, first at {mism[:3].tolist()}"
    assert colored > 0
    return frame


def small_opts(**kw):
    w = synthetic.small()
    o = bt.Options(width=w.width, height=w.height, neighbor_radius=w.radius, sample_spacing=w.spacing,
                   blur_sigma=w.sigma, blur_shrink=w.shrink)
    for k, v in kw.items():
        setattr(o, k, v)
    return w, o


def test_blank_frame_before_upload():
    gpu = bt.Gpu(bt.Options(width=100, height=60))
    f = gpu.render()
    assert f.colored_pixels == 0 and f.rgba.shape == (60, 100, 4)
    assert (f.rgba[..., :3] == (6, 6, 9)).all() and (f.rgba[..., 3] == 255).all()


@pytest.mark.parametrize("msaa", [1, 2, 4])
@pytest.mark.parametrize("color_by", [bt.COLOR_BY_DENSITY, bt.COLOR_BY_EDGE_ID])
def test_small_frame_matches_oracle(oracle, msaa, color_by):
    w, o = small_opts(msaa=msaa, color_by=color_by)
    gpu = bt.Gpu(o)
    gpu.upload((w.xy, w.starts))
    check(oracle, gpu, o)
    gpu.iterate(3)
    check(oracle, gpu, o)


@pytest.mark.parametrize("palette", [0, 1, 2, 3])
def test_palettes_and_endpoint_dots(oracle, palette):
    w, o = small_opts(palette=palette, endpoint_dots=True)
    gpu = bt.Gpu(o)
    gpu.upload((w.xy, w.starts))
    gpu.iterate(2)
    check(oracle, gpu, o)


def test_reference_canvas_mid_graph(oracle):
    # 1600 x 1600 (the reference's headless canvas), 4x MSAA, density colour.
    w = synthetic.mid()
    o = bt.Options(neighbor_radius=w.radius, sample_spacing=w.spacing, blur_sigma=w.sigma)
    gpu = bt.Gpu(o)
    gpu.upload((w.xy, w.starts))
    check(oracle, gpu, o)
    gpu.iterate(5)
    f = check(oracle, gpu, o)
    # Rendering again gives the same frame (nothing in it depends on timing).
    again = gpu.render()
    np.testing.assert_array_equal(again.rgba, f.rgba)


@pytest.mark.parametrize("size", [2100, 4200])
def test_large_frames_use_wider_tiles(oracle, size):
    # Above 16384 tiles of 16 px the bins switch to 32 px, then to 64 px.
    w = synthetic.small()
    o = bt.Options(width=size, height=size, sample_spacing=w.spacing, color_by=bt.COLOR_BY_EDGE_ID, msaa=2)
    gpu = bt.Gpu(o)
    gpu.upload((w.xy, w.starts))
    check(oracle, gpu, o)


def test_long_segments_regrow_the_bins(oracle):
    # Sample spacing of a quarter canvas: few, long segments, each in many
    # tiles, more bins than the first estimate holds.
    w = synthetic.small()
    o = bt.Options(width=1600, height=1600, sample_spacing=0.25, color_by=bt.COLOR_BY_EDGE_ID)
    gpu = bt.Gpu(o)
    gpu.upload((w.xy, w.starts))
    check(oracle, gpu, o)
    check(oracle, gpu, o)


def test_render_count_only_and_bad_buffer():
    w, o = small_opts()
    gpu = bt.Gpu(o)
    gpu.upload((w.xy, w.starts))
    full = gpu.render()
    count = gpu.render(pixels=False)
    assert count.rgba is None and count.colored_pixels == full.colored_pixels
    assert full.device_ms > 0
    with pytest.raises(ValueError):
        gpu.render(out=np.zeros((10, 10, 4), np.uint8))


def test_headless_run_writes_images_and_reports(oracle, tmp_path, capsys):
    # src/main.rs:104-221: blank-frame calibration, original.png, one image
    # per iteration, noisiness.json and distortion.json.
    from bundling_thingy_b200 import report

    w = synthetic.small()
    trl = tmp_path / "g.trl"
    synthetic.write_trl(trl, w.xy, w.starts)
    o = bt.Options(width=w.width, height=w.height, sample_spacing=w.spacing, blur_sigma=w.sigma,
                   blur_shrink=w.shrink, color_by=bt.COLOR_BY_EDGE_ID)
    out_dir = tmp_path / "out"
    r = report.headless(trl, out_dir, neighbor_radius=w.radius, iterations=2, options=o, evaluate_noisiness=True,
                        evaluate_distortion=True)
    lines = capsys.readouterr().out.splitlines()
    assert lines[0].startswith("noisiness original.png: ") and lines[0].endswith("change +0.000000")
    assert lines[1] == f"wrote {out_dir / 'original.png'}"
    assert lines[2] == "original.png distortion=0 rms_displacement_pixels=0"
    assert lines[3].startswith("noisiness iteration-01.png: ")
    assert lines[4] == f"wrote {out_dir / 'iteration-01.png'}"
    assert lines[5].startswith("iteration-01.png distortion=")
    assert lines[-1] == f"rendered {r['samples']} samples to {out_dir}"
    noise = json.loads((out_dir / "noisiness.json").read_text())
    assert noise == r["noisiness"] and noise["render"]["background_rgb"] == [6, 6, 9]
    assert [i["file"] for i in noise["images"]] == ["original.png", "iteration-01.png", "iteration-02.png"]
    assert json.loads((out_dir / "distortion.json").read_text()) == r["distortion"]
    # The last image against a fresh run of the same graph and the oracle.
    o2 = bt.Options(**{**o.__dict__, "neighbor_radius": w.radius})
    gpu = bt.Gpu(o2)
    gpu.upload(bt.Graph.load(trl))
    gpu.iterate(2)
    frame = check(oracle, gpu, o2)
    np.testing.assert_array_equal(report.read_png(out_dir / "iteration-02.png"), frame.rgba)
    assert noise["images"][-1]["colored_pixels"] == frame.colored_pixels
