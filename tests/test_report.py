"""distortion.json text and layout (src/distortion_report.rs, src/report.rs), no GPU."""
import json
import math

import pytest

from bundling_thingy_b200 import report


@pytest.mark.parametrize("value,text", [
    (0.0, "0.0"), (-0.0, "-0.0"), (1.0, "1.0"), (800.0, "800.0"), (2.0 * math.sqrt(2.0), "2.8284271247461903"),
    (0.001234, "0.001234"), (1e-5, "0.00001"), (1.5e-7, "1.5e-7"), (1e-7, "1e-7"), (1e15, "1000000000000000.0"), (1e16, "1e16"),
    (1.5e16, "1.5e16"), (1e17, "1e17"), (123456789.125, "123456789.125"), (-2.5, "-2.5"),
    (5e-324, "5e-324"), (float("nan"), "null"),
])
def test_floats_are_written_like_serde_json(value, text):
    assert report.format_f64(value) == text
    if math.isfinite(value):
        assert float(text) == value


def test_pretty_printer_sorts_keys_and_indents_two_spaces():
    text = report.to_json({"b": [1, {"d": None, "c": True}], "a": "x\"y\n", "e": {}, "f": []})
    assert text == ('{\n  "a": "x\\"y\\n",\n  "b": [\n    1,\n    {\n      "c": true,\n      "d": null\n    }\n'
                    '  ],\n  "e": {},\n  "f": []\n}')
    assert json.loads(text) == {"b": [1, {"d": None, "c": True}], "a": "x\"y\n", "e": {}, "f": []}


class _Layout:
    edge_count, skipped_count, samples = 7, 2, 123


def test_report_schema_and_publication(tmp_path):
    images = [{"file": "original.png", "iteration": 0, "distortion": 0.0, "rms_displacement_pixels": 0.0}]
    r = report.distortion_report("data/g.trl", _Layout(), images, None, 5)
    assert r["bundling"] == {"neighbor_radius": None, "iterations": 0}
    assert r["geometry"]["edges_total"] == 9 and r["geometry"]["active_samples"] == 123
    assert r["geometry"]["diagonal_clip_units"] == 2.0 * math.sqrt(2.0)
    assert r["geometry"]["pixels_per_clip_unit"] == 800.0
    report.invalidate(tmp_path, "distortion.json")          # nothing to remove: no error
    report.publish(tmp_path, "distortion.json", r)
    assert not (tmp_path / "distortion.json.tmp").exists()
    text = (tmp_path / "distortion.json").read_text()
    assert json.loads(text) == r
    assert list(json.loads(text)) == sorted(r)              # keys in serde_json's (sorted) order
    report.invalidate(tmp_path, "distortion.json")
    assert not (tmp_path / "distortion.json").exists()


# ---------------------------------------------------------------- noisiness (src/noisiness.rs)
import struct
import zlib

import numpy as np

import bundling_thingy_b200 as bt


def _frame(w, h, rgb=(6, 6, 9)):
    f = np.zeros((h, w, 4), np.uint8)
    f[..., :3] = rgb
    f[..., 3] = 255
    return f


def test_background_requires_an_opaque_uniform_frame():
    assert report.background(_frame(5, 3), 5, 3) == [6, 6, 9]
    f = _frame(5, 3)
    f[0, 0, 3] = 254
    with pytest.raises(bt.BtError, match="opaque"):
        report.background(f, 5, 3)
    f = _frame(5, 3)
    f[2, 4, 1] = 7
    with pytest.raises(bt.BtError, match="uniform"):
        report.background(f, 5, 3)
    with pytest.raises(bt.BtError, match="invalid RGBA buffer length"):
        report.background(_frame(5, 3), 5, 4)
    with pytest.raises(bt.BtError, match="nonzero"):
        report.background(_frame(5, 3), 0, 3)


def test_measure_counts_rgb_differences_and_ignores_alpha():
    f = _frame(4, 4)
    f[0, 0, 3] = 0            # alpha only: not coloured
    f[1, 1, 0] = 7
    f[2, 3] = (6, 6, 10, 255)
    m = report.measure(f, 4, 4, [6, 6, 9])
    assert m == {"colored_pixels": 2, "background_pixels": 14, "total_pixels": 16, "noisiness": 2 / 16,
                 "colored_to_background_ratio": 2 / 14}
    full = report.measure(_frame(2, 2, (1, 2, 3)), 2, 2, [6, 6, 9])
    assert full["noisiness"] == 1.0 and full["colored_to_background_ratio"] is None


def test_noisiness_report_schema_and_echo(tmp_path, capsys):
    r = report.NoisinessReport([6, 6, 9])
    a = _frame(10, 10)
    a[0, :3, 0] = 50
    b = _frame(10, 10)
    b[0, :5, 0] = 50
    r.record(a, "original.png", 0, 10, 10)
    r.record(b, "neighbor-mean.png", 1, 10, 10)
    out = capsys.readouterr().out.splitlines()
    assert out == ["noisiness original.png: 0.030000, change +0.000000",
                   "noisiness neighbor-mean.png: 0.050000, change +0.020000"]
    o = bt.Options(neighbor_radius=4, color_by=bt.COLOR_BY_EDGE_ID, palette=3, msaa=2)
    d = r.write(tmp_path, "data/g.trl", o, 10, 10)
    text = (tmp_path / "noisiness.json").read_text()
    assert json.loads(text) == d
    assert d["render"]["palette"] == "batlow" and d["render"]["color_by"] == "edge-id"
    assert d["render"]["msaa"] == 2 and d["render"]["endpoint_dots"] is False
    assert d["render"]["background_rgb"] == [6, 6, 9]
    assert d["bundling"] == {"neighbor_radius": 4, "iterations": 1}
    img = d["images"][1]
    assert sorted(img) == ["background_pixels", "change_from_original", "colored_pixels",
                           "colored_to_background_ratio", "file", "iteration", "noisiness", "total_pixels"]
    assert img["change_from_original"] == 0.05 - 0.03
    # serde_json text: "path_style" keys sorted, integers stay integers.
    assert '"endpoint_radius_pixels": 3,' in text and '"half_width_clip": 0.001,' in text


def _png_with_filters(img):
    """A PNG of img whose rows use filter types 0..4 in turn (test helper)."""
    h, w = img.shape[:2]
    rows = img.reshape(h, 4 * w).astype(np.int32)
    out = bytearray()
    prev = np.zeros(4 * w, np.int32)
    for y in range(h):
        ft = y % 5
        cur = rows[y]
        a = np.concatenate([np.zeros(4, np.int32), cur[:-4]])
        c = np.concatenate([np.zeros(4, np.int32), prev[:-4]])
        b = prev
        if ft == 0:
            p = np.zeros_like(cur)
        elif ft == 1:
            p = a
        elif ft == 2:
            p = b
        elif ft == 3:
            p = (a + b) // 2
        else:
            pa, pb, pc = np.abs(b - c), np.abs(a - c), np.abs(a + b - 2 * c)
            p = np.where((pa <= pb) & (pa <= pc), a, np.where(pb <= pc, b, c))
        out.append(ft)
        out += ((cur - p) & 0xFF).astype(np.uint8).tobytes()
        prev = cur

    def chunk(k, d):
        return struct.pack(">I", len(d)) + k + d + struct.pack(">I", zlib.crc32(k + d) & 0xFFFFFFFF)

    return (b"\x89PNG\r\n\x1a\n" + chunk(b"IHDR", struct.pack(">IIBBBBB", w, h, 8, 6, 0, 0, 0)) +
            chunk(b"IDAT", zlib.compress(bytes(out))) + chunk(b"IEND", b""))


def test_png_round_trip(tmp_path):
    rng = np.random.default_rng(3)
    img = rng.integers(0, 256, (23, 17, 4), dtype=np.uint8)
    report.write_png(tmp_path / "a.png", img)
    data = (tmp_path / "a.png").read_bytes()
    assert data[:8] == b"\x89PNG\r\n\x1a\n" and data[12:16] == b"IHDR" and data[-8:-4] == b"IEND"
    np.testing.assert_array_equal(report.read_png(tmp_path / "a.png"), img)
    (tmp_path / "b.png").write_bytes(_png_with_filters(img))
    np.testing.assert_array_equal(report.read_png(tmp_path / "b.png"), img)
