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
