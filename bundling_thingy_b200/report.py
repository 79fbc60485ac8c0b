"""The distortion report of the reference's headless run, on the B200 library.

Restates src/distortion_report.rs:6-31 (the `distortion.json` schema),
src/report.rs:4-19 (stale-report removal and atomic publication) and the
distortion part of `headless` (src/main.rs:104-191): upload, the baseline
layout and snapshot, one measurement per iteration. Rendering is not part of
this library, so no PNG is written; the image entries keep the file names
the reference gives its images (`original.png`, `neighbor-mean.png`,
`iteration-NN.png`) so that readers of the report find the same keys.

The JSON text follows serde_json's pretty printer as the reference uses it
(no `preserve_order` feature: object keys sorted, two-space indent, floats
in ryu's shortest form).
"""
from __future__ import annotations

import math
import os
from decimal import Decimal
from pathlib import Path

import numpy as np

from . import SIZE, Aggregate, BtError, Gpu, Graph, Options

__all__ = ["distortion_report", "to_json", "publish", "invalidate", "headless_distortion", "format_f64"]


# ---------------------------------------------------------------- JSON text
def format_f64(v: float) -> str:
    """An f64 as serde_json writes it: ryu's shortest round-trip digits d
    (value = d x 10^k, kk = len(d) + k), positional when kk <= 16 and either
    k >= 0 or kk > -5, else `d.ddde<kk-1>`; non-finite values are null."""
    if not math.isfinite(v):
        return "null"
    if v == 0.0:
        return "-0.0" if math.copysign(1.0, v) < 0 else "0.0"
    sign = "-" if v < 0 else ""
    t = Decimal(repr(abs(v))).normalize().as_tuple()   # repr: Python's shortest round-trip digits
    digits = "".join(map(str, t.digits))
    k = t.exponent
    n = len(digits)
    kk = n + k
    if 0 <= k and kk <= 16:
        return sign + digits + "0" * k + ".0"
    if 0 < kk <= 16:
        return sign + digits[:kk] + "." + digits[kk:]
    if -5 < kk <= 0:
        return sign + "0." + "0" * (-kk) + digits
    return sign + digits[0] + ("." + digits[1:] if n > 1 else "") + "e" + str(kk - 1)


def _string(s: str) -> str:
    out = ['"']
    for ch in s:
        c = ord(ch)
        if ch == '"':
            out.append('\\"')
        elif ch == "\\":
            out.append("\\\\")
        elif ch == "\n":
            out.append("\\n")
        elif ch == "\r":
            out.append("\\r")
        elif ch == "\t":
            out.append("\\t")
        elif ch == "\b":
            out.append("\\b")
        elif ch == "\f":
            out.append("\\f")
        elif c < 0x20:
            out.append(f"\\u{c:04x}")
        else:
            out.append(ch)
    out.append('"')
    return "".join(out)


def to_json(value, indent: int = 0) -> str:
    """serde_json::to_vec_pretty of a JSON value built by `json!`."""
    pad, inner = "  " * indent, "  " * (indent + 1)
    if value is None:
        return "null"
    if isinstance(value, bool):
        return "true" if value else "false"
    if isinstance(value, (int, np.integer)):
        return str(int(value))
    if isinstance(value, (float, np.floating)):
        return format_f64(float(value))
    if isinstance(value, str):
        return _string(value)
    if isinstance(value, dict):
        if not value:
            return "{}"
        items = [f"{inner}{_string(k)}: {to_json(value[k], indent + 1)}" for k in sorted(value)]
        return "{\n" + ",\n".join(items) + "\n" + pad + "}"
    if isinstance(value, (list, tuple)):
        if not value:
            return "[]"
        return "[\n" + ",\n".join(inner + to_json(v, indent + 1) for v in value) + "\n" + pad + "]"
    raise TypeError(f"not a JSON value: {type(value).__name__}")


# ---------------------------------------------------------------- report
def distortion_report(input_path: str, layout, images: list, neighbor_radius: int | None, iterations: int) -> dict:
    """The `distortion.json` object (src/distortion_report.rs:6-31)."""
    return {
        "schema_version": 1, "metric_version": 1, "metric": "distortion",
        "definition": ("Square root of the equal-edge mean integral of squared clip-coordinate displacement under "
                       "directed normalized arc-length correspondence, divided by the fixed canvas diagonal."),
        "interpretation": ("Lower means less geometric change from the original GPU-resampled geometry. Detours, "
                           "retracing, reversal and loop start changes affect correspondence. Splitting edges "
                           "changes equal-edge weighting. This is not Frechet or Hausdorff distance, topology, "
                           "ambiguity or overall quality. Color, MSAA, opacity and endpoint dots are excluded. "
                           "GPU ordering can cause run-to-run variation."),
        "input": str(input_path),
        "baseline": {
            "source": "gpu_resampled_iteration_0",
            "correspondence": "directed_edge_normalized_arc_length",
            "weighting": "equal_edges", "preprocessing_distortion_included": False,
        },
        "geometry": {
            "geometry_contract_version": 1, "coordinate_space": "clip",
            "width": SIZE, "height": SIZE,
            "normalization": "initial graph bounds, centered uniform 95% fit, unchanged through iterations",
            "diagonal_clip_units": 2.0 * math.sqrt(2.0),
            "pixels_per_clip_unit": float(SIZE) / 2.0,
            "edges_total": layout.edge_count + layout.skipped_count,
            "edges_evaluated": layout.edge_count, "edges_skipped": layout.skipped_count,
            "active_samples": layout.samples,
        },
        "bundling": {"neighbor_radius": neighbor_radius, "iterations": iterations if neighbor_radius is not None else 0},
        "images": images,
    }


def invalidate(directory, file: str) -> None:
    """Removes a stale report (src/report.rs:4-11)."""
    try:
        os.remove(Path(directory) / file)
    except FileNotFoundError:
        pass


def publish(directory, file: str, report: dict) -> None:
    """Writes the report to a temporary file and renames it into place
    (src/report.rs:13-19)."""
    path = Path(directory) / file
    temporary = Path(directory) / f"{file}.tmp"
    temporary.write_bytes(to_json(report).encode("utf-8"))
    os.replace(temporary, path)


def _rust_display(v: float) -> str:
    """f64 as Rust's `{}` prints it (shortest digits, never an exponent)."""
    if v == 0.0:
        return "0"
    s = format_f64(v)
    if "e" in s:
        m, e = s.split("e")
        sign = "-" if m.startswith("-") else ""
        m = m.lstrip("-")
        digits = m.replace(".", "")
        point = (m.index(".") if "." in m else len(m)) + int(e)
        if point <= 0:
            s = sign + "0." + "0" * (-point) + digits
        elif point >= len(digits):
            s = sign + digits + "0" * (point - len(digits))
        else:
            s = sign + digits[:point] + "." + digits[point:]
        return s
    return s[:-2] if s.endswith(".0") else s


def headless_distortion(input_path, out_dir, neighbor_radius: int | None = None, iterations: int = 1,
                        options: Options | None = None, measure: str = "device", echo: bool = True) -> dict:
    """The distortion part of the reference's headless run (src/main.rs:104-191):
    invalidates a stale `distortion.json`, loads and uploads the graph,
    validates the baseline, iterates `iterations` times when a radius is
    set, measures each iteration against the baseline, and publishes the
    report. `measure` = "device" computes the per-edge integrals on the GPU
    (`bt_distortion`); "host" decodes each snapshot and aggregates edge by
    edge on the host, as the reference does. Returns the report."""
    out_dir = Path(out_dir)
    out_dir.mkdir(parents=True, exist_ok=True)
    invalidate(out_dir, "distortion.json")
    o = options if options is not None else Options()
    o.neighbor_radius = neighbor_radius
    o.evaluate_distortion = True
    gpu = Gpu(o)
    try:
        graph = Graph.load(input_path)
        samples = gpu.upload(graph)
        layout = gpu.distortion_layout()
        baseline = gpu.distortion_snapshot(layout)
        for eid, points in baseline.edges():
            p = points.astype(np.float64)
            if not (np.hypot(*(p[1:] - p[:-1]).T).sum() > 0.0):
                raise BtError(3, f"baseline edge {eid} has zero length")
        images = [{"file": "original.png", "iteration": 0, "distortion": 0.0, "rms_displacement_pixels": 0.0}]
        if echo:
            print("original.png distortion=0 rms_displacement_pixels=0")
        if neighbor_radius is not None:
            for it in range(1, iterations + 1):
                gpu.iterate(1)
                name = "neighbor-mean.png" if iterations == 1 else f"iteration-{it:02d}.png"
                if measure == "host":
                    current = gpu.distortion_snapshot(layout)
                    agg = Aggregate()
                    for (_, a), (_, b) in zip(baseline.edges(), current.edges()):
                        agg.add(a, b)
                    m = agg.finish(SIZE)
                else:
                    m = gpu.distortion(SIZE)
                images.append({"file": name, "iteration": it, "distortion": m.distortion,
                               "rms_displacement_pixels": m.rms_displacement_pixels})
                if echo:
                    print(f"{name} distortion={_rust_display(m.distortion)} "
                          f"rms_displacement_pixels={_rust_display(m.rms_displacement_pixels)}")
        report = distortion_report(input_path, layout, images, neighbor_radius, iterations)
        publish(out_dir, "distortion.json", report)
        if echo:
            print(f"rendered {samples} samples to {out_dir}")
        return report
    finally:
        gpu.close()
