"""The reports and image export of the reference's headless run, on the B200 library.

Restates src/distortion_report.rs:6-31 (the `distortion.json` schema),
src/noisiness.rs:16-138 (background calibration, the occupancy measurement
and the `noisiness.json` schema), src/report.rs:4-19 (stale-report removal and
atomic publication) and `headless` with `write_image` (src/main.rs:104-221):
upload, the baseline layout and snapshot, one frame (rendered by bt_render),
PNG and measurement per image. PNG files hold the same pixels as the
reference's frames would under this library's rasterisation rules; their
compressed bytes are this module's own (zlib, no filtering).

The JSON text follows serde_json's pretty printer as the reference uses it
(no `preserve_order` feature: object keys sorted, two-space indent, floats
in ryu's shortest form).
"""
from __future__ import annotations

import dataclasses
import math
import os
import struct
import zlib
from decimal import Decimal
from pathlib import Path

import numpy as np

from . import COLOR_BY_EDGE_ID, PALETTES, SIZE, Aggregate, BtError, Gpu, Graph, Options

__all__ = ["distortion_report", "to_json", "publish", "invalidate", "headless_distortion", "format_f64",
           "background", "measure", "NoisinessReport", "write_png", "read_png", "headless"]


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


# ---------------------------------------------------------------- noisiness
def _validate_buffer(pixels, width: int, height: int) -> int:
    """src/noisiness.rs:16-26."""
    if width <= 0 or height <= 0:
        raise BtError(3, "image dimensions must be nonzero")
    total = width * height
    if np.asarray(pixels).size != total * 4:
        raise BtError(3, f"invalid RGBA buffer length for {width}x{height}")
    return total


def background(pixels, width: int, height: int) -> list[int]:
    """The clear colour of a blank frame (src/noisiness.rs:28-42): the first
    pixel must be opaque and every pixel the same."""
    _validate_buffer(pixels, width, height)
    px = np.asarray(pixels, np.uint8).reshape(-1, 4)
    first = px[0]
    if first[3] != 255:
        raise BtError(3, "blank frame must be opaque")
    if not (px == first).all():
        raise BtError(3, "blank frame must have uniform RGB and opaque alpha")
    return [int(v) for v in first[:3]]


def measure(pixels, width: int, height: int, rgb) -> dict:
    """Occupancy of one frame (src/noisiness.rs:44-74): pixels whose RGB
    differs from `rgb`; alpha is ignored."""
    total = _validate_buffer(pixels, width, height)
    px = np.asarray(pixels, np.uint8).reshape(-1, 4)
    colored = int((px[:, :3] != np.asarray(rgb, np.uint8)).any(axis=1).sum())
    background_pixels = total - colored
    return {
        "colored_pixels": colored, "background_pixels": background_pixels, "total_pixels": total,
        "noisiness": float(colored) / float(total),
        "colored_to_background_ratio": float(colored) / float(background_pixels) if background_pixels > 0 else None,
    }


class NoisinessReport:
    """src/noisiness.rs:84-138: one measurement per exported image, written
    as `noisiness.json`."""

    def __init__(self, rgb, echo: bool = True):
        self.rgb = [int(v) for v in rgb]
        self.images: list[dict] = []
        self.echo = echo

    def record(self, pixels, file: str, iteration: int, width: int = SIZE, height: int = SIZE) -> dict:
        m = measure(pixels, width, height, self.rgb)
        original = self.images[0]["noisiness"] if self.images else m["noisiness"]
        change = m["noisiness"] - original
        if self.echo:
            print(f"noisiness {file}: {m['noisiness']:.6f}, change {change:+.6f}")
        image = {"file": file, "iteration": int(iteration), **m, "change_from_original": change}
        self.images.append(image)
        return image

    def to_dict(self, input_path: str, options: Options, width: int = SIZE, height: int = SIZE) -> dict:
        return {
            "schema_version": 1, "metric_version": 1, "metric": "noisiness",
            "definition": ("Fraction of exported pixels whose RGB differs exactly from the calibrated background. "
                           "Alpha is ignored."),
            "interpretation": ("Comparisons require identical rendering settings. Lower occupancy is not total "
                               "drawing quality. For bundling comparisons, edge-id coloring and disabled endpoint "
                               "dots are recommended; density coloring can change with geometry."),
            "input": str(input_path),
            "render": {
                "render_contract_version": 1,
                "width": width, "height": height, "format": "rgba8unorm",
                "background_rgb": self.rgb, "comparison": "rgb_exact_inequality",
                "palette": PALETTES[options.palette],
                "color_by": "edge-id" if options.color_by == COLOR_BY_EDGE_ID else "density",
                "endpoint_dots": bool(options.endpoint_dots), "msaa": int(options.msaa),
                "path_style": {"half_width_clip": 0.001, "opacity": 0.1, "endpoint_radius_pixels": 3,
                               "endpoint_outline_width_pixels": 1},
                "normalization": ("Initial graph bounds; uniform fit to 95% canvas extent; centered; unchanged "
                                  "through iterations."),
            },
            "bundling": {"neighbor_radius": options.neighbor_radius,
                         "iterations": self.images[-1]["iteration"] if self.images else 0},
            "images": self.images,
        }

    def write(self, directory, input_path: str, options: Options, width: int = SIZE, height: int = SIZE) -> dict:
        report = self.to_dict(input_path, options, width, height)
        publish(directory, "noisiness.json", report)
        return report


# ---------------------------------------------------------------- PNG
def _chunk(kind: bytes, data: bytes) -> bytes:
    return struct.pack(">I", len(data)) + kind + data + struct.pack(">I", zlib.crc32(kind + data) & 0xFFFFFFFF)


def write_png(path, rgba: np.ndarray) -> None:
    """An 8-bit RGBA PNG of a height x width x 4 frame (png::ColorType::Rgba,
    BitDepth::Eight, as write_image, src/main.rs:200-221)."""
    rgba = np.ascontiguousarray(rgba, np.uint8)
    h, w = rgba.shape[:2]
    rows = np.empty((h, 1 + 4 * w), np.uint8)
    rows[:, 0] = 0                                   # filter type None
    rows[:, 1:] = rgba.reshape(h, 4 * w)
    data = (b"\x89PNG\r\n\x1a\n" + _chunk(b"IHDR", struct.pack(">IIBBBBB", w, h, 8, 6, 0, 0, 0)) +
            _chunk(b"IDAT", zlib.compress(rows.tobytes(), 6)) + _chunk(b"IEND", b""))
    Path(path).write_bytes(data)


def read_png(path) -> np.ndarray:
    """Pixels of an 8-bit RGBA, non-interlaced PNG (any filter types)."""
    data = Path(path).read_bytes()
    if data[:8] != b"\x89PNG\r\n\x1a\n":
        raise ValueError("not a PNG file")
    pos, idat = 8, b""
    w = h = None
    while pos < len(data):
        (n,) = struct.unpack(">I", data[pos:pos + 4])
        kind, body = data[pos + 4:pos + 8], data[pos + 8:pos + 8 + n]
        pos += 12 + n
        if kind == b"IHDR":
            w, h, depth, ctype, _, _, interlace = struct.unpack(">IIBBBBB", body)
            if depth != 8 or ctype != 6 or interlace:
                raise ValueError("only 8-bit RGBA, non-interlaced PNG")
        elif kind == b"IDAT":
            idat += body
        elif kind == b"IEND":
            break
    raw = np.frombuffer(zlib.decompress(idat), np.uint8).reshape(h, 1 + 4 * w)
    if not raw[:, 0].any():                         # no filtering (what write_png stores)
        return raw[:, 1:].reshape(h, w, 4).copy()
    out = np.zeros((h, 4 * w), np.int32)
    prev = np.zeros(4 * w, np.int32)
    for y in range(h):
        ft, line = raw[y, 0], raw[y, 1:].astype(np.int32)
        cur = np.zeros(4 * w, np.int32)
        for x in range(4 * w):
            a = cur[x - 4] if x >= 4 else 0
            b = prev[x]
            c = prev[x - 4] if x >= 4 else 0
            if ft == 0:
                p = 0
            elif ft == 1:
                p = a
            elif ft == 2:
                p = b
            elif ft == 3:
                p = (a + b) // 2
            else:
                pa, pb, pc = abs(b - c), abs(a - c), abs(a + b - 2 * c)
                p = a if pa <= pb and pa <= pc else (b if pb <= pc else c)
            cur[x] = (line[x] + p) & 0xFF
        out[y] = cur
        prev = cur
    return out.astype(np.uint8).reshape(h, w, 4)


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


def headless(input_path, out_dir, neighbor_radius: int | None = None, iterations: int = 1,
             options: Options | None = None, evaluate_noisiness: bool = False, evaluate_distortion: bool = False,
             measure_on: str = "device", write_images: bool = True, echo: bool = True) -> dict:
    """The reference's headless run (src/main.rs:104-221): removes stale
    reports, calibrates the noisiness background on a blank frame, loads and
    uploads the graph, validates the distortion baseline, exports
    `original.png`, then after each of `iterations` mean updates (when a
    radius is set) `neighbor-mean.png` or `iteration-NN.png`, measuring every
    frame, and publishes `noisiness.json` and `distortion.json`. Frames come
    from bt_render at the options' map size (the reference's canvas is 1600 x
    1600). `measure_on` = "device" computes the distortion integrals on the
    GPU (`bt_distortion`); "host" decodes each snapshot and aggregates edge by
    edge, as the reference does. write_images=False skips the PNG files (the
    frames are still rendered when noisiness is evaluated). Returns
    {"samples", "noisiness", "distortion"} (absent reports are None)."""
    out_dir = Path(out_dir)
    out_dir.mkdir(parents=True, exist_ok=True)
    invalidate(out_dir, "distortion.json")
    invalidate(out_dir, "noisiness.json")
    o = dataclasses.replace(options) if options is not None else Options()
    o.neighbor_radius = neighbor_radius
    o.evaluate_distortion = bool(evaluate_distortion)
    width, height = o.width, o.height
    gpu = Gpu(o)
    try:
        noise = None
        if evaluate_noisiness:
            blank = gpu.render()
            noise = NoisinessReport(background(blank.rgba, width, height), echo=echo)
        graph = Graph.load(input_path)
        samples = gpu.upload(graph)
        layout = baseline = None
        if evaluate_distortion:
            layout = gpu.distortion_layout()
            baseline = gpu.distortion_snapshot(layout)
            for eid, points in baseline.edges():
                p = points.astype(np.float64)
                if not (np.hypot(*(p[1:] - p[:-1]).T).sum() > 0.0):
                    raise BtError(3, f"baseline edge {eid} has zero length")

        def write_image(name: str, iteration: int) -> None:
            if not (write_images or noise is not None):
                return
            frame = gpu.render()
            path = out_dir / name
            if write_images:
                write_png(path, frame.rgba)
            if noise is not None:
                image = noise.record(frame.rgba, name, iteration, width, height)
                if image["colored_pixels"] != frame.colored_pixels:
                    raise BtError(7, "device and host coloured-pixel counts disagree")
            if write_images and echo:
                print(f"wrote {path}")

        write_image("original.png", 0)
        images = []
        if baseline is not None:
            images.append({"file": "original.png", "iteration": 0, "distortion": 0.0, "rms_displacement_pixels": 0.0})
            if echo:
                print("original.png distortion=0 rms_displacement_pixels=0")
        if neighbor_radius is not None:
            for it in range(1, iterations + 1):
                gpu.iterate(1)
                name = "neighbor-mean.png" if iterations == 1 else f"iteration-{it:02d}.png"
                write_image(name, it)
                if baseline is None:
                    continue
                if measure_on == "host":
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
        noisiness = noise.write(out_dir, str(input_path), o, width, height) if noise is not None else None
        distortion = None
        if layout is not None:
            distortion = distortion_report(input_path, layout, images, neighbor_radius, iterations)
            publish(out_dir, "distortion.json", distortion)
        if echo:
            print(f"rendered {samples} samples to {out_dir}")
        return {"samples": samples, "noisiness": noisiness, "distortion": distortion}
    finally:
        gpu.close()


def headless_distortion(input_path, out_dir, neighbor_radius: int | None = None, iterations: int = 1,
                        options: Options | None = None, measure: str = "device", echo: bool = True) -> dict:
    """The distortion part of the headless run (no images, no noisiness):
    `headless` with evaluate_distortion only. Returns the distortion report."""
    return headless(input_path, out_dir, neighbor_radius, iterations, options, evaluate_distortion=True,
                    measure_on=measure, write_images=False, echo=echo)["distortion"]
