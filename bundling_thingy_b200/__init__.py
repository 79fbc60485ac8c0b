"""B200-native edge bundling: Python mirror of lpstankus/bundling_thingy's API.

The compute path is ``libbt.so`` (CUDA for sm_100a, C ABI in ``include/bt.h``);
this module only binds it with ctypes. There is no CPU fallback: every call
that computes goes through the library, and constructing a :class:`Gpu` fails
loudly when the library or a CUDA device is missing.

Names follow the reference:

* :class:`Graph` — ``Graph::load/parse/normalization/points/starts``
  (src/graph.rs).
* :class:`Gpu` — ``Gpu::new/upload/iterate/distortion_layout/
  distortion_snapshot`` (src/gpu.rs), plus device readbacks.
* :class:`Layout`, :func:`squared_integral`, :class:`Aggregate` —
  ``bundling_wgpu::geometry`` and ``bundling_wgpu::distortion``.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

__all__ = [
    "BtError", "Options", "Graph", "Gpu", "Batch", "Info", "Layout", "Snapshot", "Aggregate", "Measurement",
    "squared_integral", "library", "library_path", "build", "COLOR_BY_DENSITY", "COLOR_BY_EDGE_ID", "SIZE",
    "Frame", "PALETTES",
]

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "libbt.so")
SIZE = 1600                      # headless canvas of the reference (src/gpu.rs:21)
COLOR_BY_DENSITY = 0
COLOR_BY_EDGE_ID = 1
PALETTES = ("viridis", "cividis", "plasma", "batlow")   # bt_options.palette index -> --palette name

_f32p = ctypes.POINTER(ctypes.c_float)
_u32p = ctypes.POINTER(ctypes.c_uint32)
_f64p = ctypes.POINTER(ctypes.c_double)
_vp = ctypes.c_void_p
_u8p = ctypes.POINTER(ctypes.c_uint8)

STATUS = {
    0: "ok", 1: "capacity overflow", 2: "count/emit mismatch", 3: "invalid input", 4: "no graph",
    5: "memory budget", 6: "timeout", 7: "CUDA error", 8: "not configured", 9: "cancelled",
}


class BtError(RuntimeError):
    """A non-zero bt_status with the library's message."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{message} [{STATUS.get(status, status)}]")
        self.status = status
        self.message = message


class _Options(ctypes.Structure):
    _fields_ = [
        ("width", ctypes.c_uint32), ("height", ctypes.c_uint32), ("neighbor_radius", ctypes.c_uint32),
        ("color_by", ctypes.c_uint32), ("max_graph_memory_bytes", ctypes.c_uint64),
        ("evaluate_distortion", ctypes.c_uint32), ("device", ctypes.c_int32),
        ("sample_spacing", ctypes.c_float), ("blur_sigma", ctypes.c_float), ("blur_shrink", ctypes.c_float),
        ("fine_cells", ctypes.c_uint32), ("use_graphs", ctypes.c_uint32), ("timing", ctypes.c_uint32),
        ("record_neighbors", ctypes.c_uint32), ("search_mode", ctypes.c_uint32), ("fine_cells_x", ctypes.c_uint32),
        ("palette", ctypes.c_uint32), ("msaa", ctypes.c_uint32), ("endpoint_dots", ctypes.c_uint32),
        ("advect_step", ctypes.c_float), ("advect_smooth", ctypes.c_float), ("wait_seconds", ctypes.c_float),
        ("shape_checks", ctypes.c_uint32),
    ]


class _Info(ctypes.Structure):
    _fields_ = [
        ("samples", ctypes.c_uint32), ("paths", ctypes.c_uint32), ("drawn_paths", ctypes.c_uint32),
        ("segments", ctypes.c_uint32), ("capacity", ctypes.c_uint32), ("iterations", ctypes.c_uint32),
        ("grid_width", ctypes.c_uint32), ("grid_height", ctypes.c_uint32), ("fine_cells", ctypes.c_uint32),
        ("density_passes", ctypes.c_uint32), ("device_bytes", ctypes.c_uint64), ("reserved_bytes", ctypes.c_uint64),
        ("fine_cells_x", ctypes.c_uint32), ("reserved0", ctypes.c_uint32),
    ]


class _ServerOptions(ctypes.Structure):
    _fields_ = [
        ("device", ctypes.c_int32), ("max_active", ctypes.c_uint32), ("budget_bytes", ctypes.c_uint64),
        ("max_step", ctypes.c_uint32), ("solo_samples", ctypes.c_uint32), ("reserve_bytes", ctypes.c_uint64),
        ("queue_timeout_ms", ctypes.c_uint32), ("reserved", ctypes.c_uint32 * 3),
    ]


class _RequestResult(ctypes.Structure):
    _fields_ = [
        ("id", ctypes.c_uint64), ("status", ctypes.c_int32), ("samples", ctypes.c_uint32),
        ("iterations", ctypes.c_uint32), ("reserved0", ctypes.c_uint32), ("arrival_s", ctypes.c_double),
        ("admitted_s", ctypes.c_double), ("finished_s", ctypes.c_double), ("device_bytes", ctypes.c_uint64),
        ("message", ctypes.c_char * 160),
    ]


class _ServerStats(ctypes.Structure):
    _fields_ = [
        ("submitted", ctypes.c_uint64), ("finished", ctypes.c_uint64), ("failed", ctypes.c_uint64),
        ("steps", ctypes.c_uint64), ("rebuilds", ctypes.c_uint64), ("budget_waits", ctypes.c_uint64),
        ("evictions", ctypes.c_uint64), ("queued", ctypes.c_uint32), ("active", ctypes.c_uint32),
        ("peak_active", ctypes.c_uint32), ("resident_results", ctypes.c_uint32), ("device_bytes", ctypes.c_uint64),
        ("peak_device_bytes", ctypes.c_uint64), ("launch_s", ctypes.c_double), ("upload_s", ctypes.c_double),
        ("wait_s", ctypes.c_double), ("retire_s", ctypes.c_double), ("idle_s", ctypes.c_double),
        ("contexts_created", ctypes.c_uint64), ("create_s", ctypes.c_double),
    ]


# Every entry point of include/bt.h with its ctypes signature.
SIGNATURES = {
    "bt_abi_version": ([], ctypes.c_int32),
    "bt_options_init": ([ctypes.POINTER(_Options)], None),
    "bt_create": ([ctypes.POINTER(_Options), ctypes.POINTER(_vp)], ctypes.c_int32),
    "bt_destroy": ([_vp], None),
    "bt_last_error": ([_vp], ctypes.c_char_p),
    "bt_upload": ([_vp, _f32p, ctypes.c_uint32, _u32p, ctypes.c_uint32, _u32p], ctypes.c_int32),
    "bt_upload_graph": ([_vp, _vp, _u32p], ctypes.c_int32),
    "bt_iterate": ([_vp, ctypes.c_uint32], ctypes.c_int32),
    "bt_iterate_async": ([_vp, ctypes.c_uint32], ctypes.c_int32),
    "bt_synchronize": ([_vp], ctypes.c_int32),
    "bt_iterate_timed": ([_vp, ctypes.c_uint32, _f32p], ctypes.c_int32),
    "bt_get_info": ([_vp, ctypes.POINTER(_Info)], ctypes.c_int32),
    "bt_set_wait_seconds": ([_vp, ctypes.c_float], ctypes.c_int32),
    "bt_read_points": ([_vp, _vp, ctypes.c_size_t], ctypes.c_int32),
    "bt_read_paths": ([_vp, _vp, ctypes.c_size_t], ctypes.c_int32),
    "bt_restore_points": ([_vp, _vp, ctypes.c_size_t, ctypes.c_uint32], ctypes.c_int32),
    "bt_read_segments": ([_vp, _u32p, ctypes.c_size_t], ctypes.c_int32),
    "bt_read_edges": ([_vp, _f32p, ctypes.c_size_t], ctypes.c_int32),
    "bt_read_density": ([_vp, _f32p, ctypes.c_size_t], ctypes.c_int32),
    "bt_read_density_raw": ([_vp, _f32p, ctypes.c_size_t, _f32p], ctypes.c_int32),
    "bt_read_counts": ([_vp, _u32p, ctypes.c_size_t], ctypes.c_int32),
    "bt_read_cells": ([_vp, _u32p, ctypes.c_size_t], ctypes.c_int32),
    "bt_search_stats": ([_vp, ctypes.c_uint32, ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64),
                         ctypes.POINTER(ctypes.c_uint64)], ctypes.c_int32),
    "bt_read_binning": ([_vp, _u32p, ctypes.c_size_t, _u32p, ctypes.c_size_t], ctypes.c_int32),
    "bt_read_neighbors": ([_vp, _u32p, ctypes.c_size_t], ctypes.c_int32),
    "bt_distortion": ([_vp, ctypes.c_uint32, _f64p, _f64p], ctypes.c_int32),
    "bt_render": ([_vp, _u8p, ctypes.c_size_t, ctypes.POINTER(ctypes.c_uint64), _f32p], ctypes.c_int32),
    "bt_stage_times": ([_vp, ctypes.POINTER(ctypes.c_char_p), _f32p, ctypes.c_uint32, _u32p], ctypes.c_int32),
    "bt_density_noalloc": ([_vp, _vp, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_float, _vp], ctypes.c_int32),
    "bt_autotune": ([ctypes.POINTER(_Options), _f32p, ctypes.c_uint32, _u32p, ctypes.c_uint32, ctypes.c_uint32,
                     ctypes.POINTER(_Options), _f32p], ctypes.c_int32),
    "bt_batch_create": ([ctypes.c_int32, ctypes.POINTER(_vp)], ctypes.c_int32),
    "bt_batch_destroy": ([_vp], None),
    "bt_batch_last_error": ([_vp], ctypes.c_char_p),
    "bt_batch_add": ([_vp, ctypes.POINTER(_Options), _f32p, ctypes.c_uint32, _u32p, ctypes.c_uint32, _u32p, _u32p],
                     ctypes.c_int32),
    "bt_batch_add_many": ([_vp, ctypes.c_uint32, ctypes.POINTER(_Options), ctypes.POINTER(_f32p), _u32p,
                           ctypes.POINTER(_u32p), _u32p, _u32p, _u32p], ctypes.c_int32),
    "bt_batch_remove": ([_vp, ctypes.c_uint32], ctypes.c_int32),
    "bt_batch_iterate": ([_vp, ctypes.c_uint32], ctypes.c_int32),
    "bt_batch_iterate_async": ([_vp, ctypes.c_uint32], ctypes.c_int32),
    "bt_batch_synchronize": ([_vp], ctypes.c_int32),
    "bt_batch_iterate_timed": ([_vp, ctypes.c_uint32, _f32p], ctypes.c_int32),
    "bt_batch_slot_count": ([_vp, _u32p, _u32p], ctypes.c_int32),
    "bt_batch_set_solo_samples": ([_vp, ctypes.c_uint32], ctypes.c_int32),
    "bt_batch_slot": ([_vp, ctypes.c_uint32], _vp),
    "bt_batch_set_shape": ([_vp, ctypes.c_uint32, ctypes.c_uint32], ctypes.c_int32),
    "bt_batch_get_shape": ([_vp, _u32p, _u32p], ctypes.c_int32),
    "bt_batch_autotune": ([ctypes.c_int32, ctypes.c_uint32, ctypes.POINTER(_Options), ctypes.POINTER(_f32p), _u32p,
                           ctypes.POINTER(_u32p), _u32p, ctypes.c_uint32, _u32p, _u32p, _f32p], ctypes.c_int32),
    "bt_server_options_init": ([ctypes.POINTER(_ServerOptions)], None),
    "bt_server_create": ([ctypes.POINTER(_ServerOptions), ctypes.POINTER(_vp)], ctypes.c_int32),
    "bt_server_destroy": ([_vp], None),
    "bt_server_last_error": ([_vp], ctypes.c_char_p),
    "bt_server_clock": ([_vp], ctypes.c_double),
    "bt_server_submit": ([_vp, ctypes.POINTER(_Options), _f32p, ctypes.c_uint32, _u32p, ctypes.c_uint32,
                          ctypes.c_uint32, ctypes.c_double, ctypes.POINTER(ctypes.c_uint64)], ctypes.c_int32),
    "bt_server_next": ([_vp, ctypes.c_double, ctypes.POINTER(_RequestResult)], ctypes.c_int32),
    "bt_server_read_points": ([_vp, ctypes.c_uint64, _vp, ctypes.c_size_t], ctypes.c_int32),
    "bt_server_result": ([_vp, ctypes.c_uint64], _vp),
    "bt_server_release": ([_vp, ctypes.c_uint64], ctypes.c_int32),
    "bt_server_cancel": ([_vp, ctypes.c_uint64], ctypes.c_int32),
    "bt_server_stats_get": ([_vp, ctypes.POINTER(_ServerStats)], ctypes.c_int32),
    "bt_graph_parse": ([ctypes.c_char_p, ctypes.c_size_t, ctypes.POINTER(_vp)], ctypes.c_int32),
    "bt_graph_load": ([ctypes.c_char_p, ctypes.POINTER(_vp)], ctypes.c_int32),
    "bt_graph_free": ([_vp], None),
    "bt_graph_point_count": ([_vp], ctypes.c_uint32),
    "bt_graph_start_count": ([_vp], ctypes.c_uint32),
    "bt_graph_points": ([_vp], _f32p),
    "bt_graph_starts": ([_vp], _u32p),
    "bt_graph_normalization": ([_vp, _f32p], ctypes.c_int32),
    "bt_layout_check": ([_u32p, ctypes.c_uint32, ctypes.c_uint32], ctypes.c_int32),
    "bt_decode_points": ([_u32p, ctypes.c_uint32, ctypes.c_uint32, _vp, ctypes.c_size_t, _f32p], ctypes.c_int32),
    "bt_squared_integral": ([_f32p, ctypes.c_size_t, _f32p, ctypes.c_size_t, _f64p], ctypes.c_int32),
}

_lib = None


def library_path() -> str:
    return _LIB


def build() -> None:
    """Compile libbt.so in-tree for sm_100a (nvcc cross-compiles without a GPU)."""
    subprocess.run(["make", "-s", "-C", os.path.join(_HERE, "csrc"), "-j8"], check=True)


def library():
    """The loaded libbt.so; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB):
            raise ImportError(f"libbt.so is missing at {_LIB}; build it with bundling_thingy_b200.build()")
        lib = ctypes.CDLL(_LIB)
        for name, (args, res) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.argtypes = args
            fn.restype = res
        _lib = lib
    return _lib


def _check(status: int, handle=None) -> None:
    if status:
        msg = library().bt_last_error(handle)
        raise BtError(status, msg.decode() if msg else "")


def _p(a: np.ndarray, t):
    return a.ctypes.data_as(t)


@dataclass
class Options:
    """Options of ``Gpu::new`` (src/main.rs:34-90) plus this library's extensions.

    ``sample_spacing`` (fraction of the canvas; 0 = one texel), ``blur_sigma``
    (texels; 0 = the reference's fixed sigma-6 taps) and ``blur_shrink``
    (sigma factor per density pass) default to the reference behaviour.
    """

    width: int = SIZE
    height: int = SIZE
    neighbor_radius: int | None = None
    color_by: int = COLOR_BY_DENSITY
    max_graph_memory_mib: int = 1024
    evaluate_distortion: bool = False
    device: int = 0
    sample_spacing: float = 0.0
    blur_sigma: float = 0.0
    blur_shrink: float = 1.0
    fine_cells: int = 0
    use_graphs: bool = True
    timing: bool = False
    record_neighbors: bool = False
    search_mode: int = 0     # 0: interior cells by prefix sums; 1: test every candidate (same results)
    fine_cells_x: int = 0    # search cells per grid cell along x (0 = fine_cells)
    palette: int = 0         # PALETTES index (src/palette.rs:13-23): viridis, the reference default
    msaa: int = 4            # samples per pixel: 2 or 4 as the reference (1 accepted)
    endpoint_dots: bool = False
    advect_step: float = 0.0     # > 0: density-gradient advection (texels per iteration) instead of the mean
    advect_smooth: float = 0.0   # its Laplacian relaxation along the path, in [0, 1]
    wait_seconds: float = 0.0    # host deadline of blocking calls (0 = 60 s, Gpu::wait, src/gpu.rs:484-490)
    shape_checks: bool = False   # re-check the search-cell shape during a job (iterate / iterate_timed)

    def _struct(self) -> _Options:
        o = _Options()
        library().bt_options_init(ctypes.byref(o))
        o.width, o.height = self.width, self.height
        o.neighbor_radius = self.neighbor_radius or 0
        o.color_by = self.color_by
        o.max_graph_memory_bytes = int(self.max_graph_memory_mib) * 1024 * 1024
        o.evaluate_distortion = int(bool(self.evaluate_distortion))
        o.device = self.device
        o.sample_spacing = self.sample_spacing
        o.blur_sigma = self.blur_sigma
        o.blur_shrink = self.blur_shrink
        o.fine_cells = self.fine_cells
        o.use_graphs = int(bool(self.use_graphs))
        o.timing = int(bool(self.timing))
        o.record_neighbors = int(bool(self.record_neighbors))
        o.search_mode = int(self.search_mode)
        o.fine_cells_x = self.fine_cells_x
        o.palette = int(self.palette)
        o.msaa = int(self.msaa)
        o.endpoint_dots = int(bool(self.endpoint_dots))
        o.advect_step = float(self.advect_step)
        o.advect_smooth = float(self.advect_smooth)
        o.wait_seconds = float(self.wait_seconds)
        o.shape_checks = int(bool(self.shape_checks))
        return o

    def resample_scale(self) -> tuple[float, float]:
        """The resampling texel_scale the library derives (resampling.wgsl:87)."""
        if self.sample_spacing > 0:
            s = float(np.float32(0.5 / float(np.float32(self.sample_spacing))))
            return s, s
        return (float(np.float32(self.width - 1) * np.float32(0.5)),
                float(np.float32(self.height - 1) * np.float32(0.5)))


class Graph:
    """Parsed trail graph (src/graph.rs:7-107)."""

    def __init__(self, handle):
        self._h = handle

    @classmethod
    def parse(cls, text: str | bytes) -> "Graph":
        data = text.encode() if isinstance(text, str) else bytes(text)
        h = _vp()
        _check(library().bt_graph_parse(data, len(data), ctypes.byref(h)))
        return cls(h)

    @classmethod
    def load(cls, path: str | os.PathLike) -> "Graph":
        h = _vp()
        _check(library().bt_graph_load(os.fsencode(path), ctypes.byref(h)))
        return cls(h)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and _lib is not None:
            _lib.bt_graph_free(h)
            self._h = None

    def points(self) -> np.ndarray:
        n = library().bt_graph_point_count(self._h)
        ptr = library().bt_graph_points(self._h)
        return np.ctypeslib.as_array(ptr, shape=(n * 2,)).copy().reshape(-1, 2) if n else np.zeros((0, 2), np.float32)

    def starts(self) -> np.ndarray:
        n = library().bt_graph_start_count(self._h)
        ptr = library().bt_graph_starts(self._h)
        return np.ctypeslib.as_array(ptr, shape=(n,)).copy()

    def normalization(self) -> np.ndarray:
        out = np.zeros(5, np.float32)
        _check(library().bt_graph_normalization(self._h, _p(out, _f32p)))
        return out


@dataclass
class Info:
    samples: int
    paths: int
    drawn_paths: int
    segments: int
    capacity: int
    iterations: int
    grid_width: int
    grid_height: int
    fine_cells: int
    density_passes: int
    device_bytes: int
    reserved_bytes: int
    fine_cells_x: int
    reserved0: int


class Gpu:
    """The reference's ``Gpu`` (src/gpu.rs:24-720), compute parts only."""

    def __init__(self, options: Options | None = None):
        self.options = options or Options()
        h = _vp()
        o = self.options._struct()
        _check(library().bt_create(ctypes.byref(o), ctypes.byref(h)))
        self._h = h

    def close(self) -> None:
        h = getattr(self, "_h", None)
        if h and _lib is not None:
            _lib.bt_destroy(h)
        self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _ck(self, status: int) -> None:
        _check(status, self._h)

    # -- Gpu::upload / iterate --
    def upload(self, graph: "Graph | tuple[np.ndarray, np.ndarray]") -> int:
        """Gpu::upload (src/gpu.rs:493-525); returns the sample count."""
        n = ctypes.c_uint32()
        if isinstance(graph, Graph):
            self._ck(library().bt_upload_graph(self._h, graph._h, ctypes.byref(n)))
        else:
            xy, starts = graph
            xy = np.ascontiguousarray(xy, np.float32)
            starts = np.ascontiguousarray(starts, np.uint32)
            self._ck(library().bt_upload(self._h, _p(xy, _f32p), xy.size // 2, _p(starts, _u32p), starts.size,
                                         ctypes.byref(n)))
        return n.value

    def iterate(self, n: int = 1) -> None:
        """Gpu::iterate (src/gpu.rs:527-553), n times."""
        self._ck(library().bt_iterate(self._h, n))

    def iterate_async(self, n: int = 1) -> None:
        self._ck(library().bt_iterate_async(self._h, n))

    def iterate_timed(self, n: int = 1) -> float:
        """Gpu::iterate n times; returns device milliseconds (CUDA events on
        the context's stream)."""
        ms = np.zeros(1, np.float32)
        self._ck(library().bt_iterate_timed(self._h, n, _p(ms, _f32p)))
        return float(ms[0])

    def synchronize(self) -> None:
        self._ck(library().bt_synchronize(self._h))

    def set_wait_seconds(self, seconds: float) -> None:
        """Host deadline of the blocking calls that follow (0 = 60 s, as
        Gpu::wait, src/gpu.rs:484-490); past it they raise BtError with
        status 6 and the queued work still finishes on the device."""
        self._ck(library().bt_set_wait_seconds(self._h, float(seconds)))
        self.options.wait_seconds = float(seconds)

    def info(self) -> Info:
        i = _Info()
        self._ck(library().bt_get_info(self._h, ctypes.byref(i)))
        return Info(*(getattr(i, f) for f, _ in _Info._fields_))

    # -- readbacks --
    def read_records(self, out: np.ndarray | None = None) -> np.ndarray:
        """Raw 12-byte {x, y, edge_id} records (sample order). `out`, when
        given, is a C-contiguous host array of at least 12 bytes per sample
        (pinned memory reads fastest); the view of it that was filled is
        returned."""
        n = self.info().samples
        if out is None:
            out = np.zeros(n * 12, np.uint8)
        else:
            if not out.flags.c_contiguous or out.nbytes < n * 12:
                raise ValueError("record buffer must be C-contiguous with 12 bytes per sample")
            out = out.reshape(-1).view(np.uint8)[: n * 12]
        self._ck(library().bt_read_points(self._h, out.ctypes.data, out.size))
        return out

    def read_points(self) -> tuple[np.ndarray, np.ndarray]:
        rec = self.read_records().view(np.uint32).reshape(-1, 3)
        return rec[:, :2].copy().view(np.float32), rec[:, 2].copy()

    def restore_points(self, records: np.ndarray, iterations: int) -> None:
        """Resume from a checkpoint: `records` are the 12-byte records that
        read_records returned after `iterations` iterations of this graph (it
        must be uploaded again with the same options first); iterating on
        then gives the results of an uninterrupted run."""
        rec = np.ascontiguousarray(records).reshape(-1).view(np.uint8)
        self._ck(library().bt_restore_points(self._h, rec.ctypes.data, rec.size, iterations))

    def read_paths(self) -> np.ndarray:
        n = self.info().paths
        out = np.zeros((n, 3), np.uint32)
        self._ck(library().bt_read_paths(self._h, out.ctypes.data, out.nbytes))
        return out

    def read_segments(self) -> np.ndarray:
        n = self.info().segments
        out = np.zeros(n, np.uint32)
        self._ck(library().bt_read_segments(self._h, _p(out, _u32p), n))
        return out

    def read_edges(self) -> np.ndarray:
        n = self.info().paths
        out = np.zeros((n, 4), np.float32)
        self._ck(library().bt_read_edges(self._h, _p(out, _f32p), out.size))
        return out

    def read_density(self, out: np.ndarray | None = None) -> np.ndarray:
        """The normalised density map (width * height f32); `out`, when given,
        is a C-contiguous f32 host array of that size (pinned reads fastest)."""
        o = self.options
        if out is None:
            out = np.zeros(o.width * o.height, np.float32)
        elif out.dtype != np.float32 or out.size != o.width * o.height or not out.flags.c_contiguous:
            raise ValueError("density buffer must be C-contiguous f32 of width * height")
        self._ck(library().bt_read_density(self._h, _p(out, _f32p), out.size))
        return out

    def read_density_raw(self) -> tuple[np.ndarray, float]:
        o = self.options
        out = np.zeros(o.width * o.height, np.float32)
        peak = np.zeros(1, np.float32)
        self._ck(library().bt_read_density_raw(self._h, _p(out, _f32p), out.size, _p(peak, _f32p)))
        return out, float(peak[0])

    def read_counts(self) -> np.ndarray:
        o = self.options
        out = np.zeros(o.width * o.height, np.uint32)
        self._ck(library().bt_read_counts(self._h, _p(out, _u32p), out.size))
        return out

    def read_cells(self) -> np.ndarray:
        out = np.zeros(self.info().samples, np.uint32)
        self._ck(library().bt_read_cells(self._h, _p(out, _u32p), out.size))
        return out

    def read_binning(self) -> tuple[np.ndarray, np.ndarray]:
        info = self.info()
        cells = info.grid_width * info.fine_cells_x * info.grid_height * info.fine_cells
        slots = np.zeros(info.samples, np.uint32)
        starts = np.zeros(cells + 1, np.uint32)
        self._ck(library().bt_read_binning(self._h, _p(slots, _u32p), slots.size, _p(starts, _u32p), starts.size))
        return slots, starts

    def search_stats(self, stride: int = 1) -> tuple[int, int, int]:
        """(search rows, samples in boundary cells, movable samples counted)
        of the next iteration's neighbour search over every `stride`-th slot."""
        r, b, p = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
        self._ck(library().bt_search_stats(self._h, int(stride), ctypes.byref(r), ctypes.byref(b), ctypes.byref(p)))
        return int(r.value), int(b.value), int(p.value)

    def read_neighbors(self) -> np.ndarray:
        out = np.zeros(self.info().samples, np.uint32)
        self._ck(library().bt_read_neighbors(self._h, _p(out, _u32p), out.size))
        return out

    def distortion(self, size: int = SIZE) -> "Measurement":
        d = ctypes.c_double()
        r = ctypes.c_double()
        self._ck(library().bt_distortion(self._h, size, ctypes.byref(d), ctypes.byref(r)))
        return Measurement(d.value, r.value)

    def render(self, out: np.ndarray | None = None, pixels: bool = True) -> "Frame":
        """Gpu::render + Gpu::readback (src/gpu.rs:616-655): the frame as RGBA8
        (height x width x 4, rows from the top), its count of pixels whose RGB
        differs from the clear colour, and the device time of its kernels.
        Before an upload this is the blank frame. pixels=False skips the copy."""
        o = self.options
        rgba = None
        if pixels:
            rgba = out if out is not None else np.empty((o.height, o.width, 4), np.uint8)
            if rgba.dtype != np.uint8 or rgba.size != o.width * o.height * 4 or not rgba.flags.c_contiguous:
                raise ValueError("out must be a contiguous uint8 array of height x width x 4")
        colored = ctypes.c_uint64()
        ms = np.zeros(1, np.float32)
        self._ck(library().bt_render(self._h, _p(rgba, _u8p) if rgba is not None else None,
                                     rgba.nbytes if rgba is not None else 0, ctypes.byref(colored), _p(ms, _f32p)))
        return Frame(rgba, int(colored.value), float(ms[0]))

    def stage_times(self) -> dict[str, float]:
        cap = 64
        names = (ctypes.c_char_p * cap)()
        ms = np.zeros(cap, np.float32)
        count = ctypes.c_uint32()
        self._ck(library().bt_stage_times(self._h, names, _p(ms, _f32p), cap, ctypes.byref(count)))
        return {names[i].decode(): float(ms[i]) for i in range(min(count.value, cap))}

    # -- distortion readback (src/gpu.rs:438-482) --
    def distortion_layout(self) -> "Layout":
        return Layout(self.read_paths(), self.info().samples)

    def distortion_snapshot(self, layout: "Layout") -> "Snapshot":
        return layout.decode(self.read_records())


def autotune(options: Options, xy: np.ndarray, starts: np.ndarray, iterations: int = 3) -> tuple[Options, float]:
    """bt_autotune: the search-cell size that iterates this graph fastest.
    Returns the tuned options and the time of `iterations` iterations (ms)."""
    import dataclasses

    xy = np.ascontiguousarray(xy, np.float32)
    starts = np.ascontiguousarray(starts, np.uint32)
    o = options._struct()
    tuned = _Options()
    ms = np.zeros(1, np.float32)
    _check(library().bt_autotune(ctypes.byref(o), _p(xy, _f32p), xy.size // 2, _p(starts, _u32p), starts.size,
                                 iterations, ctypes.byref(tuned), _p(ms, _f32p)))
    return (dataclasses.replace(options, fine_cells=int(tuned.fine_cells), fine_cells_x=int(tuned.fine_cells_x)),
            float(ms[0]))


class _SlotView(Gpu):
    """Read-only view of a batch slot's context (owned by the batch)."""

    def __init__(self, handle, options: Options):
        self.options = options
        self._h = handle

    def close(self) -> None:  # the batch owns the context
        self._h = None


class Batch:
    """Many independent graphs advanced together by persistent launches over
    a graph x tile work queue (bt_batch_*). Each slot keeps its own options;
    its results equal a single-graph :class:`Gpu` run bit for bit."""

    def __init__(self, device: int = 0, solo_samples: int = 0):
        """solo_samples: slots of at least this many samples iterate on their
        own context beside the persistent step (0 = never, the default)."""
        h = _vp()
        _check(library().bt_batch_create(device, ctypes.byref(h)))
        self._h = h
        self._options: dict[int, Options] = {}
        if solo_samples:
            self.set_solo_samples(solo_samples)

    def set_shape(self, mean_tile: int = 128, mean_ctas_per_sm: int = 0) -> None:
        """bt_batch_set_shape: samples per mean tile (64, 128, 256) and resident
        mean CTAs per SM (0 = as many as fit); results do not depend on it."""
        self._ck(library().bt_batch_set_shape(self._h, mean_tile, mean_ctas_per_sm))

    def shape(self) -> dict:
        t = np.zeros(1, np.uint32)
        c = np.zeros(1, np.uint32)
        self._ck(library().bt_batch_get_shape(self._h, _p(t, _u32p), _p(c, _u32p)))
        return {"mean_tile": int(t[0]), "mean_ctas_per_sm": int(c[0])}

    @staticmethod
    def autotune(jobs, iterations: int = 3, device: int = 0) -> tuple[dict, float]:
        """bt_batch_autotune over (options, xy, starts) triples: the fastest
        batch shape for these graphs and its time for `iterations` iterations."""
        jobs = list(jobs)
        n = len(jobs)
        opts = (_Options * n)(*[o._struct() for o, _, _ in jobs])
        xys = [np.ascontiguousarray(xy, np.float32) for _, xy, _ in jobs]
        sts = [np.ascontiguousarray(st, np.uint32) for _, _, st in jobs]
        xy_ptrs = (_f32p * n)(*[_p(a, _f32p) for a in xys])
        st_ptrs = (_u32p * n)(*[_p(a, _u32p) for a in sts])
        n_points = np.array([a.size // 2 for a in xys], np.uint32)
        n_starts = np.array([a.size for a in sts], np.uint32)
        t = np.zeros(1, np.uint32)
        c = np.zeros(1, np.uint32)
        ms = np.zeros(1, np.float32)
        _check(library().bt_batch_autotune(device, n, opts, xy_ptrs, _p(n_points, _u32p), st_ptrs,
                                           _p(n_starts, _u32p), iterations, _p(t, _u32p), _p(c, _u32p),
                                           _p(ms, _f32p)))
        return {"mean_tile": int(t[0]), "mean_ctas_per_sm": int(c[0])}, float(ms[0])

    def set_solo_samples(self, samples: int) -> None:
        """bt_batch_set_solo_samples: the slot size from which slots iterate on
        their own context (0 = never); from the next step."""
        self._ck(library().bt_batch_set_solo_samples(self._h, samples))

    def close(self) -> None:
        h = getattr(self, "_h", None)
        if h and _lib is not None:
            _lib.bt_batch_destroy(h)
        self._h = None

    def __del__(self):
        self.close()

    def _ck(self, status: int) -> None:
        if status:
            msg = library().bt_batch_last_error(self._h)
            raise BtError(status, msg.decode() if msg else "")

    def add(self, options: Options, xy: np.ndarray, starts: np.ndarray) -> tuple[int, int]:
        """Upload a graph into a free slot; returns (slot, samples)."""
        xy = np.ascontiguousarray(xy, np.float32)
        starts = np.ascontiguousarray(starts, np.uint32)
        o = options._struct()
        slot = ctypes.c_uint32()
        n = ctypes.c_uint32()
        self._ck(library().bt_batch_add(self._h, ctypes.byref(o), _p(xy, _f32p), xy.size // 2, _p(starts, _u32p),
                                        starts.size, ctypes.byref(slot), ctypes.byref(n)))
        self._options[slot.value] = options
        return slot.value, n.value

    def add_many(self, jobs) -> list[tuple[int, int]]:
        """Upload (options, xy, starts) triples concurrently; returns
        [(slot, samples)] in order."""
        jobs = list(jobs)
        n = len(jobs)
        opts = (_Options * n)(*[o._struct() for o, _, _ in jobs])
        xys = [np.ascontiguousarray(xy, np.float32) for _, xy, _ in jobs]
        sts = [np.ascontiguousarray(st, np.uint32) for _, _, st in jobs]
        xy_ptrs = (_f32p * n)(*[_p(a, _f32p) for a in xys])
        st_ptrs = (_u32p * n)(*[_p(a, _u32p) for a in sts])
        n_points = np.array([a.size // 2 for a in xys], np.uint32)
        n_starts = np.array([a.size for a in sts], np.uint32)
        slots = np.zeros(n, np.uint32)
        samples = np.zeros(n, np.uint32)
        self._ck(library().bt_batch_add_many(self._h, n, opts, xy_ptrs, _p(n_points, _u32p), st_ptrs,
                                             _p(n_starts, _u32p), _p(slots, _u32p), _p(samples, _u32p)))
        for (o, _, _), s in zip(jobs, slots.tolist()):
            self._options[s] = o
        return list(zip(slots.tolist(), samples.tolist()))

    def remove(self, slot: int) -> None:
        self._ck(library().bt_batch_remove(self._h, slot))
        self._options.pop(slot, None)

    def iterate(self, n: int = 1) -> None:
        self._ck(library().bt_batch_iterate(self._h, n))

    def iterate_async(self, n: int = 1) -> None:
        self._ck(library().bt_batch_iterate_async(self._h, n))

    def synchronize(self) -> None:
        self._ck(library().bt_batch_synchronize(self._h))

    def iterate_timed(self, n: int = 1) -> float:
        ms = np.zeros(1, np.float32)
        self._ck(library().bt_batch_iterate_timed(self._h, n, _p(ms, _f32p)))
        return float(ms[0])

    def active(self) -> int:
        a = ctypes.c_uint32()
        c = ctypes.c_uint32()
        self._ck(library().bt_batch_slot_count(self._h, ctypes.byref(a), ctypes.byref(c)))
        return a.value

    def slot(self, slot: int) -> Gpu:
        """The slot's context for readbacks (read_points, read_density, ...)."""
        h = library().bt_batch_slot(self._h, slot)
        if not h:
            raise BtError(3, library().bt_batch_last_error(self._h).decode())
        return _SlotView(h, self._options[slot])


@dataclass
class RequestResult:
    """A finished (or failed) serving request; times are on the server clock."""
    id: int
    status: int
    samples: int
    iterations: int
    arrival_s: float
    admitted_s: float
    finished_s: float
    device_bytes: int
    message: str

    @property
    def latency_s(self) -> float:
        return self.finished_s - self.arrival_s


class Server:
    """Continuous batching of arriving requests (bt_server_*): a native worker
    thread admits requests by a device-memory budget, uploads them while the
    batch iterates, and frees each batch slot as soon as that graph's own
    iteration count is reached. Results stay on the device until released."""

    def __init__(self, device: int = 0, max_active: int = 32, budget_bytes: int = 120_000_000_000,
                 max_step: int = 1, reserve_bytes: int = 0, solo_samples: int = 0, queue_timeout_ms: int = 0):
        """solo_samples: requests of at least this many samples iterate on
        their own context beside the batch (0 = 32768; 2**32 - 1 = never).
        queue_timeout_ms: a request not admitted this long after its arrival
        fails with status 6 (0 = no deadline)."""
        o = _ServerOptions()
        library().bt_server_options_init(ctypes.byref(o))
        o.device, o.max_active, o.budget_bytes, o.max_step = device, max_active, budget_bytes, max_step
        o.reserve_bytes = reserve_bytes
        o.solo_samples = solo_samples
        o.queue_timeout_ms = queue_timeout_ms
        h = _vp()
        _check(library().bt_server_create(ctypes.byref(o), ctypes.byref(h)))
        self._h = h
        self._options: dict[int, Options] = {}

    def close(self) -> None:
        h = getattr(self, "_h", None)
        if h and _lib is not None:
            _lib.bt_server_destroy(h)
        self._h = None

    def __del__(self):
        self.close()

    def _ck(self, status: int) -> None:
        if status:
            msg = library().bt_server_last_error(self._h)
            raise BtError(status, msg.decode() if msg else "")

    def clock(self) -> float:
        return library().bt_server_clock(self._h)

    def submit(self, options: Options, xy: np.ndarray, starts: np.ndarray, iterations: int,
               arrival_s: float | None = None) -> int:
        """Queue a request (the inputs are copied); returns its id."""
        xy = np.ascontiguousarray(xy, np.float32)
        starts = np.ascontiguousarray(starts, np.uint32)
        o = options._struct()
        rid = ctypes.c_uint64()
        self._ck(library().bt_server_submit(self._h, ctypes.byref(o), _p(xy, _f32p), xy.size // 2,
                                            _p(starts, _u32p), starts.size, iterations,
                                            -1.0 if arrival_s is None else float(arrival_s), ctypes.byref(rid)))
        self._options[rid.value] = options
        return rid.value

    def next(self, timeout_s: float = 60.0) -> RequestResult:
        """The next request to finish, in completion order."""
        r = _RequestResult()
        self._ck(library().bt_server_next(self._h, timeout_s, ctypes.byref(r)))
        return RequestResult(r.id, r.status, r.samples, r.iterations, r.arrival_s, r.admitted_s, r.finished_s,
                             r.device_bytes, r.message.decode())

    def read_records(self, rid: int, samples: int, out: np.ndarray | None = None) -> np.ndarray:
        """12-byte {x, y, edge_id} records of a finished request."""
        n = 12 * samples
        if out is None:
            out = np.zeros(n, np.uint8)
        else:
            if not out.flags.c_contiguous or out.nbytes < n:
                raise ValueError("record buffer must be C-contiguous with 12 bytes per sample")
            out = out.reshape(-1).view(np.uint8)[:n]
        self._ck(library().bt_server_read_points(self._h, rid, out.ctypes.data, n))
        return out

    def read_points(self, rid: int, samples: int) -> tuple[np.ndarray, np.ndarray]:
        rec = self.read_records(rid, samples).view(np.uint32).reshape(-1, 3)
        return rec[:, :2].copy().view(np.float32), rec[:, 2].copy()

    def result(self, rid: int) -> Gpu:
        """A finished request's context for readbacks until it is released."""
        h = library().bt_server_result(self._h, rid)
        if not h:
            raise BtError(3, "no finished request with this id")
        return _SlotView(h, self._options[rid])

    def release(self, rid: int) -> None:
        self._ck(library().bt_server_release(self._h, rid))
        self._options.pop(rid, None)

    def cancel(self, rid: int) -> None:
        """Drop a request that is still queued; it then finishes with status
        9 (cancelled) through next(). An admitted request runs to the end."""
        self._ck(library().bt_server_cancel(self._h, rid))

    def stats(self) -> dict:
        st = _ServerStats()
        self._ck(library().bt_server_stats_get(self._h, ctypes.byref(st)))
        return {name: getattr(st, name) for name, _ in _ServerStats._fields_}


@dataclass
class Frame:
    """A rendered frame (bt_render)."""
    rgba: np.ndarray | None      # height x width x 4 uint8, rows from the top
    colored_pixels: int          # pixels whose RGB differs from the clear colour
    device_ms: float


@dataclass
class Measurement:
    distortion: float
    rms_displacement_pixels: float


class Layout:
    """geometry::Layout (src/geometry.rs:19-105): validated path reservations."""

    def __init__(self, paths: np.ndarray, samples: int):
        self.paths = np.ascontiguousarray(paths, np.uint32).reshape(-1, 3)
        self.samples = int(samples)
        _check(library().bt_layout_check(_p(self.paths, _u32p), self.paths.shape[0], self.samples))
        counts = self.paths[:, 2]
        order = np.argsort(self.paths[:, 0], kind="stable")
        self.edge_ids = order[counts[order] > 0].astype(np.uint32)
        self.skipped_count = int((counts == 0).sum())
        self.edge_count = int(self.edge_ids.size)

    def decode(self, records: np.ndarray) -> "Snapshot":
        rec = np.ascontiguousarray(records, np.uint8)
        xy = np.zeros((self.samples, 2), np.float32)
        _check(library().bt_decode_points(_p(self.paths, _u32p), self.paths.shape[0], self.samples,
                                          rec.ctypes.data, rec.size, _p(xy, _f32p)))
        return Snapshot(self, xy)


@dataclass
class Snapshot:
    """geometry::Snapshot (src/geometry.rs:190-223)."""

    layout: Layout
    positions: np.ndarray

    def edges(self):
        for e in self.layout.edge_ids:
            off, _, cnt = self.layout.paths[e]
            yield int(e), self.positions[off:off + cnt]


def squared_integral(original: np.ndarray, current: np.ndarray) -> float:
    """distortion::squared_integral (src/distortion.rs:137-168)."""
    a = np.ascontiguousarray(original, np.float32)
    b = np.ascontiguousarray(current, np.float32)
    out = ctypes.c_double()
    _check(library().bt_squared_integral(_p(a, _f32p), a.size // 2, _p(b, _f32p), b.size // 2, ctypes.byref(out)))
    return out.value


@dataclass
class Aggregate:
    """distortion::Aggregate (src/distortion.rs:172-216): equal-edge mean with
    Kahan summation."""

    value: float = 0.0
    correction: float = 0.0
    edges: int = 0

    def add(self, original: np.ndarray, current: np.ndarray) -> None:
        term = squared_integral(original, current)
        adjusted = term - self.correction
        nxt = self.value + adjusted
        if not np.isfinite(nxt):
            raise BtError(3, "nonfinite distortion aggregate")
        self.correction = (nxt - self.value) - adjusted
        self.value = nxt
        self.edges += 1

    def finish(self, size: int = SIZE) -> Measurement:
        if self.edges == 0:
            raise BtError(3, "distortion requires at least one edge")
        rms = (self.value / self.edges) ** 0.5
        return Measurement(rms / (2.0 * 2.0 ** 0.5), rms * (size / 2.0))
