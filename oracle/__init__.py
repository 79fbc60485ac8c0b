"""ctypes wrapper of the CPU oracle (oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, ``__graft_entry__.smoke()`` and
the CPU-baseline leg of ``bench.py`` as the checker or the timed CPU baseline,
never by the product package.

Parity unpinned: the reference ships no golden vectors and cannot be run here
(Rust + wgpu/Vulkan, no rustc, no graphics stack); the oracle is pinned against
hand-derived known answers only.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None

_f32p = ctypes.POINTER(ctypes.c_float)
_u32p = ctypes.POINTER(ctypes.c_uint32)
_u8p = ctypes.POINTER(ctypes.c_uint8)
_f64p = ctypes.POINTER(ctypes.c_double)


class OrGraph(ctypes.Structure):
    _fields_ = [
        ("xy", _f32p),
        ("n_points", ctypes.c_uint32),
        ("starts", _u32p),
        ("n_starts", ctypes.c_uint32),
        ("min", ctypes.c_float * 2),
        ("max", ctypes.c_float * 2),
    ]


class OrConfig(ctypes.Structure):
    _fields_ = [
        ("width", ctypes.c_uint32),
        ("height", ctypes.c_uint32),
        ("radius", ctypes.c_uint32),
        ("accumulate_density", ctypes.c_uint32),
        ("resample_scale", ctypes.c_float * 2),
        ("capacity", ctypes.c_uint32),
        ("sigma", ctypes.c_double),
        ("shrink", ctypes.c_double),
        ("threads", ctypes.c_int),
    ]


def build() -> None:
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        L.or_parse_trl.argtypes = [ctypes.c_char_p, ctypes.c_size_t, ctypes.POINTER(OrGraph), ctypes.c_char_p, ctypes.c_size_t]
        L.or_graph_free.argtypes = [ctypes.POINTER(OrGraph)]
        L.or_normalization.argtypes = [_f32p, _f32p, _f32p, ctypes.c_char_p, ctypes.c_size_t]
        L.or_blur_weights.argtypes = [ctypes.c_double, _f32p, ctypes.c_int]
        L.or_create.argtypes = [ctypes.POINTER(OrConfig)]
        L.or_create.restype = ctypes.c_void_p
        L.or_destroy.argtypes = [ctypes.c_void_p]
        L.or_upload.argtypes = [ctypes.c_void_p, _f32p, ctypes.c_uint32, _u32p, ctypes.c_uint32, _u32p, ctypes.c_char_p, ctypes.c_size_t]
        L.or_iterate.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_int]
        L.or_samples.argtypes = [ctypes.c_void_p]
        L.or_samples.restype = ctypes.c_uint32
        L.or_paths.argtypes = [ctypes.c_void_p]
        L.or_paths.restype = ctypes.c_uint32
        L.or_get_points.argtypes = [ctypes.c_void_p, _f32p, _u32p]
        L.or_get_paths.argtypes = [ctypes.c_void_p, _u32p]
        L.or_get_segments.argtypes = [ctypes.c_void_p, _u32p]
        L.or_get_edges.argtypes = [ctypes.c_void_p, _f32p]
        L.or_get_counts.argtypes = [ctypes.c_void_p, _u32p]
        L.or_get_blurred.argtypes = [ctypes.c_void_p, _f32p, _f32p, _f32p]
        L.or_get_normalized.argtypes = [ctypes.c_void_p, _f32p]
        L.or_get_cells.argtypes = [ctypes.c_void_p, _u32p, _u32p, _u32p]
        L.or_get_neighbors.argtypes = [ctypes.c_void_p, _u32p]
        L.or_splat.argtypes = [_f32p, ctypes.c_size_t, ctypes.c_uint32, ctypes.c_uint32, _u32p]
        L.or_blur.argtypes = [_u32p, ctypes.c_uint32, ctypes.c_uint32, _f32p, ctypes.c_int, _f32p, _f32p, _f32p]
        L.or_normalize.argtypes = [_f32p, ctypes.c_size_t, ctypes.c_float, _f32p]
        L.or_cells.argtypes = [_f32p, ctypes.c_size_t, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, _u32p]
        L.or_neighbor_mean.argtypes = [_f32p, _u8p, ctypes.c_size_t, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32,
                                       ctypes.c_int, ctypes.c_int, _f32p, _u32p]
        L.or_neighbor_mean_sample.argtypes = [_f32p, _u8p, ctypes.c_size_t, ctypes.c_uint32, ctypes.c_uint32,
                                              ctypes.c_uint32, ctypes.c_size_t, ctypes.c_int, _f32p, _f64p]
        L.or_neighbor_mean_sample.restype = ctypes.c_size_t
        L.or_squared_integral.argtypes = [_f32p, ctypes.c_size_t, _f32p, ctypes.c_size_t, _f64p]
        L.or_distortion.argtypes = [_u32p, ctypes.c_uint32, _f32p, _f32p, ctypes.c_uint32, _f64p, _f64p]
        L.or_advect.argtypes = [_f32p, _u32p, ctypes.c_size_t, _f32p, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_float,
                                ctypes.c_float, _f32p]
        L.or_half_round.argtypes = [ctypes.c_float]
        L.or_half_round.restype = ctypes.c_float
        L.or_render.argtypes = [_f32p, _u32p, _u32p, ctypes.c_uint32, ctypes.c_uint32, _f32p, ctypes.c_uint32,
                                ctypes.c_uint32, ctypes.c_int, ctypes.c_int, ctypes.c_int, _u32p, ctypes.c_uint32,
                                ctypes.c_int, _u8p, ctypes.POINTER(ctypes.c_uint64)]
        _lib = L
    return _lib


def _p(a, t):
    return a.ctypes.data_as(t)


class OracleError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"[{status}] {message}")
        self.status = status


def parse_trl(text: str | bytes):
    """graph.rs Graph::parse -> (xy float32[P,2], starts uint32[E+1], min, max)."""
    data = text.encode() if isinstance(text, str) else text
    g = OrGraph()
    err = ctypes.create_string_buffer(256)
    rc = lib().or_parse_trl(data, len(data), ctypes.byref(g), err, 256)
    if rc:
        raise OracleError(rc, err.value.decode())
    try:
        xy = np.ctypeslib.as_array(g.xy, shape=(g.n_points * 2,)).copy().reshape(-1, 2)
        starts = np.ctypeslib.as_array(g.starts, shape=(g.n_starts,)).copy()
        return xy, starts, (g.min[0], g.min[1]), (g.max[0], g.max[1])
    finally:
        lib().or_graph_free(ctypes.byref(g))


def normalization(mn, mx):
    out = np.zeros(5, np.float32)
    a = np.asarray(mn, np.float32)
    b = np.asarray(mx, np.float32)
    err = ctypes.create_string_buffer(256)
    rc = lib().or_normalization(_p(a, _f32p), _p(b, _f32p), _p(out, _f32p), err, 256)
    if rc:
        raise OracleError(rc, err.value.decode())
    return out


def blur_weights(sigma: float) -> np.ndarray:
    w = np.zeros(4096, np.float32)
    R = lib().or_blur_weights(float(sigma), _p(w, _f32p), 4096)
    if R < 0:
        raise ValueError("invalid sigma")
    return w[: R + 1].copy()


def splat(xy, w, h, counts=None):
    xy = np.ascontiguousarray(xy, np.float32)
    if counts is None:
        counts = np.zeros(w * h, np.uint32)
    lib().or_splat(_p(xy, _f32p), xy.size // 2, w, h, _p(counts, _u32p))
    return counts


def blur(counts, w, h, taps):
    counts = np.ascontiguousarray(counts, np.uint32).reshape(-1)
    taps = np.ascontiguousarray(taps, np.float32)
    hz = np.zeros(w * h, np.float32)
    vt = np.zeros(w * h, np.float32)
    peak = np.zeros(1, np.float32)
    lib().or_blur(_p(counts, _u32p), w, h, _p(taps, _f32p), len(taps) - 1, _p(hz, _f32p), _p(vt, _f32p), _p(peak, _f32p))
    return hz, vt, float(peak[0])


def normalize(v, peak):
    v = np.ascontiguousarray(v, np.float32).reshape(-1)
    out = np.zeros_like(v)
    lib().or_normalize(_p(v, _f32p), v.size, np.float32(peak), _p(out, _f32p))
    return out


def cells(xy, w, h, radius):
    xy = np.ascontiguousarray(xy, np.float32)
    out = np.zeros(xy.size // 2, np.uint32)
    lib().or_cells(_p(xy, _f32p), xy.size // 2, w, h, radius, _p(out, _u32p))
    return out


def neighbor_mean(xy, movable, w, h, radius, mode=0, threads=0):
    xy = np.ascontiguousarray(xy, np.float32)
    mv = np.ascontiguousarray(movable, np.uint8)
    n = xy.size // 2
    out = np.zeros((n, 2), np.float32)
    nb = np.zeros(n, np.uint32)
    lib().or_neighbor_mean(_p(xy, _f32p), _p(mv, _u8p), n, w, h, radius, mode, threads, _p(out, _f32p), _p(nb, _u32p))
    return out, nb


def neighbor_mean_sample(xy, movable, w, h, radius, stride, threads=0):
    """Mean of every stride-th sample (bounded CPU-baseline sample).
    Returns (positions, samples computed, index seconds, call seconds)."""
    xy = np.ascontiguousarray(xy, np.float32)
    mv = np.ascontiguousarray(movable, np.uint8)
    n = xy.size // 2
    out = np.zeros((n, 2), np.float32)
    sec = np.zeros(2, np.float64)
    done = lib().or_neighbor_mean_sample(_p(xy, _f32p), _p(mv, _u8p), n, w, h, radius, stride, threads,
                                         _p(out, _f32p), _p(sec, _f64p))
    return out, int(done), float(sec[0]), float(sec[1])


def movable_mask(paths, n):
    """Non-endpoint samples (neighbor_mean.wgsl:61-64)."""
    mv = np.ones(n, np.uint8)
    drawn = paths[paths[:, 2] > 0]
    mv[drawn[:, 0]] = 0
    mv[drawn[:, 0] + drawn[:, 2] - 1] = 0
    return mv


def squared_integral(original, current) -> float:
    a = np.ascontiguousarray(original, np.float32)
    b = np.ascontiguousarray(current, np.float32)
    out = ctypes.c_double()
    rc = lib().or_squared_integral(_p(a, _f32p), a.size // 2, _p(b, _f32p), b.size // 2, ctypes.byref(out))
    if rc:
        raise OracleError(rc, "invalid distortion curve")
    return out.value


def distortion(paths, original_xy, current_xy, size):
    paths = np.ascontiguousarray(paths, np.uint32)
    a = np.ascontiguousarray(original_xy, np.float32)
    b = np.ascontiguousarray(current_xy, np.float32)
    d = ctypes.c_double()
    r = ctypes.c_double()
    rc = lib().or_distortion(_p(paths, _u32p), paths.size // 3, _p(a, _f32p), _p(b, _f32p), size, ctypes.byref(d), ctypes.byref(r))
    if rc:
        raise OracleError(rc, "distortion failed")
    return d.value, r.value


def advect(xy, edge_ids, density, w, h, step, smooth):
    """One density-gradient advection step (oracle.cpp or_advect)."""
    xy = np.ascontiguousarray(xy, np.float32).reshape(-1, 2)
    edge_ids = np.ascontiguousarray(edge_ids, np.uint32)
    density = np.ascontiguousarray(density, np.float32).reshape(-1)
    out = np.empty_like(xy)
    lib().or_advect(_p(xy, _f32p), _p(edge_ids, _u32p), xy.shape[0], _p(density, _f32p), w, h, np.float32(step),
                    np.float32(smooth), _p(out, _f32p))
    return out


def half_round(v: float) -> float:
    return lib().or_half_round(v)


def render(xy, edge_ids, segments, n_edges, density, w, h, color_by_edge=False, palette=0, msaa=4,
           paths=None, endpoint_dots=False):
    """Path rasterisation (render.cpp): (RGBA8 array h x w x 4, colored pixel count).
    paths: n x 3 u32 (point offset, segment offset, count), for the endpoint dots."""
    xy = np.ascontiguousarray(xy, np.float32)
    paths = np.ascontiguousarray(paths if paths is not None else np.zeros((0, 3)), np.uint32)
    edge_ids = np.ascontiguousarray(edge_ids, np.uint32)
    segments = np.ascontiguousarray(segments, np.uint32)
    density = np.ascontiguousarray(density if density is not None else np.zeros(w * h), np.float32)
    out = np.zeros((h, w, 4), np.uint8)
    colored = ctypes.c_uint64()
    rc = lib().or_render(_p(xy, _f32p), _p(edge_ids, _u32p), _p(segments, _u32p), segments.size, n_edges,
                         _p(density, _f32p), w, h, int(bool(color_by_edge)), palette, msaa, _p(paths, _u32p),
                         paths.size // 3, int(bool(endpoint_dots)), _p(out, _u8p), ctypes.byref(colored))
    if rc:
        raise OracleError(rc, "render failed")
    return out, colored.value


@dataclass
class Config:
    width: int
    height: int
    radius: int = 0
    accumulate_density: bool = True
    resample_scale: tuple | None = None  # None -> reference ((W-1)*0.5, (H-1)*0.5)
    capacity: int = 1 << 31
    sigma: float = 0.0
    shrink: float = 1.0
    threads: int = 0


class Pipeline:
    """Gpu::upload / Gpu::iterate restated on the CPU (src/gpu.rs:493-553)."""

    def __init__(self, cfg: Config):
        c = OrConfig()
        c.width, c.height, c.radius = cfg.width, cfg.height, cfg.radius
        c.accumulate_density = 1 if cfg.accumulate_density else 0
        if cfg.resample_scale is None:
            sx = np.float32(np.float32(cfg.width - 1) * np.float32(0.5))
            sy = np.float32(np.float32(cfg.height - 1) * np.float32(0.5))
        else:
            sx, sy = cfg.resample_scale
        c.resample_scale[0], c.resample_scale[1] = float(sx), float(sy)
        c.capacity = min(int(cfg.capacity), 0xFFFFFFFF)
        c.sigma, c.shrink, c.threads = float(cfg.sigma), float(cfg.shrink), int(cfg.threads)
        self.cfg = cfg
        self._h = lib().or_create(ctypes.byref(c))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            lib().or_destroy(h)
            self._h = None

    def upload(self, xy, starts) -> int:
        xy = np.ascontiguousarray(xy, np.float32)
        starts = np.ascontiguousarray(starts, np.uint32)
        n = ctypes.c_uint32()
        err = ctypes.create_string_buffer(256)
        rc = lib().or_upload(self._h, _p(xy, _f32p), xy.size // 2, _p(starts, _u32p), starts.size, ctypes.byref(n), err, 256)
        if rc:
            raise OracleError(rc, err.value.decode())
        return n.value

    def iterate(self, n: int = 1, mode: int = 0) -> None:
        rc = lib().or_iterate(self._h, n, mode)
        if rc:
            raise OracleError(rc, "iterate failed")

    @property
    def samples(self) -> int:
        return lib().or_samples(self._h)

    @property
    def path_count(self) -> int:
        return lib().or_paths(self._h)

    def points(self):
        n = self.samples
        xy = np.zeros((n, 2), np.float32)
        ids = np.zeros(n, np.uint32)
        lib().or_get_points(self._h, _p(xy, _f32p), _p(ids, _u32p))
        return xy, ids

    def paths(self):
        out = np.zeros((self.path_count, 3), np.uint32)
        lib().or_get_paths(self._h, _p(out, _u32p))
        return out

    def segments(self):
        p = self.paths()
        n = int((p[:, 2].astype(np.int64) - 1).clip(min=0)[p[:, 2] > 0].sum())
        out = np.zeros(n, np.uint32)
        lib().or_get_segments(self._h, _p(out, _u32p))
        return out

    def edges(self):
        out = np.zeros((self.path_count, 4), np.float32)
        lib().or_get_edges(self._h, _p(out, _f32p))
        return out

    def counts(self):
        out = np.zeros(self.cfg.width * self.cfg.height, np.uint32)
        lib().or_get_counts(self._h, _p(out, _u32p))
        return out

    def blurred(self):
        g = self.cfg.width * self.cfg.height
        hz = np.zeros(g, np.float32)
        vt = np.zeros(g, np.float32)
        peak = np.zeros(1, np.float32)
        lib().or_get_blurred(self._h, _p(hz, _f32p), _p(vt, _f32p), _p(peak, _f32p))
        return hz, vt, float(peak[0])

    def normalized(self):
        out = np.zeros(self.cfg.width * self.cfg.height, np.float32)
        lib().or_get_normalized(self._h, _p(out, _f32p))
        return out

    def cells(self):
        gw = ctypes.c_uint32()
        gh = ctypes.c_uint32()
        out = np.zeros(self.samples, np.uint32)
        lib().or_get_cells(self._h, _p(out, _u32p), ctypes.byref(gw), ctypes.byref(gh))
        return out, gw.value, gh.value

    def neighbors(self):
        out = np.zeros(self.samples, np.uint32)
        lib().or_get_neighbors(self._h, _p(out, _u32p))
        return out
