// geometry.cpp — CPU readers of the device geometry.
//
// Layout::new / tile (src/geometry.rs:28-73, 107-118), Decoder::push/finish
// (src/geometry.rs:131-187) and squared_integral (src/distortion.rs:137-168)
// for callers that read the 12-byte records back themselves.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <utility>
#include <vector>

#include "host.h"

namespace bt {
namespace {

struct Range {
    size_t start, end;
};

bool tile(const std::vector<Range>& ranges, size_t expected, std::string* err) {
    size_t end = 0;
    for (const Range& r : ranges) {
        if (!(r.start == end && r.end <= expected)) {
            *err = "geometry ranges have a gap, overlap or exceed active count";
            return false;
        }
        end = r.end;
    }
    if (end != expected) {
        *err = "geometry ranges do not cover active count";
        return false;
    }
    return true;
}

struct EdgeRange {
    uint32_t id;
    Range points;
};

bool build_layout(const uint32_t* paths, uint32_t n_paths, uint32_t samples, std::vector<EdgeRange>* edges,
                  std::string* err) {
    std::vector<Range> segments;
    edges->clear();
    for (uint32_t id = 0; id < n_paths; ++id) {
        const size_t off = paths[3 * id], seg = paths[3 * id + 1], count = paths[3 * id + 2];
        if (count == 0) continue;   // skipped edge
        if (count < 2) {
            *err = "edge " + std::to_string(id) + " has only one sample";
            return false;
        }
        edges->push_back(EdgeRange{id, Range{off, off + count}});
        segments.push_back(Range{seg, seg + count - 1});
    }
    if (edges->empty()) {
        *err = "no eligible edges";
        return false;
    }
    if (samples < edges->size()) {
        *err = "sample count below edge count";
        return false;
    }
    const size_t segment_count = samples - edges->size();
    std::sort(edges->begin(), edges->end(),
              [](const EdgeRange& a, const EdgeRange& b) { return a.points.start < b.points.start; });
    std::sort(segments.begin(), segments.end(), [](const Range& a, const Range& b) { return a.start < b.start; });
    std::vector<Range> pts;
    pts.reserve(edges->size());
    for (const EdgeRange& e : *edges) pts.push_back(e.points);
    return tile(pts, samples, err) && tile(segments, segment_count, err);
}

struct Cursor {
    const float* pts;
    size_t n;
    size_t next = 0;
    double total, traversed = 0.0;
    double start[2], end[2];
    double start_t = 0.0, end_t = 0.0;
    Cursor(const float* p, size_t count, double length) : pts(p), n(count), total(length) {
        start[0] = end[0] = p[0];
        start[1] = end[1] = p[1];
    }
    size_t left() const { return (n >= 2 ? n - 1 : 0) - next; }
    static double dist(const float* a, const float* b) {
        return std::hypot(static_cast<double>(b[0]) - a[0], static_cast<double>(b[1]) - a[1]);
    }
    void advance(double t) {
        while (end_t <= t && end_t < 1.0) {
            if (left() == 0) {
                start[0] = end[0];
                start[1] = end[1];
                start_t = end_t;
                end_t = 1.0;
                return;
            }
            const float* a = pts + 2 * next;
            const float* b = a + 2;
            ++next;
            const double length = dist(a, b);
            if (length == 0.0) continue;
            start[0] = a[0]; start[1] = a[1];
            end[0] = b[0]; end[1] = b[1];
            start_t = end_t;
            traversed += length;
            end_t = left() == 0 ? 1.0 : traversed / total;
        }
    }
    void position(double t, double* out) const {
        if (t >= end_t) { out[0] = end[0]; out[1] = end[1]; return; }
        if (t <= start_t) { out[0] = start[0]; out[1] = start[1]; return; }
        const double f = (t - start_t) / (end_t - start_t);
        out[0] = std::fma(f, end[0] - start[0], start[0]);
        out[1] = std::fma(f, end[1] - start[1], start[1]);
    }
};

bool curve_length(const float* pts, size_t n, double* length) {
    if (n == 0) return false;
    for (size_t i = 0; i < 2 * n; ++i)
        if (!std::isfinite(pts[i])) return false;
    double l = 0.0;
    for (size_t i = 0; i + 1 < n; ++i) l += Cursor::dist(pts + 2 * i, pts + 2 * i + 2);
    if (!std::isfinite(l)) return false;
    *length = l;
    return true;
}

}  // namespace

bool layout_check(const uint32_t* paths, uint32_t n_paths, uint32_t samples, std::string* err) {
    std::vector<EdgeRange> edges;
    return build_layout(paths, n_paths, samples, &edges, err);
}

bool decode_points(const uint32_t* paths, uint32_t n_paths, uint32_t samples, const void* records, size_t bytes,
                   float* xy, std::string* err) {
    std::vector<EdgeRange> edges;
    if (!build_layout(paths, n_paths, samples, &edges, err)) return false;
    if (bytes % 12 != 0) {
        *err = "partial GPU point record";
        return false;
    }
    const size_t n = bytes / 12;
    if (n > samples) {
        *err = "excess GPU point records";
        return false;
    }
    if (n < samples) {
        *err = "missing GPU point records";
        return false;
    }
    const unsigned char* r = static_cast<const unsigned char*>(records);
    size_t owner = 0;
    for (size_t i = 0; i < n; ++i) {
        while (owner < edges.size() && i >= edges[owner].points.end) ++owner;
        if (owner >= edges.size()) {
            *err = "missing point owner";
            return false;
        }
        float x, y;
        uint32_t id;
        std::memcpy(&x, r + 12 * i, 4);
        std::memcpy(&y, r + 12 * i + 4, 4);
        std::memcpy(&id, r + 12 * i + 8, 4);
        if (id != edges[owner].id) {
            *err = "point " + std::to_string(i) + " has incorrect edge ID";
            return false;
        }
        if (!std::isfinite(x) || !std::isfinite(y)) {
            *err = "point " + std::to_string(i) + " has nonfinite coordinates";
            return false;
        }
        xy[2 * i] = x;
        xy[2 * i + 1] = y;
    }
    return true;
}

bool squared_integral_host(const float* original, size_t n_original, const float* current, size_t n_current,
                           double* out, std::string* err) {
    double lo, lc;
    if (!curve_length(original, n_original, &lo) || !curve_length(current, n_current, &lc)) {
        *err = "invalid distortion curve";
        return false;
    }
    Cursor a(original, n_original, lo), b(current, n_current, lc);
    KahanSum sum;
    double t = 0.0;
    while (!(t >= 1.0)) {
        a.advance(t);
        b.advance(t);
        const double next = std::min(a.end_t, b.end_t);
        if (!(next > t && next <= 1.0)) {
            *err = "invalid distortion interval";
            return false;
        }
        double p[2], q[2], r[2], s[2];
        a.position(t, p);
        b.position(t, q);
        a.position(next, r);
        b.position(next, s);
        const double ax = p[0] - q[0], ay = p[1] - q[1];
        const double bx = r[0] - s[0], by = r[1] - s[1];
        const double sx = ax + bx, sy = ay + by;
        const double dx = bx - ax, dy = by - ay;
        const double mid = std::fma(sx, sx, sy * sy);
        const double chg = std::fma(dx, dx, dy * dy);
        sum.add((next - t) * (mid / 4.0 + chg / 12.0));
        t = next;
    }
    if (!(std::isfinite(sum.value) && sum.value >= 0.0)) {
        *err = "nonfinite or negative distortion integral";
        return false;
    }
    *out = sum.value;
    return true;
}

}  // namespace bt
