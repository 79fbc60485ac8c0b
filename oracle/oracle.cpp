// oracle.cpp — CPU restatement of lpstankus/bundling_thingy's bundling loop.
//
// TEST INFRASTRUCTURE ONLY (see oracle.h). Parity unpinned: the reference has
// no golden vectors and cannot be run here; this file is checked against
// hand-derived known answers only.
//
// Compile with -O2 -ffp-contract=off (no fast-math): every float expression
// below is one IEEE binary32 rounding per operation, in the reference's
// evaluation order, unless it calls fmaf() explicitly.
#include "oracle.h"

#include <algorithm>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

void set_err(char* err, size_t len, const std::string& msg) {
    if (err && len) {
        std::snprintf(err, len, "%s", msg.c_str());
    }
}

// WGSL u32(f32): truncation toward zero, saturating at the range ends.
inline uint32_t u32_sat(float v) {
    if (!(v > 0.0f)) return 0u;
    if (v >= 4294967296.0f) return 0xFFFFFFFFu;
    return static_cast<uint32_t>(v);
}

// ---------------------------------------------------------------------------
// TRL parsing (src/graph.rs:35-77, 102-107)
// ---------------------------------------------------------------------------

// Grammar of Rust's `str::parse::<f32>` (core dec2flt): optional sign, then
// inf | infinity | nan (any case), or digits with an optional '.' and an
// optional exponent, at least one digit in the mantissa.
bool rust_float_syntax(const char* s, size_t n) {
    size_t i = 0;
    if (i < n && (s[i] == '+' || s[i] == '-')) ++i;
    auto ieq = [&](const char* word) {
        size_t m = std::strlen(word);
        if (n - i != m) return false;
        for (size_t k = 0; k < m; ++k) {
            char c = s[i + k];
            if (c >= 'A' && c <= 'Z') c = static_cast<char>(c - 'A' + 'a');
            if (c != word[k]) return false;
        }
        return true;
    };
    if (ieq("inf") || ieq("infinity") || ieq("nan")) return true;
    size_t digits = 0;
    while (i < n && s[i] >= '0' && s[i] <= '9') { ++i; ++digits; }
    if (i < n && s[i] == '.') {
        ++i;
        while (i < n && s[i] >= '0' && s[i] <= '9') { ++i; ++digits; }
    }
    if (digits == 0) return false;
    if (i < n && (s[i] == 'e' || s[i] == 'E')) {
        ++i;
        if (i < n && (s[i] == '+' || s[i] == '-')) ++i;
        size_t exp_digits = 0;
        while (i < n && s[i] >= '0' && s[i] <= '9') { ++i; ++exp_digits; }
        if (exp_digits == 0) return false;
    }
    return i == n;
}

bool parse_f32(const std::string& token, float* out) {
    if (!rust_float_syntax(token.data(), token.size())) return false;
    errno = 0;
    char* end = nullptr;
    *out = std::strtof(token.c_str(), &end);  // correctly rounded (glibc)
    return end == token.c_str() + token.size();
}

}  // namespace

extern "C" int or_parse_trl(const char* text, size_t len, or_graph* out, char* err, size_t errlen) {
    std::vector<float> xy;
    std::vector<uint32_t> starts;
    float mn[2] = {INFINITY, INFINITY}, mx[2] = {-INFINITY, -INFINITY};
    // Point::MAX / Point::MIN initial bounds (graph.rs:39-40) are finite in
    // Rust (f32::MAX / f32::MIN); min/max against finite points give the same.
    mn[0] = mn[1] = 3.40282347e+38f;
    mx[0] = mx[1] = -3.40282347e+38f;
    size_t pos = 0, line = 0;
    // str::lines(): split after each '\n', strip "\n" then one "\r".
    while (pos < len) {
        size_t nl = pos;
        while (nl < len && text[nl] != '\n') ++nl;
        size_t end = nl;
        if (nl < len && end > pos && text[end - 1] == '\r') --end;
        std::string l(text + pos, end - pos);
        pos = (nl < len) ? nl + 1 : len;
        // split(' '), skipping the first token (graph.rs:43-44)
        std::vector<std::string> tokens;
        size_t a = 0;
        while (true) {
            size_t b = l.find(' ', a);
            if (b == std::string::npos) { tokens.push_back(l.substr(a)); break; }
            tokens.push_back(l.substr(a, b - a));
            a = b + 1;
        }
        size_t start = xy.size() / 2;
        size_t t = 1;
        while (t < tokens.size()) {
            const std::string& token = tokens[t++];
            if (token.empty() || token[0] == '(' || token[0] == '<') continue;
            float x, y;
            if (!parse_f32(token, &x)) {
                set_err(err, errlen, "line " + std::to_string(line + 1) + " x: invalid coordinate");
                return 3;
            }
            if (t >= tokens.size()) {
                set_err(err, errlen, "line " + std::to_string(line + 1) + " y: unexpected end of TRL line");
                return 3;
            }
            if (!parse_f32(tokens[t++], &y)) {
                set_err(err, errlen, "line " + std::to_string(line + 1) + " y: invalid coordinate");
                return 3;
            }
            if (!std::isfinite(x) || !std::isfinite(y)) {
                set_err(err, errlen, "non-finite TRL coordinate");
                return 3;
            }
            size_t have = xy.size() / 2;
            // Consecutive duplicates within an edge are dropped (graph.rs:55-58);
            // f32 equality, so -0.0 == 0.0.
            if (have > start && xy[2 * have - 2] == x && xy[2 * have - 1] == y) continue;
            xy.push_back(x);
            xy.push_back(y);
        }
        size_t have = xy.size() / 2;
        if (have - start < 2) {
            xy.resize(2 * start);
        } else {
            if (start > 0xFFFFFFFFull) {
                set_err(err, errlen, "too many control points");
                return 3;
            }
            starts.push_back(static_cast<uint32_t>(start));
            for (size_t k = start; k < have; ++k) {
                mn[0] = std::min(mn[0], xy[2 * k]);
                mn[1] = std::min(mn[1], xy[2 * k + 1]);
                mx[0] = std::max(mx[0], xy[2 * k]);
                mx[1] = std::max(mx[1], xy[2 * k + 1]);
            }
        }
        ++line;
    }
    starts.push_back(static_cast<uint32_t>(xy.size() / 2));
    if (xy.empty()) {
        set_err(err, errlen, "graph has no drawable edges");
        return 3;
    }
    out->n_points = static_cast<uint32_t>(xy.size() / 2);
    out->n_starts = static_cast<uint32_t>(starts.size());
    out->xy = static_cast<float*>(std::malloc(xy.size() * sizeof(float)));
    out->starts = static_cast<uint32_t*>(std::malloc(starts.size() * sizeof(uint32_t)));
    std::memcpy(out->xy, xy.data(), xy.size() * sizeof(float));
    std::memcpy(out->starts, starts.data(), starts.size() * sizeof(uint32_t));
    out->min[0] = mn[0]; out->min[1] = mn[1];
    out->max[0] = mx[0]; out->max[1] = mx[1];
    return 0;
}

extern "C" void or_graph_free(or_graph* g) {
    if (!g) return;
    std::free(g->xy);
    std::free(g->starts);
    g->xy = nullptr;
    g->starts = nullptr;
}

// graph.rs:79-91
extern "C" int or_normalization(const float mn[2], const float mx[2], float out[5], char* err, size_t errlen) {
    float rx = mx[0] - mn[0];
    float ry = mx[1] - mn[1];
    float span = std::fmax(rx, ry);
    if (!(span > 0.0f && std::isfinite(span))) {
        set_err(err, errlen, "graph has invalid extent");
        return 3;
    }
    float scale = 0.95f / span;
    if (!std::isfinite(scale)) {
        set_err(err, errlen, "graph normalization scale is not finite");
        return 3;
    }
    out[0] = mn[0];
    out[1] = mn[1];
    out[2] = scale;
    out[3] = (1.0f - scale * rx) / 2.0f;
    out[4] = (1.0f - scale * ry) / 2.0f;
    return 0;
}

// ---------------------------------------------------------------------------
// Blur taps (src/shaders/blur.wgsl:41-60)
// ---------------------------------------------------------------------------
extern "C" int or_blur_weights(double sigma, float* w, int max_taps) {
    static const float kReference[19] = {
        0.0666251319f, 0.0657061792f, 0.0630246744f, 0.0587964725f, 0.0533492351f,
        0.0470805347f, 0.0404101852f, 0.0337346772f, 0.0273904106f, 0.0216300135f,
        0.0166131238f, 0.0124102942f, 0.0090167311f, 0.0063716575f, 0.0043791719f,
        0.0029273040f, 0.0019031803f, 0.0012034507f, 0.0007401384f};
    if (sigma == 0.0) {
        if (max_taps < 19) return -1;
        for (int k = 0; k < 19; ++k) w[k] = kReference[k];
        return 18;
    }
    if (!(sigma > 0.0) || !std::isfinite(sigma)) return -1;
    int R = static_cast<int>(std::ceil(3.0 * sigma));
    if (R < 1) R = 1;
    if (R + 1 > max_taps) return -1;
    double total = 0.0;
    for (int k = -R; k <= R; ++k) total += std::exp(-(double)k * k / (2.0 * sigma * sigma));
    for (int k = 0; k <= R; ++k) w[k] = static_cast<float>(std::exp(-(double)k * k / (2.0 * sigma * sigma)) / total);
    return R;
}

// ---------------------------------------------------------------------------
// Pure kernels
// ---------------------------------------------------------------------------
namespace {

// Density splat of one sample (src/shaders/resampling.wgsl:70-75,
// src/shaders/neighbor_mean.wgsl:68-72). round() is half-to-even.
inline void splat_one(float x, float y, uint32_t w, uint32_t h, uint32_t* counts) {
    float ux = x * 0.5f + 0.5f;
    float uy = 0.5f - y * 0.5f;
    uint32_t cx = u32_sat(std::nearbyint(ux * static_cast<float>(w - 1)));
    uint32_t cy = u32_sat(std::nearbyint(uy * static_cast<float>(h - 1)));
    if (cx < w && cy < h) counts[static_cast<size_t>(cy) * w + cx] += 1u;
}

// spatial_grid.wgsl:59-65
inline float texel_of(float p, uint32_t size) {
    return ((p + 1.0f) * 0.5f) * static_cast<float>(size - 1u);
}
inline uint32_t grid_of(float t, uint32_t radius, uint32_t gsize) {
    uint32_t c = u32_sat(std::fmax(t / static_cast<float>(radius), 0.0f));
    return std::min(c, gsize - 1u);
}

int thread_count(int requested) {
#ifdef _OPENMP
    return requested > 0 ? requested : omp_get_max_threads();
#else
    (void)requested;
    return 1;
#endif
}

}  // namespace

extern "C" void or_splat(const float* xy, size_t n, uint32_t w, uint32_t h, uint32_t* counts) {
    for (size_t i = 0; i < n; ++i) splat_one(xy[2 * i], xy[2 * i + 1], w, h, counts);
}

// blur.wgsl:13-82. Tap sum: value = x0*w0, then for k = 1..R
// value = fmaf(x[-k] + x[k], w[k], value) — the contraction WGSL permits for
// `value += pair(...) * w`. Zero padding outside the map. Horizontal reads
// f32(count), vertical reads the horizontal result. peak = max(vertical).
extern "C" void or_blur(const uint32_t* counts, uint32_t w, uint32_t h, const float* taps, int R,
                        float* horizontal, float* vertical, float* peak) {
    const long W = w, H = h;
#pragma omp parallel for schedule(static)
    for (long y = 0; y < H; ++y) {
        for (long x = 0; x < W; ++x) {
            auto at = [&](long xx) -> float {
                return (xx >= 0 && xx < W) ? static_cast<float>(counts[y * W + xx]) : 0.0f;
            };
            float v = at(x) * taps[0];
            for (int k = 1; k <= R; ++k) v = std::fmaf(at(x - k) + at(x + k), taps[k], v);
            horizontal[y * W + x] = v;
        }
    }
    float best = 0.0f;
#pragma omp parallel for schedule(static) reduction(max : best)
    for (long y = 0; y < H; ++y) {
        for (long x = 0; x < W; ++x) {
            auto at = [&](long yy) -> float {
                return (yy >= 0 && yy < H) ? horizontal[yy * W + x] : 0.0f;
            };
            float v = at(y) * taps[0];
            for (int k = 1; k <= R; ++k) v = std::fmaf(at(y - k) + at(y + k), taps[k], v);
            vertical[y * W + x] = v;
            best = std::max(best, v);
        }
    }
    *peak = best;
}

// normalization.wgsl:11-16 (the reference stores the value in an RGBA16F
// texture; here it stays f32).
extern "C" void or_normalize(const float* v, size_t n, float peak, float* out) {
    for (size_t i = 0; i < n; ++i) {
        float value = 0.0f;
        if (peak > 0.0f) value = std::fmin(std::fmax(v[i] / peak, 0.0f), 1.0f);
        out[i] = value;
    }
}

// spatial_grid.wgsl:67-70 with the grid of neighbor_mean.rs:26-32.
extern "C" void or_cells(const float* xy, size_t n, uint32_t w, uint32_t h, uint32_t radius, uint32_t* cell_ids) {
    const uint32_t gw = (w + radius - 1) / radius, gh = (h + radius - 1) / radius;
    for (size_t i = 0; i < n; ++i) {
        uint32_t cx = grid_of(texel_of(xy[2 * i], w), radius, gw);
        uint32_t cy = grid_of(texel_of(xy[2 * i + 1], h), radius, gh);
        cell_ids[i] = cy * gw + cx;
    }
}

// Neighbour mean, sparse formulation (neighbor_mean.wgsl:164-203): every
// sample q in the cells of the reach box with
//   dot((q - p) * ts, (q - p) * ts) <= r * r
// belongs to N(p) (p itself included).
//
// mode 0 (canonical): the displacement sum is accumulated exactly as
//   D = sum_q (Q(q) - Q(p)),  Q(v) = round-half-even(v * 2^30)  (int64),
// and p' = p + f32(f64(D) / (f64(|N|) * 2^30)). The sum is independent of the
// order of N(p), which the reference leaves to atomics (spatial_grid.wgsl:135).
// mode 1: the reference's literal f32 running sum `displacement += delta`
// over cells row-major and samples by ascending index, p' = p + disp / f32(n).
extern "C" void or_neighbor_mean(const float* xy, const uint8_t* movable, size_t n, uint32_t w, uint32_t h,
                                 uint32_t radius, int mode, int threads, float* out_xy, uint32_t* neighbors) {
    const uint32_t gw = (w + radius - 1) / radius, gh = (h + radius - 1) / radius;
    const size_t cells = static_cast<size_t>(gw) * gh;
    // Stable counting sort of samples by cell.
    std::vector<uint32_t> cell_of(n), start(cells + 1, 0), order(n);
    or_cells(xy, n, w, h, radius, cell_of.data());
    for (size_t i = 0; i < n; ++i) start[cell_of[i] + 1]++;
    for (size_t c = 0; c < cells; ++c) start[c + 1] += start[c];
    {
        std::vector<uint32_t> fill(start.begin(), start.end() - 1);
        for (size_t i = 0; i < n; ++i) order[fill[cell_of[i]]++] = static_cast<uint32_t>(i);
    }
    const float tsx = static_cast<float>(w - 1u) * 0.5f;
    const float tsy = static_cast<float>(h - 1u) * 0.5f;
    const float r2 = static_cast<float>(radius) * static_cast<float>(radius);
    const float padx = static_cast<float>(w) * 0.00000024f;
    const float pady = static_cast<float>(h) * 0.00000024f;
    const float reachx = static_cast<float>(radius) + padx;
    const float reachy = static_cast<float>(radius) + pady;
    const long N = static_cast<long>(n);
#pragma omp parallel for schedule(dynamic, 1024) num_threads(thread_count(threads))
    for (long i = 0; i < N; ++i) {
        const float px = xy[2 * i], py = xy[2 * i + 1];
        if (!movable[i]) {
            out_xy[2 * i] = px;
            out_xy[2 * i + 1] = py;
            if (neighbors) neighbors[i] = 0;
            continue;
        }
        const float tx = texel_of(px, w), ty = texel_of(py, h);
        const uint32_t fx = grid_of(tx - reachx, radius, gw), lx = grid_of(tx + reachx, radius, gw);
        const uint32_t fy = grid_of(ty - reachy, radius, gh), ly = grid_of(ty + reachy, radius, gh);
        const int64_t qpx = std::llrint(px * 1073741824.0f), qpy = std::llrint(py * 1073741824.0f);
        int64_t dx_fixed = 0, dy_fixed = 0;
        float dispx = 0.0f, dispy = 0.0f;
        uint32_t count = 0;
        for (uint32_t cy = fy; cy <= ly; ++cy) {
            for (uint32_t cx = fx; cx <= lx; ++cx) {
                const uint32_t c = cy * gw + cx;
                for (uint32_t s = start[c]; s < start[c + 1]; ++s) {
                    const uint32_t j = order[s];
                    const float dx = xy[2 * j] - px, dy = xy[2 * j + 1] - py;
                    const float ex = dx * tsx, ey = dy * tsy;
                    const float d2 = ex * ex + ey * ey;
                    if (d2 <= r2) {
                        ++count;
                        if (mode == 0) {
                            dx_fixed += std::llrint(xy[2 * j] * 1073741824.0f) - qpx;
                            dy_fixed += std::llrint(xy[2 * j + 1] * 1073741824.0f) - qpy;
                        } else {
                            dispx = dispx + dx;
                            dispy = dispy + dy;
                        }
                    }
                }
            }
        }
        if (mode == 0) {
            const double denom = static_cast<double>(count) * 1073741824.0;
            out_xy[2 * i] = px + static_cast<float>(static_cast<double>(dx_fixed) / denom);
            out_xy[2 * i + 1] = py + static_cast<float>(static_cast<double>(dy_fixed) / denom);
        } else {
            const float nf = static_cast<float>(count);
            out_xy[2 * i] = px + dispx / nf;
            out_xy[2 * i + 1] = py + dispy / nf;
        }
        if (neighbors) neighbors[i] = count;
    }
}

extern "C" size_t or_neighbor_mean_sample(const float* xy, const uint8_t* movable, size_t n, uint32_t w, uint32_t h,
                                          uint32_t radius, size_t stride, int threads, float* out_xy,
                                          double* seconds) {
    if (stride == 0) stride = 1;
    // A contiguous block of n / stride samples (whole paths in sample order)
    // keeps the cache locality of a full pass.
    std::vector<uint8_t> mask(n, 0);
    size_t computed = 0;
    const size_t block = (n + stride - 1) / stride;
    for (size_t i = 0; i < block; ++i) {
        mask[i] = movable[i];
        computed += movable[i] ? 1 : 0;
    }
    // seconds[0]: grid index over all samples (time of a whole-set stable
    // counting sort, measured separately); seconds[1]: the whole call.
#ifdef _OPENMP
    double t0 = omp_get_wtime();
    {
        std::vector<uint32_t> cell_of(n);
        or_cells(xy, n, w, h, radius, cell_of.data());
        const uint32_t gw = (w + radius - 1) / radius, gh = (h + radius - 1) / radius;
        std::vector<uint32_t> start(static_cast<size_t>(gw) * gh + 1, 0), order(n);
        for (size_t i = 0; i < n; ++i) start[cell_of[i] + 1]++;
        for (size_t c = 0; c + 1 < start.size(); ++c) start[c + 1] += start[c];
        std::vector<uint32_t> fill(start.begin(), start.end() - 1);
        for (size_t i = 0; i < n; ++i) order[fill[cell_of[i]]++] = static_cast<uint32_t>(i);
    }
    double t1 = omp_get_wtime();
    or_neighbor_mean(xy, mask.data(), n, w, h, radius, 0, threads, out_xy, nullptr);
    double t2 = omp_get_wtime();
    if (seconds) {
        seconds[0] = t1 - t0;
        seconds[1] = t2 - t1;
    }
#else
    or_neighbor_mean(xy, mask.data(), n, w, h, radius, 0, threads, out_xy, nullptr);
    if (seconds) seconds[0] = seconds[1] = 0.0;
#endif
    return computed;
}

// ---------------------------------------------------------------------------
// Resampling (src/shaders/resampling.wgsl:45-183)
// ---------------------------------------------------------------------------
namespace {

struct Norm {
    float min_x, min_y, scale, tx, ty;
};

// resampling.wgsl:45-48
inline void normalized(const Norm& nm, const float* cp, uint32_t i, float* ox, float* oy) {
    float ax = (cp[2 * i] - nm.min_x) * nm.scale;
    ax = ax + nm.tx;
    ax = ax - 0.5f;
    *ox = ax * 2.0f;
    float ay = (cp[2 * i + 1] - nm.min_y) * nm.scale;
    ay = ay + nm.ty;
    ay = ay - 0.5f;
    *oy = ay * 2.0f;
}

struct PathRec {
    uint32_t point_offset, segment_offset, count;
};

struct Walk {
    const float* cp;
    const uint32_t* starts;
    Norm nm;
    float sx, sy;         // resampling texel_scale
    uint32_t capacity;
    // emit-mode outputs
    float* pts;
    uint32_t* edge_ids;
    uint32_t* segments;
    uint32_t* counts;
    uint32_t w, h;
    bool accumulate;
};

struct Cursor {
    uint32_t count;
    float lx, ly;
};

// push_sample (resampling.wgsl:50-79). Returns false when emit reports a
// count mismatch (overflow 2).
inline bool push(Cursor& c, float x, float y, bool write, const Walk& wk, const PathRec& path,
                 uint32_t edge_id, bool* mismatch) {
    if (c.count > 0u && x == c.lx && y == c.ly) return true;
    if (!write && c.count >= wk.capacity) {
        c.count = wk.capacity + 1u;
        return true;
    }
    if (write) {
        if (c.count >= path.count) {
            *mismatch = true;
            c.count = wk.capacity + 1u;
            return false;
        }
        uint32_t index = path.point_offset + c.count;
        wk.pts[2 * static_cast<size_t>(index)] = x;
        wk.pts[2 * static_cast<size_t>(index) + 1] = y;
        wk.edge_ids[index] = edge_id;
        if (c.count > 0u) wk.segments[path.segment_offset + c.count - 1u] = index - 1u;
        if (wk.accumulate) splat_one(x, y, wk.w, wk.h, wk.counts);
    }
    c.lx = x;
    c.ly = y;
    c.count += 1u;
    return true;
}

// resample (resampling.wgsl:82-136)
uint32_t resample(const Walk& wk, uint32_t p, bool write, const PathRec& path, float* edge_out, bool* mismatch) {
    const uint32_t start = wk.starts[p], end = wk.starts[p + 1];
    float fx, fy;
    normalized(wk.nm, wk.cp, start, &fx, &fy);
    Cursor c{0u, fx, fy};
    push(c, fx, fy, write, wk, path, p, mismatch);
    float prevx = fx, prevy = fy;
    float remaining = 1.0f;
    for (uint32_t i = start + 1u; i < end; ++i) {
        float cx, cy;
        normalized(wk.nm, wk.cp, i, &cx, &cy);
        const float dx = cx - prevx, dy = cy - prevy;
        const float ex = dx * wk.sx, ey = dy * wk.sy;
        const float distance = std::sqrt(ex * ex + ey * ey);
        if (distance > 0.0f) {
            const uint32_t steps = u32_sat(std::fmax(std::floor(distance - remaining) + 1.0f, 0.0f));
            if (write) {
                for (uint32_t step = 0; step < steps; ++step) {
                    const float along = remaining + static_cast<float>(step);
                    const float t = along / distance;
                    push(c, prevx + dx * t, prevy + dy * t, write, wk, path, p, mismatch);
                    if (c.count > wk.capacity) return c.count;
                }
            } else if (steps > 0u) {
                const float t0 = remaining / distance;
                const float t1 = (remaining + static_cast<float>(steps - 1u)) / distance;
                const float ax = prevx + dx * t0, ay = prevy + dy * t0;
                const float bx = prevx + dx * t1, by = prevy + dy * t1;
                // Only the first sample of a segment can repeat the prior one.
                c.count += steps - ((ax == c.lx && ay == c.ly) ? 1u : 0u);
                c.lx = bx;
                c.ly = by;
                if (c.count > wk.capacity) return wk.capacity + 1u;
            }
            remaining = remaining + static_cast<float>(steps) - distance;
        }
        prevx = cx;
        prevy = cy;
    }
    if (!write && edge_out) {
        edge_out[0] = fx; edge_out[1] = fy; edge_out[2] = prevx; edge_out[3] = prevy;
    }
    push(c, prevx, prevy, write, wk, path, p, mismatch);
    // A short closed path keeps its excursion and returning endpoint.
    if (c.count == 1u) {
        for (uint32_t i = start + 1u; i < end; ++i) {
            float nx, ny;
            normalized(wk.nm, wk.cp, i, &nx, &ny);
            if (nx != fx || ny != fy) {
                push(c, nx, ny, write, wk, path, p, mismatch);
                push(c, prevx, prevy, write, wk, path, p, mismatch);
                break;
            }
        }
    }
    return c.count;
}

}  // namespace

// ---------------------------------------------------------------------------
// Pipeline state
// ---------------------------------------------------------------------------
struct or_state {
    or_config cfg;
    uint32_t samples = 0, paths_n = 0, density_pass = 0;
    std::vector<float> xy;
    std::vector<uint32_t> edge_ids, segments, counts, neighbors;
    std::vector<PathRec> paths;
    std::vector<float> edges, horizontal, vertical, normalized;
    std::vector<uint8_t> movable;
    float peak = 0.0f;
};

extern "C" or_state* or_create(const or_config* cfg) {
    auto* s = new or_state();
    s->cfg = *cfg;
    if (s->cfg.shrink == 0.0) s->cfg.shrink = 1.0;
    size_t g = static_cast<size_t>(cfg->width) * cfg->height;
    s->counts.assign(g, 0);
    s->horizontal.assign(g, 0.0f);
    s->vertical.assign(g, 0.0f);
    s->normalized.assign(g, 0.0f);
    return s;
}

extern "C" void or_destroy(or_state* s) { delete s; }

namespace {
// Density::encode (src/density.rs:155-166): blur H, blur V + max, normalise.
void density_pass(or_state* s) {
    float taps[4096];
    double sigma = s->cfg.sigma;
    for (uint32_t i = 0; i < s->density_pass && sigma != 0.0; ++i) sigma *= s->cfg.shrink;
    int R = or_blur_weights(sigma, taps, 4096);
    or_blur(s->counts.data(), s->cfg.width, s->cfg.height, taps, R, s->horizontal.data(), s->vertical.data(),
            &s->peak);
    or_normalize(s->vertical.data(), s->vertical.size(), s->peak, s->normalized.data());
    s->density_pass++;
}
}  // namespace

extern "C" int or_upload(or_state* s, const float* cp, uint32_t n_points, const uint32_t* starts,
                         uint32_t n_starts, uint32_t* samples_out, char* err, size_t errlen) {
    if (n_starts < 2 || starts[0] != 0 || starts[n_starts - 1] != n_points) {
        set_err(err, errlen, "invalid path starts");
        return 3;
    }
    float mn[2] = {3.40282347e+38f, 3.40282347e+38f}, mx[2] = {-3.40282347e+38f, -3.40282347e+38f};
    for (uint32_t i = 0; i < n_points; ++i) {
        mn[0] = std::min(mn[0], cp[2 * i]);
        mn[1] = std::min(mn[1], cp[2 * i + 1]);
        mx[0] = std::max(mx[0], cp[2 * i]);
        mx[1] = std::max(mx[1], cp[2 * i + 1]);
    }
    float nm5[5];
    if (int rc = or_normalization(mn, mx, nm5, err, errlen)) return rc;
    const uint32_t E = n_starts - 1;
    Walk wk{};
    wk.cp = cp;
    wk.starts = starts;
    wk.nm = Norm{nm5[0], nm5[1], nm5[2], nm5[3], nm5[4]};
    wk.sx = s->cfg.resample_scale[0];
    wk.sy = s->cfg.resample_scale[1];
    wk.capacity = s->cfg.capacity;
    wk.w = s->cfg.width;
    wk.h = s->cfg.height;
    wk.accumulate = s->cfg.accumulate_density != 0;
    std::fill(s->counts.begin(), s->counts.end(), 0u);
    s->density_pass = 0;
    // count_paths (resampling.wgsl:139-159); offsets by an exclusive scan in
    // path order instead of atomics.
    std::vector<uint32_t> count(E);
    s->edges.assign(4 * static_cast<size_t>(E), 0.0f);
    PathRec none{0, 0, 0};
    bool dummy = false;
    for (uint32_t p = 0; p < E; ++p) count[p] = resample(wk, p, false, none, &s->edges[4 * p], &dummy);
    s->paths.assign(E, PathRec{0, 0, 0});
    uint64_t total = 0, segs = 0;
    bool overflow = false;
    for (uint32_t p = 0; p < E; ++p) {
        if (count[p] < 2u) continue;
        if (total >= wk.capacity || count[p] > wk.capacity - total) overflow = true;
        s->paths[p] = PathRec{static_cast<uint32_t>(total), static_cast<uint32_t>(segs), count[p]};
        total += count[p];
        segs += count[p] - 1u;
    }
    if (overflow) {
        set_err(err, errlen, "resampling exceeds the sample buffer capacity");
        return 1;
    }
    if (segs == 0) {
        set_err(err, errlen, "resampled graph has no drawable edges");
        return 3;
    }
    s->samples = static_cast<uint32_t>(total);
    s->paths_n = E;
    s->xy.assign(2 * total, 0.0f);
    s->edge_ids.assign(total, 0u);
    s->segments.assign(segs, 0u);
    wk.pts = s->xy.data();
    wk.edge_ids = s->edge_ids.data();
    wk.segments = s->segments.data();
    wk.counts = s->counts.data();
    // emit_paths (resampling.wgsl:162-183)
    bool mismatch = false;
    for (uint32_t p = 0; p < E; ++p) {
        if (s->paths[p].count < 2u) continue;
        uint32_t written = resample(wk, p, true, s->paths[p], nullptr, &mismatch);
        if (written != s->paths[p].count) mismatch = true;
    }
    if (mismatch) {
        set_err(err, errlen, "resampling count and write passes disagree");
        return 2;
    }
    // Movable samples (neighbor_mean.wgsl:61-64).
    s->movable.assign(total, 1);
    for (uint32_t p = 0; p < E; ++p) {
        const PathRec& r = s->paths[p];
        if (r.count < 2u) continue;
        s->movable[r.point_offset] = 0;
        s->movable[r.point_offset + r.count - 1u] = 0;
    }
    s->neighbors.assign(total, 0u);
    if (wk.accumulate) density_pass(s);
    *samples_out = s->samples;
    return 0;
}

// Gpu::iterate: clear density, neighbour mean + splat, density encode.
extern "C" int or_iterate(or_state* s, uint32_t n, int mode) {
    if (s->samples == 0) return 4;
    if (s->cfg.radius == 0) return 8;
    std::vector<float> next(s->xy.size());
    for (uint32_t it = 0; it < n; ++it) {
        std::fill(s->counts.begin(), s->counts.end(), 0u);
        or_neighbor_mean(s->xy.data(), s->movable.data(), s->samples, s->cfg.width, s->cfg.height, s->cfg.radius,
                         mode, s->cfg.threads, next.data(), s->neighbors.data());
        s->xy.swap(next);
        if (s->cfg.accumulate_density) {
            or_splat(s->xy.data(), s->samples, s->cfg.width, s->cfg.height, s->counts.data());
            density_pass(s);
        }
    }
    return 0;
}

extern "C" uint32_t or_samples(const or_state* s) { return s->samples; }
extern "C" uint32_t or_paths(const or_state* s) { return s->paths_n; }
extern "C" void or_get_points(const or_state* s, float* xy, uint32_t* edge_ids) {
    if (xy) std::memcpy(xy, s->xy.data(), s->xy.size() * sizeof(float));
    if (edge_ids) std::memcpy(edge_ids, s->edge_ids.data(), s->edge_ids.size() * sizeof(uint32_t));
}
extern "C" void or_get_paths(const or_state* s, uint32_t* out) {
    for (size_t p = 0; p < s->paths.size(); ++p) {
        out[3 * p] = s->paths[p].point_offset;
        out[3 * p + 1] = s->paths[p].segment_offset;
        out[3 * p + 2] = s->paths[p].count;
    }
}
extern "C" void or_get_segments(const or_state* s, uint32_t* out) {
    std::memcpy(out, s->segments.data(), s->segments.size() * sizeof(uint32_t));
}
extern "C" void or_get_edges(const or_state* s, float* out) {
    std::memcpy(out, s->edges.data(), s->edges.size() * sizeof(float));
}
extern "C" void or_get_counts(const or_state* s, uint32_t* out) {
    std::memcpy(out, s->counts.data(), s->counts.size() * sizeof(uint32_t));
}
extern "C" void or_get_blurred(const or_state* s, float* horizontal, float* vertical, float* peak) {
    if (horizontal) std::memcpy(horizontal, s->horizontal.data(), s->horizontal.size() * sizeof(float));
    if (vertical) std::memcpy(vertical, s->vertical.data(), s->vertical.size() * sizeof(float));
    if (peak) *peak = s->peak;
}
extern "C" void or_get_normalized(const or_state* s, float* out) {
    std::memcpy(out, s->normalized.data(), s->normalized.size() * sizeof(float));
}
extern "C" void or_get_cells(const or_state* s, uint32_t* cell_ids, uint32_t* gw, uint32_t* gh) {
    uint32_t r = s->cfg.radius ? s->cfg.radius : 1u;
    *gw = (s->cfg.width + r - 1) / r;
    *gh = (s->cfg.height + r - 1) / r;
    if (cell_ids) or_cells(s->xy.data(), s->samples, s->cfg.width, s->cfg.height, r, cell_ids);
}
extern "C" void or_get_neighbors(const or_state* s, uint32_t* out) {
    std::memcpy(out, s->neighbors.data(), s->neighbors.size() * sizeof(uint32_t));
}

// ---------------------------------------------------------------------------
// Distortion (src/distortion.rs:10-216), f64 throughout.
// ---------------------------------------------------------------------------
namespace {

struct Curve {
    const float* pts;
    size_t n;
    double length;
};

inline double dist(const float* a, const float* b) {
    return std::hypot(static_cast<double>(b[0]) - a[0], static_cast<double>(b[1]) - a[1]);
}

// distortion.rs:19-40
bool make_curve(const float* pts, size_t n, Curve* c) {
    if (n == 0) return false;
    for (size_t i = 0; i < 2 * n; ++i)
        if (!std::isfinite(pts[i])) return false;
    double length = 0.0;
    for (size_t i = 0; i + 1 < n; ++i) length += dist(pts + 2 * i, pts + 2 * i + 2);
    if (!std::isfinite(length)) return false;
    *c = Curve{pts, n, length};
    return true;
}

// distortion.rs:53-116
struct CurveCursor {
    const Curve* c;
    size_t next_seg;   // index of the next window (pair) to consume
    double traversed;
    double start[2], end[2];
    double start_t, end_t;
    explicit CurveCursor(const Curve* curve) : c(curve), next_seg(0), traversed(0.0) {
        start[0] = end[0] = curve->pts[0];
        start[1] = end[1] = curve->pts[1];
        start_t = end_t = 0.0;
    }
    size_t remaining_windows() const { return (c->n >= 2 ? c->n - 1 : 0) - next_seg; }
    void advance(double t) {
        while (end_t <= t && end_t < 1.0) {
            if (remaining_windows() == 0) {
                start[0] = end[0];
                start[1] = end[1];
                start_t = end_t;
                end_t = 1.0;
                return;
            }
            const float* a = c->pts + 2 * next_seg;
            const float* b = a + 2;
            ++next_seg;
            double length = dist(a, b);
            if (length == 0.0) continue;
            start[0] = a[0]; start[1] = a[1];
            end[0] = b[0]; end[1] = b[1];
            start_t = end_t;
            traversed += length;
            end_t = remaining_windows() == 0 ? 1.0 : traversed / c->length;
        }
    }
    void position(double t, double* out) const {
        if (t >= end_t) { out[0] = end[0]; out[1] = end[1]; return; }
        if (t <= start_t) { out[0] = start[0]; out[1] = start[1]; return; }
        double f = (t - start_t) / (end_t - start_t);
        out[0] = std::fma(f, end[0] - start[0], start[0]);
        out[1] = std::fma(f, end[1] - start[1], start[1]);
    }
};

struct KahanSum {
    double value = 0.0, correction = 0.0;
    void add(double term) {
        double adjusted = term - correction;
        double next = value + adjusted;
        correction = (next - value) - adjusted;
        value = next;
    }
};

// distortion.rs:137-168
bool squared_integral(const Curve& o, const Curve& c, double* out) {
    CurveCursor a(&o), b(&c);
    KahanSum sum;
    double t = 0.0;
    while (!(t >= 1.0)) {
        a.advance(t);
        b.advance(t);
        double next = std::min(a.end_t, b.end_t);
        if (!(next > t && next <= 1.0)) return false;
        double p[2], q[2], r[2], s[2];
        a.position(t, p);
        b.position(t, q);
        a.position(next, r);
        b.position(next, s);
        double ax = p[0] - q[0], ay = p[1] - q[1];
        double bx = r[0] - s[0], by = r[1] - s[1];
        double sx = ax + bx, sy = ay + by;
        double dx = bx - ax, dy = by - ay;
        double mid = std::fma(sx, sx, sy * sy);
        double chg = std::fma(dx, dx, dy * dy);
        sum.add((next - t) * (mid / 4.0 + chg / 12.0));
        t = next;
    }
    if (!(std::isfinite(sum.value) && sum.value >= 0.0)) return false;
    *out = sum.value;
    return true;
}

}  // namespace

extern "C" int or_squared_integral(const float* original, size_t n_original, const float* current,
                                   size_t n_current, double* out) {
    Curve o, c;
    if (!make_curve(original, n_original, &o) || !make_curve(current, n_current, &c)) return 3;
    return squared_integral(o, c, out) ? 0 : 3;
}

// Aggregate::add / finish (distortion.rs:172-216) over edges in point-offset
// order (geometry.rs:64 sorts the edges by offset).
extern "C" int or_distortion(const uint32_t* paths, uint32_t n_paths, const float* original_xy,
                             const float* current_xy, uint32_t size, double* distortion, double* rms_pixels) {
    std::vector<uint32_t> order;
    for (uint32_t p = 0; p < n_paths; ++p)
        if (paths[3 * p + 2] != 0) order.push_back(p);
    std::sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return paths[3 * a] < paths[3 * b]; });
    KahanSum sum;
    uint32_t edges = 0;
    for (uint32_t p : order) {
        const size_t off = paths[3 * p], cnt = paths[3 * p + 2];
        double integral;
        if (or_squared_integral(original_xy + 2 * off, cnt, current_xy + 2 * off, cnt, &integral)) return 3;
        KahanSum trial = sum;
        trial.add(integral);
        if (!std::isfinite(trial.value)) return 3;
        sum = trial;
        ++edges;
    }
    if (edges == 0 || size == 0) return 3;
    double rms = std::sqrt(sum.value / static_cast<double>(edges));
    *distortion = rms / (2.0 * 1.4142135623730951);
    *rms_pixels = rms * (static_cast<double>(size) / 2.0);
    if (!std::isfinite(*distortion) || !std::isfinite(*rms_pixels)) return 3;
    return 0;
}

// ---------------------------------------------------------------------------
// Density-gradient advection step (an extension beyond the reference, in the
// manner of kernel-density-estimation edge bundling: samples climb the
// gradient of the blurred density, then relax along their path). The CUDA
// kernel (csrc/advect.cu) follows the same operation order:
//  - map position (u, v) = ((x * 0.5 + 0.5) * (W - 1), (0.5 - y * 0.5) * (H - 1)),
//    the splat's texel space;
//  - density sampled bilinearly with clamp-to-edge; gradient by central
//    differences one texel apart, halved;
//  - a step of `step` texels along the unit gradient (none when its length is
//    not above 1e-12), back to clip units by 2 / (W - 1) and -2 / (H - 1);
//  - Laplacian relaxation a + smooth * ((a_prev + a_next) * 0.5 - a) with the
//    advected neighbours along the path; first and last samples stay fixed.
namespace {

float density_at(const float* d, uint32_t w, uint32_t h, float u, float v) {
    const float uc = std::fmin(std::fmax(u, 0.0f), static_cast<float>(w - 1u));
    const float vc = std::fmin(std::fmax(v, 0.0f), static_cast<float>(h - 1u));
    const float fx0 = std::floor(uc), fy0 = std::floor(vc);
    const float fx = uc - fx0, fy = vc - fy0;
    const uint32_t x0 = static_cast<uint32_t>(fx0), y0 = static_cast<uint32_t>(fy0);
    const uint32_t x1 = std::min(x0 + 1u, w - 1u), y1 = std::min(y0 + 1u, h - 1u);
    const float top = d[static_cast<size_t>(y0) * w + x0] * (1.0f - fx) + d[static_cast<size_t>(y0) * w + x1] * fx;
    const float bottom = d[static_cast<size_t>(y1) * w + x0] * (1.0f - fx) + d[static_cast<size_t>(y1) * w + x1] * fx;
    return top * (1.0f - fy) + bottom * fy;
}

void advected(const float* xy, size_t i, const float* d, uint32_t w, uint32_t h, float step, float sxi, float syi,
              float* out) {
    const float x = xy[2 * i], y = xy[2 * i + 1];
    const float u = (x * 0.5f + 0.5f) * static_cast<float>(w - 1u);
    const float v = (0.5f - y * 0.5f) * static_cast<float>(h - 1u);
    const float gu = (density_at(d, w, h, u + 1.0f, v) - density_at(d, w, h, u - 1.0f, v)) * 0.5f;
    const float gv = (density_at(d, w, h, u, v + 1.0f) - density_at(d, w, h, u, v - 1.0f)) * 0.5f;
    const float len = std::sqrt(gu * gu + gv * gv);
    float du = 0.0f, dv = 0.0f;
    if (len > 1e-12f) {
        du = step * (gu / len);
        dv = step * (gv / len);
    }
    out[0] = x + du * sxi;
    out[1] = y - dv * syi;
}

}  // namespace

extern "C" void or_advect(const float* xy, const uint32_t* edge_ids, size_t n, const float* density, uint32_t w,
                          uint32_t h, float step, float smooth, float* out_xy) {
    const float sxi = 2.0f / static_cast<float>(w - 1u), syi = 2.0f / static_cast<float>(h - 1u);
    auto movable = [&](size_t i) {
        return i > 0 && i + 1 < n && edge_ids[i - 1] == edge_ids[i] && edge_ids[i + 1] == edge_ids[i];
    };
#pragma omp parallel for schedule(static)
    for (long long ii = 0; ii < static_cast<long long>(n); ++ii) {
        const size_t i = static_cast<size_t>(ii);
        if (!movable(i)) {
            out_xy[2 * i] = xy[2 * i];
            out_xy[2 * i + 1] = xy[2 * i + 1];
            continue;
        }
        float a[2], p[2], q[2];
        advected(xy, i, density, w, h, step, sxi, syi, a);
        if (movable(i - 1)) {
            advected(xy, i - 1, density, w, h, step, sxi, syi, p);
        } else {
            p[0] = xy[2 * (i - 1)];
            p[1] = xy[2 * (i - 1) + 1];
        }
        if (movable(i + 1)) {
            advected(xy, i + 1, density, w, h, step, sxi, syi, q);
        } else {
            q[0] = xy[2 * (i + 1)];
            q[1] = xy[2 * (i + 1) + 1];
        }
        for (int k = 0; k < 2; ++k) out_xy[2 * i + k] = a[k] + smooth * ((p[k] + q[k]) * 0.5f - a[k]);
    }
}
