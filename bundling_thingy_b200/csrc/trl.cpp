// trl.cpp — trail-file loader (src/graph.rs:35-107).
//
// One pass over the text without per-token allocations. Rules of
// Graph::parse: lines split like str::lines(); tokens split on single spaces;
// the first token of a line is skipped, as are empty tokens and tokens that
// start with '(' or '<'; coordinates are x y pairs parsed with Rust's f32
// grammar (correctly rounded); non-finite values are errors; consecutive equal
// points of an edge are dropped; edges with fewer than two points are dropped;
// starts end with a sentinel; an empty graph is an error.
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "host.h"

namespace bt {
namespace {

bool rust_float_syntax(const char* s, size_t n) {
    size_t i = 0;
    if (i < n && (s[i] == '+' || s[i] == '-')) ++i;
    auto ieq = [&](const char* word) {
        const size_t m = std::strlen(word);
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
        size_t e = 0;
        while (i < n && s[i] >= '0' && s[i] <= '9') { ++i; ++e; }
        if (e == 0) return false;
    }
    return i == n;
}

bool parse_token(const char* s, size_t n, float* out) {
    if (!rust_float_syntax(s, n)) return false;
    char buf[128];
    std::string big;
    const char* z = buf;
    if (n < sizeof(buf)) {
        std::memcpy(buf, s, n);
        buf[n] = 0;
    } else {
        big.assign(s, n);
        z = big.c_str();
    }
    char* end = nullptr;
    *out = std::strtof(z, &end);   // correctly rounded, like Rust's parse::<f32>
    return end == z + n;
}

}  // namespace

bool parse_trl(const char* text, size_t len, HostGraph* g, std::string* err) {
    g->xy.clear();
    g->starts.clear();
    g->min[0] = g->min[1] = 3.40282347e+38f;     // Point::MAX
    g->max[0] = g->max[1] = -3.40282347e+38f;    // Point::MIN
    size_t pos = 0, line = 0;
    while (pos < len) {
        const char* nl = static_cast<const char*>(std::memchr(text + pos, '\n', len - pos));
        size_t stop = nl ? static_cast<size_t>(nl - text) : len;
        size_t end = stop;
        if (nl && end > pos && text[end - 1] == '\r') --end;   // "\r\n" only
        const size_t start = g->xy.size() / 2;
        // Tokens of [pos, end) split on ' '; the first is skipped.
        size_t a = pos;
        bool first = true;
        bool want_y = false;
        float x = 0.0f;
        while (true) {
            const char* sp = static_cast<const char*>(std::memchr(text + a, ' ', end - a));
            const size_t b = sp ? static_cast<size_t>(sp - text) : end;
            const char* tok = text + a;
            const size_t n = b - a;
            if (first) {
                first = false;
            } else if (want_y) {
                float y;
                if (!parse_token(tok, n, &y)) {
                    *err = "line " + std::to_string(line + 1) + " y: invalid coordinate";
                    return false;
                }
                want_y = false;
                if (!std::isfinite(x) || !std::isfinite(y)) {
                    *err = "non-finite TRL coordinate";
                    return false;
                }
                const size_t have = g->xy.size() / 2;
                if (!(have > start && g->xy[2 * have - 2] == x && g->xy[2 * have - 1] == y)) {
                    g->xy.push_back(x);
                    g->xy.push_back(y);
                }
            } else if (n != 0 && tok[0] != '(' && tok[0] != '<') {
                if (!parse_token(tok, n, &x)) {
                    *err = "line " + std::to_string(line + 1) + " x: invalid coordinate";
                    return false;
                }
                want_y = true;
            }
            if (!sp) break;
            a = b + 1;
        }
        if (want_y) {
            *err = "line " + std::to_string(line + 1) + " y: unexpected end of TRL line";
            return false;
        }
        const size_t have = g->xy.size() / 2;
        if (have - start < 2) {
            g->xy.resize(2 * start);
        } else {
            if (start > 0xFFFFFFFFull) {
                *err = "too many control points";
                return false;
            }
            g->starts.push_back(static_cast<uint32_t>(start));
            for (size_t k = start; k < have; ++k) {
                g->min[0] = std::fmin(g->min[0], g->xy[2 * k]);
                g->min[1] = std::fmin(g->min[1], g->xy[2 * k + 1]);
                g->max[0] = std::fmax(g->max[0], g->xy[2 * k]);
                g->max[1] = std::fmax(g->max[1], g->xy[2 * k + 1]);
            }
        }
        pos = nl ? stop + 1 : len;
        ++line;
    }
    if (g->xy.size() / 2 > 0xFFFFFFFFull) {
        *err = "too many control points";
        return false;
    }
    g->starts.push_back(static_cast<uint32_t>(g->xy.size() / 2));
    if (g->xy.empty()) {
        *err = "graph has no drawable edges";
        return false;
    }
    return true;
}

bool load_trl(const char* path, HostGraph* g, std::string* err) {
    FILE* f = std::fopen(path, "rb");
    if (!f) {
        *err = std::string("read ") + path + ": " + std::strerror(errno);
        return false;
    }
    std::string text;
    char buf[1 << 16];
    size_t n;
    while ((n = std::fread(buf, 1, sizeof(buf), f)) > 0) text.append(buf, n);
    const bool ok = !std::ferror(f);
    std::fclose(f);
    if (!ok) {
        *err = std::string("read ") + path;
        return false;
    }
    return parse_trl(text.data(), text.size(), g, err);
}

// src/graph.rs:79-91
bool normalization(const float mn[2], const float mx[2], float out[5], std::string* err) {
    const float rx = mx[0] - mn[0];
    const float ry = mx[1] - mn[1];
    const float span = std::fmax(rx, ry);
    if (!(span > 0.0f && std::isfinite(span))) {
        *err = "graph has invalid extent";
        return false;
    }
    const float scale = 0.95f / span;
    if (!std::isfinite(scale)) {
        *err = "graph normalization scale is not finite";
        return false;
    }
    out[0] = mn[0];
    out[1] = mn[1];
    out[2] = scale;
    out[3] = (1.0f - scale * rx) / 2.0f;
    out[4] = (1.0f - scale * ry) / 2.0f;
    return true;
}

}  // namespace bt
