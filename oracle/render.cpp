// render.cpp — CPU restatement of the path rasterisation behind the noisiness
// report (src/shaders/render_paths.wgsl:35-101, src/gpu.rs:572-620,
// src/noisiness.rs:30-74). TEST INFRASTRUCTURE ONLY: the oracle of the CUDA
// rasteriser (csrc/render.cu), which follows the same rules:
//
//  - each segment (i, i+1) of the segments list is a quad of half-width 0.001
//    clip around the two samples (vs_main: normal = (-dy, dx) * (0.001 /
//    max(length(d), 1e-10)), corners first +/- normal, second +/- normal),
//    drawn as the strip triangles (v0, v1, v2), (v2, v1, v3), in list order;
//  - viewport x = (X * 0.5 + 0.5) * W, y = (0.5 - Y * 0.5) * H, snapped to
//    1/256 pixel; coverage at the standard sample positions of 1, 2 or 4
//    samples per pixel, edge functions with a top-left tie rule;
//  - fs_main's colour at the pixel centre: the normalised density stored as
//    f16 and filtered bilinearly with clamp-to-edge at texel coordinate
//    uv * (size - 1), or edge_id / (max(edges, 2) - 1); 16-stop palette lerp;
//  - alpha blending (src * 0.1 + dst * 0.9) into 8-bit samples in draw
//    order, cleared to (0.025, 0.025, 0.035);
//  - endpoint dots (optional): the first and last sample of every path with
//    at least two samples; a square of +/- 3 pixels (vs_endpoint) whose
//    offset, interpolated at each covered sample by the barycentric weights
//    of the snapped triangle, discards the sample outside the unit circle
//    (outline, palette[0] * 0.1, opaque) or outside radius 2/3 (centre, the
//    palette's endpoint colour); all outlines before all centres;
//  - the resolve rounds the mean of a pixel's samples half to even.
// Exact agreement with a hardware rasteriser is not claimed: its subpixel
// snapping, filtering weights and blend precision are its own.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "oracle.h"

namespace {

// 16 evenly spaced samples of the colour maps the reference uses
// (src/palette.rs:40-144): viridis, cividis, plasma (matplotlib) and batlow
// (Crameri's scientific colour maps), with the endpoint colours of
// src/palette.rs:26-33.
const float kPalettes[4][16][3] = {
    {{0.267004f, 0.004874f, 0.329415f}, {0.282656f, 0.100196f, 0.422160f}, {0.277134f, 0.185228f, 0.489898f},
     {0.253935f, 0.265254f, 0.529983f}, {0.221989f, 0.339161f, 0.548752f}, {0.190631f, 0.407061f, 0.556089f},
     {0.163625f, 0.471133f, 0.558148f}, {0.139147f, 0.533812f, 0.555298f}, {0.120565f, 0.596422f, 0.543611f},
     {0.134692f, 0.658636f, 0.517649f}, {0.208030f, 0.718701f, 0.472873f}, {0.327796f, 0.773980f, 0.406640f},
     {0.477504f, 0.821444f, 0.318195f}, {0.647257f, 0.858400f, 0.209861f}, {0.824940f, 0.884720f, 0.106217f},
     {0.993248f, 0.906157f, 0.143936f}},
    {{0.000000f, 0.135112f, 0.304751f}, {0.000000f, 0.181610f, 0.421859f}, {0.117612f, 0.225935f, 0.434308f},
     {0.208926f, 0.272546f, 0.424809f}, {0.279411f, 0.318677f, 0.423031f}, {0.342246f, 0.364939f, 0.428559f},
     {0.401418f, 0.411790f, 0.440708f}, {0.458366f, 0.459552f, 0.460457f}, {0.517920f, 0.508454f, 0.472707f},
     {0.582087f, 0.558670f, 0.468118f}, {0.648222f, 0.610553f, 0.454801f}, {0.716177f, 0.664384f, 0.432386f},
     {0.785965f, 0.720438f, 0.399613f}, {0.857809f, 0.778969f, 0.353259f}, {0.932180f, 0.840159f, 0.285880f},
     {0.995737f, 0.909344f, 0.217772f}},
    {{0.050383f, 0.029803f, 0.527975f}, {0.200445f, 0.017902f, 0.593364f}, {0.312543f, 0.008239f, 0.635700f},
     {0.417642f, 0.000564f, 0.658390f}, {0.517933f, 0.021563f, 0.654109f}, {0.610667f, 0.090204f, 0.619951f},
     {0.692840f, 0.165141f, 0.564522f}, {0.764193f, 0.240396f, 0.502126f}, {0.826588f, 0.315714f, 0.441316f},
     {0.881443f, 0.392529f, 0.383229f}, {0.928329f, 0.472975f, 0.326067f}, {0.965024f, 0.559118f, 0.268513f},
     {0.988260f, 0.652325f, 0.211364f}, {0.994141f, 0.753137f, 0.161404f}, {0.977995f, 0.861432f, 0.142808f},
     {0.940015f, 0.975158f, 0.131326f}},
    {{0.005193f, 0.098238f, 0.349842f}, {0.050795f, 0.196274f, 0.366684f}, {0.069002f, 0.270922f, 0.378774f},
     {0.094462f, 0.332712f, 0.385116f}, {0.149706f, 0.386975f, 0.374449f}, {0.237075f, 0.428325f, 0.335634f},
     {0.339469f, 0.461685f, 0.279468f}, {0.449052f, 0.493684f, 0.221074f}, {0.570016f, 0.526186f, 0.175273f},
     {0.701421f, 0.555294f, 0.185478f}, {0.825472f, 0.577725f, 0.264197f}, {0.928323f, 0.605212f, 0.385404f},
     {0.983574f, 0.649590f, 0.538819f}, {0.993074f, 0.699161f, 0.687519f}, {0.989411f, 0.747997f, 0.829372f},
     {0.981354f, 0.800406f, 0.981267f}},
};
const float kEndpointColors[4][3] = {
    {1.0f, 0.4f, 0.7f}, {1.0f, 0.35f, 0.75f}, {0.15f, 0.9f, 1.0f}, {0.1f, 0.85f, 1.0f}};

struct Pt {
    int64_t x, y;
};

// f32 -> IEEE binary16 (round to nearest even) -> f32: the value rounded to
// the f16 quantum of its binade (2^(e-10), subnormal quantum 2^-24).
float to_half_and_back(float v) {
    if (std::isnan(v)) return v;
    const float a = std::fabs(v);
    if (a >= 65520.0f) return std::copysign(INFINITY, v);
    if (a == 0.0f) return v;
    int e = 0;
    std::frexp(a, &e);                       // a = m * 2^e, m in [0.5, 1)
    int lead = e - 1;
    if (lead < -14) lead = -14;
    const double q = std::ldexp(1.0, lead - 10);
    const double r = std::nearbyint(static_cast<double>(a) / q) * q;
    return std::copysign(static_cast<float>(r), v);
}

int samples_of(int msaa, int offs[4][2]) {
    if (msaa == 4) {
        const int o[4][2] = {{96, 32}, {224, 96}, {32, 160}, {160, 224}};
        std::memcpy(offs, o, sizeof(o));
        return 4;
    }
    if (msaa == 2) {
        const int o[2][2] = {{192, 192}, {64, 64}};
        std::memcpy(offs, o, sizeof(o));
        return 2;
    }
    offs[0][0] = offs[0][1] = 128;
    return 1;
}

bool top_left(const Pt& a, const Pt& b) {
    const int64_t dx = b.x - a.x, dy = b.y - a.y;
    return dy > 0 || (dy == 0 && dx < 0);
}

int64_t edge_fn(const Pt& a, const Pt& b, const Pt& p) { return (b.x - a.x) * (p.y - a.y) - (b.y - a.y) * (p.x - a.x); }

// The endpoint squares of all drawn paths (vs_endpoint + fs_endpoint*): every
// covered sample whose interpolated offset lies within radius2 takes the
// opaque colour.
void draw_endpoints(const float* xy, const uint32_t* paths, uint32_t n_paths, uint32_t w, uint32_t h, int ns,
                    const int offs[4][2], float radius2, const float color[3], uint8_t* samp) {
    uint8_t c8[3];
    for (int ch = 0; ch < 3; ++ch) {
        // ALPHA_BLENDING with source alpha 1: src * 1 + dst * 0.
        const float r = color[ch] * 1.0f + 0.0f;
        c8[ch] = static_cast<uint8_t>(std::fmin(std::fmax(std::nearbyint(r * 255.0f), 0.0f), 255.0f));
    }
    const float corner[4][2] = {{-1.0f, 1.0f}, {-1.0f, -1.0f}, {1.0f, 1.0f}, {1.0f, -1.0f}};
    for (uint32_t p = 0; p < n_paths; ++p) {
        const uint32_t offset = paths[3 * p], count = paths[3 * p + 2];
        if (count < 2) continue;
        for (int end = 0; end < 2; ++end) {
            const uint32_t i = end ? offset + count - 1 : offset;
            const float cx = xy[2 * i], cy = xy[2 * i + 1];
            Pt v[4];
            bool far = false;
            for (int k = 0; k < 4; ++k) {
                const float X = cx + corner[k][0] * 3.0f * 2.0f / static_cast<float>(w);
                const float Y = cy + corner[k][1] * 3.0f * 2.0f / static_cast<float>(h);
                const float fx = (X * 0.5f + 0.5f) * static_cast<float>(w);
                const float fy = (0.5f - Y * 0.5f) * static_cast<float>(h);
                if (!(std::fabs(fx) < 1.0e6f) || !(std::fabs(fy) < 1.0e6f)) far = true;
                v[k] = Pt{static_cast<int64_t>(std::nearbyint(fx * 256.0f)), static_cast<int64_t>(std::nearbyint(fy * 256.0f))};
            }
            if (far) continue;
            const int tri[2][3] = {{0, 1, 2}, {2, 1, 3}};
            for (int t = 0; t < 2; ++t) {
                int ia = tri[t][0], ib = tri[t][1], ic = tri[t][2];
                const int64_t area0 = edge_fn(v[ia], v[ib], v[ic]);
                if (area0 == 0) continue;
                if (area0 < 0) std::swap(ib, ic);
                const Pt a = v[ia], b = v[ib], c = v[ic];
                const float area = static_cast<float>(edge_fn(a, b, c));
                const int64_t minx = std::min(a.x, std::min(b.x, c.x)), maxx = std::max(a.x, std::max(b.x, c.x));
                const int64_t miny = std::min(a.y, std::min(b.y, c.y)), maxy = std::max(a.y, std::max(b.y, c.y));
                const int64_t x0 = std::max<int64_t>(0, minx >> 8), x1 = std::min<int64_t>(w - 1, maxx >> 8);
                const int64_t y0 = std::max<int64_t>(0, miny >> 8), y1 = std::min<int64_t>(h - 1, maxy >> 8);
                const bool tl_ab = top_left(a, b), tl_bc = top_left(b, c), tl_ca = top_left(c, a);
                for (int64_t y = y0; y <= y1; ++y)
                    for (int64_t x = x0; x <= x1; ++x)
                        for (int q = 0; q < ns; ++q) {
                            const Pt s{x * 256 + offs[q][0], y * 256 + offs[q][1]};
                            const int64_t wc = edge_fn(a, b, s), wa = edge_fn(b, c, s), wb = edge_fn(c, a, s);
                            if (!(wc > 0 || (wc == 0 && tl_ab))) continue;
                            if (!(wa > 0 || (wa == 0 && tl_bc))) continue;
                            if (!(wb > 0 || (wb == 0 && tl_ca))) continue;
                            const float la = static_cast<float>(wa) / area, lb = static_cast<float>(wb) / area,
                                        lc = static_cast<float>(wc) / area;
                            const float ox = la * corner[ia][0] + lb * corner[ib][0] + lc * corner[ic][0];
                            const float oy = la * corner[ia][1] + lb * corner[ib][1] + lc * corner[ic][1];
                            if (ox * ox + oy * oy > radius2) continue;
                            std::memcpy(&samp[((static_cast<size_t>(y) * w + x) * ns + q) * 3], c8, 3);
                        }
            }
        }
    }
}

}  // namespace

extern "C" float or_half_round(float v) { return to_half_and_back(v); }

extern "C" int or_render(const float* xy, const uint32_t* edge_ids, const uint32_t* segments, uint32_t n_segments,
                         uint32_t n_edges, const float* density, uint32_t w, uint32_t h, int color_by_edge,
                         int palette, int msaa, const uint32_t* paths, uint32_t n_paths, int endpoint_dots,
                         uint8_t* rgba, uint64_t* colored) {
    if (w == 0 || h == 0 || palette < 0 || palette > 3 || (msaa != 1 && msaa != 2 && msaa != 4)) return 1;
    int offs[4][2];
    const int ns = samples_of(msaa, offs);
    const uint8_t bg[3] = {static_cast<uint8_t>(std::nearbyint(0.025f * 255.0f)),
                           static_cast<uint8_t>(std::nearbyint(0.025f * 255.0f)),
                           static_cast<uint8_t>(std::nearbyint(0.035f * 255.0f))};
    std::vector<uint8_t> samp(static_cast<size_t>(w) * h * ns * 3);
    for (size_t i = 0; i < samp.size(); i += 3) std::memcpy(&samp[i], bg, 3);
    const float edge_den = static_cast<float>((n_edges > 2u ? n_edges : 2u) - 1u);
    const float alpha = 0.1f, keep = 1.0f - 0.1f;
    const float (*pal)[3] = kPalettes[palette];

    for (uint32_t s = 0; s < n_segments; ++s) {
        const uint32_t i = segments[s];
        const float px = xy[2 * i], py = xy[2 * i + 1], qx = xy[2 * i + 2], qy = xy[2 * i + 3];
        const float dx = qx - px, dy = qy - py;
        const float len = std::sqrt(dx * dx + dy * dy);
        const float k = 0.001f / std::fmax(len, 1e-10f);
        const float nx = -dy * k, ny = dx * k;
        const float cx[4] = {px + nx, px - nx, qx + nx, qx - nx};
        const float cy[4] = {py + ny, py - ny, qy + ny, qy - ny};
        Pt v[4];
        bool far = false;
        for (int c = 0; c < 4; ++c) {
            const float fx = (cx[c] * 0.5f + 0.5f) * static_cast<float>(w);
            const float fy = (0.5f - cy[c] * 0.5f) * static_cast<float>(h);
            if (!(std::fabs(fx) < 1.0e6f) || !(std::fabs(fy) < 1.0e6f)) far = true;
            v[c] = Pt{static_cast<int64_t>(std::nearbyint(fx * 256.0f)), static_cast<int64_t>(std::nearbyint(fy * 256.0f))};
        }
        if (far) continue;
        const float edge_value = static_cast<float>(edge_ids[i]) / edge_den;
        const int tri[2][3] = {{0, 1, 2}, {2, 1, 3}};
        for (int t = 0; t < 2; ++t) {
            Pt a = v[tri[t][0]], b = v[tri[t][1]], c = v[tri[t][2]];
            int64_t area = (b.x - a.x) * (c.y - a.y) - (b.y - a.y) * (c.x - a.x);
            if (area == 0) continue;
            if (area < 0) std::swap(b, c);
            const int64_t minx = std::min(a.x, std::min(b.x, c.x)), maxx = std::max(a.x, std::max(b.x, c.x));
            const int64_t miny = std::min(a.y, std::min(b.y, c.y)), maxy = std::max(a.y, std::max(b.y, c.y));
            const int64_t x0 = std::max<int64_t>(0, minx >> 8), x1 = std::min<int64_t>(w - 1, maxx >> 8);
            const int64_t y0 = std::max<int64_t>(0, miny >> 8), y1 = std::min<int64_t>(h - 1, maxy >> 8);
            const Pt e[3][2] = {{a, b}, {b, c}, {c, a}};
            bool tl[3];
            for (int j = 0; j < 3; ++j) tl[j] = top_left(e[j][0], e[j][1]);
            for (int64_t y = y0; y <= y1; ++y)
                for (int64_t x = x0; x <= x1; ++x) {
                    float color[3];
                    bool have_color = false;
                    for (int q = 0; q < ns; ++q) {
                        const Pt p{x * 256 + offs[q][0], y * 256 + offs[q][1]};
                        bool in = true;
                        for (int j = 0; j < 3 && in; ++j) {
                            const Pt& ea = e[j][0];
                            const Pt& eb = e[j][1];
                            const int64_t f = (eb.x - ea.x) * (p.y - ea.y) - (eb.y - ea.y) * (p.x - ea.x);
                            in = f > 0 || (f == 0 && tl[j]);
                        }
                        if (!in) continue;
                        if (!have_color) {
                            float value = edge_value;
                            if (!color_by_edge) {
                                const float u = (static_cast<float>(x) + 0.5f) / static_cast<float>(w);
                                const float vv = (static_cast<float>(y) + 0.5f) / static_cast<float>(h);
                                const float tx = u * static_cast<float>(w - 1u), ty = vv * static_cast<float>(h - 1u);
                                const float fx0 = std::floor(tx), fy0 = std::floor(ty);
                                const float wx = tx - fx0, wy = ty - fy0;
                                const int64_t ix0 = std::min<int64_t>(std::max<int64_t>(static_cast<int64_t>(fx0), 0), w - 1);
                                const int64_t iy0 = std::min<int64_t>(std::max<int64_t>(static_cast<int64_t>(fy0), 0), h - 1);
                                const int64_t ix1 = std::min<int64_t>(ix0 + 1, w - 1), iy1 = std::min<int64_t>(iy0 + 1, h - 1);
                                const float d00 = to_half_and_back(density[iy0 * w + ix0]);
                                const float d10 = to_half_and_back(density[iy0 * w + ix1]);
                                const float d01 = to_half_and_back(density[iy1 * w + ix0]);
                                const float d11 = to_half_and_back(density[iy1 * w + ix1]);
                                const float top = d00 * (1.0f - wx) + d10 * wx;
                                const float bottom = d01 * (1.0f - wx) + d11 * wx;
                                value = top * (1.0f - wy) + bottom * wy;
                                value = std::fmin(std::fmax(value, 0.0f), 1.0f);
                            }
                            const float stop = value * 15.0f;
                            uint32_t idx = static_cast<uint32_t>(stop);
                            if (idx > 14u) idx = 14u;
                            const float f = stop - static_cast<float>(idx);
                            for (int ch = 0; ch < 3; ++ch) color[ch] = pal[idx][ch] * (1.0f - f) + pal[idx + 1][ch] * f;
                            have_color = true;
                        }
                        uint8_t* d = &samp[((static_cast<size_t>(y) * w + x) * ns + q) * 3];
                        for (int ch = 0; ch < 3; ++ch) {
                            const float dst = static_cast<float>(d[ch]) / 255.0f;
                            const float r = color[ch] * alpha + dst * keep;
                            float z = std::nearbyint(r * 255.0f);
                            z = std::fmin(std::fmax(z, 0.0f), 255.0f);
                            d[ch] = static_cast<uint8_t>(z);
                        }
                    }
                }
        }
    }
    if (endpoint_dots) {
        const float outline[3] = {pal[0][0] * 0.1f, pal[0][1] * 0.1f, pal[0][2] * 0.1f};
        const float inner = 1.0f - 1.0f / 3.0f;
        draw_endpoints(xy, paths, n_paths, w, h, ns, offs, 1.0f, outline, samp.data());
        draw_endpoints(xy, paths, n_paths, w, h, ns, offs, inner * inner, kEndpointColors[palette], samp.data());
    }
    uint64_t count = 0;
    for (size_t pix = 0; pix < static_cast<size_t>(w) * h; ++pix) {
        bool differs = false;
        for (int ch = 0; ch < 3; ++ch) {
            uint32_t sum = 0;
            for (int q = 0; q < ns; ++q) sum += samp[(pix * ns + q) * 3 + ch];
            uint32_t v = sum / ns;
            const uint32_t rem = sum % ns;
            if (ns > 1) {
                const uint32_t half = ns / 2;
                if (rem > half || (rem == half && (v & 1u))) ++v;
            }
            rgba[pix * 4 + ch] = static_cast<uint8_t>(v);
            differs |= v != bg[ch];
        }
        rgba[pix * 4 + 3] = 255;
        count += differs ? 1 : 0;
    }
    if (colored) *colored = count;
    return 0;
}
