// render.cu — the reference's render pass (src/shaders/render_paths.wgsl:35-101,
// src/gpu.rs:572-620) into a headless RGBA8 image, and the noisiness count of
// src/noisiness.rs:44-74 (pixels whose RGB differs from the clear colour).
//
// Rules, stated identically by the oracle's rasteriser:
//  - segment s of the segments list, samples (i, i+1), is a quad of
//    half-width 0.001 clip: normal = (-dy, dx) * (0.001 / max(length(d),
//    1e-10)); corners first + n, first - n, second + n, second - n; strip
//    triangles (v0, v1, v2), (v2, v1, v3); segments are drawn in list order;
//  - viewport x = (X * 0.5 + 0.5) * W, y = (0.5 - Y * 0.5) * H, snapped to
//    1/256 pixel; the standard 1/2/4-sample positions; 64-bit edge functions
//    with a top-left tie rule;
//  - colour of a (pixel, segment): the normalised density stored as f16 and
//    filtered bilinearly with clamp-to-edge at texel coordinate
//    uv * (size - 1) of the pixel centre, or edge_id / (max(edges, 2) - 1);
//    16-stop palette lerp (fs_main);
//  - blending src * 0.1 + dst * 0.9 into 8-bit samples in draw order, from
//    the clear colour (0.025, 0.025, 0.035);
//  - optional endpoint dots: opaque outline discs (radius 3 px, palette[0] *
//    0.1) then opaque centres (radius 2 px, the palette's endpoint colour) at
//    the first and last sample of every path with two or more samples, the
//    disc test on the offset interpolated with the snapped triangle's
//    barycentric weights (vs_endpoint, fs_endpoint_outline, fs_endpoint);
//  - the resolve rounds the mean of a pixel's samples half to even.
// A hardware rasteriser snaps, filters and blends with its own precision, so
// agreement with the reference's images is approximate.
//
// GPU plan (sort-middle): each segment's pixel bounding box is binned into
// square screen tiles; a stable counting sort by tile keeps every tile's list
// in draw order; one CTA per tile walks its list, each thread holding its
// pixels' samples in registers, and writes the samples; the endpoint passes
// overwrite samples; the resolve writes RGBA8 and counts the coloured pixels.
#include <climits>

#include <cuda_fp16.h>

#include "kernels.cuh"
#include "scan.cuh"

namespace bt {
namespace {

__constant__ float kPalette[4][16][3] = {
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
__constant__ float kEndpointColor[4][3] = {
    {1.0f, 0.4f, 0.7f}, {1.0f, 0.35f, 0.75f}, {0.15f, 0.9f, 1.0f}, {0.1f, 0.85f, 1.0f}};

// Sample offsets in 1/256 pixel.
__device__ __forceinline__ void sample_offset(int ns, int q, int* ox, int* oy) {
    if (ns == 4) {
        *ox = q == 0 ? 96 : q == 1 ? 224 : q == 2 ? 32 : 160;
        *oy = q == 0 ? 32 : q == 1 ? 96 : q == 2 ? 160 : 224;
    } else if (ns == 2) {
        *ox = *oy = q == 0 ? 192 : 64;
    } else {
        *ox = *oy = 128;
    }
}

// One triangle's three edges: edge j runs from (ax, ay) by (dx, dy); a point
// p is inside when every f_j = dx*(p.y-ay) - dy*(p.x-ax) > 0, or = 0 on a
// top-left edge (dy > 0, or dy = 0 and dx < 0).
struct TriSetup {
    int ax[3], ay[3], dx[3], dy[3];
};

// A segment's two triangles, the union of their pixel boxes (clipped to the
// image; x0 > x1 when nothing can be covered) and its first sample.
struct SegSetup {
    TriSetup t[2];
    int x0, y0, x1, y1;
    uint32_t first;
    uint32_t valid;   // bit k: triangle k has nonzero area
};

__device__ __forceinline__ long long edge_fn(int ax, int ay, int dx, int dy, long long px, long long py) {
    return static_cast<long long>(dx) * (py - ay) - static_cast<long long>(dy) * (px - ax);
}

__device__ __forceinline__ bool inside(const TriSetup& t, long long px, long long py) {
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        const long long f = edge_fn(t.ax[j], t.ay[j], t.dx[j], t.dy[j], px, py);
        const bool tl = t.dy[j] > 0 || (t.dy[j] == 0 && t.dx[j] < 0);
        if (!(f > 0 || (f == 0 && tl))) return false;
    }
    return true;
}

// The viewport position of a clip point, snapped to 1/256 pixel; false when
// it is absurdly far outside the frame (such a primitive is skipped).
__device__ __forceinline__ bool snap(float X, float Y, uint32_t w, uint32_t h, int* sx, int* sy) {
    const float fx = __fmul_rn(__fadd_rn(__fmul_rn(X, 0.5f), 0.5f), static_cast<float>(w));
    const float fy = __fmul_rn(__fsub_rn(0.5f, __fmul_rn(Y, 0.5f)), static_cast<float>(h));
    const bool ok = fabsf(fx) < 1.0e6f && fabsf(fy) < 1.0e6f;
    *sx = ok ? static_cast<int>(rintf(__fmul_rn(fx, 256.0f))) : 0;
    *sy = ok ? static_cast<int>(rintf(__fmul_rn(fy, 256.0f))) : 0;
    return ok;
}

// Orients triangle (order[0], order[1], order[2]) of the snapped corners:
// swaps order[1] and order[2] when the area is negative; false for zero
// area.
__device__ __forceinline__ bool orient(const int* vx, const int* vy, int* order, long long* area) {
    const int a = order[0], b = order[1], c = order[2];
    const long long ar = static_cast<long long>(vx[b] - vx[a]) * (vy[c] - vy[a]) -
                         static_cast<long long>(vy[b] - vy[a]) * (vx[c] - vx[a]);
    if (ar == 0) return false;
    if (ar < 0) {
        order[1] = c;
        order[2] = b;
    }
    *area = ar < 0 ? -ar : ar;
    return true;
}

__device__ __forceinline__ void set_edges(const int* vx, const int* vy, const int* order, TriSetup* t) {
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        const int u = order[j], v = order[j == 2 ? 0 : j + 1];
        t->ax[j] = vx[u];
        t->ay[j] = vy[u];
        t->dx[j] = vx[v] - vx[u];
        t->dy[j] = vy[v] - vy[u];
    }
}

// The snapped corners of the quad of the segment starting at sample i
// (vs_main + the viewport); false when one is too far off screen.
__device__ __forceinline__ bool quad_corners(const RenderArgs& a, uint32_t i, int* vx, int* vy) {
    const float2 p = a.xy[i], q = a.xy[i + 1];
    const float dx = __fsub_rn(q.x, p.x), dy = __fsub_rn(q.y, p.y);
    const float len = __fsqrt_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)));
    const float k = __fdiv_rn(0.001f, fmaxf(len, 1e-10f));
    const float nx = __fmul_rn(-dy, k), ny = __fmul_rn(dx, k);
    const float cx[4] = {__fadd_rn(p.x, nx), __fsub_rn(p.x, nx), __fadd_rn(q.x, nx), __fsub_rn(q.x, nx)};
    const float cy[4] = {__fadd_rn(p.y, ny), __fsub_rn(p.y, ny), __fadd_rn(q.y, ny), __fsub_rn(q.y, ny)};
    bool ok = true;
#pragma unroll
    for (int c = 0; c < 4; ++c) ok &= snap(cx[c], cy[c], a.w, a.h, &vx[c], &vy[c]);
    return ok;
}

// Setup of segment s (vs_main + the viewport).
__device__ __forceinline__ void seg_setup(const RenderArgs& a, uint32_t s, SegSetup* g) {
    const uint32_t i = a.segments[s];
    g->first = i;
    g->valid = 0;
    g->x0 = 1;
    g->x1 = 0;
    g->y0 = 1;
    g->y1 = 0;
    int vx[4], vy[4];
    if (!quad_corners(a, i, vx, vy)) return;
    int minx = INT_MAX, maxx = INT_MIN, miny = INT_MAX, maxy = INT_MIN;
#pragma unroll
    for (int t = 0; t < 2; ++t) {
        int order[3] = {t == 0 ? 0 : 2, 1, t == 0 ? 2 : 3};
        long long area;
        if (!orient(vx, vy, order, &area)) continue;
        g->valid |= 1u << t;
        set_edges(vx, vy, order, &g->t[t]);
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            minx = min(minx, vx[order[j]]);
            maxx = max(maxx, vx[order[j]]);
            miny = min(miny, vy[order[j]]);
            maxy = max(maxy, vy[order[j]]);
        }
    }
    if (!g->valid) return;
    g->x0 = max(0, minx >> 8);
    g->x1 = min(static_cast<int>(a.w) - 1, maxx >> 8);
    g->y0 = max(0, miny >> 8);
    g->y1 = min(static_cast<int>(a.h) - 1, maxy >> 8);
}

// fs_main's palette position of the density texture at pixel (x, y): the
// same for every segment drawn there.
__device__ __forceinline__ float pixel_value(const RenderArgs& a, int x, int y) {
    const float u = __fdiv_rn(__fadd_rn(static_cast<float>(x), 0.5f), static_cast<float>(a.w));
    const float v = __fdiv_rn(__fadd_rn(static_cast<float>(y), 0.5f), static_cast<float>(a.h));
    const float tx = __fmul_rn(u, static_cast<float>(a.w - 1u)), ty = __fmul_rn(v, static_cast<float>(a.h - 1u));
    const float fx0 = floorf(tx), fy0 = floorf(ty);
    const float wx = __fsub_rn(tx, fx0), wy = __fsub_rn(ty, fy0);
    const int w1 = static_cast<int>(a.w) - 1, h1 = static_cast<int>(a.h) - 1;
    const int ix0 = min(max(static_cast<int>(fx0), 0), w1), iy0 = min(max(static_cast<int>(fy0), 0), h1);
    const int ix1 = min(ix0 + 1, w1), iy1 = min(iy0 + 1, h1);
    auto texel = [&](int yy, int xx) {
        return __half2float(__float2half_rn(__ldg(a.density + static_cast<size_t>(yy) * a.w + xx)));
    };
    const float d00 = texel(iy0, ix0), d10 = texel(iy0, ix1), d01 = texel(iy1, ix0), d11 = texel(iy1, ix1);
    const float top = __fadd_rn(__fmul_rn(d00, __fsub_rn(1.0f, wx)), __fmul_rn(d10, wx));
    const float bottom = __fadd_rn(__fmul_rn(d01, __fsub_rn(1.0f, wx)), __fmul_rn(d11, wx));
    const float value = __fadd_rn(__fmul_rn(top, __fsub_rn(1.0f, wy)), __fmul_rn(bottom, wy));
    return fminf(fmaxf(value, 0.0f), 1.0f);
}

// fs_main's palette position of a segment starting at sample `first` under
// edge-id colouring.
__device__ __forceinline__ float edge_value(const RenderArgs& a, uint32_t first) {
    return __fdiv_rn(static_cast<float>(a.edge_ids[first]), a.edge_den);
}

// The 16-stop palette lerp of fs_main.
__device__ __forceinline__ void palette_color(const float (*pal)[3], float value, float col[3]) {
    const float stop = __fmul_rn(value, 15.0f);
    uint32_t idx = static_cast<uint32_t>(stop);
    if (idx > 14u) idx = 14u;
    const float f = __fsub_rn(stop, static_cast<float>(idx));
#pragma unroll
    for (int ch = 0; ch < 3; ++ch)
        col[ch] = __fadd_rn(__fmul_rn(pal[idx][ch], __fsub_rn(1.0f, f)), __fmul_rn(pal[idx + 1][ch], f));
}

__device__ __forceinline__ uint32_t to_u8(float r) {
    return static_cast<uint32_t>(fminf(fmaxf(rintf(__fmul_rn(r, 255.0f)), 0.0f), 255.0f));
}

// One blend (alpha 0.1) into a packed RGB8 sample: src = col * 0.1 per
// channel, unorm[c] = c / 255 (IEEE quotients, tabulated).
__device__ __forceinline__ uint32_t blend(uint32_t packed, const float src[3], const float* unorm) {
    const float keep = __fsub_rn(1.0f, 0.1f);
    uint32_t out = 0;
#pragma unroll
    for (int ch = 0; ch < 3; ++ch) {
        const float dst = unorm[(packed >> (8 * ch)) & 0xFFu];
        out |= to_u8(__fadd_rn(src[ch], __fmul_rn(dst, keep))) << (8 * ch);
    }
    return out;
}

__device__ __forceinline__ uint32_t clear_color() {
    return to_u8(0.025f) | (to_u8(0.025f) << 8) | (to_u8(0.035f) << 16);
}

// ---------------------------------------------------------------- binning

// Pairs of this frame, or 0 when they exceed the bin buffers (the host
// grows them and renders again).
__device__ __forceinline__ size_t live_pairs(const RenderArgs& a) {
    const unsigned long long total = *a.pair_total;
    return total > a.pair_capacity ? 0 : static_cast<size_t>(total);
}

__global__ void __launch_bounds__(256) bin_count_kernel(RenderArgs a) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= a.n_segments) return;
    SegSetup g;
    seg_setup(a, s, &g);
    unsigned long long n = 0;
    if (g.x0 <= g.x1 && g.y0 <= g.y1) {
        const int tx0 = g.x0 >> a.tile_shift, tx1 = g.x1 >> a.tile_shift;
        const int ty0 = g.y0 >> a.tile_shift, ty1 = g.y1 >> a.tile_shift;
        n = static_cast<unsigned long long>(tx1 - tx0 + 1) * static_cast<unsigned long long>(ty1 - ty0 + 1);
    }
    a.seg_count[s] = n;
}

// (tile, segment) pairs in segment order.
__global__ void __launch_bounds__(256) bin_emit_kernel(RenderArgs a) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= a.n_segments) return;
    const unsigned long long begin = a.seg_off[s], end = a.seg_off[s + 1];
    if (begin == end || live_pairs(a) == 0) return;
    SegSetup g;
    seg_setup(a, s, &g);
    const int tx0 = g.x0 >> a.tile_shift, tx1 = g.x1 >> a.tile_shift;
    const int ty0 = g.y0 >> a.tile_shift, ty1 = g.y1 >> a.tile_shift;
    unsigned long long k = begin;
    for (int ty = ty0; ty <= ty1; ++ty)
        for (int tx = tx0; tx <= tx1 && k < end; ++tx, ++k) {
            a.pair_tile[k] = static_cast<uint32_t>(ty) * a.tiles_x + static_cast<uint32_t>(tx);
            a.pair_seg[k] = s;
        }
}

// Per block of kBinItems pairs: the count of each tile, stored tile-major
// (hist[tile * blocks + block]) so that one exclusive scan gives every
// (tile, block) its first output position.
__global__ void __launch_bounds__(256) bin_hist_kernel(RenderArgs a) {
    extern __shared__ uint32_t cnt[];
    const uint32_t tiles = a.tiles_x * a.tiles_y;
    for (uint32_t t = threadIdx.x; t < tiles; t += blockDim.x) cnt[t] = 0;
    __syncthreads();
    const size_t begin = static_cast<size_t>(blockIdx.x) * kBinItems;
    const size_t end = min(begin + kBinItems, live_pairs(a));
    for (size_t i = begin + threadIdx.x; i < end; i += blockDim.x) atomicAdd(&cnt[a.pair_tile[i]], 1u);
    __syncthreads();
    for (uint32_t t = threadIdx.x; t < tiles; t += blockDim.x)
        a.hist[static_cast<size_t>(t) * gridDim.x + blockIdx.x] = cnt[t];
}

// Stable scatter: the block's pairs in order, each placed after the earlier
// pairs of its tile (ranks from a warp-wide match on the tile). One warp
// walks the block 32 pairs at a time, with the loads of the next four
// batches in flight.
__global__ void __launch_bounds__(256) bin_rank_kernel(RenderArgs a) {
    extern __shared__ uint32_t next[];
    const uint32_t tiles = a.tiles_x * a.tiles_y;
    for (uint32_t t = threadIdx.x; t < tiles; t += blockDim.x)
        next[t] = a.hist_off[static_cast<size_t>(t) * gridDim.x + blockIdx.x];
    __syncthreads();
    if (threadIdx.x >= 32) return;
    constexpr int kAhead = 4;
    const int lane = threadIdx.x;
    const unsigned lower = (1u << lane) - 1u;
    const size_t begin = static_cast<size_t>(blockIdx.x) * kBinItems;
    const size_t end = min(begin + kBinItems, live_pairs(a));
    for (size_t base = begin; base < end; base += 32 * kAhead) {
        uint32_t tile[kAhead], seg[kAhead];
#pragma unroll
        for (int u = 0; u < kAhead; ++u) {
            const size_t i = base + 32 * u + lane;
            tile[u] = i < end ? a.pair_tile[i] : 0xFFFFFFFFu;
            seg[u] = i < end ? a.pair_seg[i] : 0u;
        }
#pragma unroll
        for (int u = 0; u < kAhead; ++u) {
            const bool valid = tile[u] != 0xFFFFFFFFu;
            const unsigned peers = __match_any_sync(0xFFFFFFFFu, tile[u]);
            if (valid) a.sorted[next[tile[u]] + __popc(peers & lower)] = seg[u];
            __syncwarp();
            if (valid && lane == 31 - __clz(peers)) next[tile[u]] += __popc(peers);
            __syncwarp();
        }
    }
}

// ---------------------------------------------------------------- raster

constexpr int kChunk = 128;
constexpr uint32_t kSlow = 1u;

// A segment as the raster kernel tests it. For a small segment (snapped
// corners less than 64 pixels apart in x and in y, so every edge function
// over its pixel box stays below 2^30 in magnitude) the six edge functions of its two triangles are kept relative to the origin
// (X0, Y0) = 256 * (x0, y0) of its pixel box, with the top-left rule folded
// in: for edge j, f_j(sx, sy) - bias_j = E_j + dx_j * (sy - Y0) - dy_j * (sx - X0),
// bias_j = 0 on a top-left edge and 1 otherwise, so a sample is inside
// triangle t when the three values of its edges are all >= 0 (their OR has
// no sign bit). K_j[q] = dx_j * oy_q - dy_j * ox_q adds sample q's offset.
// A triangle of zero area has E = -1, dx = dy = K = 0 (never inside). Other
// segments (kSlow) are tested in 64 bits from their setup.
struct __align__(16) FastSeg {
    int4 edge[6];     // dx, dy, E, 0
    int4 k[6];        // K per sample
    int4 box;         // x0, y0, x1, y1
    float4 src;       // edge-id colour * 0.1
    uint32_t seg, flags, pad0, pad1;
};

__device__ __forceinline__ void fast_setup(const RenderArgs& a, uint32_t s, const float (*pal)[3], FastSeg* f) {
    int vx[4], vy[4];
    const uint32_t first = a.segments[s];
    f->seg = s;
    // The segment is in this tile's list, so its quad is on screen and has a
    // triangle of nonzero area.
    quad_corners(a, first, vx, vy);
    int order[2][3];
    bool valid[2];
    int minx = INT_MAX, maxx = INT_MIN, miny = INT_MAX, maxy = INT_MIN;
#pragma unroll
    for (int t = 0; t < 2; ++t) {
        order[t][0] = t == 0 ? 0 : 2;
        order[t][1] = 1;
        order[t][2] = t == 0 ? 2 : 3;
        long long area;
        valid[t] = orient(vx, vy, order[t], &area);
        if (!valid[t]) continue;
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            minx = min(minx, vx[order[t][j]]);
            maxx = max(maxx, vx[order[t][j]]);
            miny = min(miny, vy[order[t][j]]);
            maxy = max(maxy, vy[order[t][j]]);
        }
    }
    const int x0 = max(0, minx >> 8), y0 = max(0, miny >> 8);
    f->box = make_int4(x0, y0, min(static_cast<int>(a.w) - 1, maxx >> 8), min(static_cast<int>(a.h) - 1, maxy >> 8));
    const bool small = maxx - minx < (1 << 14) && maxy - miny < (1 << 14);
    f->flags = small ? 0u : kSlow;
    float col[3] = {0.0f, 0.0f, 0.0f};
    if (a.color_by_edge) {
        palette_color(pal, edge_value(a, first), col);
#pragma unroll
        for (int ch = 0; ch < 3; ++ch) col[ch] = __fmul_rn(col[ch], 0.1f);
    }
    f->src = make_float4(col[0], col[1], col[2], 0.0f);
    const int X0 = x0 * 256, Y0 = y0 * 256;
#pragma unroll
    for (int t = 0; t < 2; ++t)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            int4 e = make_int4(0, 0, -1, 0), k = make_int4(0, 0, 0, 0);
            if (valid[t] && small) {
                const int u = order[t][j], v = order[t][j == 2 ? 0 : j + 1];
                const int dx = vx[v] - vx[u], dy = vy[v] - vy[u];
                const bool tl = dy > 0 || (dy == 0 && dx < 0);
                e = make_int4(dx, dy, dx * (Y0 - vy[u]) - dy * (X0 - vx[u]) - (tl ? 0 : 1), 0);
                int kq[4] = {0, 0, 0, 0};
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    if (q < a.ns) {
                        int ox, oy;
                        sample_offset(a.ns, q, &ox, &oy);
                        kq[q] = dx * oy - dy * ox;
                    }
                }
                k = make_int4(kq[0], kq[1], kq[2], kq[3]);
            }
            f->edge[3 * t + j] = e;
            f->k[3 * t + j] = k;
        }
}

// Covering triangles of each sample of pixel (px, py), 8 bits per sample,
// for a segment too large for 32-bit edge functions (rare: corners 64 or
// more pixels apart).
__device__ __noinline__ uint32_t slow_cover(const float2* xy, const uint32_t* segments, uint32_t s, uint32_t w,
                                            uint32_t h, int ns, int px, int py) {
    RenderArgs a{};
    a.xy = xy;
    a.segments = segments;
    a.w = w;
    a.h = h;
    SegSetup g;
    seg_setup(a, s, &g);
    uint32_t out = 0;
    for (int q = 0; q < ns; ++q) {
        int ox, oy;
        sample_offset(ns, q, &ox, &oy);
        const long long sx = static_cast<long long>(px) * 256 + ox, sy = static_cast<long long>(py) * 256 + oy;
        uint32_t n = 0;
        for (int t = 0; t < 2; ++t)
            if (g.valid & (1u << t)) n += inside(g.t[t], sx, sy);
        out |= n << (8 * q);
    }
    return out;
}

// One CTA per tile of T x T pixels (T = 16, 32 or 64). Warp w owns the band
// of T / 8 rows starting at row w * T / 8; its lanes own the band's pixels
// (T = 16: lane -> column lane % 16, row lane / 16; T >= 32: columns
// lane + 32 c, every row of the band) and keep their samples in registers.
// The CTA sets up kChunk segments of the tile's list at a time; each warp
// walks, in draw order, those whose box meets its band (a ballot per 32).
template <int T>
__global__ void __launch_bounds__(256, T == 16 ? 6 : 1) raster_kernel(RenderArgs a) {
    constexpr int kRows = T / 8;
    constexpr int kCols = T >= 32 ? T / 32 : 1;
    constexpr int PPT = T >= 32 ? kRows * kCols : 1;
    constexpr bool kCacheColour = PPT <= 4;
    __shared__ FastSeg segs[kChunk];
    __shared__ float pal[16][3];
    __shared__ float unorm[256];
    if (threadIdx.x < 48) pal[threadIdx.x / 3][threadIdx.x % 3] = kPalette[a.palette][threadIdx.x / 3][threadIdx.x % 3];
    unorm[threadIdx.x] = __fdiv_rn(static_cast<float>(threadIdx.x), 255.0f);
    __syncthreads();
    const int lane = static_cast<int>(threadIdx.x) & 31, warp = static_cast<int>(threadIdx.x) >> 5;
    const uint32_t tile = blockIdx.x;
    const int tx = static_cast<int>(tile % a.tiles_x), ty = static_cast<int>(tile / a.tiles_x);
    const int band0 = ty * T + warp * kRows, band1 = band0 + kRows - 1;
    int px[PPT], py[PPT];
    uint32_t samp[PPT][4];
    float pcol[kCacheColour ? PPT : 1][3];
    const uint32_t bg = clear_color();
#pragma unroll
    for (int k = 0; k < PPT; ++k) {
        if (T == 16) {
            px[k] = tx * T + (lane & 15);
            py[k] = band0 + (lane >> 4);
        } else {
            px[k] = tx * T + lane + 32 * (k % kCols);
            py[k] = band0 + k / kCols;
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) samp[k][q] = bg;
    }
    size_t begin = 0, end = 0;
    if (a.hist_off) {
        begin = a.hist_off[static_cast<size_t>(tile) * a.bin_blocks];
        end = a.hist_off[static_cast<size_t>(tile + 1) * a.bin_blocks];
    }
    // Density colour of each owned pixel, once (only a tile with segments
    // reads the density map, which exists once a graph is uploaded).
    if (kCacheColour && !a.color_by_edge && begin < end && a.density) {
#pragma unroll
        for (int k = 0; k < PPT; ++k) {
            if (px[k] >= static_cast<int>(a.w) || py[k] >= static_cast<int>(a.h)) continue;
            float c[3];
            palette_color(pal, pixel_value(a, px[k], py[k]), c);
#pragma unroll
            for (int ch = 0; ch < 3; ++ch) pcol[kCacheColour ? k : 0][ch] = __fmul_rn(c[ch], 0.1f);
        }
    }
    for (size_t chunk = begin; chunk < end; chunk += kChunk) {
        const int n = static_cast<int>(min(static_cast<size_t>(kChunk), end - chunk));
        __syncthreads();
        if (static_cast<int>(threadIdx.x) < n) fast_setup(a, a.sorted[chunk + threadIdx.x], pal, &segs[threadIdx.x]);
        __syncthreads();
        for (int base = 0; base < n; base += 32) {
            const int e0 = base + lane;
            const bool hit = e0 < n && segs[e0].box.y <= band1 && segs[e0].box.w >= band0;
            unsigned mask = __ballot_sync(0xFFFFFFFFu, hit);
            while (mask) {
                const int e = base + __ffs(mask) - 1;
                mask &= mask - 1;
                const FastSeg& g = segs[e];
                const int4 box = g.box;
#pragma unroll
                for (int k = 0; k < PPT; ++k) {
                    if (px[k] < box.x || px[k] > box.z || py[k] < box.y || py[k] > box.w) continue;
                    int cover[4] = {0, 0, 0, 0};
                    if (g.flags & kSlow) {
                        const uint32_t c = slow_cover(a.xy, a.segments, g.seg, a.w, a.h, a.ns, px[k], py[k]);
#pragma unroll
                        for (int q = 0; q < 4; ++q) cover[q] = (c >> (8 * q)) & 0xFFu;
                    } else {
                        const int rx = (px[k] - box.x) * 256, ry = (py[k] - box.y) * 256;
                        int p[6];
#pragma unroll
                        for (int j = 0; j < 6; ++j) {
                            const int4 ed = g.edge[j];
                            p[j] = ed.z + ed.x * ry - ed.y * rx;
                        }
                        int4 kk[6];
#pragma unroll
                        for (int j = 0; j < 6; ++j) kk[j] = g.k[j];
#pragma unroll
                        for (int q = 0; q < 4; ++q) {
                            if (q < a.ns) {
                                auto kq = [&](int j) { return q == 0 ? kk[j].x : q == 1 ? kk[j].y : q == 2 ? kk[j].z : kk[j].w; };
                                const int t0 = (p[0] + kq(0)) | (p[1] + kq(1)) | (p[2] + kq(2));
                                const int t1 = (p[3] + kq(3)) | (p[4] + kq(4)) | (p[5] + kq(5));
                                cover[q] = (t0 >= 0) + (t1 >= 0);
                            }
                        }
                    }
                    if ((cover[0] | cover[1] | cover[2] | cover[3]) == 0) continue;
                    float src[3];
                    if (a.color_by_edge) {
                        src[0] = g.src.x;
                        src[1] = g.src.y;
                        src[2] = g.src.z;
                    } else if (kCacheColour) {
#pragma unroll
                        for (int ch = 0; ch < 3; ++ch) src[ch] = pcol[kCacheColour ? k : 0][ch];
                    } else {
                        palette_color(pal, pixel_value(a, px[k], py[k]), src);
#pragma unroll
                        for (int ch = 0; ch < 3; ++ch) src[ch] = __fmul_rn(src[ch], 0.1f);
                    }
                    // Samples with the same history blend to the same value.
                    uint32_t last_in = 0xFFFFFFFFu, last_out = 0;
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        for (int r = 0; r < cover[q]; ++r) {
                            if (samp[k][q] != last_in) {
                                last_in = samp[k][q];
                                last_out = blend(last_in, src, unorm);
                            }
                            samp[k][q] = last_out;
                        }
                    }
                }
            }
        }
    }
#pragma unroll
    for (int k = 0; k < PPT; ++k) {
        if (px[k] >= static_cast<int>(a.w) || py[k] >= static_cast<int>(a.h)) continue;
        const size_t base = (static_cast<size_t>(py[k]) * a.w + px[k]) * a.ns;
#pragma unroll
        for (int q = 0; q < 4; ++q)
            if (q < a.ns) a.samples[base + q] = samp[k][q];
    }
}

// ---------------------------------------------------------------- endpoints

// Endpoint squares (vs_endpoint): thread = (path, end). Every covered sample
// whose interpolated offset lies within radius2 takes the opaque colour.
__global__ void __launch_bounds__(256) endpoint_kernel(RenderArgs a, float radius2, int centre) {
    const uint32_t id = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t p = id >> 1;
    if (p >= a.n_paths) return;
    const PathRec rec = a.paths[p];
    if (rec.count < 2) return;
    const uint32_t i = (id & 1u) ? rec.point_offset + rec.count - 1u : rec.point_offset;
    // ALPHA_BLENDING with source alpha 1: src * 1 + dst * 0.
    uint32_t c8 = 0;
#pragma unroll
    for (int ch = 0; ch < 3; ++ch) {
        const float col = centre ? kEndpointColor[a.palette][ch] : __fmul_rn(kPalette[a.palette][0][ch], 0.1f);
        c8 |= to_u8(__fadd_rn(__fmul_rn(col, 1.0f), 0.0f)) << (8 * ch);
    }
    const float2 c = a.xy[i];
    const float cxo[4] = {-1.0f, -1.0f, 1.0f, 1.0f}, cyo[4] = {1.0f, -1.0f, 1.0f, -1.0f};
    int vx[4], vy[4];
    bool ok = true;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const float X = __fadd_rn(c.x, __fdiv_rn(__fmul_rn(__fmul_rn(cxo[k], 3.0f), 2.0f), static_cast<float>(a.w)));
        const float Y = __fadd_rn(c.y, __fdiv_rn(__fmul_rn(__fmul_rn(cyo[k], 3.0f), 2.0f), static_cast<float>(a.h)));
        ok &= snap(X, Y, a.w, a.h, &vx[k], &vy[k]);
    }
    if (!ok) return;
    for (int t = 0; t < 2; ++t) {
        int order[3] = {t == 0 ? 0 : 2, 1, t == 0 ? 2 : 3};
        long long area_i;
        if (!orient(vx, vy, order, &area_i)) continue;
        const int ia = order[0], ib = order[1], ic = order[2];
        const float area = __ll2float_rn(area_i);
        TriSetup tri;
        set_edges(vx, vy, order, &tri);
        const int minx = min(vx[ia], min(vx[ib], vx[ic])), maxx = max(vx[ia], max(vx[ib], vx[ic]));
        const int miny = min(vy[ia], min(vy[ib], vy[ic])), maxy = max(vy[ia], max(vy[ib], vy[ic]));
        const int x0 = max(0, minx >> 8), x1 = min(static_cast<int>(a.w) - 1, maxx >> 8);
        const int y0 = max(0, miny >> 8), y1 = min(static_cast<int>(a.h) - 1, maxy >> 8);
        for (int y = y0; y <= y1; ++y)
            for (int x = x0; x <= x1; ++x)
                for (int q = 0; q < a.ns; ++q) {
                    int ox, oy;
                    sample_offset(a.ns, q, &ox, &oy);
                    const long long sx = static_cast<long long>(x) * 256 + ox, sy = static_cast<long long>(y) * 256 + oy;
                    if (!inside(tri, sx, sy)) continue;
                    // Barycentric weights: edge (a,b) weighs c, (b,c) weighs a, (c,a) weighs b.
                    const float wc = __ll2float_rn(edge_fn(tri.ax[0], tri.ay[0], tri.dx[0], tri.dy[0], sx, sy));
                    const float wa = __ll2float_rn(edge_fn(tri.ax[1], tri.ay[1], tri.dx[1], tri.dy[1], sx, sy));
                    const float wb = __ll2float_rn(edge_fn(tri.ax[2], tri.ay[2], tri.dx[2], tri.dy[2], sx, sy));
                    const float la = __fdiv_rn(wa, area), lb = __fdiv_rn(wb, area), lc = __fdiv_rn(wc, area);
                    const float ox2 =
                        __fadd_rn(__fadd_rn(__fmul_rn(la, cxo[ia]), __fmul_rn(lb, cxo[ib])), __fmul_rn(lc, cxo[ic]));
                    const float oy2 =
                        __fadd_rn(__fadd_rn(__fmul_rn(la, cyo[ia]), __fmul_rn(lb, cyo[ib])), __fmul_rn(lc, cyo[ic]));
                    if (__fadd_rn(__fmul_rn(ox2, ox2), __fmul_rn(oy2, oy2)) > radius2) continue;
                    // Every writer of this pass stores the same value.
                    a.samples[(static_cast<size_t>(y) * a.w + x) * a.ns + q] = c8;
                }
    }
}

// ---------------------------------------------------------------- resolve

__global__ void __launch_bounds__(256) resolve_kernel(RenderArgs a) {
    const size_t pix = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
    const bool valid = pix < static_cast<size_t>(a.w) * a.h;
    const uint32_t bg = clear_color();
    bool differs = false;
    if (valid) {
        uint32_t out = 0xFF000000u;
        const uint32_t n = static_cast<uint32_t>(a.ns);
#pragma unroll
        for (int ch = 0; ch < 3; ++ch) {
            uint32_t sum = 0;
            for (int q = 0; q < a.ns; ++q) sum += (a.samples[pix * a.ns + q] >> (8 * ch)) & 0xFFu;
            uint32_t v = sum / n;
            const uint32_t rem = sum % n;
            if (n > 1u) {
                const uint32_t half = n / 2u;
                if (rem > half || (rem == half && (v & 1u))) ++v;
            }
            out |= v << (8 * ch);
            differs |= v != ((bg >> (8 * ch)) & 0xFFu);
        }
        a.rgba[pix] = out;
    }
    const unsigned votes = __ballot_sync(0xFFFFFFFFu, valid && differs);
    if ((threadIdx.x & 31) == 0 && votes) atomicAdd(a.colored, static_cast<unsigned long long>(__popc(votes)));
}

}  // namespace

int render_tile_shift(uint32_t w, uint32_t h) {
    for (int shift = 4; shift <= 6; ++shift) {
        const uint64_t tx = (w + (1u << shift) - 1) >> shift, ty = (h + (1u << shift) - 1) >> shift;
        if (tx * ty <= kMaxRenderTiles) return shift;
    }
    return -1;
}

void launch_render_bin_count(const RenderArgs& a, cudaStream_t s) {
    if (a.n_segments) bin_count_kernel<<<div_up(a.n_segments, 256), 256, 0, s>>>(a);
}

void launch_render_bin_emit(const RenderArgs& a, cudaStream_t s) {
    if (a.n_segments) bin_emit_kernel<<<div_up(a.n_segments, 256), 256, 0, s>>>(a);
}

cudaError_t launch_render_bin_sort(const RenderArgs& a, uint32_t* scan_scratch, cudaStream_t s) {
    const size_t tiles = static_cast<size_t>(a.tiles_x) * a.tiles_y;
    const int smem = static_cast<int>(4 * tiles);
    cudaError_t e = cudaFuncSetAttribute(bin_hist_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(bin_rank_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    bin_hist_kernel<<<a.bin_blocks, 256, smem, s>>>(a);
    exclusive_scan<uint32_t>(a.hist, a.hist_off, tiles * a.bin_blocks, scan_scratch, s);
    bin_rank_kernel<<<a.bin_blocks, 256, smem, s>>>(a);
    return cudaSuccess;
}

void launch_render_raster(const RenderArgs& a, cudaStream_t s) {
    const unsigned tiles = a.tiles_x * a.tiles_y;
    if (a.tile_shift == 4) raster_kernel<16><<<tiles, 256, 0, s>>>(a);
    else if (a.tile_shift == 5) raster_kernel<32><<<tiles, 256, 0, s>>>(a);
    else raster_kernel<64><<<tiles, 256, 0, s>>>(a);
}

void launch_render_endpoints(const RenderArgs& a, cudaStream_t s) {
    if (!a.n_paths) return;
    const unsigned blocks = div_up(2u * a.n_paths, 256);
    const float third = 1.0f / 3.0f;
    const float inner = 1.0f - third;
    endpoint_kernel<<<blocks, 256, 0, s>>>(a, 1.0f, 0);
    endpoint_kernel<<<blocks, 256, 0, s>>>(a, inner * inner, 1);
}

void launch_render_resolve(const RenderArgs& a, cudaStream_t s) {
    resolve_kernel<<<div_up(static_cast<size_t>(a.w) * a.h, 256), 256, 0, s>>>(a);
}

}  // namespace bt
