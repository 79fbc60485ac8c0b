// common.cuh — shared device formulas and launch helpers.
//
// The library is compiled with -fmad=false: every float expression is one
// IEEE binary32 rounding per operation in source order (the reference's WGSL
// expression order), and a fused multiply-add appears only where the code
// calls __fmaf_rn explicitly. Division and sqrt are IEEE (nvcc's default
// -prec-div=true -prec-sqrt=true), denormals are kept (no -ftz).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace bt {

constexpr int kWarp = 32;
constexpr float kFixedScale = 1073741824.0f;   // 2^30, fixed-point scale of positions

// WGSL u32(f32): truncation toward zero, saturating at the range ends.
__host__ __device__ __forceinline__ uint32_t u32_sat(float v) {
    if (!(v > 0.0f)) return 0u;
    if (v >= 4294967296.0f) return 0xFFFFFFFFu;
    return static_cast<uint32_t>(v);
}

// Normalisation parameters of Graph::normalization (src/graph.rs:79-91).
struct Norm {
    float min_x, min_y, scale, tx, ty;
};

// resampling.wgsl:45-48: ((cp - min) * scale + translation - 0.5) * 2.
__device__ __forceinline__ float2 normalized(const Norm& n, float2 cp) {
    float ax = (cp.x - n.min_x) * n.scale;
    ax = ax + n.tx;
    ax = ax - 0.5f;
    float ay = (cp.y - n.min_y) * n.scale;
    ay = ay + n.ty;
    ay = ay - 0.5f;
    return make_float2(ax * 2.0f, ay * 2.0f);
}

// Map geometry shared by the splat, grid and neighbour kernels.
struct Map {
    uint32_t w, h;
    float wm1, hm1;      // f32(size - 1)
};

// Density splat cell (resampling.wgsl:70-75, neighbor_mean.wgsl:68-72):
// uv = (x/2 + 1/2, 1/2 - y/2), cell = u32(round(uv * (size - 1))) with
// round-half-to-even. Returns false for a cell outside the map.
__device__ __forceinline__ bool splat_index(float x, float y, const Map& m, uint32_t* index) {
    float ux = x * 0.5f;
    ux = ux + 0.5f;
    float uy = y * 0.5f;
    uy = 0.5f - uy;
    uint32_t cx = u32_sat(rintf(ux * m.wm1));
    uint32_t cy = u32_sat(rintf(uy * m.hm1));
    if (cx >= m.w || cy >= m.h) return false;
    *index = cy * m.w + cx;
    return true;
}

// Neighbour grid (neighbor_mean.rs:26-32, spatial_grid.wgsl:59-70) plus the
// finer search cells: each grid cell is split into kx x ky search cells.
struct Grid {
    Map map;
    uint32_t radius;
    float rf;            // f32(radius)
    uint32_t gw, gh;     // grid cells: ceil(size / radius)
    uint32_t kx, ky;     // search cells per grid cell, along x and y
    float inv_sx, inv_sy;// f32(k) / f32(radius)
    float sx, sy;        // search cell sides in texels, f32(radius) / f32(k)
    uint32_t fw, fh;     // search cells: gw * kx, gh * ky
    float tsx, tsy;      // texel_scale = f32(size - 1) * 0.5
    float r2;            // f32(radius) * f32(radius)
    float reachx, reachy;// f32(radius) + f32(size) * 2.4e-7 (neighbor_mean.wgsl:180-181)
    float margin;        // conservative slack of the search-cell bounds, texels
};

// texel_position (spatial_grid.wgsl:59-61), one axis.
__device__ __forceinline__ float texel_of(float p, float size_m1) {
    float t = p + 1.0f;
    t = t * 0.5f;
    return t * size_m1;
}

// grid_cell (spatial_grid.wgsl:63-65), one axis.
__device__ __forceinline__ uint32_t grid_of(float t, float rf, uint32_t gsize) {
    uint32_t c = u32_sat(fmaxf(t / rf, 0.0f));
    return c < gsize - 1u ? c : gsize - 1u;
}

// Search cell along one axis: the grid cell, then the sub-cell inside it, so
// that search cell / k is exactly the reference's grid cell.
__device__ __forceinline__ uint32_t search_of(float t, float rf, uint32_t gsize, uint32_t k, float inv_s) {
    uint32_t c = grid_of(t, rf, gsize);
    float rel = t - static_cast<float>(c) * rf;
    uint32_t sub = u32_sat(rel * inv_s);
    sub = sub < k - 1u ? sub : k - 1u;
    return c * k + sub;
}

__device__ __forceinline__ uint32_t search_cell(float2 p, const Grid& g) {
    uint32_t fx = search_of(texel_of(p.x, g.map.wm1), g.rf, g.gw, g.kx, g.inv_sx);
    uint32_t fy = search_of(texel_of(p.y, g.map.hm1), g.rf, g.gh, g.ky, g.inv_sy);
    return fy * g.fw + fx;
}

// Fixed-point position: round-half-even(v * 2^30).
__device__ __forceinline__ long long fixed_of(float v) { return __float2ll_rn(v * kFixedScale); }

inline unsigned int div_up(size_t n, unsigned int d) { return static_cast<unsigned int>((n + d - 1) / d); }

}  // namespace bt
