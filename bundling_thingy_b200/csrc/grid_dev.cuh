// grid_dev.cuh — per-sample bodies of the neighbour-mean and scatter kernels,
// shared by the single-graph kernels (grid.cu) and the batched persistent
// kernels (batch.cu). See grid.cu for the semantics and the layout.
#pragma once

#include "kernels.cuh"

namespace bt {
namespace dev {

// Search-cell index bounds t / s, by the reciprocal: the bounds are
// conservative by the margin, which exceeds this rounding many times over.
__device__ __forceinline__ int floor_cell(float t, float inv_s) { return static_cast<int>(floorf(t * inv_s)); }
__device__ __forceinline__ int ceil_cell(float t, float inv_s) { return static_cast<int>(ceilf(t * inv_s)); }

// Approximate square root (one MUFU op); callers widen its result by a
// relative 1e-6 plus the margin, far above its error.
__device__ __forceinline__ float sqrt_approx(float x) {
    float r;
    asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

struct Acc {
    unsigned long long sx, sy;
    uint32_t count;
};

// Exact test of every sample in slots [b, e) (neighbor_mean.wgsl:193-198).
__device__ __forceinline__ void scan_range(const float2* __restrict__ rec, uint32_t b, uint32_t e, float2 neg_p,
                                           float2 ts, float r2, Acc& acc) {
#pragma unroll 8
    for (uint32_t j = b; j < e; ++j) {
        const float2 q = __ldg(rec + j);
        const float2 d = __fadd2_rn(q, neg_p);
        const float2 t = __fmul2_rn(d, ts);
        const float2 t2 = __fmul2_rn(t, t);
        const float d2 = t2.x + t2.y;
        if (d2 <= r2) {
            acc.sx += biased_fixed(q.x);
            acc.sy += biased_fixed(q.y);
            acc.count += 1u;
        }
    }
}

// Neighbour mean of the sample in slot i (i >= a.n: an idle lane). Every
// lane of the warp must call it: the next-grid counts are warp-aggregated.
__device__ __forceinline__ void mean_sample(const MeanArgs& a, uint32_t i) {
    const bool valid = i < a.n;
    const Grid& g = a.g;
    const float2 p = valid ? a.rec[i] : make_float2(0.0f, 0.0f);
    const uint32_t tag = valid ? a.tag[i] : 0u;
    float2 np = p;
    uint32_t count = 0;
    if (tag & kMovableBit) {
        const float tx = texel_of(p.x, g.map.wm1), ty = texel_of(p.y, g.map.hm1);
        // Reach box in grid cells (neighbor_mean.wgsl:180-185), in search cells.
        const uint32_t cx0 = grid_of(tx - g.reachx, g.rf, g.gw), cx1 = grid_of(tx + g.reachx, g.rf, g.gw);
        const uint32_t cy0 = grid_of(ty - g.reachy, g.rf, g.gh), cy1 = grid_of(ty + g.reachy, g.rf, g.gh);
        const int fx_min = static_cast<int>(cx0 * g.kx), fx_max = static_cast<int>(cx1 * g.kx + g.kx - 1u);
        const int fy_min = static_cast<int>(cy0 * g.ky), fy_max = static_cast<int>(cy1 * g.ky + g.ky - 1u);
        // Candidate circle r + m; certain circle r - m (texels).
        const float R = g.rf + g.margin;
        const float Rin = g.rf - g.margin;
        const int fy_lo = max(fy_min, floor_cell(ty - R, g.inv_sy));
        const int fy_hi = min(fy_max, floor_cell(ty + R, g.inv_sy));
        const bool interior = a.mode == kSearchInterior;
        const int fw = static_cast<int>(g.fw), fh = static_cast<int>(g.fh);
        const float2 neg_p = make_float2(-p.x, -p.y);
        const float2 ts = make_float2(g.tsx, g.tsy);
        Acc acc{0ull, 0ull, 0u};
        for (int fy = fy_lo; fy <= fy_hi; ++fy) {
            const float ylo = static_cast<float>(fy) * g.sy;
            const float yhi = ylo + g.sy;
            const float near = fmaxf(fmaxf(ylo - ty, ty - yhi), 0.0f);
            const float dn = fmaxf(near - g.margin, 0.0f);
            if (dn > R) continue;
            // f32 rounding of R^2 - dn^2 is below 5e-7 R^2; widen by that.
            const float hout = sqrt_approx(fmaxf(R * R - dn * dn + 5e-7f * R * R, 0.0f)) * 1.000001f + g.margin;
            const int bx0 = max(fx_min, floor_cell(tx - hout, g.inv_sx));
            const int bx1 = min(fx_max, floor_cell(tx + hout, g.inv_sx));
            if (bx0 > bx1) continue;
            const uint32_t row = static_cast<uint32_t>(fy) * g.fw;
            const uint32_t s0 = a.cell_start[row + bx0];
            const uint32_t s3 = a.cell_start[row + bx1 + 1];
            int ix0 = 1, ix1 = 0;
            if (interior && fy > 0 && fy < fh - 1) {
                // Cells of this row whose every sample passes the f32 test:
                // the farthest point of the row band, widened by the margin.
                const float far = fmaxf(fabsf(ylo - ty), fabsf(yhi - ty)) + g.margin;
                if (far < Rin) {
                    const float h2 = Rin * Rin - far * far - 5e-7f * Rin * Rin;
                    const float hin = sqrt_approx(fmaxf(h2, 0.0f)) * 0.999999f - g.margin;
                    if (hin > 0.0f) {
                        ix0 = max(ceil_cell(tx - hin, g.inv_sx), max(bx0, 1));
                        ix1 = min(floor_cell(tx + hin, g.inv_sx) - 1, min(bx1, fw - 2));
                    }
                }
            }
            if (ix0 <= ix1) {
                const uint32_t s1 = a.cell_start[row + ix0];
                const uint32_t s2 = a.cell_start[row + ix1 + 1];
                const LL2 lo = a.prefix[s1], hi = a.prefix[s2];
                acc.sx += static_cast<unsigned long long>(hi.x - lo.x);
                acc.sy += static_cast<unsigned long long>(hi.y - lo.y);
                acc.count += s2 - s1;
                scan_range(a.rec, s0, s1, neg_p, ts, g.r2, acc);
                scan_range(a.rec, s2, s3, neg_p, ts, g.r2, acc);
            } else {
                scan_range(a.rec, s0, s3, neg_p, ts, g.r2, acc);
            }
        }
        count = acc.count;
        // Biased sums: sum (Q(q) + B) - n (Q(p) + B) = sum Q(q) - n Q(p).
        const long long dx = static_cast<long long>(acc.sx - static_cast<unsigned long long>(count) * biased_fixed(p.x));
        const long long dy = static_cast<long long>(acc.sy - static_cast<unsigned long long>(count) * biased_fixed(p.y));
        const double den = static_cast<double>(count) * 1073741824.0;
        np.x = p.x + static_cast<float>(static_cast<double>(dx) / den);
        np.y = p.y + static_cast<float>(static_cast<double>(dy) / den);
    }
    // The next grid: search cell and population. Lanes of a warp that land
    // in one cell (neighbours in slot order mostly do) add their count once.
    const uint32_t c = valid ? search_cell(np, g) : 0xFFFFFFFFu;
    const unsigned peers = __match_any_sync(0xFFFFFFFFu, c);
    const int lane = threadIdx.x & 31;
    if (a.counts) {
        // Density splat, warp-aggregated too: once bundled, the samples of a
        // warp mostly share texels, and one add per texel spares the L2 the
        // serialised same-address atomics (integer sums: the counts are the
        // same in any order).
        uint32_t d = 0xFFFFFFFFu;                          // stays so off the map
        if (valid) splat_index(np.x, np.y, g.map, &d);
        const unsigned same = __match_any_sync(0xFFFFFFFFu, d);
        if (d != 0xFFFFFFFFu && lane == __ffs(same) - 1) atomicAdd(&a.counts[d], static_cast<uint32_t>(__popc(same)));
    }
    if (!valid) return;
    if (lane == __ffs(peers) - 1) {
        atomicAdd(&a.hist[c], static_cast<uint32_t>(__popc(peers)));
        if (a.hist_tiles) atomicAdd(&a.hist_tiles[c / kCellTile], static_cast<uint32_t>(__popc(peers)));
    }
    a.out_xy[i] = np;
    a.out_tag[i] = tag;
    a.out_cell[i] = c;
    if (a.neighbors) a.neighbors[i] = count;
}

// Slot of sample i in the next order: start of its search cell plus a rank
// taken by counting the population down (order within a cell is free: the
// mean's exact sum does not depend on it). Every lane of the warp calls it.
__device__ __forceinline__ void scatter_sample(const ScatterArgs& a, uint32_t i) {
    const bool valid = i < a.n;
    const uint32_t c = valid ? a.cell[i] : 0xFFFFFFFFu;
    // Lanes of one warp that share a cell (neighbours in slot order mostly do)
    // take one reservation and consecutive slots, so their writes coalesce.
    const unsigned peers = __match_any_sync(0xFFFFFFFFu, c);
    // Cell ids and populations are consistent by construction; a failed
    // upload can leave stale entries, which are skipped and flagged.
    bool ok = valid && c < a.cells;
    if (valid && !ok) atomicOr(a.status, 8u);
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(peers) - 1;
    const uint32_t group = __popc(peers);
    const uint32_t rank = __popc(peers & ((1u << lane) - 1u));
    uint32_t top = 0;
    if (ok && lane == leader) top = atomicSub(&a.hist[c], group);
    top = __shfl_sync(0xFFFFFFFFu, top, leader);
    const uint32_t slot = ok ? a.cell_start[c] + (top - group) + rank : 0u;
    if (ok && (top < group || slot >= a.n)) {
        atomicOr(a.status, 8u);
        ok = false;
    }
    if (!ok) return;
    const float2 p = a.xy[i];
    a.out_rec[slot] = p;
    a.out_tag[slot] = a.tag[i];
}

// Slot-prefix scan input: the biased fixed-point position of a record.
struct RecordQSource {
    const float2* rec;
    __device__ __forceinline__ LL2 read(size_t j) const {
        const float2 r = rec[j];
        return LL2{static_cast<long long>(biased_fixed(r.x)), static_cast<long long>(biased_fixed(r.y))};
    }
    __device__ __forceinline__ void consume(size_t) const {}
};

}  // namespace dev
}  // namespace bt
