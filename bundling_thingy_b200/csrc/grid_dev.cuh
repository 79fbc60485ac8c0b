// grid_dev.cuh — per-sample bodies of the neighbour-mean and scatter kernels,
// shared by the single-graph kernels (grid.cu) and the batched persistent
// kernels (batch.cu). See grid.cu for the semantics and the layout.
#pragma once

#include "kernels.cuh"

namespace bt {
namespace dev {

// Search-cell index bounds floor / ceil of t * inv_s, by the reciprocal: the
// bounds are conservative by the margin, which exceeds this rounding many
// times over. The products stay far below 2^22 in magnitude, where adding
// 1.5 * 2^23 with rounding down (up) leaves floor (ceil) in the low bits.
__device__ __forceinline__ int floor_cell(float t, float inv_s) {
    return __float_as_int(__fadd_rd(t * inv_s, 12582912.0f)) - 0x4B400000;
}
__device__ __forceinline__ int ceil_cell(float t, float inv_s) {
    return __float_as_int(__fadd_ru(t * inv_s, 12582912.0f)) - 0x4B400000;
}

// Approximate square root (one MUFU op); callers widen its result by a
// relative 1e-6 plus the margin, far above its error.
__device__ __forceinline__ float sqrt_approx(float x) {
    float r;
    asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// Sums of one sample's neighbourhood. Interior runs of whole search cells
// come from the slot prefix (biased fixed point, exact in 64 bits); the
// samples of boundary cells are tested one by one and accumulated either as
// exact f32 differences (fast, see Grid) or as biased fixed point.
struct Acc {
    unsigned long long sx, sy;   // sums of biased fixed-point positions (Q + 2^30)
    uint32_t count;              // samples in sx / sy
    long long dx, dy;            // sums of Q(q) - Q(p), flushed from the f32 parts
    uint32_t dcount;             // samples in dx / dy
};

// Boundary candidates of one lane: its slot ranges in shared memory (lane-
// interleaved, rs[k * 32]) are walked kMeanGroup loads at a time, every group
// from one range; loads past a range's end read padding or the next slots
// and are masked. The test is neighbor_mean.wgsl:193-198 in f32.
template <bool kFast>
__device__ __forceinline__ void walk_ranges(const float2* __restrict__ rec, const uint2* rs, uint32_t nr,
                                            float2 p, const Grid& g, Acc& acc) {
    const float2 neg_p = make_float2(-p.x, -p.y);
    const float2 ts = make_float2(g.tsx, g.tsy);
    const float r2 = g.r2;
    const float2 split = make_float2(g.split_x, g.split_y);
    const float2 neg_split = make_float2(-g.split_x, -g.split_y);
    // Fast path: sum of (q - p) as an exact f32 pair per axis: the part on the
    // 2^(k-11) grid and the remainder on the 2^(k-23) grid. Each stays exact
    // for 4096 terms; it is flushed into 64-bit integers every 2048.
    float2 hi = make_float2(0.0f, 0.0f), lo = make_float2(0.0f, 0.0f);
    uint32_t fcount = 0, since_flush = 0;
    uint32_t k = 0, j = 0, e = 0;
    while (true) {
        if (j >= e && k < nr) {
            const uint2 r = rs[k * 32];
            j = r.x;
            e = r.y;
            ++k;
        }
        if (!__any_sync(0xFFFFFFFFu, j < e)) break;
        float2 q[kMeanGroup];
#pragma unroll
        for (int u = 0; u < kMeanGroup; ++u) q[u] = __ldg(rec + (j < e ? j + u : 0u));
#pragma unroll
        for (int u = 0; u < kMeanGroup; ++u) {
            const float2 d = __fadd2_rn(q[u], neg_p);
            const float2 t = __fmul2_rn(d, ts);
            const float2 t2 = __fmul2_rn(t, t);
            const float d2 = t2.x + t2.y;
            if (d2 <= r2 && j + u < e) {
                if (kFast) {
                    const float2 h = __fadd2_rn(__fadd2_rn(d, split), neg_split);
                    const float2 l = __fadd2_rn(d, make_float2(-h.x, -h.y));
                    hi = __fadd2_rn(hi, h);
                    lo = __fadd2_rn(lo, l);
                    ++fcount;
                } else {
                    acc.sx += biased_fixed(q[u].x);
                    acc.sy += biased_fixed(q[u].y);
                    acc.count += 1u;
                }
            }
        }
        j += kMeanGroup;
        if (kFast && (since_flush += kMeanGroup) >= 2048u) {
            acc.dx += __float2ll_rn(hi.x * kFixedScale) + __float2ll_rn(lo.x * kFixedScale);
            acc.dy += __float2ll_rn(hi.y * kFixedScale) + __float2ll_rn(lo.y * kFixedScale);
            hi = lo = make_float2(0.0f, 0.0f);
            since_flush = 0;
        }
    }
    if (kFast) {
        acc.dx += __float2ll_rn(hi.x * kFixedScale) + __float2ll_rn(lo.x * kFixedScale);
        acc.dy += __float2ll_rn(hi.y * kFixedScale) + __float2ll_rn(lo.y * kFixedScale);
        acc.dcount += fcount;
    }
}

// Neighbour mean of the sample in slot i (i >= a.n: an idle lane). Every
// lane of the warp must call it (the row set-up, the walk and the next-grid
// counts are warp-cooperative); `rs` is this warp's range buffer
// (MeanShared::ranges[warp]).
__device__ __forceinline__ void mean_sample(const MeanArgs& a, uint32_t i, uint2 (*rs)[32]) {
    const bool valid = i < a.n;
    const Grid& g = a.g;
    const int lane = threadIdx.x & 31;
    const float2 p = valid ? a.rec[i] : make_float2(0.0f, 0.0f);
    const uint32_t tag = valid ? a.tag[i] : 0u;
    const bool movable = (tag & kMovableBit) != 0;
    float2 np = p;
    uint32_t count = 0;
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
    const int rows = movable ? fy_hi - fy_lo + 1 : 0;
    const bool interior = a.mode == kSearchInterior;
    const int fw = static_cast<int>(g.fw), fh = static_cast<int>(g.fh);
    // The exact f32 accumulation when every moving lane of the warp is far
    // enough from the axes (warp-uniform, so the walk does not diverge).
    const bool fast = __all_sync(0xFFFFFFFFu, !movable || (fabsf(p.x) >= g.fast_x && fabsf(p.y) >= g.fast_y));
    Acc acc{0ull, 0ull, 0u, 0ll, 0ll, 0u};
    for (int base = 0; __any_sync(0xFFFFFFFFu, base < rows); base += kMeanChunkRows) {
        // Set-up of up to kMeanChunkRows search rows per lane, in lockstep:
        // interior cells from the slot prefix, boundary cells as ranges.
        uint32_t nr = 0;
#pragma unroll 2
        for (int jr = 0; jr < kMeanChunkRows; ++jr) {
            if (base + jr >= rows) continue;
            const int fy = fy_lo + base + jr;
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
            uint32_t s1 = s3, s2 = s3;
            if (ix0 <= ix1) {
                s1 = a.cell_start[row + ix0];
                s2 = a.cell_start[row + ix1 + 1];
                const LL2 lo = a.prefix[s1], hi = a.prefix[s2];
                acc.sx += static_cast<unsigned long long>(hi.x - lo.x);
                acc.sy += static_cast<unsigned long long>(hi.y - lo.y);
                acc.count += s2 - s1;
            }
            if (s1 > s0) rs[nr++][lane] = make_uint2(s0, s1);
            if (s3 > s2) rs[nr++][lane] = make_uint2(s2, s3);
        }
        __syncwarp();
        if (fast) {
            walk_ranges<true>(a.rec, &rs[0][lane], nr, p, g, acc);
        } else {
            walk_ranges<false>(a.rec, &rs[0][lane], nr, p, g, acc);
        }
        __syncwarp();
    }
    if (movable) {
        count = acc.count + acc.dcount;
        // Biased sums: sum (Q(q) + B) - n (Q(p) + B) = sum Q(q) - n Q(p).
        const long long dx = static_cast<long long>(acc.sx - static_cast<unsigned long long>(acc.count) *
                                                                 biased_fixed(p.x)) + acc.dx;
        const long long dy = static_cast<long long>(acc.sy - static_cast<unsigned long long>(acc.count) *
                                                                 biased_fixed(p.y)) + acc.dy;
        const double den = static_cast<double>(count) * 1073741824.0;
        np.x = p.x + static_cast<float>(static_cast<double>(dx) / den);
        np.y = p.y + static_cast<float>(static_cast<double>(dy) / den);
    }
    // The next grid: search cell and population. Lanes of a warp that land
    // in one cell (neighbours in slot order mostly do) add their count once.
    const uint32_t c = valid ? search_cell(np, g) : 0xFFFFFFFFu;
    const unsigned peers = __match_any_sync(0xFFFFFFFFu, c);
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
