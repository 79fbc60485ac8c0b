// grid.cu — neighbour-grid binning and the fused neighbour-mean step.
//
// Restates count_cells / reserve_cells / scatter_points
// (src/shaders/spatial_grid.wgsl:72-138) and neighbor_mean_sparse
// (src/shaders/neighbor_mean.wgsl:164-203) with write_point's splat (66-73).
//
// Semantics (identical to the oracle): N(p) = every sample q whose grid cell
// lies in p's reach box (grid_cell(texel(p) -/+ reach)) and that passes the
// reference's f32 test dot((q-p)*ts, (q-p)*ts) <= r*r. The displacement is
// accumulated exactly in 2^-30 fixed point (64-bit integers), so the result
// does not depend on the order of N(p) — which the reference leaves to
// atomics — nor on how N(p) is enumerated:
//   p' = p + f32(f64(sum_q Q(q) - |N| Q(p)) / (f64(|N|) * 2^30)).
//
// B200 layout: samples live in slot order as 16-byte records
// {x, y, Q(x) + 2^30, Q(y) + 2^30}, sorted by search cell (each grid cell side
// split into k search cells, search cells row-major over the whole map), so a
// row of search cells [a, b] is one contiguous slot range. An exclusive prefix
// sum of the biased fixed-point positions over slots turns any such range into
// one subtraction. Per search row, a thread takes the cells that lie entirely
// inside its circle (by conservative bounds, with a margin far above every
// f32 rounding involved) from the prefix sums — the role of the reference's
// fully-contained cell summaries (neighbor_mean.wgsl:40-59) — and tests only
// the samples of the boundary cells, exactly. The kernel writes the new
// position in the same slot order (coalesced), its next search cell and the
// population count (fusing count_cells of the next iteration), and its density
// splat. The scatter then moves the samples into the next slot order,
// counting the populations back down to zero for reuse.
#include "kernels.cuh"

namespace bt {
namespace {

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
__device__ __forceinline__ void scan_range(const uint4* __restrict__ rec, uint32_t b, uint32_t e, float2 neg_p,
                                           float2 ts, float r2, Acc& acc) {
#pragma unroll 4
    for (uint32_t j = b; j < e; ++j) {
        const uint4 q = __ldg(rec + j);
        const float2 d = __fadd2_rn(make_float2(__uint_as_float(q.x), __uint_as_float(q.y)), neg_p);
        const float2 t = __fmul2_rn(d, ts);
        const float2 t2 = __fmul2_rn(t, t);
        const float d2 = t2.x + t2.y;
        if (d2 <= r2) {
            acc.sx += q.z;
            acc.sy += q.w;
            acc.count += 1u;
        }
    }
}

// Six resident 256-thread CTAs per SM (at most 42 registers) hide more of
// the cell-table and record load latency than five.
__global__ void __launch_bounds__(256, 6) neighbor_mean_kernel(MeanArgs a) {
    const uint32_t slot = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = slot < a.n;
    const Grid& g = a.g;
    const uint4 me = valid ? a.rec[slot] : make_uint4(0u, 0u, 0u, 0u);
    const float2 p = make_float2(__uint_as_float(me.x), __uint_as_float(me.y));
    const uint32_t tag = valid ? a.tag[slot] : 0u;
    float2 np = p;
    uint32_t count = 0;
    if (tag & kMovableBit) {
        const float tx = texel_of(p.x, g.map.wm1), ty = texel_of(p.y, g.map.hm1);
        // Reach box in grid cells (neighbor_mean.wgsl:180-185), in search cells.
        const uint32_t cx0 = grid_of(tx - g.reachx, g.rf, g.gw), cx1 = grid_of(tx + g.reachx, g.rf, g.gw);
        const uint32_t cy0 = grid_of(ty - g.reachy, g.rf, g.gh), cy1 = grid_of(ty + g.reachy, g.rf, g.gh);
        const int fx_min = static_cast<int>(cx0 * g.k), fx_max = static_cast<int>(cx1 * g.k + g.k - 1u);
        const int fy_min = static_cast<int>(cy0 * g.k), fy_max = static_cast<int>(cy1 * g.k + g.k - 1u);
        // Candidate circle r + m; certain circle r - m (texels).
        const float R = g.rf + g.margin;
        const float Rin = g.rf - g.margin;
        const int fy_lo = max(fy_min, floor_cell(ty - R, g.inv_s));
        const int fy_hi = min(fy_max, floor_cell(ty + R, g.inv_s));
        const bool interior = a.mode == kSearchInterior;
        const int fw = static_cast<int>(g.fw), fh = static_cast<int>(g.fh);
        const float2 neg_p = make_float2(-p.x, -p.y);
        const float2 ts = make_float2(g.tsx, g.tsy);
        Acc acc{0ull, 0ull, 0u};
        for (int fy = fy_lo; fy <= fy_hi; ++fy) {
            const float ylo = static_cast<float>(fy) * g.s;
            const float yhi = ylo + g.s;
            const float near = fmaxf(fmaxf(ylo - ty, ty - yhi), 0.0f);
            const float dn = fmaxf(near - g.margin, 0.0f);
            if (dn > R) continue;
            // f32 rounding of R^2 - dn^2 is below 5e-7 R^2; widen by that.
            const float hout = sqrt_approx(fmaxf(R * R - dn * dn + 5e-7f * R * R, 0.0f)) * 1.000001f + g.margin;
            const int bx0 = max(fx_min, floor_cell(tx - hout, g.inv_s));
            const int bx1 = min(fx_max, floor_cell(tx + hout, g.inv_s));
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
                        ix0 = max(ceil_cell(tx - hin, g.inv_s), max(bx0, 1));
                        ix1 = min(floor_cell(tx + hin, g.inv_s) - 1, min(bx1, fw - 2));
                    }
                }
            }
            if (ix0 <= ix1) {
                const uint32_t s1 = a.cell_start[row + ix0];
                const uint32_t s2 = a.cell_start[row + ix1 + 1];
                const LL2 lo = a.cell_prefix[row + ix0], hi = a.cell_prefix[row + ix1 + 1];
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
        const long long dx = static_cast<long long>(acc.sx - static_cast<unsigned long long>(count) * me.z);
        const long long dy = static_cast<long long>(acc.sy - static_cast<unsigned long long>(count) * me.w);
        const double den = static_cast<double>(count) * 1073741824.0;
        np.x = p.x + static_cast<float>(static_cast<double>(dx) / den);
        np.y = p.y + static_cast<float>(static_cast<double>(dy) / den);
    }
    // The next grid: search cell, population and biased position sum. Lanes
    // of a warp that land in one cell (neighbours in slot order mostly do)
    // add their counts and sums once.
    const uint32_t c = valid ? search_cell(np, g) : 0xFFFFFFFFu;
    const unsigned peers = __match_any_sync(0xFFFFFFFFu, c);
    if (!valid) return;
    const uint32_t qx = biased_fixed(np.x), qy = biased_fixed(np.y);
    // Group sums in 16-bit halves so each 32-bit reduction cannot overflow.
    const uint32_t xl = __reduce_add_sync(peers, qx & 0xFFFFu), xh = __reduce_add_sync(peers, qx >> 16);
    const uint32_t yl = __reduce_add_sync(peers, qy & 0xFFFFu), yh = __reduce_add_sync(peers, qy >> 16);
    if ((threadIdx.x & 31) == __ffs(peers) - 1) {
        atomicAdd(&a.hist[c], static_cast<uint32_t>(__popc(peers)));
        atomicAdd(reinterpret_cast<unsigned long long*>(&a.cellsum[c].x),
                  (static_cast<unsigned long long>(xh) << 16) + xl);
        atomicAdd(reinterpret_cast<unsigned long long*>(&a.cellsum[c].y),
                  (static_cast<unsigned long long>(yh) << 16) + yl);
    }
    a.out_xy[slot] = np;
    a.out_tag[slot] = tag;
    a.out_cell[slot] = c;
    if (a.counts) {
        uint32_t d;
        if (splat_index(np.x, np.y, g.map, &d)) atomicAdd(&a.counts[d], 1u);
    }
    if (a.neighbors) a.neighbors[slot] = count;
}

// Slot of each sample in the next order: start of its search cell plus a
// rank taken by counting the population down (order within a cell is free:
// the mean's exact sum does not depend on it).
__global__ void __launch_bounds__(256) scatter_kernel(ScatterArgs a) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = i < a.n;
    const uint32_t c = valid ? a.cell[i] : 0xFFFFFFFFu;
    // Lanes of one warp that share a cell (neighbours in slot order mostly do)
    // take one reservation and consecutive slots, so their writes coalesce.
    const unsigned peers = __match_any_sync(0xFFFFFFFFu, c);
    if (!valid) return;
    // Cell ids and populations are consistent by construction; a failed
    // upload can leave stale entries, which are skipped and flagged.
    if (c >= a.cells) {
        atomicOr(a.status, 8u);
        return;
    }
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(peers) - 1;
    const uint32_t group = __popc(peers);
    const uint32_t rank = __popc(peers & ((1u << lane) - 1u));
    uint32_t top = 0;
    if (lane == leader) top = atomicSub(&a.hist[c], group);
    top = __shfl_sync(peers, top, leader);
    const uint32_t slot = a.cell_start[c] + (top - group) + rank;
    if (top < group || slot >= a.n) {
        atomicOr(a.status, 8u);
        return;
    }
    const float2 p = a.xy[i];
    a.out_rec[slot] = make_uint4(__float_as_uint(p.x), __float_as_uint(p.y), biased_fixed(p.x), biased_fixed(p.y));
    a.out_tag[slot] = a.tag[i];
}

__global__ void unsort_records_kernel(const uint4* rec, const uint32_t* tag, const uint32_t* edge_ids, uint32_t n,
                                      uint32_t* records) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const uint32_t i = tag[s] & ~kMovableBit;
    const uint4 r = rec[s];
    records[3 * static_cast<size_t>(i)] = r.x;
    records[3 * static_cast<size_t>(i) + 1] = r.y;
    records[3 * static_cast<size_t>(i) + 2] = edge_ids[i];
}

__global__ void unsort_u32_kernel(const uint32_t* values, const uint32_t* tag, uint32_t n, uint32_t* out) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    out[tag[s] & ~kMovableBit] = values[s];
}

__global__ void records_kernel(const float2* xy, const uint32_t* edge_ids, uint32_t n, uint32_t* records) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float2 p = xy[i];
    records[3 * static_cast<size_t>(i)] = __float_as_uint(p.x);
    records[3 * static_cast<size_t>(i) + 1] = __float_as_uint(p.y);
    records[3 * static_cast<size_t>(i) + 2] = edge_ids[i];
}

// cell_index (spatial_grid.wgsl:67-70) of each sample, sample order.
__global__ void grid_cells_kernel(const uint4* rec, const uint32_t* tag, uint32_t n, Grid g, uint32_t* out) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const uint4 r = rec[s];
    const uint32_t cx = grid_of(texel_of(__uint_as_float(r.x), g.map.wm1), g.rf, g.gw);
    const uint32_t cy = grid_of(texel_of(__uint_as_float(r.y), g.map.hm1), g.rf, g.gh);
    out[tag[s] & ~kMovableBit] = cy * g.gw + cx;
}

__global__ void positions_kernel(const uint4* rec, const uint32_t* tag, uint32_t n, float2* out) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const uint4 r = rec[s];
    out[tag[s] & ~kMovableBit] = make_float2(__uint_as_float(r.x), __uint_as_float(r.y));
}

}  // namespace

void launch_neighbor_mean(const MeanArgs& a, cudaStream_t s) {
    if (a.n == 0) return;
    neighbor_mean_kernel<<<div_up(a.n, 256), 256, 0, s>>>(a);
}

void launch_scatter(const ScatterArgs& a, cudaStream_t s) {
    if (a.n == 0) return;
    scatter_kernel<<<div_up(a.n, 256), 256, 0, s>>>(a);
}

namespace {
// Scan input: a cell's population and position sums; the sums are cleared
// after their last read so the next iteration accumulates from zero.
struct CellAccSource {
    const uint32_t* hist;
    LL2* cellsum;
    __device__ __forceinline__ LL3 read(size_t j) const {
        const LL2 s = cellsum[j];
        return LL3{static_cast<long long>(hist[j]), s.x, s.y};
    }
    __device__ __forceinline__ void consume(size_t j) const { cellsum[j] = LL2{0, 0}; }
};

struct CellTableSink {
    uint32_t* cell_start;
    LL2* cell_prefix;
    __device__ __forceinline__ void store(size_t j, LL3 v) const {
        cell_start[j] = static_cast<uint32_t>(v.c);
        cell_prefix[j] = LL2{v.x, v.y};
    }
};
}  // namespace

size_t cell_table_scratch(size_t cells) { return scan_scratch_elems<LL3>(cells); }
int cell_table_launches(size_t cells) { return scan_launch_count<LL3>(cells); }

void launch_cell_table(const uint32_t* hist, LL2* cellsum, size_t cells, uint32_t* cell_start, LL2* cell_prefix,
                       LL3* scratch, cudaStream_t s) {
    exclusive_scan_with<LL3>(CellAccSource{hist, cellsum}, CellTableSink{cell_start, cell_prefix}, cells, scratch, s);
}

void launch_unsort_records(const uint4* rec, const uint32_t* tag, const uint32_t* edge_ids, uint32_t n,
                           uint32_t* records, cudaStream_t s) {
    if (n == 0) return;
    unsort_records_kernel<<<div_up(n, 256), 256, 0, s>>>(rec, tag, edge_ids, n, records);
}

void launch_unsort_u32(const uint32_t* values, const uint32_t* tag, uint32_t n, uint32_t* out, cudaStream_t s) {
    if (n == 0) return;
    unsort_u32_kernel<<<div_up(n, 256), 256, 0, s>>>(values, tag, n, out);
}

void launch_records_from_sample_order(const float2* xy, const uint32_t* edge_ids, uint32_t n, uint32_t* records,
                                      cudaStream_t s) {
    if (n == 0) return;
    records_kernel<<<div_up(n, 256), 256, 0, s>>>(xy, edge_ids, n, records);
}

void launch_grid_cells(const uint4* rec, const uint32_t* tag, uint32_t n, const Grid& g, uint32_t* out,
                       cudaStream_t s) {
    if (n == 0) return;
    grid_cells_kernel<<<div_up(n, 256), 256, 0, s>>>(rec, tag, n, g, out);
}

void launch_positions_from_slots(const uint4* rec, const uint32_t* tag, uint32_t n, float2* out, cudaStream_t s) {
    if (n == 0) return;
    positions_kernel<<<div_up(n, 256), 256, 0, s>>>(rec, tag, n, out);
}

}  // namespace bt
