// grid.cu — neighbour-grid binning and the fused neighbour-mean step.
//
// Restates count_cells / reserve_cells / scatter_points
// (src/shaders/spatial_grid.wgsl:72-138) and neighbor_mean_sparse
// (src/shaders/neighbor_mean.wgsl:164-203) with write_point's splat (66-73).
//
// Semantics (identical to the oracle): N(p) = every sample q whose grid cell
// lies in p's reach box (grid_cell(texel(p) -/+ reach)) and that passes the
// reference's f32 test dot((q-p)*ts, (q-p)*ts) <= r*r. The displacement is
// accumulated exactly in 2^-30 fixed point (int64), so the result does not
// depend on the order of N(p) — which the reference leaves to atomics — and
// p' = p + f32(f64(sum) / (f64(|N|) * 2^30)).
//
// B200 layout: samples live in slot order, sorted by search cell (each grid
// cell side split into k search cells, search cells row-major over the whole
// map). A search row of cells [a, b] is then one contiguous slot range, so a
// thread walks, row by row, only the search cells that can meet its circle
// (conservative chord bounds), testing every sample there exactly. The kernel
// writes the new position in the same slot order (coalesced), its next search
// cell and population count (fusing count_cells of the next iteration), and
// its density splat. The scatter then moves the samples into the next slot
// order, counting the populations back down to zero for reuse.
#include "kernels.cuh"

namespace bt {
namespace {

__device__ __forceinline__ int floor_div(float t, float s) { return static_cast<int>(floorf(t / s)); }

__global__ void __launch_bounds__(256) neighbor_mean_kernel(MeanArgs a) {
    const uint32_t slot = blockIdx.x * blockDim.x + threadIdx.x;
    if (slot >= a.n) return;
    const Grid& g = a.g;
    const float2 p = a.xy[slot];
    const uint32_t tag = a.tag[slot];
    float2 np = p;
    uint32_t count = 0;
    if (tag & kMovableBit) {
        const float tx = texel_of(p.x, g.map.wm1), ty = texel_of(p.y, g.map.hm1);
        // Reach box in grid cells (neighbor_mean.wgsl:180-185).
        const uint32_t cx0 = grid_of(tx - g.reachx, g.rf, g.gw), cx1 = grid_of(tx + g.reachx, g.rf, g.gw);
        const uint32_t cy0 = grid_of(ty - g.reachy, g.rf, g.gh), cy1 = grid_of(ty + g.reachy, g.rf, g.gh);
        const int fx_min = static_cast<int>(cx0 * g.k), fx_max = static_cast<int>(cx1 * g.k + g.k - 1u);
        const int fy_min = static_cast<int>(cy0 * g.k), fy_max = static_cast<int>(cy1 * g.k + g.k - 1u);
        // Conservative circle: radius r + margin around the texel position.
        const float R = g.rf + g.margin;
        const int fy_lo = max(fy_min, floor_div(ty - R, g.s));
        const int fy_hi = min(fy_max, floor_div(ty + R, g.s));
        const int2 qp = a.q[slot];
        long long sx = 0, sy = 0;
        for (int fy = fy_lo; fy <= fy_hi; ++fy) {
            const float ylo = static_cast<float>(fy) * g.s;
            const float yhi = ylo + g.s;
            float dy = fmaxf(fmaxf(ylo - ty, ty - yhi), 0.0f) - g.margin;
            dy = fmaxf(dy, 0.0f);
            if (dy > R) continue;
            const float half = sqrtf(fmaxf(R * R - dy * dy, 0.0f)) + g.margin;
            const int fx_lo = max(fx_min, floor_div(tx - half, g.s));
            const int fx_hi = min(fx_max, floor_div(tx + half, g.s));
            if (fx_lo > fx_hi) continue;
            const uint32_t row = static_cast<uint32_t>(fy) * g.fw;
            const uint32_t b = a.cell_start[row + fx_lo];
            const uint32_t e = a.cell_start[row + fx_hi + 1];
            for (uint32_t j = b; j < e; ++j) {
                const float2 qq = a.xy[j];
                const float dx = qq.x - p.x, ddy = qq.y - p.y;
                const float ex = dx * g.tsx, ey = ddy * g.tsy;
                const float d2 = ex * ex + ey * ey;
                if (d2 <= g.r2) {
                    const int2 qj = a.q[j];
                    sx += static_cast<long long>(qj.x) - static_cast<long long>(qp.x);
                    sy += static_cast<long long>(qj.y) - static_cast<long long>(qp.y);
                    ++count;
                }
            }
        }
        const double den = static_cast<double>(count) * 1073741824.0;
        np.x = p.x + static_cast<float>(static_cast<double>(sx) / den);
        np.y = p.y + static_cast<float>(static_cast<double>(sy) / den);
    }
    a.out_xy[slot] = np;
    a.out_tag[slot] = tag;
    const uint32_t c = search_cell(np, g);
    a.out_cell[slot] = c;
    atomicAdd(&a.hist[c], 1u);
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
    if (i >= a.n) return;
    const uint32_t c = a.cell[i];
    // Cell ids and populations are consistent by construction; a failed
    // upload can leave stale entries, which are skipped and flagged.
    if (c >= a.cells) {
        atomicOr(a.status, 8u);
        return;
    }
    const uint32_t rank = atomicSub(&a.hist[c], 1u);
    const uint32_t slot = a.cell_start[c] + rank - 1u;
    if (rank == 0u || slot >= a.n) {
        atomicOr(a.status, 8u);
        return;
    }
    const float2 p = a.xy[i];
    a.out_xy[slot] = p;
    a.out_q[slot] = make_int2(__float2int_rn(p.x * kFixedScale), __float2int_rn(p.y * kFixedScale));
    a.out_tag[slot] = a.tag[i];
}

__global__ void unsort_records_kernel(const float2* xy, const uint32_t* tag, const uint32_t* edge_ids, uint32_t n,
                                      uint32_t* records) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const uint32_t i = tag[s] & ~kMovableBit;
    const float2 p = xy[s];
    records[3 * static_cast<size_t>(i)] = __float_as_uint(p.x);
    records[3 * static_cast<size_t>(i) + 1] = __float_as_uint(p.y);
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
__global__ void grid_cells_kernel(const float2* xy, const uint32_t* tag, uint32_t n, Grid g, uint32_t* out) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const float2 p = xy[s];
    const uint32_t cx = grid_of(texel_of(p.x, g.map.wm1), g.rf, g.gw);
    const uint32_t cy = grid_of(texel_of(p.y, g.map.hm1), g.rf, g.gh);
    const uint32_t i = tag ? (tag[s] & ~kMovableBit) : s;
    out[i] = cy * g.gw + cx;
}

__global__ void positions_kernel(const float2* xy, const uint32_t* tag, uint32_t n, float2* out) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    out[tag[s] & ~kMovableBit] = xy[s];
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

void launch_unsort_records(const float2* xy, const uint32_t* tag, const uint32_t* edge_ids, uint32_t n,
                           uint32_t* records, cudaStream_t s) {
    if (n == 0) return;
    unsort_records_kernel<<<div_up(n, 256), 256, 0, s>>>(xy, tag, edge_ids, n, records);
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

void launch_grid_cells(const float2* xy, const uint32_t* tag, uint32_t n, const Grid& g, uint32_t* out,
                       cudaStream_t s) {
    if (n == 0) return;
    grid_cells_kernel<<<div_up(n, 256), 256, 0, s>>>(xy, tag, n, g, out);
}

void launch_positions_from_slots(const float2* xy, const uint32_t* tag, uint32_t n, float2* out, cudaStream_t s) {
    if (n == 0) return;
    positions_kernel<<<div_up(n, 256), 256, 0, s>>>(xy, tag, n, out);
}

}  // namespace bt
