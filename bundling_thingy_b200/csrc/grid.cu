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
// B200 layout: samples live in slot order as 8-byte position records (their
// biased fixed-point values Q + 2^30 recomputed where a sum needs them: an
// exact conversion, cheaper than moving 16-byte records through the
// candidate loads), sorted by search cell (each grid cell split
// into kx x ky search cells, search cells row-major over the whole map), so a
// row of search cells [a, b] is one contiguous slot range. The cell table (a
// scan of the search-cell populations) gives each cell's first slot, and the
// slot prefix (a scan of the records) the sum of the biased fixed-point
// positions of all earlier slots, which turns any such range into one
// subtraction. Per search row, a thread takes the cells that lie entirely
// inside its circle (by conservative bounds, with a margin far above every f32
// rounding involved) from the prefix — the role of the reference's
// fully-contained cell summaries (neighbor_mean.wgsl:40-59) — and tests only
// the samples of the boundary cells, exactly. Flat search cells (kx > ky) cut
// the boundary band: its area per circle is about 4 r (sy + sx) texels. The
// kernel writes the new position in the same slot order (coalesced), the new
// search cell's population (warp-aggregated; this fuses count_cells of the
// next iteration), and its density splat. The scatter then moves the samples
// into the next slot order, counting the populations back down to zero.
// The per-sample bodies live in grid_dev.cuh (shared with batch.cu).
#include <algorithm>

#include "grid_dev.cuh"

namespace bt {
namespace {

// Forty resident warps per SM at 48 registers: with 8-byte records and eight
// candidate loads in flight per lane, the registers are worth more than a
// sixth 256-thread CTA (0.86 against 0.90 ms per steady-state iteration of
// the large workload; four: 0.92). Ten CTAs of 128 rather than five of 256:
// samples of very different neighbourhood sizes share an SM at a finer
// grain, which trims the tail (0.845 against 0.863 ms; 64 threads: 0.849).
// Persistent: one grid of SMs x 10 CTAs, each warp taking 32-slot chunks
// (its first by warp id, the rest from an atomic queue), so a warp that
// finishes early takes more work instead of holding its CTA's slot idle
// until the CTA's slowest warp is done (36.5 against 37.3 ms per
// 30-iteration job of the large workload; 64-slot chunks: 40.1 ms).
constexpr uint32_t kMeanChunk = 32;
__global__ void __launch_bounds__(128, 10) neighbor_mean_kernel(MeanArgs a) {
    const int lane = threadIdx.x & 31;
    const uint32_t warps = gridDim.x * (blockDim.x / 32u);
    uint32_t base = (blockIdx.x * (blockDim.x / 32u) + (threadIdx.x >> 5)) * kMeanChunk;
    while (base < a.n) {
        dev::mean_sample(a, base + lane);
        uint32_t next = 0;
        if (lane == 0) next = atomicAdd(a.chunk_counter, kMeanChunk);
        base = warps * kMeanChunk + __shfl_sync(0xFFFFFFFFu, next, 0);
    }
}

__global__ void __launch_bounds__(256) scatter_kernel(ScatterArgs a) {
    dev::scatter_sample(a, blockIdx.x * blockDim.x + threadIdx.x);
}

__global__ void unsort_records_kernel(const float2* rec, const uint32_t* tag, const uint32_t* edge_ids, uint32_t n,
                                      uint32_t* records) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const uint32_t i = tag[s] & ~kMovableBit;
    const float2 r = rec[s];
    records[3 * static_cast<size_t>(i)] = __float_as_uint(r.x);
    records[3 * static_cast<size_t>(i) + 1] = __float_as_uint(r.y);
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
__global__ void grid_cells_kernel(const float2* rec, const uint32_t* tag, uint32_t n, Grid g, uint32_t* out) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const float2 r = rec[s];
    const uint32_t cx = grid_of(texel_of(r.x, g.map.wm1), g.rf, g.gw);
    const uint32_t cy = grid_of(texel_of(r.y, g.map.hm1), g.rf, g.gh);
    out[tag[s] & ~kMovableBit] = cy * g.gw + cx;
}

// Populations of the reference's grid cells (r x r) from the search-cell
// populations; counts is zero before the launch.
__global__ void __launch_bounds__(256) grid_counts_kernel(const uint32_t* hist, Grid g, uint32_t* counts) {
    const size_t cells = static_cast<size_t>(g.fw) * g.fh;
    for (size_t c = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; c < cells;
         c += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const uint32_t n = hist[c];
        if (n == 0) continue;
        const uint32_t fx = static_cast<uint32_t>(c % g.fw), fy = static_cast<uint32_t>(c / g.fw);
        atomicAdd(&counts[(fy / g.ky) * g.gw + fx / g.kx], n);
    }
}

__global__ void __launch_bounds__(256) grid_pairs_kernel(const uint32_t* counts, uint32_t n_cells,
                                                         unsigned long long* out) {
    __shared__ unsigned long long warp_sums[8];
    unsigned long long acc = 0;
    for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < n_cells; c += gridDim.x * blockDim.x) {
        const unsigned long long n = counts[c];
        acc += n * (n ? n - 1 : 0);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xFFFFFFFFu, acc, o);
    if ((threadIdx.x & 31) == 0) warp_sums[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long total = 0;
        for (int w = 0; w < 8; ++w) total += warp_sums[w];
        atomicAdd(out, total);
    }
}

__global__ void __launch_bounds__(256) rebin_kernel(const float2* rec, const uint32_t* tag, uint32_t n, Grid g,
                                                    float2* xy, uint32_t* out_tag, uint32_t* cell, uint32_t* hist) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = s < n;
    const float2 p = valid ? rec[s] : make_float2(0.0f, 0.0f);
    const uint32_t c = valid ? search_cell(p, g) : 0xFFFFFFFFu;
    const unsigned peers = __match_any_sync(0xFFFFFFFFu, c);
    if (!valid) return;
    if ((threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(&hist[c], static_cast<uint32_t>(__popc(peers)));
    xy[s] = p;
    out_tag[s] = tag[s];
    cell[s] = c;
}

__global__ void positions_kernel(const float2* rec, const uint32_t* tag, uint32_t n, float2* out) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    out[tag[s] & ~kMovableBit] = rec[s];
}

__global__ void restore_kernel(const uint32_t* records, const uint32_t* edge_ids, const uint32_t* slot_tag, uint32_t n,
                               float2* xy, uint32_t* tag_out, uint32_t* status) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    uint32_t i = s;
    if (slot_tag) {
        const uint32_t t = slot_tag[s];
        i = t & ~kMovableBit;
        tag_out[i] = t;
    }
    const float x = __uint_as_float(records[3 * static_cast<size_t>(i)]);
    const float y = __uint_as_float(records[3 * static_cast<size_t>(i) + 1]);
    if (records[3 * static_cast<size_t>(i) + 2] != edge_ids[i] || !isfinite(x) || !isfinite(y)) atomicOr(status, 32u);
    xy[i] = make_float2(x, y);
}

}  // namespace

void launch_restore_records(const uint32_t* records, const uint32_t* edge_ids, const uint32_t* slot_tag, uint32_t n,
                            float2* xy, uint32_t* tag_out, uint32_t* status, cudaStream_t s) {
    if (n == 0) return;
    restore_kernel<<<div_up(n, 256), 256, 0, s>>>(records, edge_ids, slot_tag, n, xy, tag_out, status);
}

void launch_neighbor_mean(const MeanArgs& a, cudaStream_t s) {
    if (a.n == 0) return;
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaMemsetAsync(a.chunk_counter, 0, sizeof(uint32_t), s);
    const unsigned grid = std::min<unsigned>(div_up(a.n, 128), static_cast<unsigned>(sms) * 10u);
    neighbor_mean_kernel<<<grid, 128, 0, s>>>(a);
}

namespace {

// Work of the neighbour search on every `stride`-th slot: its search rows
// and the samples of its boundary cells (those the mean tests exactly), with
// the row bounds of mean_sample. out[0] += rows, out[1] += boundary samples,
// out[2] += movable samples probed.
__global__ void __launch_bounds__(256) search_probe_kernel(const float2* rec, const uint32_t* tag,
                                                           const uint32_t* cell_start, uint32_t n, Grid g,
                                                           uint32_t stride, unsigned long long* out) {
    const uint64_t s = (static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x) * stride;
    uint32_t rows = 0, tests = 0, probed = 0;
    if (s < n && (tag[s] & kMovableBit)) {
        const float2 p = rec[s];
        const float tx = texel_of(p.x, g.map.wm1), ty = texel_of(p.y, g.map.hm1);
        const uint32_t cx0 = grid_of(tx - g.reachx, g.rf, g.gw), cx1 = grid_of(tx + g.reachx, g.rf, g.gw);
        const uint32_t cy0 = grid_of(ty - g.reachy, g.rf, g.gh), cy1 = grid_of(ty + g.reachy, g.rf, g.gh);
        const int fx_min = static_cast<int>(cx0 * g.kx), fx_max = static_cast<int>(cx1 * g.kx + g.kx - 1u);
        const int fy_min = static_cast<int>(cy0 * g.ky), fy_max = static_cast<int>(cy1 * g.ky + g.ky - 1u);
        const float R = g.rf + g.margin, Rin = g.rf - g.margin;
        const int fw = static_cast<int>(g.fw), fh = static_cast<int>(g.fh);
        const int fy_lo = max(fy_min, static_cast<int>(floorf((ty - R) * g.inv_sy)));
        const int fy_hi = min(fy_max, static_cast<int>(floorf((ty + R) * g.inv_sy)));
        probed = 1;
        for (int fy = fy_lo; fy <= fy_hi; ++fy) {
            const float ylo = static_cast<float>(fy) * g.sy, yhi = ylo + g.sy;
            const float dn = fmaxf(fmaxf(fmaxf(ylo - ty, ty - yhi), 0.0f) - g.margin, 0.0f);
            if (dn > R) continue;
            const float hout = sqrtf(fmaxf(R * R - dn * dn, 0.0f)) + g.margin;
            const int bx0 = max(fx_min, static_cast<int>(floorf((tx - hout) * g.inv_sx)));
            const int bx1 = min(fx_max, static_cast<int>(floorf((tx + hout) * g.inv_sx)));
            if (bx0 > bx1) continue;
            ++rows;
            const uint32_t row = static_cast<uint32_t>(fy) * g.fw;
            const uint32_t s0 = cell_start[row + bx0], s3 = cell_start[row + bx1 + 1];
            uint32_t inner = 0;
            const float far = fmaxf(fabsf(ylo - ty), fabsf(yhi - ty)) + g.margin;
            if (fy > 0 && fy < fh - 1 && far < Rin) {
                const float hin = sqrtf(fmaxf(Rin * Rin - far * far, 0.0f)) - g.margin;
                if (hin > 0.0f) {
                    const int ix0 = max(static_cast<int>(ceilf((tx - hin) * g.inv_sx)), max(bx0, 1));
                    const int ix1 = min(static_cast<int>(floorf((tx + hin) * g.inv_sx)) - 1, min(bx1, fw - 2));
                    if (ix0 <= ix1) inner = cell_start[row + ix1 + 1] - cell_start[row + ix0];
                }
            }
            tests += (s3 - s0) - inner;
        }
    }
    // One atomic per warp and counter.
    for (int o = 16; o > 0; o >>= 1) {
        rows += __shfl_xor_sync(0xFFFFFFFFu, rows, o);
        tests += __shfl_xor_sync(0xFFFFFFFFu, tests, o);
        probed += __shfl_xor_sync(0xFFFFFFFFu, probed, o);
    }
    if ((threadIdx.x & 31) == 0 && probed) {
        atomicAdd(&out[0], static_cast<unsigned long long>(rows));
        atomicAdd(&out[1], static_cast<unsigned long long>(tests));
        atomicAdd(&out[2], static_cast<unsigned long long>(probed));
    }
}

}  // namespace

void launch_search_probe(const float2* rec, const uint32_t* tag, const uint32_t* cell_start, uint32_t n,
                         const Grid& g, uint32_t stride, unsigned long long* out, cudaStream_t s) {
    cudaMemsetAsync(out, 0, 3 * sizeof(unsigned long long), s);
    if (n == 0 || stride == 0) return;
    const uint64_t probes = (static_cast<uint64_t>(n) + stride - 1) / stride;   // >= 1, <= n
    search_probe_kernel<<<div_up(probes, 256), 256, 0, s>>>(rec, tag, cell_start, n, g, stride, out);
}

void launch_scatter(const ScatterArgs& a, cudaStream_t s) {
    if (a.n == 0) return;
    scatter_kernel<<<div_up(a.n, 256), 256, 0, s>>>(a);
}

void launch_cell_table(const uint32_t* hist, size_t cells, uint32_t* cell_start, uint32_t* hist_tiles,
                       bool tiles_ready, cudaStream_t s) {
    if (!tiles_ready) reduce_tiles<uint32_t>(ArraySource<uint32_t>{hist}, cells, hist_tiles, s);
    exclusive_scan_presummed<uint32_t>(ArraySource<uint32_t>{hist}, ArraySink<uint32_t>{cell_start}, cells,
                                       hist_tiles, s);
}

void launch_slot_prefix(const float2* rec, uint32_t n, LL2* prefix, LL2* prefix_tiles, cudaStream_t s) {
    reduce_tiles<LL2>(dev::RecordQSource{rec}, n, prefix_tiles, s);
    exclusive_scan_presummed<LL2>(dev::RecordQSource{rec}, ArraySink<LL2>{prefix}, n, prefix_tiles, s);
}

void launch_grid_pairs(const uint32_t* hist, const Grid& g, uint32_t* scratch, unsigned long long* out,
                       cudaStream_t s) {
    const uint32_t grid_cells = g.gw * g.gh;
    const size_t cells = static_cast<size_t>(g.fw) * g.fh;
    cudaMemsetAsync(scratch, 0, 4ull * grid_cells, s);
    grid_counts_kernel<<<static_cast<unsigned>(std::min<size_t>((cells + 255) / 256, 148 * 16)), 256, 0, s>>>(
        hist, g, scratch);
    grid_pairs_kernel<<<std::min(div_up(grid_cells, 256), 1184u), 256, 0, s>>>(scratch, grid_cells, out);
}

void launch_rebin(const float2* rec, const uint32_t* tag, uint32_t n, const Grid& g, float2* xy, uint32_t* out_tag,
                  uint32_t* cell, uint32_t* hist, cudaStream_t s) {
    if (n == 0) return;
    rebin_kernel<<<div_up(n, 256), 256, 0, s>>>(rec, tag, n, g, xy, out_tag, cell, hist);
}

void launch_unsort_records(const float2* rec, const uint32_t* tag, const uint32_t* edge_ids, uint32_t n,
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

void launch_grid_cells(const float2* rec, const uint32_t* tag, uint32_t n, const Grid& g, uint32_t* out,
                       cudaStream_t s) {
    if (n == 0) return;
    grid_cells_kernel<<<div_up(n, 256), 256, 0, s>>>(rec, tag, n, g, out);
}

void launch_positions_from_slots(const float2* rec, const uint32_t* tag, uint32_t n, float2* out, cudaStream_t s) {
    if (n == 0) return;
    positions_kernel<<<div_up(n, 256), 256, 0, s>>>(rec, tag, n, out);
}

}  // namespace bt
