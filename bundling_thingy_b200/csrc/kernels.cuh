// kernels.cuh — launchers of the bundling kernels (one stream per context).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"
#include "scan.cuh"

namespace bt {

// 12-byte path reservation (graph.wgsl Path; src/geometry.rs:8-12).
struct PathRec {
    uint32_t point_offset, segment_offset, count;
};

constexpr uint32_t kMovableBit = 0x80000000u;

// ---- resampling (resample.cu) ----
struct ResampleCountArgs {
    const float2* cp;
    const uint32_t* starts;
    uint32_t paths;
    Norm norm;
    float sx, sy;            // resampling texel_scale
    uint32_t capacity;
    unsigned long long* packed;   // (count << 32) | 1 for paths with >= 2 samples, else 0
    float4* edges;           // {first, last} control point per path
    unsigned long long* totals;   // [0] samples, [1] drawn paths
};
void launch_resample_count(const ResampleCountArgs& a, cudaStream_t s);

// Builds PathRec from the packed values and their exclusive scan.
void launch_paths_from_scan(const unsigned long long* packed, const unsigned long long* scan, uint32_t paths,
                            PathRec* out, cudaStream_t s);

struct ResampleEmitArgs {
    const float2* cp;
    const uint32_t* starts;
    const PathRec* paths;
    uint32_t n_paths;
    Norm norm;
    float sx, sy;
    Map map;
    float2* xy;              // sample order
    uint32_t* edge_ids;
    uint32_t* segments;
    uint32_t* counts;        // density splat (nullptr = off)
    // binning for the first iteration (nullptr = no neighbour grid)
    const Grid* grid_host;   // host copy (passed by value to the kernel)
    uint32_t* tag;           // sample index | movable bit, sample order
    uint32_t* cell;          // search cell of each sample
    uint32_t* hist;          // search-cell populations
    uint32_t* status;        // bit 1: count/emit mismatch
};
void launch_resample_emit(const ResampleEmitArgs& a, cudaStream_t s);

// ---- density (density.cu) ----
constexpr int kMaxTaps = 129;   // R <= 128
struct Taps {
    float w[kMaxTaps];
    int R;
};
cudaError_t prepare_density_kernels();
void launch_blur_horizontal(const uint32_t* counts, float* out, uint32_t w, uint32_t h, const Taps& taps,
                            cudaStream_t s);
void launch_blur_vertical(const float* in, float* out, uint32_t w, uint32_t h, const Taps& taps, uint32_t* peak,
                          cudaStream_t s);
void launch_normalize(const float* in, const uint32_t* peak, float* out, size_t n, cudaStream_t s);
// TMA-staged passes (blur_tma.cu), for maps whose rows and columns are whole
// 16-byte units, 16-byte aligned buffers and halos up to 48 texels
// (blur_tma_eligible); same results as the element-staged passes. The
// horizontal pass writes its result transposed (out_t[x * h + y]) and the
// vertical pass reads it so. A copy wait that runs out sets bit 16 of *status.
bool blur_tma_eligible(const void* in, const void* out, uint32_t w, uint32_t h, int R);
cudaError_t prepare_blur_tma_kernels();
cudaError_t launch_blur_horizontal_tma(const uint32_t* counts, float* out_t, uint32_t w, uint32_t h,
                                       const Taps& taps, uint32_t* status, cudaStream_t s);
cudaError_t launch_blur_vertical_tma(const float* in_t, float* out, uint32_t w, uint32_t h, const Taps& taps,
                                     uint32_t* peak, uint32_t* status, cudaStream_t s);

// ---- neighbour grid and mean (grid.cu) ----
// Slot-order sample records hold the position alone (float2, 8 bytes); the
// exact neighbour sums use Q(v) = round-half-even(v * 2^30), recomputed from
// it and biased by 2^30 so that the values are unsigned.
constexpr uint32_t kFixedBias = 1u << 30;


__device__ __forceinline__ uint32_t biased_fixed(float v) {
    return static_cast<uint32_t>(__float2int_rn(v * kFixedScale)) + kFixedBias;
}

enum SearchMode : int {
    kSearchInterior = 0,   // interior search cells from the prefix sums, boundary ring tested exactly
    kSearchScanAll = 1,    // every sample of the candidate search cells tested exactly
};

struct MeanArgs {
    const float2* rec;       // slot order (sorted by search cell)
    const uint32_t* tag;     // sample index | movable bit, slot order
    const uint32_t* cell_start;   // cell table: first slot of each search cell (cells + 1)
    const LL2* prefix;       // sum of the biased positions of all earlier slots (n + 1)
    float2* out_xy;          // new positions, same slot order
    uint32_t* out_tag;
    uint32_t* out_cell;      // search cell of the new position
    uint32_t* hist;          // populations of the next grid
    uint32_t* hist_tiles;    // their sums per cell-table tile (zero before the launch)
    uint32_t* counts;        // density splat (nullptr = off)
    uint32_t* neighbors;     // |N(p)| per slot (nullptr = off)
    uint32_t* chunk_counter; // work-queue head of the persistent single-graph kernel (reset by its launcher)
    uint32_t n;
    Grid g;
    int mode;                // SearchMode
};
void launch_neighbor_mean(const MeanArgs& a, cudaStream_t s);

// Sampled work of the neighbour search under grid g (slot order rec/tag with
// its cell table): over every `stride`-th slot that is movable, out[0] =
// search rows, out[1] = samples in boundary cells (tested exactly), out[2] =
// slots probed (out is cleared first, on s).
void launch_search_probe(const float2* rec, const uint32_t* tag, const uint32_t* cell_start, uint32_t n,
                         const Grid& g, uint32_t stride, unsigned long long* out, cudaStream_t s);

// Tiles of the cell table (search cells) and of the slot prefix (slots).
constexpr uint32_t kCellTile = static_cast<uint32_t>(scan_tile<uint32_t>());
constexpr uint32_t kPrefixTile = static_cast<uint32_t>(scan_tile<LL2>());

// Cell table of the next slot order: the first slot of each search cell, an
// exclusive scan of the populations (which stay for the scatter's count-down).
// hist_tiles (scan_tiles(cells) + 1 entries) holds the populations' sums per
// tile when tiles_ready (the mean kernel accumulates them), else they are
// reduced here.
void launch_cell_table(const uint32_t* hist, size_t cells, uint32_t* cell_start, uint32_t* hist_tiles,
                       bool tiles_ready, cudaStream_t s);

// Pairs of samples sharing a grid cell (r x r texels): sum over grid cells of
// n (n - 1), from the search-cell populations; added to *out. scratch holds
// gw * gh u32 (any contents).
void launch_grid_pairs(const uint32_t* hist, const Grid& g, uint32_t* scratch, unsigned long long* out,
                       cudaStream_t s);

// Re-bins slot-order records under another search-cell shape: positions,
// tags and new search cells in slot order (the scatter's input) and the new
// populations (hist must be zero).
void launch_rebin(const float2* rec, const uint32_t* tag, uint32_t n, const Grid& g, float2* xy, uint32_t* out_tag,
                  uint32_t* cell, uint32_t* hist, cudaStream_t s);

// Slot prefix of the scattered records: prefix[j] = sum over slots < j of the
// biased fixed-point positions (n + 1 entries); prefix_tiles (scan_tiles(n) +
// 1 entries) is its scratch.
void launch_slot_prefix(const float2* rec, uint32_t n, LL2* prefix, LL2* prefix_tiles, cudaStream_t s);

struct ScatterArgs {
    const float2* xy;
    const uint32_t* tag;
    const uint32_t* cell;
    const uint32_t* cell_start;
    uint32_t* hist;          // counted down to zero
    float2* out_rec;
    uint32_t* out_tag;
    uint32_t n;
    uint32_t cells;          // search cells
    uint32_t* status;        // bit 3 (value 8): inconsistent binning input
};
void launch_scatter(const ScatterArgs& a, cudaStream_t s);

// Sample-order records {x, y, edge_id} from slot order.
void launch_unsort_records(const float2* rec, const uint32_t* tag, const uint32_t* edge_ids, uint32_t n,
                           uint32_t* records, cudaStream_t s);
void launch_unsort_u32(const uint32_t* values, const uint32_t* tag, uint32_t n, uint32_t* out, cudaStream_t s);
void launch_records_from_sample_order(const float2* xy, const uint32_t* edge_ids, uint32_t n, uint32_t* records,
                                      cudaStream_t s);
void launch_grid_cells(const float2* rec, const uint32_t* tag, uint32_t n, const Grid& g, uint32_t* out,
                       cudaStream_t s);
void launch_positions_from_slots(const float2* rec, const uint32_t* tag, uint32_t n, float2* out, cudaStream_t s);
// Checkpointed 12-byte {x, y, edge_id} records (sample order) back into
// sample-order positions; with slot_tag (the current slot order's tags) also
// each sample's tag in sample order (tag_out). A record whose edge id differs
// from the uploaded graph's, or whose position is not finite, sets bit 5
// (value 32) of *status.
void launch_restore_records(const uint32_t* records, const uint32_t* edge_ids, const uint32_t* slot_tag, uint32_t n,
                            float2* xy, uint32_t* tag_out, uint32_t* status, cudaStream_t s);
// Density splat of n sample positions (counts zero before the launch).
void launch_splat_positions(const float2* xy, uint32_t n, Map map, uint32_t* counts, cudaStream_t s);

// ---- distortion (distortion.cu) ----
// Per-edge squared_integral of original vs current (sample order); status bit
// 2 (value 4) flags an invalid curve or interval.
void launch_edge_integrals(const PathRec* paths, uint32_t n_paths, const float2* original, const float2* current,
                           double* out, uint32_t* status, cudaStream_t s);

// ---- density-gradient advection (advect.cu) ----
struct AdvectArgs {
    const float2* xy;            // current positions, sample order
    const uint32_t* edge_ids;    // per sample (paths are contiguous)
    uint32_t n;
    const float* density;        // normalised density of xy, map.w x map.h
    Map map;
    float step;                  // texels per iteration
    float smooth;                // Laplacian relaxation weight
    float sx_inv, sy_inv;        // 2 / (W - 1), 2 / (H - 1)
    float2* out;                 // new positions, sample order
    uint32_t* counts;            // splat of the new positions (zero before)
};
void launch_advect(const AdvectArgs& a, cudaStream_t s);

// ---- rendering (render.cu) ----
// Pairs per block of the stable tile sort; tiles per frame at most (the sort
// keeps one 4-byte counter per tile in shared memory).
constexpr uint32_t kBinItems = 16384;
constexpr uint32_t kMaxRenderTiles = 16384;

struct RenderArgs {
    const float2* xy;            // current positions, sample order
    const uint32_t* edge_ids;    // per sample
    const uint32_t* segments;    // first sample of each segment, draw order
    uint32_t n_segments;
    const PathRec* paths;        // endpoint dots
    uint32_t n_paths;
    const float* density;        // normalised density, w x h (density colouring)
    uint32_t w, h;
    float edge_den;              // max(edges, 2) - 1
    int color_by_edge, palette, ns;
    int tile_shift;              // tiles of (1 << tile_shift) pixels square
    uint32_t tiles_x, tiles_y;
    unsigned long long* seg_count;   // n_segments: tiles per segment
    unsigned long long* seg_off;     // n_segments + 1
    uint32_t* pair_tile;         // pairs, segment order
    uint32_t* pair_seg;
    unsigned long long pair_capacity;         // pairs the bin buffers hold
    const unsigned long long* pair_total;     // device: pairs of this frame (above the
                                              // capacity: nothing is binned)
    uint32_t bin_blocks;         // ceil(pair_capacity / kBinItems)
    uint32_t* hist;              // tiles * bin_blocks
    uint32_t* hist_off;          // tiles * bin_blocks + 1 (null: no segments)
    uint32_t* sorted;            // pairs: segment ids, tile-major, draw order
    uint32_t* samples;           // w * h * ns packed RGB8
    uint32_t* rgba;              // w * h
    unsigned long long* colored;
};

// Tile size for a w x h frame (4, 5 or 6), or -1 when it has too many tiles.
int render_tile_shift(uint32_t w, uint32_t h);
void launch_render_bin_count(const RenderArgs& a, cudaStream_t s);
void launch_render_bin_emit(const RenderArgs& a, cudaStream_t s);
// Histogram, scan and stable scatter of the pairs by tile; scan_scratch holds
// scan_scratch_elems<uint32_t>(tiles * bin_blocks) elements.
cudaError_t launch_render_bin_sort(const RenderArgs& a, uint32_t* scan_scratch, cudaStream_t s);
void launch_render_raster(const RenderArgs& a, cudaStream_t s);
void launch_render_endpoints(const RenderArgs& a, cudaStream_t s);
void launch_render_resolve(const RenderArgs& a, cudaStream_t s);

}  // namespace bt
