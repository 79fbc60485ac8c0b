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
    LL2* cellsum;            // search-cell sums of the biased fixed-point positions
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

// ---- neighbour grid and mean (grid.cu) ----
// Slot-order sample record: {f32 x bits, f32 y bits, Qx + 2^30, Qy + 2^30}
// with Q(v) = round-half-even(v * 2^30), so the biased values are unsigned.
constexpr uint32_t kFixedBias = 1u << 30;

__device__ __forceinline__ uint32_t biased_fixed(float v) {
    return static_cast<uint32_t>(__float2int_rn(v * kFixedScale)) + kFixedBias;
}

// Adds a sample's biased fixed-point position to its cell's sums.
__device__ __forceinline__ void add_cell_sum(LL2* cellsum, uint32_t c, uint32_t qx, uint32_t qy) {
    atomicAdd(reinterpret_cast<unsigned long long*>(&cellsum[c].x), static_cast<unsigned long long>(qx));
    atomicAdd(reinterpret_cast<unsigned long long*>(&cellsum[c].y), static_cast<unsigned long long>(qy));
}

enum SearchMode : int {
    kSearchInterior = 0,   // interior search cells from the prefix sums, boundary ring tested exactly
    kSearchScanAll = 1,    // every sample of the candidate search cells tested exactly
};

struct MeanArgs {
    const uint4* rec;        // slot order (sorted by search cell)
    const uint32_t* tag;     // sample index | movable bit, slot order
    const uint32_t* cell_start;   // cell table: first slot of each search cell (cells + 1)
    const LL2* cell_prefix;  // cell table: sum of the biased positions of all earlier slots (cells + 1)
    float2* out_xy;          // new positions, same slot order
    uint32_t* out_tag;
    uint32_t* out_cell;      // search cell of the new position
    uint32_t* hist;          // populations of the next grid
    LL2* cellsum;            // biased position sums of the next grid
    uint32_t* counts;        // density splat (nullptr = off)
    uint32_t* neighbors;     // |N(p)| per slot (nullptr = off)
    uint32_t n;
    Grid g;
    int mode;                // SearchMode
};
void launch_neighbor_mean(const MeanArgs& a, cudaStream_t s);

// Cell table of the next slot order from the populations and sums (the sums
// are cleared for reuse; the populations stay for the scatter's count-down).
void launch_cell_table(const uint32_t* hist, LL2* cellsum, size_t cells, uint32_t* cell_start, LL2* cell_prefix,
                       LL3* scratch, cudaStream_t s);
size_t cell_table_scratch(size_t cells);
int cell_table_launches(size_t cells);

struct ScatterArgs {
    const float2* xy;
    const uint32_t* tag;
    const uint32_t* cell;
    const uint32_t* cell_start;
    uint32_t* hist;          // counted down to zero
    uint4* out_rec;
    uint32_t* out_tag;
    uint32_t n;
    uint32_t cells;          // search cells
    uint32_t* status;        // bit 3 (value 8): inconsistent binning input
};
void launch_scatter(const ScatterArgs& a, cudaStream_t s);

// Sample-order records {x, y, edge_id} from slot order.
void launch_unsort_records(const uint4* rec, const uint32_t* tag, const uint32_t* edge_ids, uint32_t n,
                           uint32_t* records, cudaStream_t s);
void launch_unsort_u32(const uint32_t* values, const uint32_t* tag, uint32_t n, uint32_t* out, cudaStream_t s);
void launch_records_from_sample_order(const float2* xy, const uint32_t* edge_ids, uint32_t n, uint32_t* records,
                                      cudaStream_t s);
void launch_grid_cells(const uint4* rec, const uint32_t* tag, uint32_t n, const Grid& g, uint32_t* out,
                       cudaStream_t s);
void launch_positions_from_slots(const uint4* rec, const uint32_t* tag, uint32_t n, float2* out, cudaStream_t s);

// ---- distortion (distortion.cu) ----
// Per-edge squared_integral of original vs current (sample order); status bit
// 2 (value 4) flags an invalid curve or interval.
void launch_edge_integrals(const PathRec* paths, uint32_t n_paths, const float2* original, const float2* current,
                           double* out, uint32_t* status, cudaStream_t s);

}  // namespace bt
