// context.h — the per-graph device context (the reference's `Gpu`,
// src/gpu.rs:24-57), shared by the single-graph C ABI (context.cu) and the
// batch engine (batch.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "bt.h"
#include "host.h"
#include "kernels.cuh"

namespace bt {

struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    template <typename T>
    T* as() const {
        return static_cast<T*>(p);
    }
};

struct StageRec {
    const char* name;
    cudaEvent_t start, stop;
};

// Shared helpers of context.cu.
bool make_blur_taps(double sigma, Taps* taps);
double sigma_for_pass(const bt_options& options, uint32_t pass);
void set_thread_error(const char* message);

}  // namespace bt

struct bt_graph {
    bt::HostGraph g;
};

struct bt_ctx {
    bt_options opt{};
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    std::string err;

    bt::Map map{};
    bt::Grid grid{};
    bool has_grid = false, accumulate = false;
    float rsx = 0.f, rsy = 0.f;
    uint64_t grid_bytes_ref = 0, staging_ref = 0;
    size_t cells = 0, texels = 0;

    bt::DevBuf cp, starts, packed, offsets, scan64, edges, paths, totals, status;
    bt::DevBuf edge_ids, segments, tmp_xy, tmp_tag, tmp_cell, neighbors, baseline, current;
    bt::DevBuf sorted_rec[2], sorted_tag[2];
    bt::DevBuf hist, cellsum, cell_start, cell_prefix, table_scratch;
    bt::DevBuf counts, himg, vimg, norm, peak;
    bt::DevBuf records, integrals;
    unsigned long long* h_totals = nullptr;   // pinned
    uint32_t* h_status = nullptr;             // pinned
    size_t device_bytes = 0;

    bool uploaded = false;
    uint32_t samples = 0, n_paths = 0, drawn = 0, capacity = 0;
    uint64_t reserved_bytes = 0;
    uint32_t iterations = 0, density_passes = 0;
    int cur = 0;

    cudaGraphExec_t graphs[2] = {nullptr, nullptr};

    std::vector<bt::StageRec> stage_pool;
    size_t stage_used = 0;
};
