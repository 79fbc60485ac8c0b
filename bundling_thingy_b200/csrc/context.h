// context.h — the per-graph device context (the reference's `Gpu`,
// src/gpu.rs:24-57), shared by the single-graph C ABI (context.cu) and the
// batch engine (batch.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <string>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "bt.h"
#include "host.h"
#include "kernels.cuh"

namespace bt {

// An NVTX range over a public call (named after the reference's `Gpu`
// method it replaces), for timelines of profilers; without one attached the
// NVTX calls do nothing.
struct NvtxRange {
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};


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

struct bt_ctx;

struct bt_batch;

namespace bt {
// Device-memory account shared by many contexts: every allocation a context
// makes is charged against `limit` before it is made, and fails with
// BT_ERR_BUDGET (nothing allocated) when it would not fit.
struct MemAccount {
    std::atomic<uint64_t> used{0};
    uint64_t limit = 0;
};

// 64-byte host words in page-locked memory for the contexts' small status
// and count read-backs, carved from shared slabs (one cudaMallocHost per 256
// contexts instead of two per context). Thread-safe.
void* pinned_slot();
void release_pinned_slot(void* p);

// Once per device: the stream-ordered allocator keeps freed memory for
// reuse instead of returning it to the driver at each synchronisation, and
// reuses it across streams only where the streams are already ordered.
cudaError_t prepare_device_memory(int device);

// bt_create with an optional shared account (nullptr = unaccounted).
bt_status create_context(const bt_options* options, MemAccount* account, bt_ctx** out);

// Gpu::upload in phases (bt_upload = begin, wait, finish, wait, check). A
// phase that fails with BT_ERR_BUDGET before launching work may be retried.
bt_status upload_begin(bt_ctx* c, const float* xy, uint32_t n_points, const uint32_t* starts, uint32_t n_starts);
bt_status upload_finish(bt_ctx* c);
bt_status upload_check(bt_ctx* c, uint32_t* out_samples);
// After the check: re-bins the graph under a search-cell shape chosen for
// its density when the options leave the shape open (asynchronous; a refused
// allocation keeps the current shape).
bt_status upload_adapt(bt_ctx* c);
bt_status upload_wait(bt_ctx* c);

// Unsort the current positions into 12-byte records on the context's stream
// (what bt_read_points copies out), and the copy itself.
bt_status reserve_records(bt_ctx* c);   // the records buffer alone
bt_status prepare_records(bt_ctx* c);
bt_status copy_records(bt_ctx* c, void* dst, size_t bytes);

// Hand an uploaded context to a batch (the batch advances it from then on)
// and take it back without destroying it; detach waits for the batch.
bt_status batch_attach(bt_batch* b, bt_ctx* c, uint32_t* slot);
bt_ctx* batch_detach(bt_batch* b, uint32_t slot);
// The stream the batch's steps run on.
cudaStream_t batch_stream(bt_batch* b);
}  // namespace bt

struct bt_graph {
    bt::HostGraph g;
};

struct bt_ctx {
    bt_options opt{};
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t side = nullptr;              // density passes, overlapped with the binning
    cudaEvent_t fork = nullptr, join = nullptr;
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
    bt::DevBuf hist, cell_start, hist_tiles, slot_prefix, prefix_tiles;
    bt::DevBuf counts, himg, vimg, norm, peak;
    bt::DevBuf records, integrals;
    bt::DevBuf adv_xy;                          // advection mode: next positions, sample order
    bt::DevBuf ckpt_tag;                        // bt_restore_points: tags in sample order
    bt::DevBuf chunk_counter;                   // the mean kernel's work-queue head
    bt::DevBuf probe;                           // sampled search work (rows, boundary samples, probed)
    // bt_render: tile bins, samples, image, and {colored pixels, pairs}.
    bt::DevBuf r_seg_count, r_seg_off, r_scan64, r_pair_tile, r_pair_seg, r_sorted, r_hist, r_hist_off, r_scan32;
    bt::DevBuf r_samples, r_rgba, r_misc;
    uint64_t render_cap = 0;   // (tile, segment) pairs the bin buffers hold
    unsigned long long* h_totals = nullptr;   // pinned
    uint32_t* h_status = nullptr;             // pinned
    size_t device_bytes = 0;
    bt::MemAccount* account = nullptr;          // shared budget (serving), or none

    bool uploaded = false;
    bt::Norm norm_params{};   // normalisation of the graph being uploaded
    uint32_t samples = 0, n_paths = 0, drawn = 0, capacity = 0;
    uint64_t reserved_bytes = 0;
    uint32_t iterations = 0, density_passes = 0;
    uint32_t next_shape_check = 0;              // iteration count of the next search-shape check (0: none)
    int cur = 0;

    cudaGraphExec_t graphs[2] = {nullptr, nullptr};
    bool graph_stale[2] = {false, false};   // a new upload changed sizes or buffers

    std::vector<bt::StageRec> stage_pool;
    size_t stage_used = 0;
};
