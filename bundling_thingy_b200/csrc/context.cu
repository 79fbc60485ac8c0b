// context.cu — bt_ctx (the reference's `Gpu`, src/gpu.rs) and the C ABI.
//
// One context = one device, one CUDA stream and the device buffers of one
// graph. Upload and iterate enqueue the kernels of resample.cu, density.cu and
// grid.cu on that stream; blocking calls wait with a deadline. With a constant
// blur sigma the iteration is captured once per ping-pong parity as a CUDA
// graph and replayed.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "bt.h"
#include "context.h"
#include "host.h"
#include "kernels.cuh"
#include "scan.cuh"

namespace {

using bt::DevBuf;
using bt::StageRec;

thread_local std::string g_thread_error;

constexpr uint64_t kMiB = 1024ull * 1024ull;
constexpr uint64_t kDistortionStagingBytes = 4194300;   // resampling.rs:16
constexpr uint32_t kMaxDimension = 32768;
constexpr double kWaitSeconds = 60.0;                   // gpu.rs:484-490

bt_status fail(bt_ctx* c, bt_status code, const std::string& msg) {
    if (c) c->err = msg;
    g_thread_error = msg;
    return code;
}

// Bounds of the control points (graph.rs:39-40, 79-91) with the result of
// a sequential std::min / std::max fold (the earlier value stays on ties);
// false when a coordinate is not finite. Sixteen interleaved lanes (even: x,
// odd: y) let the compiler vectorise the pass; a bound that comes out as a
// zero is refolded in order, since lanes could pick the other zero sign.
bool point_bounds(const float* xy, uint32_t n, float mn[2], float mx[2]) {
    constexpr int kLanes = 16;
    float lo[kLanes], hi[kLanes];
    uint32_t bad[kLanes];
    for (int j = 0; j < kLanes; ++j) {
        lo[j] = 3.40282347e+38f;
        hi[j] = -3.40282347e+38f;
        bad[j] = 0;
    }
    const size_t m = 2ull * n, body = m / kLanes * kLanes;
    for (size_t k = 0; k < body; k += kLanes)
        for (int j = 0; j < kLanes; ++j) {
            const float v = xy[k + j];
            uint32_t b;
            std::memcpy(&b, &v, 4);
            bad[j] |= static_cast<uint32_t>((b & 0x7F800000u) == 0x7F800000u);
            lo[j] = v < lo[j] ? v : lo[j];
            hi[j] = hi[j] < v ? v : hi[j];
        }
    uint32_t nonfinite = 0;
    for (int j = 0; j < kLanes; ++j) nonfinite |= bad[j];
    for (size_t k = body; k < m; ++k) nonfinite |= static_cast<uint32_t>(!std::isfinite(xy[k]));
    if (nonfinite) return false;
    for (int d = 0; d < 2; ++d) {
        float a = 3.40282347e+38f, b = -3.40282347e+38f;
        for (int j = d; j < kLanes; j += 2) {
            a = lo[j] < a ? lo[j] : a;
            b = b < hi[j] ? hi[j] : b;
        }
        for (size_t k = body + d; k < m; k += 2) {
            a = xy[k] < a ? xy[k] : a;
            b = b < xy[k] ? xy[k] : b;
        }
        if (a == 0.0f || b == 0.0f) {
            a = 3.40282347e+38f;
            b = -3.40282347e+38f;
            for (size_t k = d; k < m; k += 2) {
                a = xy[k] < a ? xy[k] : a;
                b = b < xy[k] ? xy[k] : b;
            }
        }
        mn[d] = a;
        mx[d] = b;
    }
    return true;
}

bt_status cuda_fail(bt_ctx* c, cudaError_t e, const char* what) {
    const bt_status code = (e == cudaErrorMemoryAllocation) ? BT_ERR_BUDGET : BT_ERR_CUDA;
    return fail(c, code, std::string(what) + ": " + cudaGetErrorString(e));
}

#define BT_CUDA(ctx, call)                                        \
    do {                                                          \
        cudaError_t e_ = (call);                                  \
        if (e_ != cudaSuccess) return cuda_fail((ctx), e_, #call);\
    } while (0)

bt_status ensure(bt_ctx* c, DevBuf& b, size_t bytes) {
    if (bytes == 0) bytes = 16;
    if (b.bytes >= bytes) return BT_OK;
    const uint64_t growth = bytes - b.bytes;
    if (c->account) {
        // Charge the growth before allocating; give it back on failure.
        uint64_t used = c->account->used.load();
        do {
            if (used + growth > c->account->limit)
                return fail(c, BT_ERR_BUDGET, "device memory budget of the server is exhausted");
        } while (!c->account->used.compare_exchange_weak(used, used + growth));
    }
    // Stream-ordered: neither the free nor the allocation waits for the rest
    // of the device (a serving worker allocates while batches run).
    if (b.p) {
        cudaFreeAsync(b.p, c->stream);
        c->device_bytes -= b.bytes;
        b.p = nullptr;
        b.bytes = 0;
    }
    cudaError_t e = cudaMallocAsync(&b.p, bytes, c->stream);
    if (e != cudaSuccess) {
        cudaGetLastError();
        if (c->account) c->account->used -= bytes;   // the old buffer is gone too
        return cuda_fail(c, e, "device allocation");
    }
    b.bytes = bytes;
    c->device_bytes += bytes;
    return BT_OK;
}

void release(DevBuf& b, cudaStream_t stream) {
    if (b.p) cudaFreeAsync(b.p, stream);
    b.p = nullptr;
    b.bytes = 0;
}

// Blur taps for sigma (0 = the reference's fixed sigma-6 table, blur.wgsl:41-60).
bool blur_taps(double sigma, bt::Taps* t) {
    static const float kReference[19] = {
        0.0666251319f, 0.0657061792f, 0.0630246744f, 0.0587964725f, 0.0533492351f,
        0.0470805347f, 0.0404101852f, 0.0337346772f, 0.0273904106f, 0.0216300135f,
        0.0166131238f, 0.0124102942f, 0.0090167311f, 0.0063716575f, 0.0043791719f,
        0.0029273040f, 0.0019031803f, 0.0012034507f, 0.0007401384f};
    std::memset(t, 0, sizeof(*t));
    if (sigma == 0.0) {
        for (int k = 0; k < 19; ++k) t->w[k] = kReference[k];
        t->R = 18;
        return true;
    }
    if (!(sigma > 0.0) || !std::isfinite(sigma)) return false;
    int R = static_cast<int>(std::ceil(3.0 * sigma));
    if (R < 1) R = 1;
    if (R > bt::kMaxTaps - 1) return false;
    double total = 0.0;
    for (int k = -R; k <= R; ++k) total += std::exp(-(double)k * k / (2.0 * sigma * sigma));
    for (int k = 0; k <= R; ++k) t->w[k] = static_cast<float>(std::exp(-(double)k * k / (2.0 * sigma * sigma)) / total);
    t->R = R;
    return true;
}

double sigma_for_pass(const bt_options& o, uint32_t pass) {
    double sigma = o.blur_sigma;
    const double shrink = (o.blur_shrink == 0.0f) ? 1.0 : static_cast<double>(o.blur_shrink);
    for (uint32_t i = 0; i < pass && sigma != 0.0; ++i) sigma *= shrink;
    return sigma;
}

// Search-cell shape chosen per graph (the options fix none).
bool adaptive(const bt_ctx* c) { return c->opt.fine_cells == 0 && c->opt.fine_cells_x == 0; }

// Iteration count of a graph's first search-shape check (check_shape).
constexpr uint32_t kFirstShapeCheck = 5;

bool constant_sigma(const bt_options& o) {
    return o.blur_sigma == 0.0f || o.blur_shrink == 0.0f || o.blur_shrink == 1.0f;
}

// GridParameters (neighbor_mean.rs:26-46) byte accounting of the reference.
uint64_t reference_grid_bytes(uint32_t w, uint32_t h, uint32_t r) {
    const uint64_t cells = static_cast<uint64_t>((w + r - 1) / r) * ((h + r - 1) / r);
    return cells * 8 + 8 + cells * 24 + 52;
}

void set_search_shape(bt::Grid& g, uint32_t ky, uint32_t kx) {
    g.ky = ky;
    g.kx = kx;
    g.inv_sx = static_cast<float>(kx) / g.rf;
    g.inv_sy = static_cast<float>(ky) / g.rf;
    g.sx = g.rf / static_cast<float>(kx);
    g.sy = g.rf / static_cast<float>(ky);
    g.fw = g.gw * kx;
    g.fh = g.gh * ky;
}

// Search-cell shape for a graph from the pairs of samples that share a grid
// cell (sum of n (n - 1) over r x r cells). With rho the mean density around a
// sample (samples per texel^2), a search costs about 2r / sy row lookups plus
// rho 4r (sy + sx) exact tests per sample, and the cell table about 8 bytes a
// cell per iteration: the best row height goes as 1 / sqrt(rho), and cells
// about 8 times narrower than high pay for their table. The constant 2.7 is
// fitted on B200 to the first ten iterations after an upload, which hold a
// job's costliest iterations. Per-iteration timings of 4 to 6 shapes on each
// of seven graphs (radius 2 to 16, 0.6M to 12M samples, maps of 256^2 to
// 2048^2) put the fastest rows 1.5 to 2 times lower than 4.5 / sqrt(rho),
// with little change beyond. The earlier constant 4.5 was fitted after the
// eighth iteration. It was 8 to 12% slower on the ten-iteration jobs and
// equal on a 30-iteration job of 5M samples.
void shape_for_rows(const bt_ctx* c, double sy, uint32_t* ky_out, uint32_t* kx_out);

void adaptive_shape(const bt_ctx* c, unsigned long long pairs, uint32_t* ky_out, uint32_t* kx_out) {
    const double r = c->grid.rf, n = static_cast<double>(c->samples);
    const double rho = std::max(static_cast<double>(pairs) / (r * r * n), 1e-4);
    shape_for_rows(c, 2.7 / std::sqrt(rho), ky_out, kx_out);
}

// Search cells of rows about sy texels high (at least 1/4 texel, at most
// min(4, r)), 8 times narrower than high.
void shape_for_rows(const bt_ctx* c, double sy, uint32_t* ky_out, uint32_t* kx_out) {
    const bt::Grid& g = c->grid;
    const double r = g.rf;
    sy = std::min(std::max(sy, 0.25), std::min(4.0, r));
    uint32_t ky = static_cast<uint32_t>(std::min(std::max(std::lround(r / sy), 1L), 4096L));
    uint32_t kx = std::min(8u * ky, 4096u);
    // At most 64 Mi search cells (8 bytes each per iteration) and 8 per sample.
    const uint64_t grid_cells = static_cast<uint64_t>(g.gw) * g.gh;
    const uint64_t cap = std::min<uint64_t>(64ull << 20, std::max<uint64_t>(grid_cells, 8ull * c->samples));
    if (grid_cells * ky * kx > cap) kx = static_cast<uint32_t>(std::max<uint64_t>(ky, cap / (grid_cells * ky)));
    if (grid_cells * ky * kx > cap)
        ky = kx = static_cast<uint32_t>(std::max(1.0, std::floor(std::sqrt(static_cast<double>(cap) / grid_cells))));
    *ky_out = ky;
    *kx_out = kx;
}

// Stage timing (GpuTimings, src/profiling.rs:35-136).
void stage_begin(bt_ctx* c, const char* name, cudaStream_t stream = nullptr) {
    if (!c->opt.timing) return;
    if (c->stage_used == c->stage_pool.size()) {
        StageRec r{name, nullptr, nullptr};
        cudaEventCreate(&r.start);
        cudaEventCreate(&r.stop);
        c->stage_pool.push_back(r);
    }
    StageRec& r = c->stage_pool[c->stage_used++];
    r.name = name;
    cudaEventRecord(r.start, stream ? stream : c->stream);
}

void stage_end(bt_ctx* c, cudaStream_t stream = nullptr) {
    if (!c->opt.timing || c->stage_used == 0) return;
    cudaEventRecord(c->stage_pool[c->stage_used - 1].stop, stream ? stream : c->stream);
}

bt_status wait(bt_ctx* c) {
    cudaError_t e = cudaEventRecord(c->done, c->stream);
    if (e != cudaSuccess) return cuda_fail(c, e, "cudaEventRecord");
    const auto start = std::chrono::steady_clock::now();
    const double limit = c->opt.wait_seconds > 0.0f ? static_cast<double>(c->opt.wait_seconds) : kWaitSeconds;
    int spins = 0;
    while (true) {
        e = cudaEventQuery(c->done);
        if (e == cudaSuccess) break;
        if (e != cudaErrorNotReady) return cuda_fail(c, e, "device execution");
        const double waited = std::chrono::duration<double>(std::chrono::steady_clock::now() - start).count();
        if (waited > limit) {
            char msg[96];
            std::snprintf(msg, sizeof(msg), "device wait exceeded %g s", limit);
            return fail(c, BT_ERR_TIMEOUT, msg);
        }
        if (++spins < 2000) {
            std::this_thread::yield();
        } else {
            std::this_thread::sleep_for(std::chrono::microseconds(50));
        }
    }
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(c, e, "kernel launch");
    return BT_OK;
}

void drop_graphs(bt_ctx* c) {
    for (auto& g : c->graphs) {
        if (g) cudaGraphExecDestroy(g);
        g = nullptr;
    }
}

// Density::encode (density.rs:155-166) for density pass `pass`, on `stream`.
bt_status enqueue_density(bt_ctx* c, uint32_t pass, cudaStream_t stream) {
    bt::Taps taps;
    if (!blur_taps(sigma_for_pass(c->opt, pass), &taps)) return fail(c, BT_ERR_INVALID, "invalid blur sigma");
    // TMA-staged passes (blur_tma.cu) when the map's rows are whole 16-byte
    // units; element-staged ones (density.cu) otherwise. Same results.
    const bool tma = bt::blur_tma_eligible(c->counts.p, c->himg.p, c->map.w, c->map.h, taps.R) &&
                     bt::blur_tma_eligible(c->himg.p, c->vimg.p, c->map.w, c->map.h, taps.R);
    stage_begin(c, "density.blur_horizontal", stream);
    if (tma) {
        BT_CUDA(c, bt::launch_blur_horizontal_tma(c->counts.as<uint32_t>(), c->himg.as<float>(), c->map.w, c->map.h,
                                                   taps, c->status.as<uint32_t>(), stream));
    } else {
        bt::launch_blur_horizontal(c->counts.as<uint32_t>(), c->himg.as<float>(), c->map.w, c->map.h, taps, stream);
    }
    stage_end(c, stream);
    stage_begin(c, "density.blur_vertical_and_maximum", stream);
    if (tma) {
        BT_CUDA(c, bt::launch_blur_vertical_tma(c->himg.as<float>(), c->vimg.as<float>(), c->map.w, c->map.h, taps,
                                                 c->peak.as<uint32_t>(), c->status.as<uint32_t>(), stream));
    } else {
        bt::launch_blur_vertical(c->himg.as<float>(), c->vimg.as<float>(), c->map.w, c->map.h, taps,
                                 c->peak.as<uint32_t>(), stream);
    }
    stage_end(c, stream);
    stage_begin(c, "density.normalize", stream);
    bt::launch_normalize(c->vimg.as<float>(), c->peak.as<uint32_t>(), c->norm.as<float>(), c->texels, stream);
    stage_end(c, stream);
    return BT_OK;
}

// Cell table of the search-cell populations (their tile sums accumulated by
// the mean kernel when tiles_ready), the scatter into slot order `dst`, and
// the slot prefix.
void enqueue_binning(bt_ctx* c, int dst, bool tiles_ready) {
    stage_begin(c, "graph.grid_scan");
    bt::launch_cell_table(c->hist.as<uint32_t>(), c->cells, c->cell_start.as<uint32_t>(),
                          c->hist_tiles.as<uint32_t>(), tiles_ready, c->stream);
    stage_end(c);
    stage_begin(c, "graph.grid_scatter");
    bt::ScatterArgs s{};
    s.xy = c->tmp_xy.as<float2>();
    s.tag = c->tmp_tag.as<uint32_t>();
    s.cell = c->tmp_cell.as<uint32_t>();
    s.cell_start = c->cell_start.as<uint32_t>();
    s.hist = c->hist.as<uint32_t>();
    s.out_rec = c->sorted_rec[dst].as<float2>();
    s.out_tag = c->sorted_tag[dst].as<uint32_t>();
    s.n = c->samples;
    s.cells = static_cast<uint32_t>(c->cells);
    s.status = c->status.as<uint32_t>();
    bt::launch_scatter(s, c->stream);
    stage_end(c);
    stage_begin(c, "graph.slot_prefix");
    bt::launch_slot_prefix(c->sorted_rec[dst].as<float2>(), c->samples, c->slot_prefix.as<bt::LL2>(),
                           c->prefix_tiles.as<bt::LL2>(), c->stream);
    stage_end(c);
}

// One Gpu::iterate (gpu.rs:527-553) starting from slot order `src`.
bt_status enqueue_iteration(bt_ctx* c, int src, uint32_t pass) {
    if (c->accumulate) {
        cudaMemsetAsync(c->counts.p, 0, c->texels * sizeof(uint32_t), c->stream);
        cudaMemsetAsync(c->peak.p, 0, sizeof(uint32_t), c->stream);
    }
    cudaMemsetAsync(c->hist_tiles.p, 0, c->hist_tiles.bytes, c->stream);
    stage_begin(c, "graph.neighbor_mean");
    bt::MeanArgs m{};
    m.rec = c->sorted_rec[src].as<float2>();
    m.tag = c->sorted_tag[src].as<uint32_t>();
    m.cell_start = c->cell_start.as<uint32_t>();
    m.prefix = c->slot_prefix.as<bt::LL2>();
    m.mode = static_cast<int>(c->opt.search_mode);
    m.out_xy = c->tmp_xy.as<float2>();
    m.out_tag = c->tmp_tag.as<uint32_t>();
    m.out_cell = c->tmp_cell.as<uint32_t>();
    m.hist = c->hist.as<uint32_t>();
    m.hist_tiles = c->hist_tiles.as<uint32_t>();
    m.counts = c->accumulate ? c->counts.as<uint32_t>() : nullptr;
    m.neighbors = c->opt.record_neighbors ? c->neighbors.as<uint32_t>() : nullptr;
    m.chunk_counter = c->chunk_counter.as<uint32_t>();
    m.n = c->samples;
    m.g = c->grid;
    bt::launch_neighbor_mean(m, c->stream);
    stage_end(c);
    if (!c->accumulate) {
        enqueue_binning(c, src ^ 1, true);
        return BT_OK;
    }
    // The density passes read only the splat counts and the binning never
    // touches the density images: the two branches run concurrently, joined
    // before the next iteration clears the counts.
    BT_CUDA(c, cudaEventRecord(c->fork, c->stream));
    BT_CUDA(c, cudaStreamWaitEvent(c->side, c->fork, 0));
    bt_status s = enqueue_density(c, pass, c->side);
    BT_CUDA(c, cudaEventRecord(c->join, c->side));
    enqueue_binning(c, src ^ 1, true);
    BT_CUDA(c, cudaStreamWaitEvent(c->stream, c->join, 0));
    return s;
}

// One density-gradient advection step (advect.cu) from the current
// positions (sample order, tmp_xy) into adv_xy, fused with their splat, then
// density pass `pass` of the new positions; the buffers swap afterwards.
bt_status enqueue_advection(bt_ctx* c, uint32_t pass) {
    BT_CUDA(c, cudaMemsetAsync(c->counts.p, 0, c->texels * sizeof(uint32_t), c->stream));
    BT_CUDA(c, cudaMemsetAsync(c->peak.p, 0, sizeof(uint32_t), c->stream));
    stage_begin(c, "graph.advect");
    bt::AdvectArgs a{};
    a.xy = c->tmp_xy.as<float2>();
    a.edge_ids = c->edge_ids.as<uint32_t>();
    a.n = c->samples;
    a.density = c->norm.as<float>();
    a.map = c->map;
    a.step = c->opt.advect_step;
    a.smooth = c->opt.advect_smooth;
    a.sx_inv = 2.0f / static_cast<float>(c->map.w - 1u);
    a.sy_inv = 2.0f / static_cast<float>(c->map.h - 1u);
    a.out = c->adv_xy.as<float2>();
    a.counts = c->counts.as<uint32_t>();
    bt::launch_advect(a, c->stream);
    stage_end(c);
    if (bt_status s = enqueue_density(c, pass, c->stream)) return s;
    std::swap(c->tmp_xy, c->adv_xy);
    return BT_OK;
}

bt_status validate_options(const bt_options* o, bt_ctx* c) {
    if (o->width == 0 || o->height == 0) return fail(c, BT_ERR_INVALID, "density map dimensions must be nonzero");
    if (o->width > kMaxDimension || o->height > kMaxDimension)
        return fail(c, BT_ERR_INVALID, "density map exceeds GPU texture limits");
    if (o->max_graph_memory_bytes == 0) return fail(c, BT_ERR_INVALID, "graph memory budget must be nonzero");
    if (o->color_by > BT_COLOR_BY_EDGE_ID) return fail(c, BT_ERR_INVALID, "unknown color_by");
    if (!(o->blur_sigma >= 0.0f) || !std::isfinite(o->blur_sigma) || !(o->blur_shrink >= 0.0f) ||
        !std::isfinite(o->blur_shrink))
        return fail(c, BT_ERR_INVALID, "invalid blur sigma or shrink");
    bt::Taps t;
    if (!blur_taps(o->blur_sigma, &t)) return fail(c, BT_ERR_INVALID, "blur sigma above 42.6 texels (128 taps)");
    if (!(o->sample_spacing >= 0.0f) || !std::isfinite(o->sample_spacing))
        return fail(c, BT_ERR_INVALID, "invalid sample spacing");
    if (o->sample_spacing > 0.0f && !std::isfinite(0.5 / static_cast<double>(o->sample_spacing)))
        return fail(c, BT_ERR_INVALID, "invalid sample spacing");
    if (o->neighbor_radius > 0 && (o->fine_cells > 4096 || o->fine_cells_x > 4096))
        return fail(c, BT_ERR_INVALID, "fine_cells too large");
    if (o->shape_checks > 1) return fail(c, BT_ERR_INVALID, "shape_checks must be 0 or 1");
    if (o->search_mode > 1) return fail(c, BT_ERR_INVALID, "unknown search_mode");
    if (o->palette > BT_PALETTE_BATLOW) return fail(c, BT_ERR_INVALID, "unknown palette");
    if (!(o->advect_step >= 0.0f) || !std::isfinite(o->advect_step) || !(o->advect_smooth >= 0.0f) ||
        !(o->advect_smooth <= 1.0f))
        return fail(c, BT_ERR_INVALID, "advection step must be finite and >= 0, smoothing in [0, 1]");
    if (o->advect_step > 0.0f && o->neighbor_radius > 0)
        return fail(c, BT_ERR_INVALID, "choose one bundling step: the neighbour mean or density advection");
    if (o->advect_step > 0.0f && (o->width < 2 || o->height < 2))
        return fail(c, BT_ERR_INVALID, "density advection needs a map of at least 2 x 2 texels");
    if (!(o->wait_seconds >= 0.0f) || !std::isfinite(o->wait_seconds))
        return fail(c, BT_ERR_INVALID, "wait_seconds must be finite and >= 0");
    if (o->msaa != 0 && o->msaa != 1 && o->msaa != 2 && o->msaa != 4)
        return fail(c, BT_ERR_INVALID, "msaa must be 1, 2 or 4 samples");
    const uint64_t grid = o->neighbor_radius ? reference_grid_bytes(o->width, o->height, o->neighbor_radius) : 0;
    const uint64_t staging = o->evaluate_distortion ? kDistortionStagingBytes : 0;
    // resampling.rs:85-89
    if (!(grid + staging < o->max_graph_memory_bytes))
        return fail(c, BT_ERR_BUDGET,
                    "neighbor grid and optional distortion staging exceed --max-graph-memory-mib; increase the "
                    "budget or --neighbor-radius");
    return BT_OK;
}

}  // namespace

namespace bt {

namespace {
std::mutex g_pinned_mu;
std::vector<void*> g_pinned_free;
std::mutex g_device_mu;
std::vector<bool> g_device_ready;
}  // namespace

void* pinned_slot() {
    std::lock_guard<std::mutex> lk(g_pinned_mu);
    if (g_pinned_free.empty()) {
        constexpr size_t kSlot = 64, kSlots = 256;
        void* slab = nullptr;
        if (cudaMallocHost(&slab, kSlot * kSlots) != cudaSuccess) return nullptr;   // held until exit
        for (size_t i = 0; i < kSlots; ++i) g_pinned_free.push_back(static_cast<char*>(slab) + i * kSlot);
    }
    void* p = g_pinned_free.back();
    g_pinned_free.pop_back();
    std::memset(p, 0, 64);
    return p;
}

void release_pinned_slot(void* p) {
    if (!p) return;
    std::lock_guard<std::mutex> lk(g_pinned_mu);
    g_pinned_free.push_back(p);
}

cudaError_t prepare_device_memory(int device) {
    std::lock_guard<std::mutex> lk(g_device_mu);
    if (device < 0) return cudaErrorInvalidDevice;
    if (g_device_ready.size() <= static_cast<size_t>(device)) g_device_ready.resize(device + 1, false);
    if (g_device_ready[device]) return cudaSuccess;
    cudaMemPool_t pool = nullptr;
    cudaError_t e = cudaDeviceGetDefaultMemPool(&pool, device);
    if (e != cudaSuccess) return e;
    uint64_t keep = UINT64_MAX;
    e = cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    if (e != cudaSuccess) return e;
    // Memory freed on one context's stream is not handed to another stream by
    // making that stream wait for the first: with hundreds of contexts
    // uploading at once those hidden waits chained every stream together
    // (256 batched uploads took 4.8 s instead of 0.1 s).
    int off = 0;
    if ((e = cudaMemPoolSetAttribute(pool, cudaMemPoolReuseAllowInternalDependencies, &off)) != cudaSuccess) return e;
    if ((e = cudaMemPoolSetAttribute(pool, cudaMemPoolReuseAllowOpportunistic, &off)) != cudaSuccess) return e;
    g_device_ready[device] = true;
    return cudaSuccess;
}

// Shared with the allocation-free density entry point (density_noalloc.cu).
bool make_blur_taps(double sigma, Taps* taps) { return blur_taps(sigma, taps); }
void set_thread_error(const char* message) { g_thread_error = message; }
double sigma_for_pass(const bt_options& options, uint32_t pass) { return ::sigma_for_pass(options, pass); }
}  // namespace bt

extern "C" {

int32_t bt_abi_version(void) { return BT_ABI_VERSION; }

void bt_options_init(bt_options* o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->width = 1600;   // gpu.rs:21 (headless SIZE)
    o->height = 1600;
    o->color_by = BT_COLOR_BY_DENSITY;
    o->max_graph_memory_bytes = 1024 * kMiB;   // main.rs:87-89
    o->use_graphs = 1;
}

const char* bt_last_error(const bt_ctx* ctx) { return ctx ? ctx->err.c_str() : g_thread_error.c_str(); }

bt_status bt_create(const bt_options* options, bt_ctx** out) { return bt::create_context(options, nullptr, out); }

void bt_destroy(bt_ctx* c) {
    if (!c) return;
    if (c->stream) cudaStreamSynchronize(c->stream);
    if (c->side) cudaStreamSynchronize(c->side);
    drop_graphs(c);
    DevBuf* bufs[] = {&c->cp, &c->starts, &c->packed, &c->offsets, &c->scan64, &c->edges, &c->paths, &c->totals,
                      &c->status, &c->edge_ids, &c->segments, &c->tmp_xy, &c->tmp_tag, &c->tmp_cell,
                      &c->neighbors, &c->baseline, &c->current, &c->sorted_rec[0], &c->sorted_rec[1],
                      &c->slot_prefix, &c->prefix_tiles, &c->sorted_tag[0], &c->sorted_tag[1], &c->hist,
                      &c->cell_start, &c->hist_tiles, &c->counts, &c->himg, &c->vimg, &c->norm, &c->peak,
                      &c->records, &c->integrals, &c->r_seg_count, &c->r_seg_off, &c->r_scan64,
                      &c->r_pair_tile, &c->r_pair_seg, &c->r_sorted, &c->r_hist, &c->r_hist_off, &c->r_scan32,
                      &c->r_samples, &c->r_rgba, &c->r_misc, &c->adv_xy, &c->ckpt_tag, &c->chunk_counter,
                      &c->probe};
    for (DevBuf* b : bufs) release(*b, c->stream);
    if (c->stream) cudaStreamSynchronize(c->stream);
    if (c->account) c->account->used -= c->device_bytes;
    for (StageRec& r : c->stage_pool) {
        cudaEventDestroy(r.start);
        cudaEventDestroy(r.stop);
    }
    bt::release_pinned_slot(c->h_totals);
    if (c->done) cudaEventDestroy(c->done);
    if (c->t0) cudaEventDestroy(c->t0);
    if (c->t1) cudaEventDestroy(c->t1);
    if (c->fork) cudaEventDestroy(c->fork);
    if (c->join) cudaEventDestroy(c->join);
    if (c->side) cudaStreamDestroy(c->side);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
}

}  // extern "C"

bt_status bt::create_context(const bt_options* options, bt::MemAccount* account, bt_ctx** out) {
    if (!options || !out) return fail(nullptr, BT_ERR_INVALID, "null argument");
    *out = nullptr;
    if (bt_status s = validate_options(options, nullptr)) return s;
    auto* c = new bt_ctx();
    c->opt = *options;
    c->device = options->device;
    c->account = account;
    auto bail = [&](bt_status s) {
        std::string msg = c->err;
        bt_destroy(c);
        g_thread_error = msg;
        return s;
    };
    cudaError_t e = cudaSetDevice(c->device);
    if (e != cudaSuccess) return bail(cuda_fail(c, e, "cudaSetDevice"));
    if ((e = bt::prepare_density_kernels()) != cudaSuccess) return bail(cuda_fail(c, e, "kernel attributes"));
    if ((e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaStreamCreateWithFlags(&c->side, cudaStreamNonBlocking)) != cudaSuccess)
        return bail(cuda_fail(c, e, "cudaStreamCreate"));
    if ((e = cudaEventCreateWithFlags(&c->fork, cudaEventDisableTiming)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&c->join, cudaEventDisableTiming)) != cudaSuccess)
        return bail(cuda_fail(c, e, "cudaEventCreate"));
    if ((e = cudaEventCreateWithFlags(&c->done, cudaEventDisableTiming)) != cudaSuccess)
        return bail(cuda_fail(c, e, "cudaEventCreate"));
    if ((e = bt::prepare_device_memory(c->device)) != cudaSuccess) return bail(cuda_fail(c, e, "memory pool"));
    // One pinned 64-byte slot: four u64 totals, then four u32 status words.
    c->h_totals = static_cast<unsigned long long*>(bt::pinned_slot());
    if (!c->h_totals) return bail(fail(c, BT_ERR_BUDGET, "pinned host memory"));
    c->h_status = reinterpret_cast<uint32_t*>(c->h_totals + 4);

    const uint32_t W = options->width, H = options->height;
    c->map = bt::Map{W, H, static_cast<float>(W - 1u), static_cast<float>(H - 1u)};
    c->texels = static_cast<size_t>(W) * H;
    c->accumulate = options->color_by == BT_COLOR_BY_DENSITY || options->advect_step > 0.0f;
    if (options->sample_spacing > 0.0f) {
        c->rsx = c->rsy = static_cast<float>(0.5 / static_cast<double>(options->sample_spacing));
    } else {
        // texel_scale of resampling.wgsl:87
        c->rsx = static_cast<float>(W - 1u) * 0.5f;
        c->rsy = static_cast<float>(H - 1u) * 0.5f;
    }
    c->staging_ref = options->evaluate_distortion ? kDistortionStagingBytes : 0;
    const uint32_t r = options->neighbor_radius;
    c->has_grid = r > 0;
    if (c->has_grid) {
        bt::Grid& g = c->grid;
        g.map = c->map;
        g.radius = r;
        g.rf = static_cast<float>(r);
        g.gw = (W + r - 1) / r;
        g.gh = (H + r - 1) / r;
        // Square search cells of about two texels until the first upload picks
        // a shape for the graph's density (unless the options fix one).
        const uint32_t ky = options->fine_cells ? options->fine_cells : std::max(1u, r / 2u);
        set_search_shape(g, ky, options->fine_cells_x ? options->fine_cells_x : ky);
        g.tsx = static_cast<float>(W - 1u) * 0.5f;
        g.tsy = static_cast<float>(H - 1u) * 0.5f;
        g.r2 = g.rf * g.rf;
        g.reachx = g.rf + static_cast<float>(W) * 0.00000024f;
        g.reachy = g.rf + static_cast<float>(H) * 0.00000024f;
        g.margin = 1e-3f + 1e-6f * static_cast<float>(std::max(W, H)) + 1e-5f * g.rf;
        c->cells = static_cast<size_t>(g.fw) * g.fh;
        if (c->cells > 0x7FFFFFFFull) return bail(fail(c, BT_ERR_INVALID, "neighbour search grid too large"));
        c->grid_bytes_ref = reference_grid_bytes(W, H, r);
        if (bt_status s = ensure(c, c->hist, c->cells * 4)) return bail(s);
        if (bt_status s = ensure(c, c->cell_start, (c->cells + 1) * 4)) return bail(s);
        if (bt_status s = ensure(c, c->hist_tiles, 4 * (bt::scan_tiles<uint32_t>(c->cells) + 1))) return bail(s);
        if ((e = cudaMemsetAsync(c->hist.p, 0, c->cells * 4, c->stream)) != cudaSuccess)
            return bail(cuda_fail(c, e, "cudaMemset"));
    }
    if (bt_status s = ensure(c, c->counts, c->texels * 4)) return bail(s);
    if (bt_status s = ensure(c, c->himg, c->texels * 4)) return bail(s);
    if (bt_status s = ensure(c, c->vimg, c->texels * 4)) return bail(s);
    if (bt_status s = ensure(c, c->norm, c->texels * 4)) return bail(s);
    if (bt_status s = ensure(c, c->peak, 16)) return bail(s);
    if (bt_status s = ensure(c, c->totals, 32)) return bail(s);
    if (bt_status s = ensure(c, c->status, 16)) return bail(s);
    if (bt_status s = ensure(c, c->chunk_counter, 16)) return bail(s);
    if (bt_status s = ensure(c, c->probe, 32)) return bail(s);
    cudaMemsetAsync(c->counts.p, 0, c->texels * 4, c->stream);
    cudaMemsetAsync(c->vimg.p, 0, c->texels * 4, c->stream);
    cudaMemsetAsync(c->norm.p, 0, c->texels * 4, c->stream);
    cudaMemsetAsync(c->peak.p, 0, 16, c->stream);
    // Everything that uses these buffers is ordered after the clears on this
    // stream (or by events from it), so creation does not wait for them.
    if ((e = cudaGetLastError()) != cudaSuccess) return bail(cuda_fail(c, e, "cudaMemsetAsync"));
    *out = c;
    return BT_OK;
}

// Gpu::upload in three phases so that a batch can run many uploads
// concurrently with two host waits in total: begin (validate, copy in, count
// kernel, totals read back asynchronously) — wait — finish (offsets, emit,
// density, first binning, status read back) — wait — check.
bt_status bt::upload_begin(bt_ctx* c, const float* xy, uint32_t n_points, const uint32_t* starts,
                           uint32_t n_starts) {
    if (!c) return fail(nullptr, BT_ERR_INVALID, "null context");
    if (!xy || !starts) return fail(c, BT_ERR_INVALID, "null argument");
    cudaSetDevice(c->device);
    // The previous graph is released first (gpu.rs:494-497).
    c->uploaded = false;
    c->samples = 0;
    c->iterations = 0;
    c->next_shape_check = kFirstShapeCheck;
    c->density_passes = 0;
    // The iteration graphs are refreshed at the next iteration (an update of
    // the executable graph when the new capture has the same shape).
    c->graph_stale[0] = c->graph_stale[1] = true;
    c->stage_used = 0;
    // Input contract of Graph (graph.rs:7-12, 60-77).
    if (n_starts < 2 || starts[0] != 0 || starts[n_starts - 1] != n_points)
        return fail(c, BT_ERR_INVALID, "path starts must begin at 0 and end at the point count");
    for (uint32_t e = 0; e + 1 < n_starts; ++e)
        if (starts[e + 1] < starts[e] || starts[e + 1] - starts[e] < 2)
            return fail(c, BT_ERR_INVALID, "every edge needs at least two control points");
    float mn[2], mx[2];
    if (!point_bounds(xy, n_points, mn, mx)) return fail(c, BT_ERR_INVALID, "non-finite TRL coordinate");
    float nm[5];
    std::string err;
    if (!bt::normalization(mn, mx, nm, &err)) return fail(c, BT_ERR_INVALID, err);
    const uint32_t E = n_starts - 1;

    // Allocation::new (resampling.rs:321-397): capacity from the budget.
    const uint64_t sample_bytes = 16 + (c->has_grid ? 32 : 0);
    const uint64_t fixed = 8ull * n_points + 4ull * n_starts + 12ull * E + 16ull * E + 8ull * E + 32 + 16 + 48 + 16 +
                           c->grid_bytes_ref + c->staging_ref;
    if (fixed > c->opt.max_graph_memory_bytes)
        return fail(c, BT_ERR_BUDGET,
                    "control points, path metadata, and neighbor grid exceed --max-graph-memory-mib");
    const uint64_t available = c->opt.max_graph_memory_bytes - fixed;
    const uint64_t binding_limit = 0xFFFFFFFFull;   // u32-indexed storage bindings
    uint64_t capacity = std::min(available / sample_bytes, binding_limit / 12);
    capacity = std::min<uint64_t>(capacity, 0x7FFFFFFFull);   // sample index + movable bit in 32 bits
    if (capacity < 3) return fail(c, BT_ERR_BUDGET, "graph memory budget has no room for resampled geometry");
    c->capacity = static_cast<uint32_t>(capacity);
    c->reserved_bytes = fixed + capacity * sample_bytes;

    if (bt_status s = ensure(c, c->cp, 8ull * n_points)) return s;
    if (bt_status s = ensure(c, c->starts, 4ull * n_starts)) return s;
    if (bt_status s = ensure(c, c->packed, 8ull * E)) return s;
    if (bt_status s = ensure(c, c->offsets, 8ull * (E + 1))) return s;
    if (bt_status s = ensure(c, c->scan64, 8ull * bt::scan_scratch_elems<unsigned long long>(E))) return s;
    if (bt_status s = ensure(c, c->edges, 16ull * E)) return s;
    if (bt_status s = ensure(c, c->paths, 12ull * E)) return s;
    BT_CUDA(c, cudaMemcpyAsync(c->cp.p, xy, 8ull * n_points, cudaMemcpyHostToDevice, c->stream));
    BT_CUDA(c, cudaMemcpyAsync(c->starts.p, starts, 4ull * n_starts, cudaMemcpyHostToDevice, c->stream));
    BT_CUDA(c, cudaMemsetAsync(c->totals.p, 0, 32, c->stream));
    BT_CUDA(c, cudaMemsetAsync(c->status.p, 0, 16, c->stream));

    c->norm_params = bt::Norm{nm[0], nm[1], nm[2], nm[3], nm[4]};
    c->n_paths = E;
    stage_begin(c, "graph.count");
    bt::ResampleCountArgs ca{};
    ca.cp = c->cp.as<float2>();
    ca.starts = c->starts.as<uint32_t>();
    ca.paths = E;
    ca.norm = c->norm_params;
    ca.sx = c->rsx;
    ca.sy = c->rsy;
    ca.capacity = c->capacity;
    ca.packed = c->packed.as<unsigned long long>();
    ca.edges = c->edges.as<float4>();
    ca.totals = c->totals.as<unsigned long long>();
    bt::launch_resample_count(ca, c->stream);
    stage_end(c);
    BT_CUDA(c, cudaMemcpyAsync(c->h_totals, c->totals.p, 16, cudaMemcpyDeviceToHost, c->stream));
    return BT_OK;
}

bt_status bt::upload_finish(bt_ctx* c) {
    cudaSetDevice(c->device);
    const uint32_t E = c->n_paths;
    const bt::Norm norm = c->norm_params;
    const unsigned long long total = c->h_totals[0], drawn = c->h_totals[1];
    // count_paths overflow 1 (resampling.wgsl:151-156), PendingGraph::finish (resampling.rs:294-308).
    if (total > c->capacity)
        return fail(c, BT_ERR_CAPACITY,
                    "GPU resampling exceeds the " + std::to_string(c->capacity) +
                        "-sample buffer capacity; increase --max-graph-memory-mib or reduce the graph or render "
                        "dimensions");
    if (total - drawn == 0) return fail(c, BT_ERR_INVALID, "resampled graph has no drawable edges");
    const uint32_t N = static_cast<uint32_t>(total);
    const uint32_t segs = static_cast<uint32_t>(total - drawn);

    // Every allocation before the first launch, so that a phase refused by a
    // memory budget launched nothing and can be retried.
    if (bt_status s = ensure(c, c->edge_ids, 4ull * N)) return s;
    if (bt_status s = ensure(c, c->segments, 4ull * segs)) return s;
    if (bt_status s = ensure(c, c->tmp_xy, 8ull * N)) return s;
    if (bt_status s = ensure(c, c->tmp_tag, 4ull * N)) return s;
    if (bt_status s = ensure(c, c->tmp_cell, 4ull * N)) return s;
    if (c->has_grid) {
        for (int b = 0; b < 2; ++b) {
            if (bt_status s = ensure(c, c->sorted_rec[b], 8ull * N)) return s;
            if (bt_status s = ensure(c, c->sorted_tag[b], 4ull * N)) return s;
        }
        if (bt_status s = ensure(c, c->slot_prefix, 16ull * (N + 1ull))) return s;
        if (bt_status s = ensure(c, c->prefix_tiles, 16 * (bt::scan_tiles<bt::LL2>(N) + 1))) return s;
        if (c->opt.record_neighbors)
            if (bt_status s = ensure(c, c->neighbors, 4ull * N)) return s;
    }
    if (c->opt.evaluate_distortion)
        if (bt_status s = ensure(c, c->baseline, 8ull * N)) return s;

    stage_begin(c, "graph.emit");
    bt::exclusive_scan<unsigned long long>(c->packed.as<unsigned long long>(), c->offsets.as<unsigned long long>(), E,
                                           c->scan64.as<unsigned long long>(), c->stream);
    bt::launch_paths_from_scan(c->packed.as<unsigned long long>(), c->offsets.as<unsigned long long>(), E,
                               c->paths.as<bt::PathRec>(), c->stream);
    if (c->has_grid) {
        BT_CUDA(c, cudaMemsetAsync(c->hist.p, 0, c->cells * 4, c->stream));
    }
    if (c->accumulate) {
        BT_CUDA(c, cudaMemsetAsync(c->counts.p, 0, c->texels * 4, c->stream));
        BT_CUDA(c, cudaMemsetAsync(c->peak.p, 0, 4, c->stream));
    }
    bt::ResampleEmitArgs ea{};
    ea.cp = c->cp.as<float2>();
    ea.starts = c->starts.as<uint32_t>();
    ea.paths = c->paths.as<bt::PathRec>();
    ea.n_paths = E;
    ea.norm = norm;
    ea.sx = c->rsx;
    ea.sy = c->rsy;
    ea.map = c->map;
    ea.xy = c->tmp_xy.as<float2>();
    ea.edge_ids = c->edge_ids.as<uint32_t>();
    ea.segments = c->segments.as<uint32_t>();
    ea.counts = c->accumulate ? c->counts.as<uint32_t>() : nullptr;
    ea.grid_host = c->has_grid ? &c->grid : nullptr;
    ea.tag = c->tmp_tag.as<uint32_t>();
    ea.cell = c->tmp_cell.as<uint32_t>();
    ea.hist = c->hist.as<uint32_t>();
    ea.status = c->status.as<uint32_t>();
    bt::launch_resample_emit(ea, c->stream);
    stage_end(c);
    if (c->has_grid && adaptive(c))
        bt::launch_grid_pairs(c->hist.as<uint32_t>(), c->grid, c->cell_start.as<uint32_t>(),   // scratch until binned
                              c->totals.as<unsigned long long>() + 2, c->stream);
    c->samples = N;
    c->n_paths = E;
    c->drawn = static_cast<uint32_t>(drawn);
    if (c->opt.evaluate_distortion)
        BT_CUDA(c, cudaMemcpyAsync(c->baseline.p, c->tmp_xy.p, 8ull * N, cudaMemcpyDeviceToDevice, c->stream));
    if (c->accumulate) {
        if (bt_status s = enqueue_density(c, 0, c->stream)) return s;
        c->density_passes = 1;
    }
    if (c->has_grid) {
        enqueue_binning(c, 0, false);
        c->cur = 0;
    }
    BT_CUDA(c, cudaMemcpyAsync(c->h_status, c->status.p, 4, cudaMemcpyDeviceToHost, c->stream));
    BT_CUDA(c, cudaMemcpyAsync(c->h_totals + 2, c->totals.as<unsigned long long>() + 2, 8, cudaMemcpyDeviceToHost,
                               c->stream));
    return BT_OK;
}

bt_status reshape(bt_ctx* c, uint32_t ky, uint32_t kx);

bt_status bt::upload_adapt(bt_ctx* c) {
    if (!c->has_grid || !adaptive(c) || c->samples == 0) return BT_OK;
    uint32_t ky = 0, kx = 0;
    adaptive_shape(c, c->h_totals[2], &ky, &kx);
    return reshape(c, ky, kx);
}

// Re-bins the current slot order under ky x kx search cells per grid cell
// (every shape gives the same neighbour sets and sums). When an allocation is
// refused (a memory budget), the graph keeps the shape it has.
bt_status reshape(bt_ctx* c, uint32_t ky, uint32_t kx) {
    if (ky == c->grid.ky && kx == c->grid.kx) return BT_OK;
    bt::Grid g = c->grid;
    set_search_shape(g, ky, kx);
    const size_t cells = static_cast<size_t>(g.fw) * g.fh;
    // Allocations first: when one is refused (a memory budget), the graph
    // keeps the shape it was binned with. New memory is not zero and the
    // scatter left the rest of the populations zero, so all of it is cleared.
    const bool room = ensure(c, c->hist, cells * 4) == BT_OK && ensure(c, c->cell_start, (cells + 1) * 4) == BT_OK &&
                      ensure(c, c->hist_tiles, 4 * (bt::scan_tiles<uint32_t>(cells) + 1)) == BT_OK;
    BT_CUDA(c, cudaMemsetAsync(c->hist.p, 0, c->hist.bytes, c->stream));
    if (!room) return BT_OK;
    c->grid = g;
    c->cells = cells;
    c->graph_stale[0] = c->graph_stale[1] = true;   // their kernels hold the old grid
    stage_begin(c, "graph.rebin");
    bt::launch_rebin(c->sorted_rec[c->cur].as<float2>(), c->sorted_tag[c->cur].as<uint32_t>(), c->samples, c->grid,
                     c->tmp_xy.as<float2>(), c->tmp_tag.as<uint32_t>(), c->tmp_cell.as<uint32_t>(),
                     c->hist.as<uint32_t>(), c->stream);
    stage_end(c);
    enqueue_binning(c, c->cur ^ 1, false);
    c->cur ^= 1;
    return BT_OK;
}

// Search-shape checks during a job (options.shape_checks). Early iterations
// test many boundary samples per search row and favour low rows; as a graph
// bundles its boundary bands empty, the rows dominate and tall rows win (on
// the large workload 2-texel rows are fastest at first and 4-texel rows from
// about the tenth iteration). After 5, 10, 20, 40, ... iterations of an
// upload, the synchronous calls (bt_iterate, bt_iterate_timed) count the
// search rows and the boundary samples of every 64th slot under the current
// shape, predict the best row height and re-bin when the prediction saves
// more than 8%. The cost model: per sample, kRowCost exact tests' worth per
// search row (about 2R / sy + 1 rows) plus the boundary samples, whose count
// scales with the band's width sy + sx. kRowCost is fitted to per-iteration
// times of five shapes on the large workload at iterations 1 and 30. Fitted
// over eight graphs the ratio ranges from 4.8 to 8.4, and no single value
// chooses well on all of them (30-iteration jobs 4% faster on the large
// workload, up to 15% slower on small-radius graphs), so the checks are an
// option, off by default.
constexpr uint32_t kProbeStride = 64;
constexpr double kRowCost = 10.0;
constexpr double kReshapeGain = 0.92;

bt_status check_shape(bt_ctx* c) {
    c->next_shape_check = std::max(c->iterations, kFirstShapeCheck) * 2u;
    if (!c->has_grid || !adaptive(c) || c->samples == 0) return BT_OK;
    bt::launch_search_probe(c->sorted_rec[c->cur].as<float2>(), c->sorted_tag[c->cur].as<uint32_t>(),
                            c->cell_start.as<uint32_t>(), c->samples, c->grid, kProbeStride,
                            c->probe.as<unsigned long long>(), c->stream);
    BT_CUDA(c, cudaMemcpyAsync(c->h_totals + 5, c->probe.p, 24, cudaMemcpyDeviceToHost, c->stream));
    // A check is only an optimisation: past the wait deadline the call goes
    // on without it (the queued work completes, as for any expired wait).
    if (bt_status s = wait(c)) return s == BT_ERR_TIMEOUT ? BT_OK : s;
    const double probed = static_cast<double>(c->h_totals[7]);
    if (probed < 64.0) return BT_OK;
    const double tests = static_cast<double>(c->h_totals[6]) / probed;
    const bt::Grid& g = c->grid;
    const double R = static_cast<double>(g.rf) + g.margin;
    const double band = static_cast<double>(g.sy) + g.sx;
    auto cost = [&](double sy, double sx) { return kRowCost * (2.0 * R / sy + 1.0) + tests * (sy + sx) / band; };
    // Minimum of kRowCost 2R / sy + tests (sy + sy / 8) / band.
    const double sy_best = std::sqrt(2.0 * R * kRowCost * band / (1.125 * std::max(tests, 1e-3)));
    uint32_t ky = 0, kx = 0;
    shape_for_rows(c, sy_best, &ky, &kx);
    if (ky == g.ky && kx == g.kx) return BT_OK;
    const double sy_new = static_cast<double>(g.rf) / ky, sx_new = static_cast<double>(g.rf) / kx;
    if (cost(sy_new, sx_new) > kReshapeGain * cost(g.sy, g.sx)) return BT_OK;
    return reshape(c, ky, kx);
}

bt_status bt::upload_check(bt_ctx* c, uint32_t* out_samples) {
    if (c->h_status[0] & 2u) return fail(c, BT_ERR_MISMATCH, "GPU resampling count and write passes disagree");
    if (c->h_status[0] & 8u) return fail(c, BT_ERR_CUDA, "inconsistent neighbour-grid binning");
    if (c->h_status[0] & 16u) return fail(c, BT_ERR_TIMEOUT, "a density tile copy did not complete on the device");
    c->uploaded = true;
    *out_samples = c->samples;
    return BT_OK;
}

bt_status bt::upload_wait(bt_ctx* c) { return wait(c); }

bt_status bt::copy_records(bt_ctx* c, void* dst, size_t bytes) {
    if (!dst || bytes != 12ull * c->samples) return fail(c, BT_ERR_INVALID, "point buffer must hold 12 bytes per sample");
    cudaSetDevice(c->device);
    BT_CUDA(c, cudaMemcpyAsync(dst, c->records.p, bytes, cudaMemcpyDeviceToHost, c->stream));
    return wait(c);
}

bt_status bt::reserve_records(bt_ctx* c) { return ensure(c, c->records, 12ull * c->samples); }

bt_status bt::prepare_records(bt_ctx* c) {
    cudaSetDevice(c->device);
    if (bt_status s = ensure(c, c->records, 12ull * c->samples)) return s;
    if (c->has_grid) {
        bt::launch_unsort_records(c->sorted_rec[c->cur].as<float2>(), c->sorted_tag[c->cur].as<uint32_t>(),
                                  c->edge_ids.as<uint32_t>(), c->samples, c->records.as<uint32_t>(), c->stream);
    } else {
        bt::launch_records_from_sample_order(c->tmp_xy.as<float2>(), c->edge_ids.as<uint32_t>(), c->samples,
                                             c->records.as<uint32_t>(), c->stream);
    }
    return BT_OK;
}

extern "C" {

bt_status bt_upload(bt_ctx* c, const float* xy, uint32_t n_points, const uint32_t* starts, uint32_t n_starts,
                    uint32_t* out_samples) {
    bt::NvtxRange range("Gpu::upload");
    if (!out_samples) return fail(c, BT_ERR_INVALID, "null argument");
    if (bt_status s = bt::upload_begin(c, xy, n_points, starts, n_starts)) return s;
    if (bt_status s = wait(c)) return s;
    if (bt_status s = bt::upload_finish(c)) return s;
    if (bt_status s = wait(c)) return s;
    if (bt_status s = bt::upload_check(c, out_samples)) return s;
    return bt::upload_adapt(c);
}

bt_status bt_upload_graph(bt_ctx* c, const bt_graph* g, uint32_t* out_samples) {
    if (!g) return fail(c, BT_ERR_INVALID, "null graph");
    return bt_upload(c, g->g.xy.data(), static_cast<uint32_t>(g->g.xy.size() / 2), g->g.starts.data(),
                     static_cast<uint32_t>(g->g.starts.size()), out_samples);
}

// Enqueues n iterations; reset_stages starts a new set of stage records
// (timing mode), otherwise they add to the current one.
bt_status iterate_enqueue(bt_ctx* c, uint32_t n, bool reset_stages) {
    bt::NvtxRange range("Gpu::iterate");
    if (!c) return fail(nullptr, BT_ERR_INVALID, "null context");
    const bool advect = c->opt.advect_step > 0.0f;
    if (!c->has_grid && !advect) return fail(c, BT_ERR_NOT_CONFIGURED, "neighbor radius is not configured");
    if (!c->uploaded) return fail(c, BT_ERR_NO_GRAPH, "no uploaded graph");
    cudaSetDevice(c->device);
    if (reset_stages) c->stage_used = 0;
    if (advect) {
        if (bt_status s = ensure(c, c->adv_xy, 8ull * c->samples)) return s;
        for (uint32_t i = 0; i < n; ++i) {
            if (bt_status s = enqueue_advection(c, c->density_passes)) return s;
            c->iterations++;
            c->density_passes++;
        }
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return cuda_fail(c, e, "kernel launch");
        return BT_OK;
    }
    const bool use_graphs = c->opt.use_graphs && !c->opt.timing && constant_sigma(c->opt);
    for (uint32_t i = 0; i < n; ++i) {
        const uint32_t pass = c->density_passes;
        if (use_graphs) {
            cudaGraphExec_t& exec = c->graphs[c->cur];
            if (!exec || c->graph_stale[c->cur]) {
                cudaGraph_t graph = nullptr;
                BT_CUDA(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
                bt_status s = enqueue_iteration(c, c->cur, pass);
                cudaError_t e = cudaStreamEndCapture(c->stream, &graph);
                if (s) {
                    if (graph) cudaGraphDestroy(graph);
                    return s;
                }
                if (e != cudaSuccess) return cuda_fail(c, e, "cudaStreamEndCapture");
                if (exec) {
                    // Same kernels and dependencies as before: update the
                    // parameters in place; otherwise build it anew.
                    cudaGraphExecUpdateResultInfo info{};
                    if (cudaGraphExecUpdate(exec, graph, &info) != cudaSuccess) {
                        cudaGetLastError();
                        cudaGraphExecDestroy(exec);
                        exec = nullptr;
                    }
                }
                if (!exec) e = cudaGraphInstantiate(&exec, graph, 0);
                cudaGraphDestroy(graph);
                if (e != cudaSuccess) {
                    exec = nullptr;
                    return cuda_fail(c, e, "cudaGraphInstantiate");
                }
                c->graph_stale[c->cur] = false;
            }
            BT_CUDA(c, cudaGraphLaunch(exec, c->stream));
        } else {
            if (bt_status s = enqueue_iteration(c, c->cur, pass)) return s;
        }
        c->cur ^= 1;
        c->iterations++;
        if (c->accumulate) c->density_passes++;
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(c, e, "kernel launch");
    return BT_OK;
}

bt_status bt_set_wait_seconds(bt_ctx* c, float seconds) {
    if (!c) return fail(nullptr, BT_ERR_INVALID, "null context");
    if (!(seconds >= 0.0f) || !std::isfinite(seconds))
        return fail(c, BT_ERR_INVALID, "wait_seconds must be finite and >= 0");
    c->opt.wait_seconds = seconds;
    return BT_OK;
}

bt_status bt_synchronize(bt_ctx* c) {
    if (!c) return fail(nullptr, BT_ERR_INVALID, "null context");
    cudaSetDevice(c->device);
    return wait(c);
}

namespace {
// Device status word after iterations (scatter guard, bit 3).
bt_status check_iteration_status(bt_ctx* c) {
    BT_CUDA(c, cudaMemcpyAsync(c->h_status, c->status.p, 4, cudaMemcpyDeviceToHost, c->stream));
    if (bt_status s = wait(c)) return s;
    if (c->h_status[0] & 8u) {
        c->uploaded = false;
        return fail(c, BT_ERR_CUDA, "inconsistent neighbour-grid binning");
    }
    if (c->h_status[0] & 16u) return fail(c, BT_ERR_TIMEOUT, "a density tile copy did not complete on the device");
    return BT_OK;
}
}  // namespace

bt_status bt_iterate_async(bt_ctx* c, uint32_t n) { return iterate_enqueue(c, n, true); }

// bt_iterate_async in pieces, with the search-shape checks that fall due
// on the way (check_shape).
bt_status iterate_checked(bt_ctx* c, uint32_t n) {
    if (!c || !c->uploaded) return iterate_enqueue(c, n, true);   // its errors
    const bool checks = c->opt.shape_checks && c->has_grid && c->opt.advect_step <= 0.0f && adaptive(c);
    c->stage_used = 0;
    if (n == 0) return iterate_enqueue(c, 0, false);
    while (n > 0) {
        if (checks && c->next_shape_check && c->iterations >= c->next_shape_check)
            if (bt_status s = check_shape(c)) return s;
        uint32_t chunk = n;
        if (checks && c->next_shape_check > c->iterations) chunk = std::min(n, c->next_shape_check - c->iterations);
        if (bt_status s = iterate_enqueue(c, chunk, false)) return s;
        n -= chunk;
    }
    return BT_OK;
}

bt_status bt_iterate(bt_ctx* c, uint32_t n) {
    if (bt_status s = iterate_checked(c, n)) return s;
    return check_iteration_status(c);
}

bt_status bt_iterate_timed(bt_ctx* c, uint32_t n, float* device_ms) {
    if (!c || !device_ms) return fail(c, BT_ERR_INVALID, "null argument");
    cudaSetDevice(c->device);
    if (!c->t0) {
        BT_CUDA(c, cudaEventCreate(&c->t0));
        BT_CUDA(c, cudaEventCreate(&c->t1));
    }
    BT_CUDA(c, cudaEventRecord(c->t0, c->stream));
    if (bt_status s = iterate_checked(c, n)) return s;
    BT_CUDA(c, cudaEventRecord(c->t1, c->stream));
    if (bt_status s = wait(c)) return s;
    BT_CUDA(c, cudaEventElapsedTime(device_ms, c->t0, c->t1));
    return check_iteration_status(c);
}

bt_status bt_autotune(const bt_options* options, const float* xy, uint32_t n_points, const uint32_t* starts,
                      uint32_t n_starts, uint32_t iterations, bt_options* tuned, float* best_ms) {
    if (!options || !tuned) return fail(nullptr, BT_ERR_INVALID, "null argument");
    *tuned = *options;
    if (best_ms) *best_ms = 0.0f;
    const uint32_t r = options->neighbor_radius;
    if (r == 0 || iterations == 0) return BT_OK;
    // Search rows of 4, 2, 1 and 1/2 texels; cells as wide as high, or 2 or 4
    // times narrower (a thinner boundary band for dense neighbourhoods).
    std::vector<std::pair<uint32_t, uint32_t>> candidates;   // (ky, kx)
    const uint64_t grid_cells = static_cast<uint64_t>((options->width + r - 1) / r) * ((options->height + r - 1) / r);
    for (uint32_t ky : {std::max(1u, r / 4u), std::max(1u, r / 2u), r, 2u * r})
        for (uint32_t m : {1u, 2u, 4u}) {
            const uint32_t kx = ky * m;
            const std::pair<uint32_t, uint32_t> kk{ky, kx};
            if (kx > 4096 || grid_cells * ky * kx > (32ull << 20)) continue;
            if (std::find(candidates.begin(), candidates.end(), kk) == candidates.end()) candidates.push_back(kk);
        }
    float best = -1.0f;
    for (const auto& kk : candidates) {
        bt_options o = *options;
        o.fine_cells = kk.first;
        o.fine_cells_x = kk.second;
        o.timing = 0;
        o.use_graphs = 1;
        bt_ctx* c = nullptr;
        if (bt_status s = bt_create(&o, &c)) return s;
        uint32_t samples = 0;
        float ms = 0.0f;
        bt_status s = bt_upload(c, xy, n_points, starts, n_starts, &samples);
        if (!s) s = bt_iterate(c, 1);
        if (!s) s = bt_iterate_timed(c, iterations, &ms);
        if (s) {
            std::string msg = c->err;
            bt_destroy(c);
            return fail(nullptr, s, msg);
        }
        bt_destroy(c);
        if (best < 0.0f || ms < best) {
            best = ms;
            *tuned = o;
        }
    }
    tuned->timing = options->timing;
    tuned->use_graphs = options->use_graphs;
    if (best_ms) *best_ms = best;
    return BT_OK;
}

bt_status bt_get_info(bt_ctx* c, bt_info* info) {
    if (!c || !info) return fail(c, BT_ERR_INVALID, "null argument");
    std::memset(info, 0, sizeof(*info));
    info->samples = c->samples;
    info->paths = c->n_paths;
    info->drawn_paths = c->drawn;
    info->segments = c->samples ? c->samples - c->drawn : 0;
    info->capacity = c->capacity;
    info->iterations = c->iterations;
    info->grid_width = c->has_grid ? c->grid.gw : 0;
    info->grid_height = c->has_grid ? c->grid.gh : 0;
    info->fine_cells = c->has_grid ? c->grid.ky : 0;
    info->fine_cells_x = c->has_grid ? c->grid.kx : 0;
    info->density_passes = c->density_passes;
    info->device_bytes = c->device_bytes;
    info->reserved_bytes = c->reserved_bytes;
    return BT_OK;
}

namespace {

bt_status need_graph(bt_ctx* c) {
    if (!c) return fail(nullptr, BT_ERR_INVALID, "null context");
    if (!c->uploaded) return fail(c, BT_ERR_NO_GRAPH, "no uploaded graph");
    cudaSetDevice(c->device);
    return BT_OK;
}

bt_status copy_out(bt_ctx* c, void* dst, const void* src, size_t bytes) {
    BT_CUDA(c, cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, c->stream));
    return wait(c);
}

// Current positions in sample order (device buffer).
bt_status current_positions(bt_ctx* c, const float2** out) {
    if (!c->has_grid) {
        *out = c->tmp_xy.as<float2>();
        return BT_OK;
    }
    if (bt_status s = ensure(c, c->current, 8ull * c->samples)) return s;
    bt::launch_positions_from_slots(c->sorted_rec[c->cur].as<float2>(), c->sorted_tag[c->cur].as<uint32_t>(),
                                    c->samples, c->current.as<float2>(), c->stream);
    *out = c->current.as<float2>();
    return BT_OK;
}

}  // namespace

bt_status bt_read_points(bt_ctx* c, void* dst, size_t bytes) {
    if (bt_status s = need_graph(c)) return s;
    if (!dst || bytes != 12ull * c->samples) return fail(c, BT_ERR_INVALID, "point buffer must hold 12 bytes per sample");
    if (bt_status s = bt::prepare_records(c)) return s;
    return copy_out(c, dst, c->records.p, bytes);
}

bt_status bt_restore_points(bt_ctx* c, const void* records, size_t bytes, uint32_t iterations) {
    bt::NvtxRange range("restore_points");
    if (bt_status s = need_graph(c)) return s;
    if (!records || bytes != 12ull * c->samples)
        return fail(c, BT_ERR_INVALID, "checkpoint must hold 12 bytes per sample of the uploaded graph");
    const bool advect = c->opt.advect_step > 0.0f;
    cudaSetDevice(c->device);
    c->stage_used = 0;
    if (bt_status s = ensure(c, c->records, bytes)) return s;
    if (bt_status s = ensure(c, c->current, 8ull * c->samples)) return s;
    if (c->has_grid)
        if (bt_status s = ensure(c, c->ckpt_tag, 4ull * c->samples)) return s;
    BT_CUDA(c, cudaMemsetAsync(c->status.p, 0, 4, c->stream));
    BT_CUDA(c, cudaMemcpyAsync(c->records.p, records, bytes, cudaMemcpyHostToDevice, c->stream));
    // Sample-order positions (and tags) into scratch, checked against the
    // graph before anything the context iterates on changes.
    float2* xy = c->current.as<float2>();
    bt::launch_restore_records(c->records.as<uint32_t>(), c->edge_ids.as<uint32_t>(),
                               c->has_grid ? c->sorted_tag[c->cur].as<uint32_t>() : nullptr, c->samples, xy,
                               c->has_grid ? c->ckpt_tag.as<uint32_t>() : nullptr, c->status.as<uint32_t>(),
                               c->stream);
    BT_CUDA(c, cudaMemcpyAsync(c->h_status, c->status.p, 4, cudaMemcpyDeviceToHost, c->stream));
    if (bt_status s = wait(c)) return s;
    if (c->h_status[0] & 32u)
        return fail(c, BT_ERR_INVALID, "checkpoint does not match the uploaded graph (edge ids or positions)");
    if (advect) {
        // The advection mode iterates on sample-order positions.
        BT_CUDA(c, cudaMemcpyAsync(c->tmp_xy.p, xy, 8ull * c->samples, cudaMemcpyDeviceToDevice, c->stream));
        xy = c->tmp_xy.as<float2>();
    }
    if (c->has_grid) {
        // Bin the positions for the next iteration, as after a mean step.
        BT_CUDA(c, cudaMemsetAsync(c->hist.p, 0, c->cells * 4, c->stream));
        bt::launch_rebin(xy, c->ckpt_tag.as<uint32_t>(), c->samples, c->grid, c->tmp_xy.as<float2>(),
                         c->tmp_tag.as<uint32_t>(), c->tmp_cell.as<uint32_t>(), c->hist.as<uint32_t>(), c->stream);
        enqueue_binning(c, c->cur ^ 1, false);
        c->cur ^= 1;
    }
    // The density of the restored positions: pass `iterations`, as the
    // iteration that produced them ran it.
    const bool density = advect || c->accumulate;
    if (density) {
        BT_CUDA(c, cudaMemsetAsync(c->counts.p, 0, c->texels * sizeof(uint32_t), c->stream));
        BT_CUDA(c, cudaMemsetAsync(c->peak.p, 0, sizeof(uint32_t), c->stream));
        bt::launch_splat_positions(xy, c->samples, c->map, c->counts.as<uint32_t>(), c->stream);
        if (bt_status s = enqueue_density(c, iterations, c->stream)) return s;
    }
    c->iterations = iterations;
    c->next_shape_check = std::max(iterations, kFirstShapeCheck);
    c->density_passes = density ? iterations + 1 : 0;
    BT_CUDA(c, cudaGetLastError());
    return check_iteration_status(c);
}

bt_status bt_read_paths(bt_ctx* c, void* dst, size_t bytes) {
    if (bt_status s = need_graph(c)) return s;
    if (!dst || bytes != 12ull * c->n_paths) return fail(c, BT_ERR_INVALID, "path buffer must hold 12 bytes per edge");
    return copy_out(c, dst, c->paths.p, bytes);
}

bt_status bt_read_segments(bt_ctx* c, uint32_t* dst, size_t count) {
    if (bt_status s = need_graph(c)) return s;
    if (!dst || count != c->samples - c->drawn) return fail(c, BT_ERR_INVALID, "segment buffer size");
    return copy_out(c, dst, c->segments.p, 4 * count);
}

bt_status bt_read_edges(bt_ctx* c, float* dst, size_t count) {
    if (bt_status s = need_graph(c)) return s;
    if (!dst || count != 4ull * c->n_paths) return fail(c, BT_ERR_INVALID, "edge buffer must hold 4 floats per edge");
    return copy_out(c, dst, c->edges.p, 4 * count);
}

bt_status bt_read_density(bt_ctx* c, float* dst, size_t count) {
    if (bt_status s = need_graph(c)) return s;
    if (!c->accumulate) return fail(c, BT_ERR_NOT_CONFIGURED, "density is only accumulated when coloring by density");
    if (!dst || count != c->texels) return fail(c, BT_ERR_INVALID, "density buffer must hold width*height floats");
    return copy_out(c, dst, c->norm.p, 4 * count);
}

bt_status bt_read_density_raw(bt_ctx* c, float* dst, size_t count, float* peak) {
    if (bt_status s = need_graph(c)) return s;
    if (!c->accumulate) return fail(c, BT_ERR_NOT_CONFIGURED, "density is only accumulated when coloring by density");
    if (!dst || !peak || count != c->texels) return fail(c, BT_ERR_INVALID, "density buffer size");
    BT_CUDA(c, cudaMemcpyAsync(dst, c->vimg.p, 4 * count, cudaMemcpyDeviceToHost, c->stream));
    uint32_t bits = 0;
    BT_CUDA(c, cudaMemcpyAsync(c->h_status + 1, c->peak.p, 4, cudaMemcpyDeviceToHost, c->stream));
    if (bt_status s = wait(c)) return s;
    bits = c->h_status[1];
    std::memcpy(peak, &bits, 4);
    return BT_OK;
}

bt_status bt_read_counts(bt_ctx* c, uint32_t* dst, size_t count) {
    if (bt_status s = need_graph(c)) return s;
    if (!c->accumulate) return fail(c, BT_ERR_NOT_CONFIGURED, "density is only accumulated when coloring by density");
    if (!dst || count != c->texels) return fail(c, BT_ERR_INVALID, "count buffer must hold width*height values");
    return copy_out(c, dst, c->counts.p, 4 * count);
}

bt_status bt_read_cells(bt_ctx* c, uint32_t* dst, size_t count) {
    if (bt_status s = need_graph(c)) return s;
    if (!c->has_grid) return fail(c, BT_ERR_NOT_CONFIGURED, "neighbor radius is not configured");
    if (!dst || count != c->samples) return fail(c, BT_ERR_INVALID, "cell buffer must hold one id per sample");
    if (bt_status s = ensure(c, c->records, 12ull * c->samples)) return s;
    bt::launch_grid_cells(c->sorted_rec[c->cur].as<float2>(), c->sorted_tag[c->cur].as<uint32_t>(), c->samples,
                          c->grid, c->records.as<uint32_t>(), c->stream);
    return copy_out(c, dst, c->records.p, 4 * count);
}

bt_status bt_search_stats(bt_ctx* c, uint32_t stride, uint64_t* rows, uint64_t* boundary, uint64_t* probed) {
    if (bt_status s = need_graph(c)) return s;
    if (!c->has_grid) return fail(c, BT_ERR_NOT_CONFIGURED, "neighbor radius is not configured");
    if (!rows || !boundary || !probed || stride == 0) return fail(c, BT_ERR_INVALID, "null argument or zero stride");
    if (c->opt.advect_step > 0.0f) return fail(c, BT_ERR_NOT_CONFIGURED, "the advection mode has no neighbour search");
    bt::launch_search_probe(c->sorted_rec[c->cur].as<float2>(), c->sorted_tag[c->cur].as<uint32_t>(),
                            c->cell_start.as<uint32_t>(), c->samples, c->grid, stride,
                            c->probe.as<unsigned long long>(), c->stream);
    BT_CUDA(c, cudaMemcpyAsync(c->h_totals + 5, c->probe.p, 24, cudaMemcpyDeviceToHost, c->stream));
    if (bt_status s = wait(c)) return s;
    *rows = c->h_totals[5];
    *boundary = c->h_totals[6];
    *probed = c->h_totals[7];
    return BT_OK;
}

bt_status bt_read_binning(bt_ctx* c, uint32_t* slot_samples, size_t count, uint32_t* cell_starts, size_t cell_count) {
    if (bt_status s = need_graph(c)) return s;
    if (!c->has_grid) return fail(c, BT_ERR_NOT_CONFIGURED, "neighbor radius is not configured");
    if (!slot_samples || !cell_starts || count != c->samples || cell_count != c->cells + 1)
        return fail(c, BT_ERR_INVALID, "binning buffer sizes");
    BT_CUDA(c, cudaMemcpyAsync(slot_samples, c->sorted_tag[c->cur].p, 4 * count, cudaMemcpyDeviceToHost, c->stream));
    BT_CUDA(c, cudaMemcpyAsync(cell_starts, c->cell_start.p, 4 * cell_count, cudaMemcpyDeviceToHost, c->stream));
    if (bt_status s = wait(c)) return s;
    for (size_t i = 0; i < count; ++i) slot_samples[i] &= ~bt::kMovableBit;
    return BT_OK;
}

bt_status bt_read_neighbors(bt_ctx* c, uint32_t* dst, size_t count) {
    if (bt_status s = need_graph(c)) return s;
    if (!c->has_grid) return fail(c, BT_ERR_NOT_CONFIGURED, "neighbor radius is not configured");
    if (!c->opt.record_neighbors) return fail(c, BT_ERR_NOT_CONFIGURED, "neighbour counts are not recorded");
    if (!dst || count != c->samples) return fail(c, BT_ERR_INVALID, "neighbor buffer size");
    if (c->iterations == 0) {
        std::memset(dst, 0, 4 * count);
        return BT_OK;
    }
    if (bt_status s = ensure(c, c->records, 12ull * c->samples)) return s;
    bt::launch_unsort_u32(c->neighbors.as<uint32_t>(), c->tmp_tag.as<uint32_t>(), c->samples,
                          c->records.as<uint32_t>(), c->stream);
    return copy_out(c, dst, c->records.p, 4 * count);
}

bt_status bt_distortion(bt_ctx* c, uint32_t size, double* distortion, double* rms_px) {
    bt::NvtxRange range("distortion");
    if (bt_status s = need_graph(c)) return s;
    if (!c->opt.evaluate_distortion) return fail(c, BT_ERR_NOT_CONFIGURED, "distortion staging disabled");
    if (!distortion || !rms_px || size == 0) return fail(c, BT_ERR_INVALID, "distortion viewport must be nonzero");
    const float2* current = nullptr;
    if (bt_status s = current_positions(c, &current)) return s;
    if (bt_status s = ensure(c, c->integrals, 8ull * c->n_paths)) return s;
    BT_CUDA(c, cudaMemsetAsync(c->status.p, 0, 4, c->stream));
    bt::launch_edge_integrals(c->paths.as<bt::PathRec>(), c->n_paths, c->baseline.as<float2>(), current,
                              c->integrals.as<double>(), c->status.as<uint32_t>(), c->stream);
    std::vector<double> per_edge(c->n_paths);
    std::vector<bt::PathRec> paths(c->n_paths);
    BT_CUDA(c, cudaMemcpyAsync(per_edge.data(), c->integrals.p, 8ull * c->n_paths, cudaMemcpyDeviceToHost, c->stream));
    BT_CUDA(c, cudaMemcpyAsync(paths.data(), c->paths.p, 12ull * c->n_paths, cudaMemcpyDeviceToHost, c->stream));
    BT_CUDA(c, cudaMemcpyAsync(c->h_status, c->status.p, 4, cudaMemcpyDeviceToHost, c->stream));
    if (bt_status s = wait(c)) return s;
    if (c->h_status[0] & 4u) return fail(c, BT_ERR_INVALID, "nonfinite distortion curve or interval");
    // Aggregate::add over edges in point-offset order (geometry.rs:64).
    std::vector<uint32_t> order;
    for (uint32_t e = 0; e < c->n_paths; ++e)
        if (paths[e].count) order.push_back(e);
    std::sort(order.begin(), order.end(),
              [&](uint32_t a, uint32_t b) { return paths[a].point_offset < paths[b].point_offset; });
    bt::KahanSum sum;
    for (uint32_t e : order) {
        bt::KahanSum trial = sum;
        trial.add(per_edge[e]);
        if (!std::isfinite(trial.value)) return fail(c, BT_ERR_INVALID, "nonfinite distortion aggregate");
        sum = trial;
    }
    if (order.empty()) return fail(c, BT_ERR_INVALID, "distortion requires at least one edge");
    // Aggregate::finish (distortion.rs:201-215)
    const double rms = std::sqrt(sum.value / static_cast<double>(order.size()));
    *distortion = rms / (2.0 * 1.4142135623730951);
    *rms_px = rms * (static_cast<double>(size) / 2.0);
    if (!std::isfinite(*distortion) || !std::isfinite(*rms_px))
        return fail(c, BT_ERR_INVALID, "nonfinite distortion measurement");
    return BT_OK;
}

namespace {

// One frame of bt_render with bin buffers for c->render_cap pairs; *pairs
// receives the pairs the frame needed (above the capacity: nothing valid was
// drawn and the caller grows the buffers and renders again).
bt_status render_frame(bt_ctx* c, const float2* xy, bool timed, uint8_t* rgba, uint64_t* colored, uint64_t* pairs) {
    const uint32_t w = c->opt.width, h = c->opt.height;
    const size_t pixels = static_cast<size_t>(w) * h;
    bt::RenderArgs a{};
    a.w = w;
    a.h = h;
    a.ns = c->opt.msaa ? static_cast<int>(c->opt.msaa) : 4;
    a.palette = static_cast<int>(c->opt.palette);
    a.color_by_edge = c->opt.color_by == BT_COLOR_BY_EDGE_ID;
    a.tile_shift = bt::render_tile_shift(w, h);
    a.tiles_x = (w + (1u << a.tile_shift) - 1) >> a.tile_shift;
    a.tiles_y = (h + (1u << a.tile_shift) - 1) >> a.tile_shift;
    const size_t tiles = static_cast<size_t>(a.tiles_x) * a.tiles_y;
    if (bt_status s = ensure(c, c->r_samples, 4 * pixels * a.ns)) return s;
    if (bt_status s = ensure(c, c->r_rgba, 4 * pixels)) return s;
    if (bt_status s = ensure(c, c->r_misc, 16)) return s;
    a.samples = c->r_samples.as<uint32_t>();
    a.rgba = c->r_rgba.as<uint32_t>();
    a.colored = c->r_misc.as<unsigned long long>();
    BT_CUDA(c, cudaMemsetAsync(c->r_misc.p, 0, 16, c->stream));
    const uint32_t n = c->uploaded ? c->samples - c->drawn : 0;
    if (c->uploaded) {
        a.xy = xy;
        a.edge_ids = c->edge_ids.as<uint32_t>();
        a.segments = c->segments.as<uint32_t>();
        a.n_segments = n;
        a.paths = c->paths.as<bt::PathRec>();
        a.n_paths = c->n_paths;
        a.density = c->accumulate ? c->norm.as<float>() : nullptr;
        a.edge_den = static_cast<float>((c->n_paths > 2u ? c->n_paths : 2u) - 1u);   // arrayLength(&edges)
    }
    if (n > 0) {
        const uint64_t cap = c->render_cap;
        a.bin_blocks = static_cast<uint32_t>((cap + bt::kBinItems - 1) / bt::kBinItems);
        const size_t hist_n = tiles * a.bin_blocks;
        if (bt_status s = ensure(c, c->r_seg_count, 8ull * (n + 1))) return s;
        if (bt_status s = ensure(c, c->r_seg_off, 8ull * (n + 1))) return s;
        if (bt_status s = ensure(c, c->r_scan64, 8ull * bt::scan_scratch_elems<unsigned long long>(n))) return s;
        if (bt_status s = ensure(c, c->r_pair_tile, 4 * cap)) return s;
        if (bt_status s = ensure(c, c->r_pair_seg, 4 * cap)) return s;
        if (bt_status s = ensure(c, c->r_sorted, 4 * cap)) return s;
        if (bt_status s = ensure(c, c->r_hist, 4 * hist_n)) return s;
        if (bt_status s = ensure(c, c->r_hist_off, 4 * (hist_n + 1))) return s;
        if (bt_status s = ensure(c, c->r_scan32, 4 * bt::scan_scratch_elems<uint32_t>(hist_n))) return s;
        a.seg_count = c->r_seg_count.as<unsigned long long>();
        a.seg_off = c->r_seg_off.as<unsigned long long>();
        a.pair_tile = c->r_pair_tile.as<uint32_t>();
        a.pair_seg = c->r_pair_seg.as<uint32_t>();
        a.sorted = c->r_sorted.as<uint32_t>();
        a.hist = c->r_hist.as<uint32_t>();
        a.hist_off = c->r_hist_off.as<uint32_t>();
        a.pair_capacity = cap;
        a.pair_total = a.seg_off + n;
        bt::launch_render_bin_count(a, c->stream);
        bt::exclusive_scan<unsigned long long>(a.seg_count, a.seg_off, n, c->r_scan64.as<unsigned long long>(),
                                               c->stream);
        bt::launch_render_bin_emit(a, c->stream);
        BT_CUDA(c, bt::launch_render_bin_sort(a, c->r_scan32.as<uint32_t>(), c->stream));
        BT_CUDA(c, cudaMemcpyAsync(c->r_misc.as<unsigned long long>() + 1, a.pair_total, 8, cudaMemcpyDeviceToDevice,
                                   c->stream));
    }
    bt::launch_render_raster(a, c->stream);
    if (n > 0 && c->opt.endpoint_dots) bt::launch_render_endpoints(a, c->stream);
    bt::launch_render_resolve(a, c->stream);
    if (timed) BT_CUDA(c, cudaEventRecord(c->t1, c->stream));
    BT_CUDA(c, cudaMemcpyAsync(c->h_totals + 2, c->r_misc.p, 16, cudaMemcpyDeviceToHost, c->stream));
    if (bt_status s = wait(c)) return s;
    *pairs = c->h_totals[3];
    *colored = c->h_totals[2];
    if (*pairs > c->render_cap) return BT_OK;
    if (rgba) BT_CUDA(c, cudaMemcpyAsync(rgba, c->r_rgba.p, 4 * pixels, cudaMemcpyDeviceToHost, c->stream));
    return rgba ? wait(c) : BT_OK;
}

}  // namespace

bt_status bt_render(bt_ctx* c, uint8_t* rgba, size_t rgba_bytes, uint64_t* colored_pixels, float* device_ms) {
    bt::NvtxRange range("Gpu::render");
    if (!c) return fail(nullptr, BT_ERR_INVALID, "null context");
    cudaSetDevice(c->device);
    const size_t pixels = static_cast<size_t>(c->opt.width) * c->opt.height;
    if (rgba && rgba_bytes != 4 * pixels) return fail(c, BT_ERR_INVALID, "RGBA buffer must hold 4*width*height bytes");
    if (bt::render_tile_shift(c->opt.width, c->opt.height) < 0)
        return fail(c, BT_ERR_INVALID, "frame too large to render (at most 16384 tiles of 64x64 pixels)");
    if (device_ms && !c->t0) {
        BT_CUDA(c, cudaEventCreate(&c->t0));
        BT_CUDA(c, cudaEventCreate(&c->t1));
    }
    if (device_ms) BT_CUDA(c, cudaEventRecord(c->t0, c->stream));
    const float2* xy = nullptr;
    if (c->uploaded) {
        if (bt_status s = current_positions(c, &xy)) return s;
        if (c->render_cap == 0) c->render_cap = 4ull * (c->samples - c->drawn) + 4096;
    }
    uint64_t colored = 0, pairs = 0;
    if (bt_status s = render_frame(c, xy, device_ms != nullptr, rgba, &colored, &pairs)) return s;
    if (pairs > c->render_cap) {
        // The bins were too small: grow them and draw again.
        if (pairs >= (1ull << 32)) return fail(c, BT_ERR_INVALID, "frame needs more than 2^32 tile bins");
        c->render_cap = pairs + pairs / 4;
        if (device_ms) BT_CUDA(c, cudaEventRecord(c->t0, c->stream));
        if (bt_status s = render_frame(c, xy, device_ms != nullptr, rgba, &colored, &pairs)) return s;
        if (pairs > c->render_cap) return fail(c, BT_ERR_CUDA, "render bin count changed between passes");
    } else if (pairs + pairs / 2 < c->render_cap) {
        // Fewer bins than provided for: size the next frame's histogram for
        // this one's (the buffers keep their size).
        c->render_cap = pairs + pairs / 4 + 4096;
    }
    if (device_ms) BT_CUDA(c, cudaEventElapsedTime(device_ms, c->t0, c->t1));
    if (colored_pixels) *colored_pixels = colored;
    return BT_OK;
}

bt_status bt_stage_times(bt_ctx* c, const char** names, float* ms, uint32_t capacity, uint32_t* count) {
    if (!c || !count) return fail(c, BT_ERR_INVALID, "null argument");
    if (bt_status s = wait(c)) return s;
    // Sum per stage name over the last call, in first-seen order.
    std::vector<const char*> seen;
    std::vector<float> totals;
    for (size_t i = 0; i < c->stage_used; ++i) {
        const StageRec& r = c->stage_pool[i];
        float t = 0.f;
        cudaEventElapsedTime(&t, r.start, r.stop);
        size_t k = 0;
        while (k < seen.size() && std::strcmp(seen[k], r.name) != 0) ++k;
        if (k == seen.size()) {
            seen.push_back(r.name);
            totals.push_back(0.f);
        }
        totals[k] += t;
    }
    *count = static_cast<uint32_t>(seen.size());
    for (size_t k = 0; k < seen.size() && k < capacity; ++k) {
        if (names) names[k] = seen[k];
        if (ms) ms[k] = totals[k];
    }
    return BT_OK;
}

// ---- graph loader ----

bt_status bt_graph_parse(const char* text, size_t len, bt_graph** out) {
    if (!out || (!text && len)) return fail(nullptr, BT_ERR_INVALID, "null argument");
    *out = nullptr;
    auto* g = new bt_graph();
    std::string err;
    if (!bt::parse_trl(text ? text : "", len, &g->g, &err)) {
        delete g;
        return fail(nullptr, BT_ERR_INVALID, err);
    }
    *out = g;
    return BT_OK;
}

bt_status bt_graph_load(const char* path, bt_graph** out) {
    if (!out || !path) return fail(nullptr, BT_ERR_INVALID, "null argument");
    *out = nullptr;
    auto* g = new bt_graph();
    std::string err;
    if (!bt::load_trl(path, &g->g, &err)) {
        delete g;
        return fail(nullptr, BT_ERR_INVALID, err);
    }
    *out = g;
    return BT_OK;
}

void bt_graph_free(bt_graph* g) { delete g; }
uint32_t bt_graph_point_count(const bt_graph* g) { return g ? static_cast<uint32_t>(g->g.xy.size() / 2) : 0; }
uint32_t bt_graph_start_count(const bt_graph* g) { return g ? static_cast<uint32_t>(g->g.starts.size()) : 0; }
const float* bt_graph_points(const bt_graph* g) { return g ? g->g.xy.data() : nullptr; }
const uint32_t* bt_graph_starts(const bt_graph* g) { return g ? g->g.starts.data() : nullptr; }

bt_status bt_graph_normalization(const bt_graph* g, float out[5]) {
    if (!g || !out) return fail(nullptr, BT_ERR_INVALID, "null argument");
    std::string err;
    if (!bt::normalization(g->g.min, g->g.max, out, &err)) return fail(nullptr, BT_ERR_INVALID, err);
    return BT_OK;
}

// ---- geometry readers ----

bt_status bt_layout_check(const uint32_t* paths, uint32_t n_paths, uint32_t samples) {
    if (!paths && n_paths) return fail(nullptr, BT_ERR_INVALID, "null argument");
    std::string err;
    if (!bt::layout_check(paths, n_paths, samples, &err)) return fail(nullptr, BT_ERR_INVALID, err);
    return BT_OK;
}

bt_status bt_decode_points(const uint32_t* paths, uint32_t n_paths, uint32_t samples, const void* records,
                           size_t bytes, float* xy) {
    if ((!paths && n_paths) || (!records && bytes) || !xy) return fail(nullptr, BT_ERR_INVALID, "null argument");
    std::string err;
    if (!bt::decode_points(paths, n_paths, samples, records, bytes, xy, &err)) return fail(nullptr, BT_ERR_INVALID, err);
    return BT_OK;
}

bt_status bt_squared_integral(const float* original, size_t n_original, const float* current, size_t n_current,
                              double* out) {
    if (!original || !current || !out) return fail(nullptr, BT_ERR_INVALID, "null argument");
    std::string err;
    if (!bt::squared_integral_host(original, n_original, current, n_current, out, &err))
        return fail(nullptr, BT_ERR_INVALID, err);
    return BT_OK;
}

}  // extern "C"
