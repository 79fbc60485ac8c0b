// batch.cu — many independent graphs bundled by one set of persistent launches.
//
// Each graph lives in a slot: a per-graph context (context.h) that uploads it
// with the single-graph path (resample, splat, blur, first binning) and owns
// its buffers. An iteration of the whole batch is one CUDA graph of persistent
// kernels, one per stage, sized to the GPU (148 SMs x resident CTAs) and fed
// by a work queue over graph x tile: every CTA takes the next (slot, tile)
// pair from an atomic counter, stages that slot's descriptor in shared memory
// and runs the same per-sample / per-tile bodies as the single-graph kernels
// (grid_dev.cuh, density_dev.cuh), so every slot's results equal a
// single-graph run bit for bit. Each slot's ping-pong parity, density pass
// and iteration count live on the device, so one captured graph serves every
// iteration; the descriptors, tile lists and graph are rebuilt only when the
// set of slots changes. Slots do not share atomics or sums: a graph's result
// does not depend on the other graphs in the batch.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "bt.h"
#include "context.h"
#include "density_dev.cuh"
#include "grid_dev.cuh"
#include "scan.cuh"

namespace bt {
namespace {

constexpr uint32_t kSampleTile = 128;     // samples per mean / scatter tile (and their CTA size)
constexpr uint32_t kTexelTile = 4096;     // texels per clear / normalise tile
constexpr uint32_t kTapsHorizon = 64;     // density passes of taps kept ahead

struct BlurSlot {
    uint32_t* counts;
    float* himg;
    float* vimg;
    float* norm;
    uint32_t* peak;
    uint32_t w, h;
    unsigned long long texels;
    const Taps* taps;        // taps of density pass i at taps[min(i, taps_count - 1)]
    uint32_t taps_count;
    uint32_t accumulate;
};

struct SlotDesc {
    MeanArgs mean[2];        // by slot parity
    ScatterArgs scatter[2];  // by slot parity (writes the other order)
    const uint32_t* hist;
    uint32_t* cell_start;
    uint32_t* cell_sums;     // population sums per cell tile (from the mean), scanned in place (cell_tiles + 1)
    const float2* rec[2];    // records by slot parity
    LL2* slot_prefix;
    LL2* prefix_sums;        // position sums per prefix tile, scanned in place (prefix_tiles + 1)
    uint32_t cells;
    uint32_t cell_tiles;
    uint32_t samples;
    uint32_t prefix_tiles;
    BlurSlot blur;
};

struct SlotState {
    uint32_t cur, pass, iterations, pad;
};

enum List : int { kSamples, kMeanTiles, kCells, kSlots, kPrefix, kBlurH, kBlurV, kTexels, kLists };
enum Counter : int {
    cClear, cMean, cCellScan, cCellApply, cScatter, cPrefixReduce, cPrefixScan, cPrefixApply, cBlurH, cBlurV,
    cNormalize, cCounters
};

struct BatchArgs {
    const SlotDesc* slots;
    SlotState* state;
    const uint2* lists[kLists];
    const uint32_t* counts;  // entries per list
    uint32_t* counters;      // work-queue heads, zeroed each iteration
    uint32_t* status;        // batch status word (bit 3: inconsistent binning)
};

// Next tile of a work queue for the whole CTA; false when the queue is empty.
__device__ __forceinline__ bool next_tile(uint32_t* counter, uint32_t n, uint32_t* shared_t, uint32_t* t) {
    __syncthreads();
    if (threadIdx.x == 0) *shared_t = atomicAdd(counter, 1u);
    __syncthreads();
    *t = *shared_t;
    return *t < n;
}

template <typename T>
__device__ __forceinline__ void stage_words(T* dst, const T* src) {
    static_assert(sizeof(T) % 4 == 0, "word copy");
    constexpr int words = static_cast<int>(sizeof(T) / 4);
    for (int i = threadIdx.x; i < words; i += blockDim.x)
        reinterpret_cast<uint32_t*>(dst)[i] = reinterpret_cast<const uint32_t*>(src)[i];
}

__global__ void __launch_bounds__(256) batch_clear_kernel(BatchArgs b) {
    __shared__ uint32_t t_sh;
    uint32_t t;
    while (next_tile(&b.counters[cClear], b.counts[kTexels], &t_sh, &t)) {
        const uint2 tile = b.lists[kTexels][t];
        const BlurSlot& s = b.slots[tile.x].blur;
        const unsigned long long start = static_cast<unsigned long long>(tile.y) * kTexelTile;
        const unsigned long long end = min(start + kTexelTile, s.texels);
        for (unsigned long long i = start + threadIdx.x; i < end; i += blockDim.x) s.counts[i] = 0u;
        if (tile.y == 0 && threadIdx.x == 0) *s.peak = 0u;
    }
}

// One mean tile per CTA of kThreads samples, at most 1,280 resident threads
// per SM (forty warps; the staged descriptor costs registers that more
// would spill). A CTA waits for its slowest warp before it takes the next
// tile, so smaller tiles waste less on graphs whose samples have very
// different neighbourhoods, and larger ones stage fewer descriptors: the
// tile size and the resident CTAs per SM are chosen per batch
// (bt_batch_set_shape, bt_batch_autotune).
template <int kThreads>
__global__ void __launch_bounds__(kThreads, 1280 / kThreads) batch_mean_kernel(BatchArgs b) {
    __shared__ uint32_t t_sh;
    __shared__ MeanArgs args;
    uint32_t t;
    while (next_tile(&b.counters[cMean], b.counts[kMeanTiles], &t_sh, &t)) {
        const uint2 tile = b.lists[kMeanTiles][t];
        stage_words(&args, &b.slots[tile.x].mean[b.state[tile.x].cur]);
        __syncthreads();
        dev::mean_sample(args, tile.y + threadIdx.x);
    }
}

template <int kThreads>
const void* mean_kernel_fn() {
    return reinterpret_cast<const void*>(batch_mean_kernel<kThreads>);
}

const void* mean_kernel_for(uint32_t tile) {
    return tile == 64 ? mean_kernel_fn<64>() : tile == 256 ? mean_kernel_fn<256>() : mean_kernel_fn<128>();
}

// Cell table: the population sums per tile (accumulated by the mean kernel)
// scanned per slot, then each tile scanned from its offset into cell_start.
// Each tile clears its sum after use, ready for the next iteration.
__global__ void __launch_bounds__(kScanBlock) batch_cell_scan_kernel(BatchArgs b) {
    __shared__ uint32_t t_sh;
    __shared__ ScanShared<uint32_t> sh;
    uint32_t t;
    while (next_tile(&b.counters[cCellScan], b.counts[kSlots], &t_sh, &t)) {
        const SlotDesc& d = b.slots[b.lists[kSlots][t].x];
        block_scan_all<uint32_t>(ArraySource<uint32_t>{d.cell_sums}, ArraySink<uint32_t>{d.cell_sums}, d.cell_tiles,
                                 sh);
    }
}

__global__ void __launch_bounds__(kScanBlock) batch_cell_apply_kernel(BatchArgs b) {
    __shared__ uint32_t t_sh;
    __shared__ ScanShared<uint32_t> sh;
    uint32_t t;
    while (next_tile(&b.counters[cCellApply], b.counts[kCells], &t_sh, &t)) {
        const uint2 tile = b.lists[kCells][t];
        const SlotDesc& d = b.slots[tile.x];
        const uint32_t offset = d.cell_sums[tile.y];
        tile_apply<uint32_t>(ArraySource<uint32_t>{d.hist}, ArraySink<uint32_t>{d.cell_start},
                             static_cast<size_t>(tile.y) * kCellTile, d.cells, offset, sh);
        if (threadIdx.x == 0) {
            d.cell_sums[tile.y] = 0u;
            if (tile.y + 1 == d.cell_tiles) d.cell_sums[d.cell_tiles] = 0u;
        }
    }
}

// Slot prefix of the records the scatter just wrote (the other parity):
// position sums per tile, scanned per slot, then each tile from its offset.
__global__ void __launch_bounds__(kScanBlock) batch_prefix_reduce_kernel(BatchArgs b) {
    __shared__ uint32_t t_sh;
    __shared__ ScanShared<LL2> sh;
    uint32_t t;
    while (next_tile(&b.counters[cPrefixReduce], b.counts[kPrefix], &t_sh, &t)) {
        const uint2 tile = b.lists[kPrefix][t];
        const SlotDesc& d = b.slots[tile.x];
        const LL2 total = tile_reduce<LL2>(dev::RecordQSource{d.rec[b.state[tile.x].cur ^ 1u]},
                                           static_cast<size_t>(tile.y) * kPrefixTile, d.samples, sh);
        if (threadIdx.x == 0) d.prefix_sums[tile.y] = total;
    }
}

__global__ void __launch_bounds__(kScanBlock) batch_prefix_scan_kernel(BatchArgs b) {
    __shared__ uint32_t t_sh;
    __shared__ ScanShared<LL2> sh;
    uint32_t t;
    while (next_tile(&b.counters[cPrefixScan], b.counts[kSlots], &t_sh, &t)) {
        const SlotDesc& d = b.slots[b.lists[kSlots][t].x];
        block_scan_all<LL2>(ArraySource<LL2>{d.prefix_sums}, ArraySink<LL2>{d.prefix_sums}, d.prefix_tiles, sh);
    }
}

__global__ void __launch_bounds__(kScanBlock) batch_prefix_apply_kernel(BatchArgs b) {
    __shared__ uint32_t t_sh;
    __shared__ ScanShared<LL2> sh;
    uint32_t t;
    while (next_tile(&b.counters[cPrefixApply], b.counts[kPrefix], &t_sh, &t)) {
        const uint2 tile = b.lists[kPrefix][t];
        const SlotDesc& d = b.slots[tile.x];
        const LL2 offset = d.prefix_sums[tile.y];
        tile_apply<LL2>(dev::RecordQSource{d.rec[b.state[tile.x].cur ^ 1u]}, ArraySink<LL2>{d.slot_prefix},
                        static_cast<size_t>(tile.y) * kPrefixTile, d.samples, offset, sh);
    }
}

__global__ void __launch_bounds__(256) batch_scatter_kernel(BatchArgs b) {
    __shared__ uint32_t t_sh;
    __shared__ ScatterArgs args;
    uint32_t t;
    while (next_tile(&b.counters[cScatter], b.counts[kSamples], &t_sh, &t)) {
        const uint2 tile = b.lists[kSamples][t];
        stage_words(&args, &b.slots[tile.x].scatter[b.state[tile.x].cur]);
        __syncthreads();
        dev::scatter_sample(args, tile.y + threadIdx.x);
    }
}

__device__ __forceinline__ const Taps& pass_taps(const BlurSlot& s, uint32_t pass) {
    return s.taps[pass < s.taps_count ? pass : s.taps_count - 1];
}

__global__ void __launch_bounds__(dev::kBlurThreads, dev::kBlurMinCtas) batch_blur_h_kernel(BatchArgs b) {
    extern __shared__ float smem[];
    __shared__ uint32_t t_sh;
    __shared__ int rp_sh;
    uint32_t t;
    while (next_tile(&b.counters[cBlurH], b.counts[kBlurH], &t_sh, &t)) {
        const uint2 tile = b.lists[kBlurH][t];
        const BlurSlot& s = b.slots[tile.x].blur;
        const Taps& taps = pass_taps(s, b.state[tile.x].pass);
        if (threadIdx.x == 0) rp_sh = dev::blur_padded(taps.R);
        __syncthreads();
        const int RP = rp_sh;
        dev::load_taps(smem, taps, RP);
        dev::blur_h_tile(s.counts, s.himg, s.w, s.h, smem, RP, static_cast<int>(tile.y & 0xFFFFu),
                         static_cast<int>(tile.y >> 16), smem + ((RP + 1 + 3) & ~3));
    }
}

__global__ void __launch_bounds__(dev::kBlurThreads, dev::kBlurMinCtas) batch_blur_v_kernel(BatchArgs b) {
    extern __shared__ float smem[];
    __shared__ uint32_t t_sh;
    __shared__ int rp_sh;
    __shared__ float warp_max[dev::kBlurSegs];
    uint32_t t;
    while (next_tile(&b.counters[cBlurV], b.counts[kBlurV], &t_sh, &t)) {
        const uint2 tile = b.lists[kBlurV][t];
        const BlurSlot& s = b.slots[tile.x].blur;
        const Taps& taps = pass_taps(s, b.state[tile.x].pass);
        if (threadIdx.x == 0) rp_sh = dev::blur_padded(taps.R);
        __syncthreads();
        const int RP = rp_sh;
        dev::load_taps(smem, taps, RP);
        dev::blur_v_tile(s.himg, s.vimg, s.w, s.h, smem, RP, static_cast<int>(tile.y & 0xFFFFu),
                         static_cast<int>(tile.y >> 16), smem + ((RP + 1 + 3) & ~3), warp_max, s.peak);
    }
}

__global__ void __launch_bounds__(256) batch_normalize_kernel(BatchArgs b) {
    __shared__ uint32_t t_sh;
    uint32_t t;
    while (next_tile(&b.counters[cNormalize], b.counts[kTexels], &t_sh, &t)) {
        const uint2 tile = b.lists[kTexels][t];
        const BlurSlot& s = b.slots[tile.x].blur;
        if (!s.accumulate) continue;
        const float peak = __uint_as_float(*s.peak);
        const unsigned long long start = static_cast<unsigned long long>(tile.y) * kTexelTile;
        const unsigned long long end = min(start + kTexelTile, s.texels);
        for (unsigned long long i = start + threadIdx.x; i < end; i += blockDim.x)
            s.norm[i] = dev::normalized_value(s.vimg[i], peak);
    }
}

// End of an iteration: flip each slot's parity, count the pass.
__global__ void batch_advance_kernel(BatchArgs b) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < b.counts[kSlots]; i += gridDim.x * blockDim.x) {
        const uint32_t slot = b.lists[kSlots][i].x;
        SlotState& st = b.state[slot];
        st.cur ^= 1u;
        st.iterations += 1u;
        if (b.slots[slot].blur.accumulate) st.pass += 1u;
    }
}

// Slots of at least bt_batch::solo_samples samples iterate on their own
// context's stream and CUDA graphs, beside the persistent step, instead of
// joining its work lists (opt-in: large dense graphs run the single-graph
// kernels faster, while mid-size graphs on small maps do better in the step).
constexpr uint32_t kNeverSolo = UINT32_MAX;

struct Slot {
    bt_ctx* ctx = nullptr;
    bool active = false;
    bool solo = false;       // iterates on its own context (not in the work lists)
    DevBuf taps;             // Taps per density pass
    uint32_t taps_count = 0;
    uint32_t taps_first_pass = 0;   // taps[i] is pass i (tables start at pass 0)
};

}  // namespace
}  // namespace bt

struct bt_batch {
    int device = 0;
    int sms = 148;
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr, t0 = nullptr, t1 = nullptr;
    cudaEvent_t fork = nullptr;   // start of a step, for the solo slots' streams
    std::string err;
    std::vector<bt::Slot> slots;
    bt::DevBuf descs, state, counts, counters, status, lists[bt::kLists];
    unsigned long long list_capacity[bt::kLists] = {};
    bool dirty = true;
    cudaGraphExec_t graph = nullptr;
    int grid_blocks[bt::cCounters] = {};
    size_t blur_smem = 0;
    uint32_t* h_status = nullptr;
    uint32_t max_pass = 0;     // highest density pass the taps tables cover
    uint32_t solo_samples = bt::kNeverSolo;
    uint32_t mean_tile = 128;        // samples per mean tile (= its CTA size): 64, 128 or 256
    uint32_t mean_ctas_per_sm = 0;   // resident mean CTAs per SM (0 = as many as fit)
};

namespace bt {
namespace {

bt_status bfail(bt_batch* b, bt_status code, const std::string& msg) {
    if (b) b->err = msg;
    set_thread_error(msg.c_str());
    return code;
}

bt_status bcuda(bt_batch* b, cudaError_t e, const char* what) {
    return bfail(b, e == cudaErrorMemoryAllocation ? BT_ERR_BUDGET : BT_ERR_CUDA,
                 std::string(what) + ": " + cudaGetErrorString(e));
}

#define BB_CUDA(b, call)                                       \
    do {                                                       \
        cudaError_t e_ = (call);                               \
        if (e_ != cudaSuccess) return bcuda((b), e_, #call);   \
    } while (0)

bt_status bgrow(bt_batch* b, DevBuf& buf, size_t bytes) {
    if (bytes == 0) bytes = 16;
    if (buf.bytes >= bytes) return BT_OK;
    // Stream-ordered, like the contexts' buffers: no device-wide wait.
    if (buf.p) cudaFreeAsync(buf.p, b->stream);
    buf.p = nullptr;
    buf.bytes = 0;
    cudaError_t e = cudaMallocAsync(&buf.p, bytes, b->stream);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return bcuda(b, e, "device allocation");
    }
    buf.bytes = bytes;
    return BT_OK;
}

bt_status bwait(bt_batch* b) {
    // The batch stream already waits for the solo slots' queued work after
    // each step; work queued on them since (a re-upload) is joined here.
    for (const Slot& s : b->slots) {
        if (!s.active || !s.solo) continue;
        cudaError_t j = cudaEventRecord(s.ctx->done, s.ctx->stream);
        if (j == cudaSuccess) j = cudaStreamWaitEvent(b->stream, s.ctx->done, 0);
        if (j != cudaSuccess) return bcuda(b, j, "stream ordering");
    }
    cudaError_t e = cudaEventRecord(b->done, b->stream);
    if (e != cudaSuccess) return bcuda(b, e, "cudaEventRecord");
    const auto start = std::chrono::steady_clock::now();
    int spins = 0;
    while (true) {
        e = cudaEventQuery(b->done);
        if (e == cudaSuccess) break;
        if (e != cudaErrorNotReady) return bcuda(b, e, "device execution");
        if (std::chrono::duration<double>(std::chrono::steady_clock::now() - start).count() > 60.0)
            return bfail(b, BT_ERR_TIMEOUT, "device wait exceeded 60 s");
        if (++spins < 2000)
            std::this_thread::yield();
        else
            std::this_thread::sleep_for(std::chrono::microseconds(50));
    }
    return BT_OK;
}

// Taps of a slot for density passes 0 .. upto (σ_i = σ · shrink^i).
bt_status fill_taps(bt_batch* b, Slot& s, uint32_t upto) {
    const bt_options& o = s.ctx->opt;
    const bool constant = o.blur_sigma == 0.0f || o.blur_shrink == 0.0f || o.blur_shrink == 1.0f;
    const uint32_t count = constant ? 1u : upto + 1u;
    if (s.taps_count >= count) return BT_OK;
    std::vector<Taps> taps(count);
    for (uint32_t i = 0; i < count; ++i)
        if (!make_blur_taps(sigma_for_pass(o, i), &taps[i])) return bfail(b, BT_ERR_INVALID, "invalid blur sigma");
    if (bt_status st = bgrow(b, s.taps, sizeof(Taps) * count)) return st;
    // Stream-ordered like the allocation (the host copy is staged before the call returns).
    BB_CUDA(b, cudaMemcpyAsync(s.taps.p, taps.data(), sizeof(Taps) * count, cudaMemcpyHostToDevice, b->stream));
    s.taps_count = count;
    return BT_OK;
}

MeanArgs mean_args(bt_ctx* c, int src) {
    MeanArgs m{};
    m.rec = c->sorted_rec[src].as<float2>();
    m.tag = c->sorted_tag[src].as<uint32_t>();
    m.cell_start = c->cell_start.as<uint32_t>();
    m.prefix = c->slot_prefix.as<LL2>();
    m.mode = static_cast<int>(c->opt.search_mode);
    m.out_xy = c->tmp_xy.as<float2>();
    m.out_tag = c->tmp_tag.as<uint32_t>();
    m.out_cell = c->tmp_cell.as<uint32_t>();
    m.hist = c->hist.as<uint32_t>();
    m.hist_tiles = c->hist_tiles.as<uint32_t>();
    m.counts = c->accumulate ? c->counts.as<uint32_t>() : nullptr;
    m.neighbors = c->opt.record_neighbors ? c->neighbors.as<uint32_t>() : nullptr;
    m.n = c->samples;
    m.g = c->grid;
    return m;
}

ScatterArgs scatter_args(bt_ctx* c, int src, uint32_t* status) {
    ScatterArgs s{};
    s.xy = c->tmp_xy.as<float2>();
    s.tag = c->tmp_tag.as<uint32_t>();
    s.cell = c->tmp_cell.as<uint32_t>();
    s.cell_start = c->cell_start.as<uint32_t>();
    s.hist = c->hist.as<uint32_t>();
    s.out_rec = c->sorted_rec[src ^ 1].as<float2>();
    s.out_tag = c->sorted_tag[src ^ 1].as<uint32_t>();
    s.n = c->samples;
    s.cells = static_cast<uint32_t>(c->cells);
    s.status = status;
    return s;
}

BatchArgs batch_args(bt_batch* b) {
    BatchArgs a{};
    a.slots = b->descs.as<SlotDesc>();
    a.state = b->state.as<SlotState>();
    for (int l = 0; l < kLists; ++l) a.lists[l] = b->lists[l].as<uint2>();
    a.counts = b->counts.as<uint32_t>();
    a.counters = b->counters.as<uint32_t>();
    a.status = b->status.as<uint32_t>();
    return a;
}

// One iteration of every slot: the kernels of Gpu::iterate as persistent
// work-queue launches.
void enqueue_batch_iteration(bt_batch* b) {
    const BatchArgs a = batch_args(b);
    cudaMemsetAsync(b->counters.p, 0, sizeof(uint32_t) * cCounters, b->stream);
    batch_clear_kernel<<<b->grid_blocks[cClear], 256, 0, b->stream>>>(a);
    switch (b->mean_tile) {
        case 64: batch_mean_kernel<64><<<b->grid_blocks[cMean], 64, 0, b->stream>>>(a); break;
        case 256: batch_mean_kernel<256><<<b->grid_blocks[cMean], 256, 0, b->stream>>>(a); break;
        default: batch_mean_kernel<128><<<b->grid_blocks[cMean], 128, 0, b->stream>>>(a); break;
    }
    batch_cell_scan_kernel<<<b->grid_blocks[cCellScan], kScanBlock, 0, b->stream>>>(a);
    batch_cell_apply_kernel<<<b->grid_blocks[cCellApply], kScanBlock, 0, b->stream>>>(a);
    batch_scatter_kernel<<<b->grid_blocks[cScatter], kSampleTile, 0, b->stream>>>(a);
    batch_prefix_reduce_kernel<<<b->grid_blocks[cPrefixReduce], kScanBlock, 0, b->stream>>>(a);
    batch_prefix_scan_kernel<<<b->grid_blocks[cPrefixScan], kScanBlock, 0, b->stream>>>(a);
    batch_prefix_apply_kernel<<<b->grid_blocks[cPrefixApply], kScanBlock, 0, b->stream>>>(a);
    batch_blur_h_kernel<<<b->grid_blocks[cBlurH], dev::kBlurThreads, b->blur_smem, b->stream>>>(a);
    batch_blur_v_kernel<<<b->grid_blocks[cBlurV], dev::kBlurThreads, b->blur_smem, b->stream>>>(a);
    batch_normalize_kernel<<<b->grid_blocks[cNormalize], 256, 0, b->stream>>>(a);
    batch_advance_kernel<<<1, 256, 0, b->stream>>>(a);
}

// Descriptors, device state and work lists of the active slots.
bt_status rebuild(bt_batch* b) {
    const size_t n = b->slots.size();
    std::vector<SlotDesc> descs(n);
    std::vector<SlotState> state(n);
    std::vector<uint2> lists[kLists];
    for (size_t i = 0; i < n; ++i) {
        Slot& s = b->slots[i];
        std::memset(&descs[i], 0, sizeof(SlotDesc));
        if (!s.active || s.solo) continue;
        bt_ctx* c = s.ctx;
        if (bt_status st = fill_taps(b, s, std::max(b->max_pass, c->density_passes) + kTapsHorizon)) return st;
        const uint32_t cell_tiles = static_cast<uint32_t>(scan_tiles<uint32_t>(c->cells));
        const uint32_t prefix_tiles = static_cast<uint32_t>(scan_tiles<LL2>(c->samples));
        // The population sums start from zero (each iteration's cell-table
        // apply clears them after use).
        BB_CUDA(b, cudaMemsetAsync(c->hist_tiles.p, 0, c->hist_tiles.bytes, b->stream));
        SlotDesc& d = descs[i];
        for (int p = 0; p < 2; ++p) {
            d.mean[p] = mean_args(c, p);
            d.scatter[p] = scatter_args(c, p, b->status.as<uint32_t>());
        }
        d.hist = c->hist.as<uint32_t>();
        d.cell_start = c->cell_start.as<uint32_t>();
        d.cell_sums = c->hist_tiles.as<uint32_t>();
        d.rec[0] = c->sorted_rec[0].as<float2>();
        d.rec[1] = c->sorted_rec[1].as<float2>();
        d.slot_prefix = c->slot_prefix.as<LL2>();
        d.prefix_sums = c->prefix_tiles.as<LL2>();
        d.cells = static_cast<uint32_t>(c->cells);
        d.cell_tiles = cell_tiles;
        d.samples = c->samples;
        d.prefix_tiles = prefix_tiles;
        d.blur = BlurSlot{c->counts.as<uint32_t>(), c->himg.as<float>(), c->vimg.as<float>(), c->norm.as<float>(),
                          c->peak.as<uint32_t>(), c->map.w, c->map.h, c->texels, s.taps.as<Taps>(), s.taps_count,
                          c->accumulate ? 1u : 0u};
        state[i] = SlotState{static_cast<uint32_t>(c->cur), c->density_passes, c->iterations, 0u};
        const uint32_t slot = static_cast<uint32_t>(i);
        for (uint32_t t = 0; t < (c->samples + kSampleTile - 1) / kSampleTile; ++t)
            lists[kSamples].push_back(make_uint2(slot, t * kSampleTile));
        for (uint32_t t = 0; t < (c->samples + b->mean_tile - 1) / b->mean_tile; ++t)
            lists[kMeanTiles].push_back(make_uint2(slot, t * b->mean_tile));
        for (uint32_t t = 0; t < cell_tiles; ++t) lists[kCells].push_back(make_uint2(slot, t));
        for (uint32_t t = 0; t < prefix_tiles; ++t) lists[kPrefix].push_back(make_uint2(slot, t));
        lists[kSlots].push_back(make_uint2(slot, 0u));
        if (c->accumulate) {
            const uint32_t hx = div_up(c->map.w, dev::kBlurSpan), hy = div_up(c->map.h, dev::kBlurLines);
            for (uint32_t y = 0; y < hy; ++y)
                for (uint32_t x = 0; x < hx; ++x) lists[kBlurH].push_back(make_uint2(slot, x | (y << 16)));
            const uint32_t vx = div_up(c->map.w, dev::kBlurLines), vy = div_up(c->map.h, dev::kBlurSpan);
            for (uint32_t y = 0; y < vy; ++y)
                for (uint32_t x = 0; x < vx; ++x) lists[kBlurV].push_back(make_uint2(slot, x | (y << 16)));
            const unsigned long long tt = (c->texels + kTexelTile - 1) / kTexelTile;
            for (unsigned long long t = 0; t < tt; ++t)
                lists[kTexels].push_back(make_uint2(slot, static_cast<uint32_t>(t)));
        }
    }
    if (bt_status st = bgrow(b, b->descs, sizeof(SlotDesc) * std::max<size_t>(n, 1))) return st;
    if (bt_status st = bgrow(b, b->state, sizeof(SlotState) * std::max<size_t>(n, 1))) return st;
    BB_CUDA(b, cudaMemcpyAsync(b->descs.p, descs.data(), sizeof(SlotDesc) * n, cudaMemcpyHostToDevice, b->stream));
    BB_CUDA(b, cudaMemcpyAsync(b->state.p, state.data(), sizeof(SlotState) * n, cudaMemcpyHostToDevice, b->stream));
    uint32_t counts[kLists];
    for (int l = 0; l < kLists; ++l) {
        counts[l] = static_cast<uint32_t>(lists[l].size());
        if (bt_status st = bgrow(b, b->lists[l], sizeof(uint2) * std::max<size_t>(lists[l].size(), 1))) return st;
        if (!lists[l].empty())
            BB_CUDA(b, cudaMemcpyAsync(b->lists[l].p, lists[l].data(), sizeof(uint2) * lists[l].size(),
                                       cudaMemcpyHostToDevice, b->stream));
    }
    BB_CUDA(b, cudaMemcpyAsync(b->counts.p, counts, sizeof(counts), cudaMemcpyHostToDevice, b->stream));
    if (bt_status st = bwait(b)) return st;   // the host vectors go out of scope
    {
        // The mean's persistent grid for the batch's shape.
        int per_sm = 0;
        cudaError_t oe = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, mean_kernel_for(b->mean_tile),
                                                                       static_cast<int>(b->mean_tile), 0);
        if (oe != cudaSuccess) return bcuda(b, oe, "occupancy");
        per_sm = std::max(1, per_sm);
        if (b->mean_ctas_per_sm) per_sm = std::min(per_sm, static_cast<int>(b->mean_ctas_per_sm));
        b->grid_blocks[cMean] = per_sm * b->sms;
    }
    if (b->graph) {
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
    }
    cudaGraph_t g = nullptr;
    BB_CUDA(b, cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    enqueue_batch_iteration(b);
    BB_CUDA(b, cudaStreamEndCapture(b->stream, &g));
    cudaError_t e = cudaGraphInstantiate(&b->graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
        b->graph = nullptr;
        return bcuda(b, e, "cudaGraphInstantiate");
    }
    b->dirty = false;
    return BT_OK;
}

// Host copies of each slot's counters follow the device state after n
// iterations (all active slots advance together).
void advance_hosts(bt_batch* b, uint32_t n) {
    for (Slot& s : b->slots) {
        if (!s.active || s.solo) continue;   // solo contexts keep their own counts
        bt_ctx* c = s.ctx;
        c->cur ^= static_cast<int>(n & 1u);
        c->iterations += n;
        if (c->accumulate) c->density_passes += n;
        b->max_pass = std::max(b->max_pass, c->density_passes);
    }
}

bt_status need_slot(bt_batch* b, uint32_t slot, bt_ctx** c) {
    if (!b) return bfail(nullptr, BT_ERR_INVALID, "null batch");
    if (slot >= b->slots.size() || !b->slots[slot].active) return bfail(b, BT_ERR_INVALID, "no such slot");
    *c = b->slots[slot].ctx;
    return BT_OK;
}

}  // namespace

bt_status batch_attach(bt_batch* b, bt_ctx* c, uint32_t* slot) {
    if (!b || !c || !slot) return bfail(b, BT_ERR_INVALID, "null argument");
    if (!c->uploaded || !c->has_grid)
        return bfail(b, BT_ERR_INVALID, "a batch slot needs an uploaded graph with a neighbour radius");
    if (c->device != b->device) return bfail(b, BT_ERR_INVALID, "the graph lives on another device");
    // The batch's next launches come after the work still queued on the
    // context's stream (an upload's re-binning runs asynchronously).
    cudaSetDevice(b->device);
    cudaError_t e = cudaEventRecord(c->done, c->stream);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(b->stream, c->done, 0);
    if (e != cudaSuccess) return bcuda(b, e, "stream ordering");
    // Reuse a free slot index, else append.
    uint32_t idx = 0;
    while (idx < b->slots.size() && b->slots[idx].active) ++idx;
    if (idx == b->slots.size()) b->slots.emplace_back();
    Slot& s = b->slots[idx];
    if (s.ctx) bt_destroy(s.ctx);
    s.ctx = c;
    s.active = true;
    s.solo = c->samples >= b->solo_samples;
    s.taps_count = 0;
    b->dirty = true;
    *slot = idx;
    return BT_OK;
}

cudaStream_t batch_stream(bt_batch* b) { return b->stream; }

bt_ctx* batch_detach(bt_batch* b, uint32_t slot) {
    bt_ctx* c = nullptr;
    if (need_slot(b, slot, &c)) return nullptr;
    cudaSetDevice(b->device);
    if (bwait(b)) return nullptr;
    b->slots[slot].active = false;
    b->slots[slot].ctx = nullptr;
    b->dirty = true;
    return c;
}

}  // namespace bt

using namespace bt;

extern "C" {

bt_status bt_batch_create(int32_t device, bt_batch** out) {
    if (!out) return bfail(nullptr, BT_ERR_INVALID, "null argument");
    *out = nullptr;
    auto* b = new bt_batch();
    b->device = device;
    auto bail = [&](bt_status s) {
        std::string msg = b->err;
        bt_batch_destroy(b);
        set_thread_error(msg.c_str());
        return s;
    };
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return bail(bcuda(b, e, "cudaSetDevice"));
    if ((e = prepare_density_kernels()) != cudaSuccess) return bail(bcuda(b, e, "kernel attributes"));
    b->blur_smem = dev::blur_smem_bytes(dev::blur_padded(kMaxTaps - 1));
    const void* blur_kernels[2] = {reinterpret_cast<const void*>(batch_blur_h_kernel),
                                   reinterpret_cast<const void*>(batch_blur_v_kernel)};
    for (const void* k : blur_kernels)
        if ((e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      static_cast<int>(b->blur_smem))) != cudaSuccess)
            return bail(bcuda(b, e, "kernel attributes"));
    cudaDeviceProp prop{};
    if ((e = cudaGetDeviceProperties(&prop, device)) != cudaSuccess) return bail(bcuda(b, e, "device properties"));
    b->sms = prop.multiProcessorCount;
    // Persistent grids: every SM filled to its resident-CTA limit.
    struct K {
        Counter c;
        const void* f;
        int threads;
        size_t smem;
    } ks[] = {
        {cClear, reinterpret_cast<const void*>(batch_clear_kernel), 256, 0},
        {cCellScan, reinterpret_cast<const void*>(batch_cell_scan_kernel), kScanBlock, 0},
        {cCellApply, reinterpret_cast<const void*>(batch_cell_apply_kernel), kScanBlock, 0},
        {cScatter, reinterpret_cast<const void*>(batch_scatter_kernel), kSampleTile, 0},
        {cPrefixReduce, reinterpret_cast<const void*>(batch_prefix_reduce_kernel), kScanBlock, 0},
        {cPrefixScan, reinterpret_cast<const void*>(batch_prefix_scan_kernel), kScanBlock, 0},
        {cPrefixApply, reinterpret_cast<const void*>(batch_prefix_apply_kernel), kScanBlock, 0},
        {cBlurH, reinterpret_cast<const void*>(batch_blur_h_kernel), dev::kBlurThreads, b->blur_smem},
        {cBlurV, reinterpret_cast<const void*>(batch_blur_v_kernel), dev::kBlurThreads, b->blur_smem},
        {cNormalize, reinterpret_cast<const void*>(batch_normalize_kernel), 256, 0},
    };
    for (const K& k : ks) {
        int per_sm = 0;
        if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k.f, k.threads, k.smem)) != cudaSuccess)
            return bail(bcuda(b, e, "occupancy"));
        b->grid_blocks[k.c] = std::max(1, per_sm) * b->sms;
    }
    if ((e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking)) != cudaSuccess)
        return bail(bcuda(b, e, "cudaStreamCreate"));
    if ((e = cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming)) != cudaSuccess)
        return bail(bcuda(b, e, "cudaEventCreate"));
    if ((e = cudaEventCreateWithFlags(&b->done, cudaEventDisableTiming)) != cudaSuccess)
        return bail(bcuda(b, e, "cudaEventCreate"));
    if ((e = cudaEventCreate(&b->t0)) != cudaSuccess || (e = cudaEventCreate(&b->t1)) != cudaSuccess)
        return bail(bcuda(b, e, "cudaEventCreate"));
    if ((e = cudaMallocHost(&b->h_status, 16)) != cudaSuccess) return bail(bcuda(b, e, "cudaMallocHost"));
    if (bt_status s = bgrow(b, b->counts, sizeof(uint32_t) * kLists)) return bail(s);
    if (bt_status s = bgrow(b, b->counters, sizeof(uint32_t) * cCounters)) return bail(s);
    if (bt_status s = bgrow(b, b->status, 16)) return bail(s);
    cudaMemsetAsync(b->status.p, 0, 16, b->stream);
    if (bt_status s = bwait(b)) return bail(s);
    *out = b;
    return BT_OK;
}

void bt_batch_destroy(bt_batch* b) {
    if (!b) return;
    if (b->stream) cudaStreamSynchronize(b->stream);
    if (b->graph) cudaGraphExecDestroy(b->graph);
    for (Slot& s : b->slots) {
        bt_destroy(s.ctx);
        if (s.taps.p) cudaFreeAsync(s.taps.p, b->stream);
    }
    DevBuf* bufs[] = {&b->descs, &b->state, &b->counts, &b->counters, &b->status};
    for (DevBuf* x : bufs)
        if (x->p) cudaFreeAsync(x->p, b->stream);
    for (DevBuf& x : b->lists)
        if (x.p) cudaFreeAsync(x.p, b->stream);
    if (b->stream) cudaStreamSynchronize(b->stream);   // the frees above
    if (b->h_status) cudaFreeHost(b->h_status);
    if (b->done) cudaEventDestroy(b->done);
    if (b->fork) cudaEventDestroy(b->fork);
    if (b->t0) cudaEventDestroy(b->t0);
    if (b->t1) cudaEventDestroy(b->t1);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
}

const char* bt_batch_last_error(const bt_batch* b) { return b ? b->err.c_str() : bt_last_error(nullptr); }

bt_status bt_batch_add(bt_batch* b, const bt_options* options, const float* xy, uint32_t n_points,
                       const uint32_t* starts, uint32_t n_starts, uint32_t* slot, uint32_t* samples) {
    if (!b || !options || !slot || !samples) return bfail(b, BT_ERR_INVALID, "null argument");
    if (options->neighbor_radius == 0) return bfail(b, BT_ERR_NOT_CONFIGURED, "neighbor radius is not configured");
    bt_options o = *options;
    o.device = b->device;
    o.timing = 0;
    bt_ctx* c = nullptr;
    if (bt_status s = bt_create(&o, &c)) return bfail(b, s, bt_last_error(nullptr));
    if (bt_status s = bt_upload(c, xy, n_points, starts, n_starts, samples)) {
        std::string msg = bt_last_error(c);
        bt_destroy(c);
        return bfail(b, s, msg);
    }
    if (bt_status s = batch_attach(b, c, slot)) {
        bt_destroy(c);
        return s;
    }
    return BT_OK;
}

bt_status bt_batch_add_many(bt_batch* b, uint32_t count, const bt_options* options, const float* const* xy,
                            const uint32_t* n_points, const uint32_t* const* starts, const uint32_t* n_starts,
                            uint32_t* slots, uint32_t* samples) {
    if (!b || (count && (!options || !xy || !n_points || !starts || !n_starts || !slots || !samples)))
        return bfail(b, BT_ERR_INVALID, "null argument");
    std::vector<bt_ctx*> ctxs(count, nullptr);
    auto unwind = [&](bt_status s, std::string msg) {   // by value: msg may live in a context destroyed here
        for (bt_ctx* c : ctxs) bt_destroy(c);
        return bfail(b, s, msg);
    };
    for (uint32_t i = 0; i < count; ++i) {
        if (options[i].neighbor_radius == 0) return unwind(BT_ERR_NOT_CONFIGURED, "neighbor radius is not configured");
        bt_options o = options[i];
        o.device = b->device;
        o.timing = 0;
        if (bt_status s = bt_create(&o, &ctxs[i])) return unwind(s, bt_last_error(nullptr));
    }
    // Every graph's phase on its own stream, one host wait per phase.
    for (uint32_t i = 0; i < count; ++i)
        if (bt_status s = upload_begin(ctxs[i], xy[i], n_points[i], starts[i], n_starts[i]))
            return unwind(s, ctxs[i]->err);
    for (uint32_t i = 0; i < count; ++i)
        if (bt_status s = upload_wait(ctxs[i])) return unwind(s, ctxs[i]->err);
    for (uint32_t i = 0; i < count; ++i)
        if (bt_status s = upload_finish(ctxs[i])) return unwind(s, ctxs[i]->err);
    for (uint32_t i = 0; i < count; ++i)
        if (bt_status s = upload_wait(ctxs[i])) return unwind(s, ctxs[i]->err);
    for (uint32_t i = 0; i < count; ++i) {
        if (bt_status s = upload_check(ctxs[i], &samples[i])) return unwind(s, ctxs[i]->err);
        if (bt_status s = upload_adapt(ctxs[i])) return unwind(s, ctxs[i]->err);
    }
    for (uint32_t i = 0; i < count; ++i) {
        batch_attach(b, ctxs[i], &slots[i]);   // cannot fail: every check above passed
        ctxs[i] = nullptr;
    }
    return BT_OK;
}

bt_status bt_batch_remove(bt_batch* b, uint32_t slot) {
    bt_ctx* c = nullptr;
    if (bt_status s = need_slot(b, slot, &c)) return s;
    cudaSetDevice(b->device);
    if (bt_status s = bwait(b)) return s;
    b->slots[slot].active = false;
    bt_destroy(c);
    b->slots[slot].ctx = nullptr;
    b->dirty = true;
    return BT_OK;
}

bt_status bt_batch_iterate_async(bt_batch* b, uint32_t n) {
    NvtxRange range("batch_iterate");
    if (!b) return bfail(nullptr, BT_ERR_INVALID, "null batch");
    cudaSetDevice(b->device);
    bool any = false, any_solo = false;
    uint32_t reach = 0;
    for (Slot& s : b->slots) {
        if (!s.active) continue;
        if (s.solo) {
            any_solo = true;
            continue;
        }
        any = true;
        reach = std::max(reach, s.ctx->density_passes + n);
        if (s.taps_count > 1 && reach >= s.taps_count) b->dirty = true;   // extend shrinking-σ tables
    }
    if (any_solo && n > 0) {
        // Solo slots start after the batch's earlier work and run beside
        // this step; the batch stream waits for them after its own launches.
        BB_CUDA(b, cudaEventRecord(b->fork, b->stream));
        for (Slot& s : b->slots) {
            if (!s.active || !s.solo) continue;
            BB_CUDA(b, cudaStreamWaitEvent(s.ctx->stream, b->fork, 0));
            if (bt_status st = bt_iterate_async(s.ctx, n)) return bfail(b, st, s.ctx->err);
        }
    }
    if (any) {
        b->max_pass = std::max(b->max_pass, reach);
        if (b->dirty)
            if (bt_status s = rebuild(b)) return s;
        for (uint32_t i = 0; i < n; ++i) BB_CUDA(b, cudaGraphLaunch(b->graph, b->stream));
        advance_hosts(b, n);
    }
    if (any_solo && n > 0) {
        for (Slot& s : b->slots) {
            if (!s.active || !s.solo) continue;
            BB_CUDA(b, cudaEventRecord(s.ctx->done, s.ctx->stream));
            BB_CUDA(b, cudaStreamWaitEvent(b->stream, s.ctx->done, 0));
        }
    }
    return BT_OK;
}

bt_status bt_batch_synchronize(bt_batch* b) {
    if (!b) return bfail(nullptr, BT_ERR_INVALID, "null batch");
    cudaSetDevice(b->device);
    if (bt_status s = bwait(b)) return s;
    BB_CUDA(b, cudaMemcpy(b->h_status, b->status.p, 4, cudaMemcpyDeviceToHost));
    for (const Slot& s : b->slots) {
        if (!s.active || !s.solo) continue;
        BB_CUDA(b, cudaMemcpy(b->h_status + 1, s.ctx->status.p, 4, cudaMemcpyDeviceToHost));
        b->h_status[0] |= b->h_status[1];
    }
    if (b->h_status[0] & 8u) return bfail(b, BT_ERR_CUDA, "inconsistent neighbour-grid binning");
    return BT_OK;
}

bt_status bt_batch_iterate(bt_batch* b, uint32_t n) {
    if (bt_status s = bt_batch_iterate_async(b, n)) return s;
    return bt_batch_synchronize(b);
}

bt_status bt_batch_iterate_timed(bt_batch* b, uint32_t n, float* device_ms) {
    if (!b || !device_ms) return bfail(b, BT_ERR_INVALID, "null argument");
    cudaSetDevice(b->device);
    // Rebuild outside the timed region.
    if (bt_status s = bt_batch_iterate_async(b, 0)) return s;
    BB_CUDA(b, cudaEventRecord(b->t0, b->stream));
    if (bt_status s = bt_batch_iterate_async(b, n)) return s;
    BB_CUDA(b, cudaEventRecord(b->t1, b->stream));
    if (bt_status s = bt_batch_synchronize(b)) return s;
    BB_CUDA(b, cudaEventElapsedTime(device_ms, b->t0, b->t1));
    return BT_OK;
}

bt_status bt_batch_set_solo_samples(bt_batch* b, uint32_t samples) {
    if (!b) return bfail(nullptr, BT_ERR_INVALID, "null batch");
    cudaSetDevice(b->device);
    if (bt_status s = bwait(b)) return s;   // no step in flight while slots change lanes
    b->solo_samples = samples ? samples : kNeverSolo;
    for (Slot& s : b->slots)
        if (s.active) s.solo = s.ctx->samples >= b->solo_samples;
    b->dirty = true;
    return BT_OK;
}

bt_status bt_batch_set_shape(bt_batch* b, uint32_t mean_tile, uint32_t mean_ctas_per_sm) {
    if (!b) return bfail(nullptr, BT_ERR_INVALID, "null batch");
    if (mean_tile != 64 && mean_tile != 128 && mean_tile != 256)
        return bfail(b, BT_ERR_INVALID, "mean_tile must be 64, 128 or 256 samples");
    if (mean_ctas_per_sm > 1280 / mean_tile)
        return bfail(b, BT_ERR_INVALID, "mean_ctas_per_sm above the 1,280 resident threads of the mean kernel");
    cudaSetDevice(b->device);
    if (bt_status s = bwait(b)) return s;   // no step in flight while the work lists change
    b->mean_tile = mean_tile;
    b->mean_ctas_per_sm = mean_ctas_per_sm;
    b->dirty = true;
    return BT_OK;
}

bt_status bt_batch_get_shape(bt_batch* b, uint32_t* mean_tile, uint32_t* mean_ctas_per_sm) {
    if (!b || !mean_tile || !mean_ctas_per_sm) return bfail(b, BT_ERR_INVALID, "null argument");
    *mean_tile = b->mean_tile;
    *mean_ctas_per_sm = b->mean_ctas_per_sm;
    return BT_OK;
}

bt_status bt_batch_autotune(int32_t device, uint32_t count, const bt_options* options, const float* const* xy,
                            const uint32_t* n_points, const uint32_t* const* starts, const uint32_t* n_starts,
                            uint32_t iterations, uint32_t* mean_tile, uint32_t* mean_ctas_per_sm, float* best_ms) {
    if (!mean_tile || !mean_ctas_per_sm || count == 0 || iterations == 0)
        return bfail(nullptr, BT_ERR_INVALID, "null argument, no graph or no iteration");
    // Each candidate on a fresh scratch batch of the same graphs, so that
    // every candidate times the same iterations (the work per iteration
    // changes as the graphs bundle); the caller's batch is not touched.
    struct Cand {
        uint32_t tile, ctas;
    };
    const Cand cands[] = {{64, 0}, {64, 14}, {128, 0}, {128, 7}, {256, 0}, {256, 3}};
    std::vector<uint32_t> slots(count), samples(count);
    float best = -1.0f;
    for (const Cand& k : cands) {
        bt_batch* b = nullptr;
        if (bt_status s = bt_batch_create(device, &b)) return s;
        bt_status s = bt_batch_add_many(b, count, options, xy, n_points, starts, n_starts, slots.data(),
                                        samples.data());
        if (!s) s = bt_batch_set_shape(b, k.tile, k.ctas);
        float ms = 0.0f;
        if (!s) s = bt_batch_iterate_timed(b, iterations, &ms);
        if (s) {
            const std::string msg = b->err;
            bt_batch_destroy(b);
            return bfail(nullptr, s, msg);
        }
        bt_batch_destroy(b);
        if (best < 0.0f || ms < best) {
            best = ms;
            *mean_tile = k.tile;
            *mean_ctas_per_sm = k.ctas;
        }
    }
    if (best_ms) *best_ms = best;
    return BT_OK;
}

bt_status bt_batch_slot_count(bt_batch* b, uint32_t* active, uint32_t* capacity) {
    if (!b) return bfail(nullptr, BT_ERR_INVALID, "null batch");
    uint32_t n = 0;
    for (const Slot& s : b->slots) n += s.active ? 1u : 0u;
    if (active) *active = n;
    if (capacity) *capacity = static_cast<uint32_t>(b->slots.size());
    return BT_OK;
}

bt_ctx* bt_batch_slot(bt_batch* b, uint32_t slot) {
    bt_ctx* c = nullptr;
    if (need_slot(b, slot, &c)) return nullptr;
    if (bwait(b)) return nullptr;
    return c;
}

}  // extern "C"
