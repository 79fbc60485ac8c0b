// blur_tma.cu — the separable blur passes staged by the Tensor Memory
// Accelerator (TMA) for maps whose rows are whole 16-byte units.
//
// Same arithmetic as density.cu (blur.wgsl:13-82 with a general tap count:
// out[x] = w0*in[x] + sum_{k=1..R} fma(in[x-k] + in[x+k], w_k, ...), k = 1..R
// in order, zero outside the map), so results are bit-identical to the
// element-staged kernels; only the movement of the tiles changes:
//  - Persistent CTAs (two per SM) walk the tiles; each owns two shared-memory
//    stages. While the CTA convolves the tile in one stage, one thread has the
//    TMA copy the next tile into the other (2-D `cp.async.bulk.tensor`, one
//    mbarrier per stage counting the bytes). The halo's zero padding is the
//    TMA's fill of coordinates outside the map; no global load is issued by
//    the convolving threads.
//  - Horizontal pass (u32 counts -> f32): a tile is 32 rows x 128 outputs plus
//    an RP-texel halo on either side, copied as boxes of 32 x 32 with the
//    128-byte swizzle, so that the float4 reads of 32 rows by one warp spread
//    over all banks. The counts are converted to f32 in place once per tile.
//  - Vertical pass (f32 -> f32 and the maximum): a tile is 32 columns x 128
//    outputs plus the halo, one box of 32 columns (two when the halo is long);
//    each lane reads its own column, so consecutive lanes hit consecutive
//    banks without a transposed copy.
//  - Every wait on an mbarrier is bounded: past the limit the kernel sets bit
//    16 of the status word, waits (again bounded) for its own copies in
//    flight, and returns.
// No copy uses cluster multicast: every tensor map covers this GPU's own
// buffers.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>

#include "density_dev.cuh"

namespace bt {
namespace {

using dev::kBlurLines;
using dev::kBlurOut;
using dev::kBlurSegs;
using dev::kBlurSpan;
using dev::kBlurThreads;

constexpr int kStages = 2;
constexpr uint32_t kStatusCopyTimeout = 16u;
// try_wait rounds of at most kWaitHintNs each: about 1.3 s in all, far above
// any copy of a tile (microseconds).
constexpr uint32_t kWaitLimit = 1u << 17;
constexpr uint32_t kWaitHintNs = 10000;

// ---- PTX wrappers (sm_90+ TMA and mbarrier) ----
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

// One bounded try_wait round: true once the phase with this parity completed.
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(parity), "r"(kWaitHintNs)
        : "memory");
    return done != 0;
}

__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
    for (uint32_t i = 0; i < kWaitLimit; ++i)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
        "[%4];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void fence_proxy_async() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Exact u32 -> f32 (round to nearest, as f32(count)): below 2^23 by the
// exponent trick, above it by the conversion instruction.
__device__ __forceinline__ float count_to_float(uint32_t u) {
    if (u < (1u << 23)) return __int_as_float(static_cast<int>(u | 0x4B000000u)) - 8388608.0f;
    return static_cast<float>(u);
}

// Horizontal stage layout: box b (32 columns) at b * 4096 bytes, row r at
// r * 128, 16-byte chunk q of the row at (q ^ (r & 7)) * 16 (the TMA's
// 128-byte swizzle; the stage is 1024-byte aligned).
__device__ __forceinline__ const float4* h_chunk(const char* stage, int r, int col) {
    const int b = col >> 5, q = (col >> 2) & 7;
    return reinterpret_cast<const float4*>(stage + b * 4096 + r * 128 + ((q ^ (r & 7)) << 4));
}

struct HTile {
    int nb;         // boxes of 32 columns per tile
    int bytes;      // bytes of one stage
};

__host__ __device__ inline HTile h_tile(int RP) {
    const int width = kBlurSpan + 2 * RP;
    HTile t;
    t.nb = (width + 31) / 32;
    t.bytes = t.nb * 4096;
    return t;
}

struct VTile {
    int rows;       // rows of the halo'd tile
    int box_rows;   // rows per box (at most 256)
    int nb;         // boxes
    int bytes;      // bytes of one stage
};

__host__ __device__ inline VTile v_tile(int RP) {
    VTile t;
    t.rows = kBlurSpan + 2 * RP;
    t.nb = (t.rows + 255) / 256;
    t.box_rows = (t.rows + t.nb - 1) / t.nb;
    t.box_rows = (t.box_rows + 7) & ~7;
    t.bytes = t.nb * t.box_rows * 128;
    return t;
}

// Per-CTA shared layout: two stages, then the taps and two mbarriers.
__host__ __device__ inline size_t tma_smem_bytes(int stage_bytes, int RP) {
    return 1024 + 2 * static_cast<size_t>(stage_bytes) + 16 * 2 + 4 * static_cast<size_t>((RP + 1 + 3) & ~3);
}

// Convolve the 8 outputs at logical indices c..c+7 of one line (c, RP
// multiples of 8); chunk(i) returns the line's values i..i+3 for i a multiple
// of 4 (indices c - RP .. c + RP + 15 are read).
template <class Chunk>
__device__ __forceinline__ void convolve8_lines(Chunk chunk, int c, int RP, const float* taps,
                                                float acc[kBlurOut]) {
    const float w0 = taps[0];
    {
        const float4 m0 = chunk(c), m1 = chunk(c + 4);
        acc[0] = m0.x * w0; acc[1] = m0.y * w0; acc[2] = m0.z * w0; acc[3] = m0.w * w0;
        acc[4] = m1.x * w0; acc[5] = m1.y * w0; acc[6] = m1.z * w0; acc[7] = m1.w * w0;
    }
    for (int kb = 0; kb < RP; kb += 8) {
        float L[16], Rv[16];
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            const float4 l4 = chunk(c - kb - 8 + 4 * v), r4 = chunk(c + kb + 4 * v);
            L[4 * v] = l4.x; L[4 * v + 1] = l4.y; L[4 * v + 2] = l4.z; L[4 * v + 3] = l4.w;
            Rv[4 * v] = r4.x; Rv[4 * v + 1] = r4.y; Rv[4 * v + 2] = r4.z; Rv[4 * v + 3] = r4.w;
        }
        float wk[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) wk[j] = taps[kb + 1 + j];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
#pragma unroll
            for (int b = 0; b < kBlurOut; ++b) acc[b] = __fmaf_rn(L[b + 7 - j] + Rv[b + 1 + j], wk[j], acc[b]);
        }
    }
}

struct TmaBlurArgs {
    uint32_t W, H;
    int RP;
    Taps taps;
    float* out;
    uint32_t* peak;       // vertical pass only
    uint32_t* status;     // bit 16: an mbarrier wait ran out
};

__global__ void __launch_bounds__(kBlurThreads, 2)
    blur_h_tma_kernel(const __grid_constant__ CUtensorMap map, TmaBlurArgs a) {
    extern __shared__ unsigned char smem_raw[];
    char* base = reinterpret_cast<char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    const HTile ht = h_tile(a.RP);
    char* const stage0 = base;
    char* const stage1 = base + ht.bytes;
    uint64_t* bar = reinterpret_cast<uint64_t*>(base + kStages * ht.bytes);
    float* taps = reinterpret_cast<float*>(bar + 2);
    const int tid = threadIdx.x;
    dev::load_taps(taps, a.taps, a.RP);
    const int tiles_x = static_cast<int>((a.W + kBlurSpan - 1) / kBlurSpan);
    const int tiles = tiles_x * static_cast<int>((a.H + kBlurLines - 1) / kBlurLines);
    auto issue = [&](int t, int s) {
        const int bx = t % tiles_x, by = t / tiles_x;
        const int x0 = bx * kBlurSpan - a.RP, y0 = by * kBlurLines;
        char* dst = s ? stage1 : stage0;
        mbar_expect_tx(&bar[s], static_cast<uint32_t>(ht.bytes));
        for (int b = 0; b < ht.nb; ++b) tma_load_2d(dst + b * 4096, &map, x0 + 32 * b, y0, &bar[s]);
    };
    if (tid == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        fence_mbar_init();
        if (static_cast<int>(blockIdx.x) < tiles) issue(blockIdx.x, 0);
    }
    __syncthreads();
    const int lane = tid & 31, seg = tid >> 5;
    uint32_t phase = 0u;                                                       // bit s: parity of stage s
    uint32_t inflight = static_cast<int>(blockIdx.x) < tiles ? 1u : 0u;       // bit s: thread 0's copies
    int it = 0;
    bool failed = false;
    for (int t = blockIdx.x; t < tiles; t += gridDim.x, ++it) {
        const int s = it & 1;
        if (tid == 0) {
            // The other stage was released by every thread at the end of the
            // previous tile; order those generic-proxy accesses before the
            // copy's writes.
            const int tn = t + static_cast<int>(gridDim.x);
            if (tn < tiles) {
                fence_proxy_async();
                issue(tn, s ^ 1);
                inflight |= 1u << (s ^ 1);
            }
        }
        const bool got = mbar_wait(&bar[s], (phase >> s) & 1u);
        if (got) {
            // Counts to f32 in place, each element by one thread.
            uint32_t* words = reinterpret_cast<uint32_t*>(s ? stage1 : stage0);
            for (int i = tid; i < ht.bytes / 4; i += kBlurThreads) {
                const uint32_t u = words[i];
                reinterpret_cast<float*>(words)[i] = count_to_float(u);
            }
        }
        if (__syncthreads_or(!got)) {
            failed = true;
            break;
        }
        phase ^= 1u << s;
        inflight &= ~(1u << s);
        const int bx = t % tiles_x, by = t / tiles_x;
        const long y = static_cast<long>(by) * kBlurLines + lane;
        const long xs = static_cast<long>(bx) * kBlurSpan + seg * kBlurOut;
        if (y < a.H && xs < a.W) {
            const char* st = s ? stage1 : stage0;
            const int r = lane;
            auto chunk = [&](int col) -> float4 { return *h_chunk(st, r, col); };
            float acc[kBlurOut];
            convolve8_lines(chunk, a.RP + seg * kBlurOut, a.RP, taps, acc);
            float* o = a.out + static_cast<size_t>(y) * a.W + xs;
            if (xs + kBlurOut <= a.W) {
                reinterpret_cast<float4*>(o)[0] = make_float4(acc[0], acc[1], acc[2], acc[3]);
                reinterpret_cast<float4*>(o)[1] = make_float4(acc[4], acc[5], acc[6], acc[7]);
            } else {
#pragma unroll
                for (int b = 0; b < kBlurOut; ++b)
                    if (xs + b < a.W) o[b] = acc[b];
            }
        }
        __syncthreads();
    }
    if (failed && tid == 0) {
        atomicOr(a.status, kStatusCopyTimeout);
        // Copies this CTA started must land before its shared memory goes.
        for (int s = 0; s < kStages; ++s)
            if ((inflight >> s) & 1u) mbar_wait(&bar[s], (phase >> s) & 1u);
    }
}

__global__ void __launch_bounds__(kBlurThreads, 2)
    blur_v_tma_kernel(const __grid_constant__ CUtensorMap map, TmaBlurArgs a) {
    extern __shared__ unsigned char smem_raw[];
    __shared__ float warp_max[kBlurSegs];
    char* base = reinterpret_cast<char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    const VTile vt = v_tile(a.RP);
    char* const stage0 = base;
    char* const stage1 = base + vt.bytes;
    uint64_t* bar = reinterpret_cast<uint64_t*>(base + kStages * vt.bytes);
    float* taps = reinterpret_cast<float*>(bar + 2);
    const int tid = threadIdx.x;
    dev::load_taps(taps, a.taps, a.RP);
    const int tiles_x = static_cast<int>((a.W + kBlurLines - 1) / kBlurLines);
    const int tiles = tiles_x * static_cast<int>((a.H + kBlurSpan - 1) / kBlurSpan);
    auto issue = [&](int t, int s) {
        const int bx = t % tiles_x, by = t / tiles_x;
        const int x0 = bx * kBlurLines, y0 = by * kBlurSpan - a.RP;
        char* dst = s ? stage1 : stage0;
        mbar_expect_tx(&bar[s], static_cast<uint32_t>(vt.bytes));
        for (int b = 0; b < vt.nb; ++b)
            tma_load_2d(dst + b * vt.box_rows * 128, &map, x0, y0 + b * vt.box_rows, &bar[s]);
    };
    if (tid == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        fence_mbar_init();
        if (static_cast<int>(blockIdx.x) < tiles) issue(blockIdx.x, 0);
    }
    __syncthreads();
    const int lane = tid & 31, seg = tid >> 5;
    uint32_t phase = 0u;                                                       // bit s: parity of stage s
    uint32_t inflight = static_cast<int>(blockIdx.x) < tiles ? 1u : 0u;       // bit s: thread 0's copies
    int it = 0;
    bool failed = false;
    float best = 0.0f;
    for (int t = blockIdx.x; t < tiles; t += gridDim.x, ++it) {
        const int s = it & 1;
        if (tid == 0) {
            const int tn = t + static_cast<int>(gridDim.x);
            if (tn < tiles) {
                fence_proxy_async();
                issue(tn, s ^ 1);
                inflight |= 1u << (s ^ 1);
            }
        }
        const bool got = mbar_wait(&bar[s], (phase >> s) & 1u);
        if (__syncthreads_or(!got)) {
            failed = true;
            break;
        }
        phase ^= 1u << s;
        inflight &= ~(1u << s);
        const int bx = t % tiles_x, by = t / tiles_x;
        const long x = static_cast<long>(bx) * kBlurLines + lane;
        const long ys = static_cast<long>(by) * kBlurSpan + seg * kBlurOut;
        if (x < a.W && ys < a.H) {
            const float* col = reinterpret_cast<const float*>(s ? stage1 : stage0) + lane;
            auto chunk = [&](int row) -> float4 {
                return make_float4(col[row * 32], col[(row + 1) * 32], col[(row + 2) * 32], col[(row + 3) * 32]);
            };
            float acc[kBlurOut];
            convolve8_lines(chunk, a.RP + seg * kBlurOut, a.RP, taps, acc);
#pragma unroll
            for (int b = 0; b < kBlurOut; ++b) {
                if (ys + b < a.H) {
                    a.out[static_cast<size_t>(ys + b) * a.W + x] = acc[b];
                    best = fmaxf(best, acc[b]);
                }
            }
        }
        __syncthreads();
    }
    if (failed) {
        if (tid == 0) {
            atomicOr(a.status, kStatusCopyTimeout);
            for (int s = 0; s < kStages; ++s)
                if ((inflight >> s) & 1u) mbar_wait(&bar[s], (phase >> s) & 1u);
        }
        return;
    }
    // The CTA's maximum over all its tiles (blur.wgsl:67-82): ordered f32 bits.
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) best = fmaxf(best, __shfl_xor_sync(0xFFFFFFFFu, best, o));
    if (lane == 0) warp_max[seg] = best;
    __syncthreads();
    if (tid == 0) {
        float m = 0.0f;
        for (int s = 0; s < kBlurSegs; ++s) m = fmaxf(m, warp_max[s]);
        if (m > 0.0f) atomicMax(a.peak, __float_as_uint(m));
    }
}

// ---- host side ----
using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                 const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiled encoder() {
    static EncodeTiled fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiled>(p);
    });
    return fn;
}

int sm_count() {
    int dev = 0, n = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    return n;
}

bool encode(CUtensorMap* map, CUtensorMapDataType type, const void* base, uint32_t W, uint32_t H, uint32_t box_x,
            uint32_t box_y, CUtensorMapSwizzle swizzle) {
    EncodeTiled fn = encoder();
    if (!fn) return false;
    const cuuint64_t dims[2] = {W, H};
    const cuuint64_t strides[1] = {static_cast<cuuint64_t>(W) * 4};
    const cuuint32_t box[2] = {box_x, box_y};
    const cuuint32_t elem[2] = {1, 1};
    return fn(map, type, 2, const_cast<void*>(base), dims, strides, box, elem, CU_TENSOR_MAP_INTERLEAVE_NONE,
              swizzle, CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

}  // namespace

bool blur_tma_eligible(const void* in, const void* out, uint32_t w, uint32_t h) {
    // Rows of whole 16-byte units (the tensor map's stride rule) and 16-byte
    // aligned buffers (its base rule and the float4 stores).
    return w % 4 == 0 && w > 0 && h > 0 && (reinterpret_cast<uintptr_t>(in) & 15) == 0 &&
           (reinterpret_cast<uintptr_t>(out) & 15) == 0 && encoder() != nullptr;
}

cudaError_t prepare_blur_tma_kernels() {
    const int RP = dev::blur_padded(kMaxTaps - 1);
    const int hb = static_cast<int>(tma_smem_bytes(h_tile(RP).bytes, RP));
    const int vb = static_cast<int>(tma_smem_bytes(v_tile(RP).bytes, RP));
    cudaError_t e = cudaFuncSetAttribute(reinterpret_cast<const void*>(blur_h_tma_kernel),
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, hb);
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(reinterpret_cast<const void*>(blur_v_tma_kernel),
                                cudaFuncAttributeMaxDynamicSharedMemorySize, vb);
}

cudaError_t launch_blur_horizontal_tma(const uint32_t* counts, float* out, uint32_t w, uint32_t h, const Taps& taps,
                                       uint32_t* status, cudaStream_t s) {
    TmaBlurArgs a{};
    a.W = w;
    a.H = h;
    a.RP = dev::blur_padded(taps.R);
    a.taps = taps;
    a.out = out;
    a.status = status;
    CUtensorMap map;
    if (!encode(&map, CU_TENSOR_MAP_DATA_TYPE_UINT32, counts, w, h, 32, kBlurLines, CU_TENSOR_MAP_SWIZZLE_128B))
        return cudaErrorInvalidValue;
    const int tiles = static_cast<int>(div_up(w, kBlurSpan) * div_up(h, kBlurLines));
    const int grid = std::min(tiles, 2 * sm_count());
    blur_h_tma_kernel<<<grid, kBlurThreads, tma_smem_bytes(h_tile(a.RP).bytes, a.RP), s>>>(map, a);
    return cudaGetLastError();
}

cudaError_t launch_blur_vertical_tma(const float* in, float* out, uint32_t w, uint32_t h, const Taps& taps,
                                     uint32_t* peak, uint32_t* status, cudaStream_t s) {
    TmaBlurArgs a{};
    a.W = w;
    a.H = h;
    a.RP = dev::blur_padded(taps.R);
    a.taps = taps;
    a.out = out;
    a.peak = peak;
    a.status = status;
    const VTile vt = v_tile(a.RP);
    CUtensorMap map;
    if (!encode(&map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, in, w, h, kBlurLines, static_cast<uint32_t>(vt.box_rows),
                CU_TENSOR_MAP_SWIZZLE_NONE))
        return cudaErrorInvalidValue;
    const int tiles = static_cast<int>(div_up(w, kBlurLines) * div_up(h, kBlurSpan));
    const int grid = std::min(tiles, 2 * sm_count());
    blur_v_tma_kernel<<<grid, kBlurThreads, tma_smem_bytes(vt.bytes, a.RP), s>>>(map, a);
    return cudaGetLastError();
}

}  // namespace bt
