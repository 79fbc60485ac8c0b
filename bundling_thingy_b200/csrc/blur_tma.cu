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
//  - One kernel serves both passes: it convolves along the rows of its input
//    (32 rows x 128 outputs plus the halo per tile, one box whose row length
//    is padded to 4 mod 32 words, so that float4 reads of 32 rows by one warp
//    spread over all banks) and writes its result transposed, lanes of a warp
//    on consecutive words. The first pass takes the u32 counts (converted to
//    f32 in place once per tile) and writes the intermediate transposed; the
//    second convolves that along its rows, the image's columns, and writes
//    the image in row order with its maximum. Halos up to 48 texels (sigma
//    up to 16) fit one box of 256 elements; wider ones use density.cu.
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

// Horizontal stage layout: 32 rows of `pitch` words, the row length of the
// halo'd tile rounded up to 4 mod 32 (conflict-free float4 reads down a
// column of rows).
// The widest halo whose padded line fits one box of 256 elements: 128 + 2 * 48
// = 224, padded to 228.
constexpr int kMaxHalo = 48;

struct HTile {
    int pitch;      // words per line (the box width)
    int bytes;      // bytes of one stage
};

__host__ __device__ inline HTile h_tile(int RP) {
    int p = kBlurSpan + 2 * RP;
    while (p % 32 != 4) ++p;
    HTile t;
    t.pitch = p;
    t.bytes = kBlurLines * p * 4;
    return t;
}

__host__ __device__ inline int stage_stride(int RP) { return (h_tile(RP).bytes + 127) & ~127; }
static_assert(kBlurSpan + 2 * kMaxHalo + 4 <= 256, "one box per line tile");

// Per-CTA shared layout: two stages, then two mbarriers and the taps.
__host__ __device__ inline size_t tma_smem_bytes(int RP) {
    return 128 + 2 * static_cast<size_t>(stage_stride(RP)) + 16 + 4 * static_cast<size_t>((RP + 1 + 3) & ~3);
}

// Convolve the 8 outputs at logical indices c..c+7 of one line (c, RP
// multiples of 8) from `line` in shared memory (indices c - RP .. c + RP + 15
// are read), in float4 chunks: out[x] = w0*in[x] + sum_k fma(in[x-k] + in[x+k], w_k, .).
__device__ __forceinline__ void convolve8_line(const float* line, int c, int RP, const float* taps,
                                               float acc[kBlurOut]) {
    const float w0 = taps[0];
    const float4 m0 = *reinterpret_cast<const float4*>(line + c);
    const float4 m1 = *reinterpret_cast<const float4*>(line + c + 4);
    acc[0] = m0.x * w0; acc[1] = m0.y * w0; acc[2] = m0.z * w0; acc[3] = m0.w * w0;
    acc[4] = m1.x * w0; acc[5] = m1.y * w0; acc[6] = m1.z * w0; acc[7] = m1.w * w0;
    for (int kb = 0; kb < RP; kb += 8) {
        const float4* lp = reinterpret_cast<const float4*>(line + c - kb - 8);
        const float4* rp = reinterpret_cast<const float4*>(line + c + kb);
        float L[16], Rv[16];
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            const float4 l4 = lp[v], r4 = rp[v];
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
    uint32_t lines, along;   // the input is `lines` rows of `along` texels
    int RP;
    Taps taps;
    float* out;              // out[along_index * lines + line_index]
    uint32_t* peak;          // the second pass's maximum (null: none)
    uint32_t* status;        // bit 16: an mbarrier wait ran out
};

// One pass of the separable blur along the rows of its input, written
// transposed: a tile is 32 input rows ("lines") x 128 outputs along them
// plus the halo. kCounts: the input is the u32 splat counts (converted to f32
// in place after each copy); otherwise f32. The first pass takes the counts
// (lines = image rows) and writes the transposed intermediate; the second
// takes that (lines = image columns) and writes the image in row order,
// with its maximum (blur.wgsl:67-82).
template <bool kCounts>
__global__ void __launch_bounds__(kBlurThreads, 2)
    blur_line_tma_kernel(const __grid_constant__ CUtensorMap map, TmaBlurArgs a) {
    extern __shared__ unsigned char smem_raw[];
    __shared__ float warp_max[kBlurSegs];
    char* base = reinterpret_cast<char*>((reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~uintptr_t(127));
    const HTile ht = h_tile(a.RP);
    const int stride = stage_stride(a.RP);
    uint64_t* bar = reinterpret_cast<uint64_t*>(base + 2 * stride);
    float* taps = reinterpret_cast<float*>(bar + 2);
    const int tid = threadIdx.x;
    dev::load_taps(taps, a.taps, a.RP);
    const int tiles_x = static_cast<int>((a.along + kBlurSpan - 1) / kBlurSpan);
    const int tiles = tiles_x * static_cast<int>((a.lines + kBlurLines - 1) / kBlurLines);
    auto issue = [&](int t, int s) {
        const int bx = t % tiles_x, by = t / tiles_x;
        mbar_expect_tx(&bar[s], static_cast<uint32_t>(ht.bytes));
        tma_load_2d(base + s * stride, &map, bx * kBlurSpan - a.RP, by * kBlurLines, &bar[s]);
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
        char* stage = base + s * stride;
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
        if (kCounts && got) {
            // Counts to f32 in place, each element by one thread.
            uint32_t* words = reinterpret_cast<uint32_t*>(stage);
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
        const uint32_t line = static_cast<uint32_t>(by) * kBlurLines + lane;
        const uint32_t xs = static_cast<uint32_t>(bx) * kBlurSpan + seg * kBlurOut;
        if (line < a.lines && xs < a.along) {
            float acc[kBlurOut];
            convolve8_line(reinterpret_cast<const float*>(stage) + lane * ht.pitch, a.RP + seg * kBlurOut, a.RP,
                           taps, acc);
            // Transposed: consecutive lanes write consecutive words.
#pragma unroll
            for (int b = 0; b < kBlurOut; ++b) {
                if (xs + b < a.along) {
                    a.out[static_cast<size_t>(xs + b) * a.lines + line] = acc[b];
                    best = fmaxf(best, acc[b]);
                }
            }
        }
        __syncthreads();
    }
    if (failed) {
        if (tid == 0) {
            atomicOr(a.status, kStatusCopyTimeout);
            // Copies this CTA started must land before its shared memory goes.
            for (int s = 0; s < kStages; ++s)
                if ((inflight >> s) & 1u) mbar_wait(&bar[s], (phase >> s) & 1u);
        }
        return;
    }
    if (!a.peak) return;
    // The CTA's maximum over its tiles: non-negative finite f32 values keep
    // their order as u32 bits.
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) best = fmaxf(best, __shfl_xor_sync(0xFFFFFFFFu, best, o));
    if (lane == 0) warp_max[seg] = best;
    __syncthreads();
    if (tid == 0) {
        float m = 0.0f;
        for (int w = 0; w < kBlurSegs; ++w) m = fmaxf(m, warp_max[w]);
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

bool blur_tma_eligible(const void* in, const void* out, uint32_t w, uint32_t h, int R) {
    // Lines of whole 16-byte units in both orientations (the tensor maps'
    // stride rule), 16-byte aligned buffers (their base rule), a halo that
    // fits one box.
    return w % 4 == 0 && h % 4 == 0 && w > 0 && h > 0 && dev::blur_padded(R) <= kMaxHalo &&
           (reinterpret_cast<uintptr_t>(in) & 15) == 0 && (reinterpret_cast<uintptr_t>(out) & 15) == 0 &&
           encoder() != nullptr;
}

cudaError_t prepare_blur_tma_kernels() {
    const int bytes = static_cast<int>(tma_smem_bytes(kMaxHalo));
    cudaError_t e = cudaFuncSetAttribute(reinterpret_cast<const void*>(blur_line_tma_kernel<true>),
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(reinterpret_cast<const void*>(blur_line_tma_kernel<false>),
                                cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
}

namespace {
template <bool kCounts>
cudaError_t launch_line_pass(const void* in, uint32_t lines, uint32_t along, const Taps& taps, float* out,
                             uint32_t* peak, uint32_t* status, cudaStream_t s) {
    TmaBlurArgs a{};
    a.lines = lines;
    a.along = along;
    a.RP = dev::blur_padded(taps.R);
    a.taps = taps;
    a.out = out;
    a.peak = peak;
    a.status = status;
    if (a.RP > kMaxHalo) return cudaErrorInvalidValue;
    CUtensorMap map;
    if (!encode(&map, kCounts ? CU_TENSOR_MAP_DATA_TYPE_UINT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, in, along, lines,
                static_cast<uint32_t>(h_tile(a.RP).pitch), kBlurLines, CU_TENSOR_MAP_SWIZZLE_NONE))
        return cudaErrorInvalidValue;
    const int tiles = static_cast<int>(div_up(along, kBlurSpan) * div_up(lines, kBlurLines));
    const int grid = std::min(tiles, 2 * sm_count());
    blur_line_tma_kernel<kCounts><<<grid, kBlurThreads, tma_smem_bytes(a.RP), s>>>(map, a);
    return cudaGetLastError();
}
}  // namespace

cudaError_t launch_blur_horizontal_tma(const uint32_t* counts, float* out_t, uint32_t w, uint32_t h,
                                       const Taps& taps, uint32_t* status, cudaStream_t s) {
    // Rows of the counts; the result is written transposed (out_t[x * h + y]).
    return launch_line_pass<true>(counts, h, w, taps, out_t, nullptr, status, s);
}

cudaError_t launch_blur_vertical_tma(const float* in_t, float* out, uint32_t w, uint32_t h, const Taps& taps,
                                     uint32_t* peak, uint32_t* status, cudaStream_t s) {
    // Rows of the transposed intermediate (image columns); the result comes
    // out in row order (out[y * w + x]).
    return launch_line_pass<false>(in_t, w, h, taps, out, peak, status, s);
}

}  // namespace bt
