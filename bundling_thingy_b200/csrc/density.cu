// density.cu — separable Gaussian blur of the splat counts and normalisation.
//
// Restates src/shaders/blur.wgsl:13-82 and normalization.wgsl:5-17 with a
// general tap count: out[x] = w0*in[x] + sum_{k=1..R} (in[x-k] + in[x+k]) * w_k,
// accumulated k = 1..R with a fused multiply-add per tap (the contraction WGSL
// allows for `value += pair(...) * w`), zero padding outside the map.
//
// B200 layout: a CTA blurs 32 lines (rows for the horizontal pass, columns for
// the vertical one) x 128 outputs. The line segments plus an RP-texel halo
// (RP = R rounded up to 8) are staged in shared memory with one line per lane
// (pitch = 4 mod 32 words, so 16-byte loads across a warp are conflict-free).
// Each thread keeps 8 outputs in registers and walks the taps 8 at a time:
// 16 + 16 staged values feed 64 add+FMA pairs. Taps beyond R have weight 0,
// which leaves the sum unchanged, so RP > R is exact. The per-tile bodies live
// in density_dev.cuh (shared with batch.cu).
#include <cuda_runtime.h>

#include "density_dev.cuh"

namespace bt {
namespace {

using dev::kBlurLines;
using dev::kBlurSpan;
using dev::kBlurThreads;

__global__ void __launch_bounds__(kBlurThreads, dev::kBlurMinCtas) blur_h_kernel(const uint32_t* __restrict__ in, float* __restrict__ out,
                                                              uint32_t W, uint32_t H, Taps taps_arg, int RP) {
    extern __shared__ float smem[];
    float* taps = smem;
    float* tile = smem + ((RP + 1 + 3) & ~3);
    dev::load_taps(taps, taps_arg, RP);
    dev::blur_h_tile(in, out, W, H, taps, RP, blockIdx.x, blockIdx.y, tile);
}

__global__ void __launch_bounds__(kBlurThreads, dev::kBlurMinCtas) blur_v_kernel(const float* __restrict__ in, float* __restrict__ out,
                                                              uint32_t W, uint32_t H, Taps taps_arg, int RP,
                                                              uint32_t* peak) {
    extern __shared__ float smem[];
    __shared__ float warp_max[dev::kBlurSegs];
    float* taps = smem;
    float* tile = smem + ((RP + 1 + 3) & ~3);
    dev::load_taps(taps, taps_arg, RP);
    dev::blur_v_tile(in, out, W, H, taps, RP, blockIdx.x, blockIdx.y, tile, warp_max, peak);
}

__global__ void normalize_kernel(const float4* __restrict__ in, const uint32_t* peak_bits, float4* __restrict__ out,
                                 size_t n4) {
    const float peak = __uint_as_float(*peak_bits);
    for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n4;
         i += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const float4 v = in[i];
        out[i] = make_float4(dev::normalized_value(v.x, peak), dev::normalized_value(v.y, peak),
                             dev::normalized_value(v.z, peak), dev::normalized_value(v.w, peak));
    }
}

__global__ void normalize_tail_kernel(const float* in, const uint32_t* peak_bits, float* out, size_t start, size_t n) {
    const float peak = __uint_as_float(*peak_bits);
    const size_t i = start + threadIdx.x;
    if (i < n) out[i] = dev::normalized_value(in[i], peak);
}

__global__ void splat_positions_kernel(const float2* xy, uint32_t n, Map map, uint32_t* counts) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float2 p = xy[i];
    uint32_t d;
    if (splat_index(p.x, p.y, map, &d)) atomicAdd(&counts[d], 1u);
}

}  // namespace

void launch_splat_positions(const float2* xy, uint32_t n, Map map, uint32_t* counts, cudaStream_t s) {
    if (n) splat_positions_kernel<<<div_up(n, 256), 256, 0, s>>>(xy, n, map, counts);
}

// Opt the blur kernels into the shared memory of the widest tap count
// (R = 128). Called once per device before any launch or graph capture.
cudaError_t prepare_density_kernels() {
    const int bytes = static_cast<int>(dev::blur_smem_bytes(dev::blur_padded(kMaxTaps - 1)));
    cudaError_t e = cudaFuncSetAttribute(reinterpret_cast<const void*>(blur_h_kernel),
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(reinterpret_cast<const void*>(blur_v_kernel),
                             cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e != cudaSuccess) return e;
    return prepare_blur_tma_kernels();
}

void launch_blur_horizontal(const uint32_t* counts, float* out, uint32_t w, uint32_t h, const Taps& taps,
                            cudaStream_t s) {
    const int RP = dev::blur_padded(taps.R);
    dim3 grid(div_up(w, kBlurSpan), div_up(h, kBlurLines));
    blur_h_kernel<<<grid, kBlurThreads, dev::blur_smem_bytes(RP), s>>>(counts, out, w, h, taps, RP);
}

void launch_blur_vertical(const float* in, float* out, uint32_t w, uint32_t h, const Taps& taps, uint32_t* peak,
                          cudaStream_t s) {
    const int RP = dev::blur_padded(taps.R);
    dim3 grid(div_up(w, kBlurLines), div_up(h, kBlurSpan));
    blur_v_kernel<<<grid, kBlurThreads, dev::blur_smem_bytes(RP), s>>>(in, out, w, h, taps, RP, peak);
}

void launch_normalize(const float* in, const uint32_t* peak, float* out, size_t n, cudaStream_t s) {
    const size_t n4 = n / 4;
    if (n4) {
        unsigned blocks = div_up(n4, 256);
        if (blocks > 148u * 8u) blocks = 148u * 8u;
        normalize_kernel<<<blocks, 256, 0, s>>>(reinterpret_cast<const float4*>(in), peak,
                                                reinterpret_cast<float4*>(out), n4);
    }
    if (n % 4) normalize_tail_kernel<<<1, 32, 0, s>>>(in, peak, out, n4 * 4, n);
}

}  // namespace bt
