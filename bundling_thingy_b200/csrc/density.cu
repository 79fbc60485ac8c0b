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
// which leaves the sum unchanged, so RP > R is exact.
#include <cuda_runtime.h>

#include "kernels.cuh"

namespace bt {
namespace {

constexpr int kLines = 32;        // lanes: one line each
constexpr int kSegs = 16;         // warps: 8 outputs each
constexpr int kOut = 8;
constexpr int kSpan = kSegs * kOut;   // outputs per line per CTA

__host__ __device__ inline int pitch_for(int RP) {
    int p = kSpan + 2 * RP;
    while (p % 32 != 4) ++p;
    return p;
}

__device__ __forceinline__ float load_value(const uint32_t* p, size_t i) { return static_cast<float>(p[i]); }

// Convolve the thread's 8 outputs on one staged line.
__device__ __forceinline__ void convolve8(const float* line, int c, int RP, const float* taps, float acc[kOut]) {
    const float4 m0 = *reinterpret_cast<const float4*>(line + c);
    const float4 m1 = *reinterpret_cast<const float4*>(line + c + 4);
    const float w0 = taps[0];
    acc[0] = m0.x * w0; acc[1] = m0.y * w0; acc[2] = m0.z * w0; acc[3] = m0.w * w0;
    acc[4] = m1.x * w0; acc[5] = m1.y * w0; acc[6] = m1.z * w0; acc[7] = m1.w * w0;
    for (int kb = 0; kb < RP; kb += 8) {
        float L[16], Rv[16];
        const float4* lp = reinterpret_cast<const float4*>(line + c - kb - 8);
        const float4* rp = reinterpret_cast<const float4*>(line + c + kb);
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
            for (int b = 0; b < kOut; ++b) {
                // tap k = kb + 1 + j: in[x-k] = L[b + 7 - j], in[x+k] = Rv[b + 1 + j]
                acc[b] = __fmaf_rn(L[b + 7 - j] + Rv[b + 1 + j], wk[j], acc[b]);
            }
        }
    }
}

// Horizontal pass: lines are rows. Input u32 counts, output f32.
__global__ void __launch_bounds__(kLines * kSegs) blur_h_kernel(const uint32_t* __restrict__ in, float* __restrict__ out,
                                                                uint32_t W, uint32_t H, Taps taps_arg, int RP) {
    extern __shared__ float smem[];
    const int P = pitch_for(RP);
    float* taps = smem;                   // RP + 1 weights (zero-padded)
    float* tile = smem + ((RP + 1 + 3) & ~3);
    const int tid = threadIdx.x;
    for (int k = tid; k <= RP; k += blockDim.x) taps[k] = k <= taps_arg.R ? taps_arg.w[k] : 0.0f;
    const long x0 = static_cast<long>(blockIdx.x) * kSpan;
    const long y0 = static_cast<long>(blockIdx.y) * kLines;
    const int width = kSpan + 2 * RP;
    for (int i = tid; i < kLines * width; i += blockDim.x) {
        const int line = i / width, col = i - line * width;
        const long y = y0 + line, x = x0 - RP + col;
        float v = 0.0f;
        if (y < H && x >= 0 && x < W) v = load_value(in, static_cast<size_t>(y) * W + x);
        tile[line * P + col] = v;
    }
    __syncthreads();
    const int lane = tid & 31, seg = tid >> 5;
    const long y = y0 + lane;
    const long xs = x0 + seg * kOut;
    if (y >= H || xs >= W) return;
    float acc[kOut];
    convolve8(tile + lane * P, RP + seg * kOut, RP, taps, acc);
    float* o = out + static_cast<size_t>(y) * W + xs;
    if (xs + kOut <= W && (reinterpret_cast<uintptr_t>(o) & 15) == 0) {
        reinterpret_cast<float4*>(o)[0] = make_float4(acc[0], acc[1], acc[2], acc[3]);
        reinterpret_cast<float4*>(o)[1] = make_float4(acc[4], acc[5], acc[6], acc[7]);
    } else {
#pragma unroll
        for (int b = 0; b < kOut; ++b)
            if (xs + b < W) o[b] = acc[b];
    }
}

// Vertical pass: lines are columns (staged transposed). Input f32, output f32,
// plus the global maximum as ordered f32 bits (blur.wgsl:67-82).
__global__ void __launch_bounds__(kLines * kSegs) blur_v_kernel(const float* __restrict__ in, float* __restrict__ out,
                                                                uint32_t W, uint32_t H, Taps taps_arg, int RP,
                                                                uint32_t* peak) {
    extern __shared__ float smem[];
    __shared__ float warp_max[kSegs];
    const int P = pitch_for(RP);
    float* taps = smem;
    float* tile = smem + ((RP + 1 + 3) & ~3);
    const int tid = threadIdx.x;
    for (int k = tid; k <= RP; k += blockDim.x) taps[k] = k <= taps_arg.R ? taps_arg.w[k] : 0.0f;
    const long x0 = static_cast<long>(blockIdx.x) * kLines;
    const long y0 = static_cast<long>(blockIdx.y) * kSpan;
    const int height = kSpan + 2 * RP;
    for (int i = tid; i < kLines * height; i += blockDim.x) {
        const int row = i >> 5, col = i & 31;
        const long y = y0 - RP + row, x = x0 + col;
        float v = 0.0f;
        if (x < W && y >= 0 && y < H) v = in[static_cast<size_t>(y) * W + x];
        tile[col * P + row] = v;
    }
    __syncthreads();
    const int lane = tid & 31, seg = tid >> 5;
    const long x = x0 + lane;
    const long ys = y0 + seg * kOut;
    float best = 0.0f;
    if (x < W && ys < H) {
        float acc[kOut];
        convolve8(tile + lane * P, RP + seg * kOut, RP, taps, acc);
#pragma unroll
        for (int b = 0; b < kOut; ++b) {
            if (ys + b < H) {
                out[static_cast<size_t>(ys + b) * W + x] = acc[b];
                best = fmaxf(best, acc[b]);
            }
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) best = fmaxf(best, __shfl_xor_sync(0xFFFFFFFFu, best, o));
    if (lane == 0) warp_max[seg] = best;
    __syncthreads();
    if (tid == 0) {
        float m = 0.0f;
        for (int s = 0; s < kSegs; ++s) m = fmaxf(m, warp_max[s]);
        // Non-negative finite f32 values keep their order as u32 bits.
        if (m > 0.0f) atomicMax(peak, __float_as_uint(m));
    }
}

__global__ void normalize_kernel(const float4* __restrict__ in, const uint32_t* peak_bits, float4* __restrict__ out,
                                 size_t n4) {
    const float peak = __uint_as_float(*peak_bits);
    for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n4;
         i += static_cast<size_t>(gridDim.x) * blockDim.x) {
        float4 v = in[i];
        float4 r = make_float4(0.f, 0.f, 0.f, 0.f);
        if (peak > 0.0f) {
            r.x = fminf(fmaxf(v.x / peak, 0.0f), 1.0f);
            r.y = fminf(fmaxf(v.y / peak, 0.0f), 1.0f);
            r.z = fminf(fmaxf(v.z / peak, 0.0f), 1.0f);
            r.w = fminf(fmaxf(v.w / peak, 0.0f), 1.0f);
        }
        out[i] = r;
    }
}

__global__ void normalize_tail_kernel(const float* in, const uint32_t* peak_bits, float* out, size_t start, size_t n) {
    const float peak = __uint_as_float(*peak_bits);
    const size_t i = start + threadIdx.x;
    if (i < n) out[i] = peak > 0.0f ? fminf(fmaxf(in[i] / peak, 0.0f), 1.0f) : 0.0f;
}

size_t smem_bytes(int RP) {
    return (static_cast<size_t>((RP + 1 + 3) & ~3) + static_cast<size_t>(kLines) * pitch_for(RP)) * sizeof(float);
}

int padded(int R) { return (R + 7) & ~7; }

}  // namespace

// Opt the blur kernels into the shared memory of the widest tap count
// (R = 128). Called once per device before any launch or graph capture.
cudaError_t prepare_density_kernels() {
    const int bytes = static_cast<int>(smem_bytes(padded(kMaxTaps - 1)));
    cudaError_t e = cudaFuncSetAttribute(reinterpret_cast<const void*>(blur_h_kernel),
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(reinterpret_cast<const void*>(blur_v_kernel),
                                cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
}

void launch_blur_horizontal(const uint32_t* counts, float* out, uint32_t w, uint32_t h, const Taps& taps,
                            cudaStream_t s) {
    const int RP = padded(taps.R);
    const size_t bytes = smem_bytes(RP);
    dim3 grid(div_up(w, kSpan), div_up(h, kLines));
    blur_h_kernel<<<grid, kLines * kSegs, bytes, s>>>(counts, out, w, h, taps, RP);
}

void launch_blur_vertical(const float* in, float* out, uint32_t w, uint32_t h, const Taps& taps, uint32_t* peak,
                          cudaStream_t s) {
    const int RP = padded(taps.R);
    const size_t bytes = smem_bytes(RP);
    dim3 grid(div_up(w, kLines), div_up(h, kSpan));
    blur_v_kernel<<<grid, kLines * kSegs, bytes, s>>>(in, out, w, h, taps, RP, peak);
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
