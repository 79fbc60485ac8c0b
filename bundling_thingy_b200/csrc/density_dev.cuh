// density_dev.cuh — per-tile bodies of the blur and normalisation kernels,
// shared by the single-graph kernels (density.cu) and the batched persistent
// kernels (batch.cu). See density.cu for the arithmetic and the layout.
#pragma once

#include "kernels.cuh"

namespace bt {
namespace dev {

constexpr int kBlurLines = 32;                        // lanes: one line each
constexpr int kBlurSegs = 16;                         // warps: 8 outputs each
constexpr int kBlurOut = 8;
constexpr int kBlurSpan = kBlurSegs * kBlurOut;       // outputs per line per CTA
constexpr int kBlurThreads = kBlurLines * kBlurSegs;
// Three resident CTAs per SM (40 registers): the staging loads of one CTA
// overlap the arithmetic of the others. Unbounded, the kernels took 56-70
// registers and ran two CTAs per SM, or one (the batch's vertical pass):
// 13.1 against 11.9 ms per iteration of 256 mixed graphs in a batch. The
// horizontal passes spill a few bytes (4 single-graph, 20 batched); they ran
// no slower than a spill-free variant with taps four at a time.
constexpr int kBlurMinCtas = 3;

__host__ __device__ inline int blur_padded(int R) { return (R + 7) & ~7; }

__host__ __device__ inline int blur_pitch(int RP) {
    int p = kBlurSpan + 2 * RP;
    while (p % 32 != 4) ++p;
    return p;
}

// Shared memory of one blur CTA: RP + 1 taps (rounded to 4) and the tile.
__host__ __device__ inline size_t blur_smem_bytes(int RP) {
    return (static_cast<size_t>((RP + 1 + 3) & ~3) + static_cast<size_t>(kBlurLines) * blur_pitch(RP)) * sizeof(float);
}

// Taps 0..RP into shared memory, zero beyond R. The caller synchronises.
__device__ __forceinline__ void load_taps(float* taps, const Taps& t, int RP) {
    for (int k = threadIdx.x; k <= RP; k += blockDim.x) taps[k] = k <= t.R ? t.w[k] : 0.0f;
}

// Convolve the thread's 8 outputs on one staged line.
__device__ __forceinline__ void convolve8(const float* line, int c, int RP, const float* taps, float acc[kBlurOut]) {
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
            for (int b = 0; b < kBlurOut; ++b) {
                // tap k = kb + 1 + j: in[x-k] = L[b + 7 - j], in[x+k] = Rv[b + 1 + j]
                acc[b] = __fmaf_rn(L[b + 7 - j] + Rv[b + 1 + j], wk[j], acc[b]);
            }
        }
    }
}

// Horizontal pass over tile (bx, by): 32 rows x 128 outputs; input u32
// counts, output f32. Taps already staged; synchronises internally.
__device__ __forceinline__ void blur_h_tile(const uint32_t* __restrict__ in, float* __restrict__ out, uint32_t W,
                                            uint32_t H, const float* taps, int RP, int bx, int by, float* tile) {
    const int P = blur_pitch(RP);
    const int tid = threadIdx.x;
    const long x0 = static_cast<long>(bx) * kBlurSpan;
    const long y0 = static_cast<long>(by) * kBlurLines;
    const int width = kBlurSpan + 2 * RP;
    const int lane = tid & 31, seg = tid >> 5;
    // Warp per line, lanes along it: coalesced, and no division per element.
    for (int line = seg; line < kBlurLines; line += kBlurSegs) {
        const long yl = y0 + line;
        const bool row = yl < H;
        const uint32_t* src = in + static_cast<size_t>(row ? yl : 0) * W;
        for (int col = lane; col < width; col += 32) {
            const long x = x0 - RP + col;
            float v = 0.0f;
            if (row && x >= 0 && x < W) v = static_cast<float>(src[x]);
            tile[line * P + col] = v;
        }
    }
    __syncthreads();
    const long y = y0 + lane;
    const long xs = x0 + seg * kBlurOut;
    if (y < H && xs < W) {
        float acc[kBlurOut];
        convolve8(tile + lane * P, RP + seg * kBlurOut, RP, taps, acc);
        float* o = out + static_cast<size_t>(y) * W + xs;
        if (xs + kBlurOut <= W && (reinterpret_cast<uintptr_t>(o) & 15) == 0) {
            reinterpret_cast<float4*>(o)[0] = make_float4(acc[0], acc[1], acc[2], acc[3]);
            reinterpret_cast<float4*>(o)[1] = make_float4(acc[4], acc[5], acc[6], acc[7]);
        } else {
#pragma unroll
            for (int b = 0; b < kBlurOut; ++b)
                if (xs + b < W) o[b] = acc[b];
        }
    }
}

// Vertical pass over tile (bx, by): 32 columns (staged transposed) x 128
// outputs; input and output f32; the tile's maximum goes into *peak as
// ordered f32 bits (blur.wgsl:67-82). Synchronises internally.
__device__ __forceinline__ void blur_v_tile(const float* __restrict__ in, float* __restrict__ out, uint32_t W,
                                            uint32_t H, const float* taps, int RP, int bx, int by, float* tile,
                                            float* warp_max, uint32_t* peak) {
    const int P = blur_pitch(RP);
    const int tid = threadIdx.x;
    const long x0 = static_cast<long>(bx) * kBlurLines;
    const long y0 = static_cast<long>(by) * kBlurSpan;
    const int height = kBlurSpan + 2 * RP;
    for (int i = tid; i < kBlurLines * height; i += kBlurThreads) {
        const int row = i >> 5, col = i & 31;
        const long y = y0 - RP + row, x = x0 + col;
        float v = 0.0f;
        if (x < W && y >= 0 && y < H) v = in[static_cast<size_t>(y) * W + x];
        tile[col * P + row] = v;
    }
    __syncthreads();
    const int lane = tid & 31, seg = tid >> 5;
    const long x = x0 + lane;
    const long ys = y0 + seg * kBlurOut;
    float best = 0.0f;
    if (x < W && ys < H) {
        float acc[kBlurOut];
        convolve8(tile + lane * P, RP + seg * kBlurOut, RP, taps, acc);
#pragma unroll
        for (int b = 0; b < kBlurOut; ++b) {
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
        for (int s = 0; s < kBlurSegs; ++s) m = fmaxf(m, warp_max[s]);
        // Non-negative finite f32 values keep their order as u32 bits.
        if (m > 0.0f) atomicMax(peak, __float_as_uint(m));
    }
}

// normalization.wgsl:11-16 for one element.
__device__ __forceinline__ float normalized_value(float v, float peak) {
    return peak > 0.0f ? fminf(fmaxf(v / peak, 0.0f), 1.0f) : 0.0f;
}

}  // namespace dev
}  // namespace bt
