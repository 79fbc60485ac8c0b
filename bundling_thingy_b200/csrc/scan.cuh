// scan.cuh — device-wide exclusive prefix sum (reduce-then-scan).
//
// Deterministic replacement for the reference's atomic reservations
// (resampling.wgsl:151,157 and spatial_grid.wgsl:110,119): offsets come out in
// index order. Three launches per level; levels recurse on the block sums.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"

namespace bt {

constexpr int kScanBlock = 256;
constexpr int kScanItems = 8;
constexpr size_t kScanTile = static_cast<size_t>(kScanBlock) * kScanItems;

template <typename T>
__device__ __forceinline__ T block_sum(T v, T* warp_sums) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xFFFFFFFFu, v, o);
    if (lane == 0) warp_sums[warp] = v;
    __syncthreads();
    T total = 0;
    if (threadIdx.x == 0) {
        for (int w = 0; w < kScanBlock / 32; ++w) total += warp_sums[w];
        warp_sums[0] = total;
    }
    __syncthreads();
    total = warp_sums[0];
    __syncthreads();
    return total;
}

// Exclusive scan of one value per thread across the block; returns the prefix
// and stores the block total in *total.
template <typename T>
__device__ __forceinline__ T block_exclusive(T v, T* warp_sums, T* total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    T x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        T y = __shfl_up_sync(0xFFFFFFFFu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[warp] = x;
    __syncthreads();
    if (warp == 0) {
        T w = lane < kScanBlock / 32 ? warp_sums[lane] : T(0);
        T s = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            T y = __shfl_up_sync(0xFFFFFFFFu, s, o);
            if (lane >= o) s += y;
        }
        if (lane < kScanBlock / 32) warp_sums[lane] = s - w;
        if (lane == kScanBlock / 32 - 1) warp_sums[kScanBlock / 32] = s;
    }
    __syncthreads();
    T prefix = warp_sums[warp] + (x - v);
    *total = warp_sums[kScanBlock / 32];
    __syncthreads();
    return prefix;
}

template <typename T>
__global__ void __launch_bounds__(kScanBlock) scan_reduce_kernel(const T* in, size_t n, T* sums) {
    __shared__ T warp_sums[kScanBlock / 32 + 1];
    const size_t base = static_cast<size_t>(blockIdx.x) * kScanTile;
    T acc = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        size_t j = base + static_cast<size_t>(i) * kScanBlock + threadIdx.x;
        if (j < n) acc += in[j];
    }
    acc = block_sum(acc, warp_sums);
    if (threadIdx.x == 0) sums[blockIdx.x] = acc;
}

// out[j] = offsets[block] + sum(in[tile start .. j)); out[n] = total when
// write_total is set.
template <typename T>
__global__ void __launch_bounds__(kScanBlock) scan_apply_kernel(const T* in, size_t n, const T* offsets, T* out,
                                                                int write_total) {
    __shared__ T tile[kScanTile + kScanTile / 32];
    __shared__ T warp_sums[kScanBlock / 32 + 1];
    const size_t base = static_cast<size_t>(blockIdx.x) * kScanTile;
    auto pad = [](int i) { return i + (i >> 5); };
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        int t = i * kScanBlock + threadIdx.x;
        size_t j = base + t;
        tile[pad(t)] = j < n ? in[j] : T(0);
    }
    __syncthreads();
    T local[kScanItems];
    T sum = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        local[i] = tile[pad(threadIdx.x * kScanItems + i)];
        sum += local[i];
    }
    T block_total;
    T prefix = block_exclusive(sum, warp_sums, &block_total);
    const T offset = offsets ? offsets[blockIdx.x] : T(0);
    prefix += offset;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        tile[pad(threadIdx.x * kScanItems + i)] = prefix;
        prefix += local[i];
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        int t = i * kScanBlock + threadIdx.x;
        size_t j = base + t;
        if (j < n) out[j] = tile[pad(t)];
    }
    if (write_total && threadIdx.x == 0 && base + kScanTile >= n) out[n] = offset + block_total;
}

// Scratch elements needed by exclusive_scan for n inputs.
// Each level keeps its block sums and their scan (blocks + 1 entries each).
inline size_t scan_scratch_elems(size_t n) {
    size_t total = 0;
    while (n > kScanTile) {
        n = (n + kScanTile - 1) / kScanTile;
        total += 2 * (n + 1);
    }
    return total + 1;
}

// out has n + 1 elements; out[n] receives the total. in and out may not alias.
template <typename T>
void exclusive_scan(const T* in, T* out, size_t n, T* scratch, cudaStream_t stream) {
    if (n == 0) {
        cudaMemsetAsync(out, 0, sizeof(T), stream);
        return;
    }
    const size_t blocks = (n + kScanTile - 1) / kScanTile;
    if (blocks == 1) {
        scan_apply_kernel<T><<<1, kScanBlock, 0, stream>>>(in, n, nullptr, out, 1);
        return;
    }
    T* sums = scratch;              // blocks + 1 entries
    T* rest = scratch + blocks + 1;
    scan_reduce_kernel<T><<<static_cast<unsigned>(blocks), kScanBlock, 0, stream>>>(in, n, sums);
    // Exclusive scan of the block sums, in place through a second buffer level.
    exclusive_scan<T>(sums, rest, blocks, rest + blocks + 1, stream);
    scan_apply_kernel<T><<<static_cast<unsigned>(blocks), kScanBlock, 0, stream>>>(in, n, rest, out, 1);
}

}  // namespace bt
