// scan.cuh — device-wide exclusive prefix sum (reduce-then-scan).
//
// Deterministic replacement for the reference's atomic reservations
// (resampling.wgsl:151,157 and spatial_grid.wgsl:110,119): offsets come out in
// index order. Three launches per level; levels recurse on the block sums.
// Sums are integers, so any association order gives the same result.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"

namespace bt {

constexpr int kScanBlock = 256;
constexpr int kScanItems = 8;
constexpr size_t kScanTile = static_cast<size_t>(kScanBlock) * kScanItems;

// Pair of 64-bit sums (fixed-point x and y).
struct LL2 {
    long long x, y;
};
__host__ __device__ __forceinline__ LL2 operator+(LL2 a, LL2 b) { return LL2{a.x + b.x, a.y + b.y}; }
__host__ __device__ __forceinline__ LL2 operator-(LL2 a, LL2 b) { return LL2{a.x - b.x, a.y - b.y}; }
__host__ __device__ __forceinline__ LL2& operator+=(LL2& a, LL2 b) {
    a.x += b.x;
    a.y += b.y;
    return a;
}

template <typename T>
__device__ __forceinline__ T zero() {
    return T(0);
}
template <>
__device__ __forceinline__ LL2 zero<LL2>() {
    return LL2{0, 0};
}

template <typename T>
__device__ __forceinline__ T shfl_up(T v, int o) {
    return __shfl_up_sync(0xFFFFFFFFu, v, o);
}
template <>
__device__ __forceinline__ LL2 shfl_up<LL2>(LL2 v, int o) {
    return LL2{__shfl_up_sync(0xFFFFFFFFu, v.x, o), __shfl_up_sync(0xFFFFFFFFu, v.y, o)};
}
template <typename T>
__device__ __forceinline__ T shfl_down(T v, int o) {
    return __shfl_down_sync(0xFFFFFFFFu, v, o);
}
template <>
__device__ __forceinline__ LL2 shfl_down<LL2>(LL2 v, int o) {
    return LL2{__shfl_down_sync(0xFFFFFFFFu, v.x, o), __shfl_down_sync(0xFFFFFFFFu, v.y, o)};
}

// Input conversions.
__device__ __forceinline__ uint32_t widen(uint32_t v, uint32_t*) { return v; }
__device__ __forceinline__ unsigned long long widen(unsigned long long v, unsigned long long*) { return v; }
__device__ __forceinline__ LL2 widen(int2 v, LL2*) { return LL2{v.x, v.y}; }
// Slot record {x, y, biased Qx, biased Qy}: the fixed-point half.
__device__ __forceinline__ LL2 widen(uint4 v, LL2*) {
    return LL2{static_cast<long long>(v.z), static_cast<long long>(v.w)};
}
__device__ __forceinline__ LL2 widen(LL2 v, LL2*) { return v; }

template <typename T>
__device__ __forceinline__ T block_sum(T v, T* warp_sums) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += shfl_down(v, o);
    if (lane == 0) warp_sums[warp] = v;
    __syncthreads();
    T total = zero<T>();
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
        T y = shfl_up(x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[warp] = x;
    __syncthreads();
    if (warp == 0) {
        T w = lane < kScanBlock / 32 ? warp_sums[lane] : zero<T>();
        T s = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            T y = shfl_up(s, o);
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

template <typename In, typename T>
__global__ void __launch_bounds__(kScanBlock) scan_reduce_kernel(const In* in, size_t n, T* sums) {
    __shared__ T warp_sums[kScanBlock / 32 + 1];
    const size_t base = static_cast<size_t>(blockIdx.x) * kScanTile;
    T acc = zero<T>();
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        size_t j = base + static_cast<size_t>(i) * kScanBlock + threadIdx.x;
        if (j < n) acc += widen(in[j], static_cast<T*>(nullptr));
    }
    acc = block_sum(acc, warp_sums);
    if (threadIdx.x == 0) sums[blockIdx.x] = acc;
}

// out[j] = offsets[block] + sum(in[tile start .. j)); out[n] = total.
template <typename In, typename T>
__global__ void __launch_bounds__(kScanBlock) scan_apply_kernel(const In* in, size_t n, const T* offsets, T* out) {
    __shared__ T tile[kScanTile + kScanTile / 32];
    __shared__ T warp_sums[kScanBlock / 32 + 1];
    const size_t base = static_cast<size_t>(blockIdx.x) * kScanTile;
    auto pad = [](int i) { return i + (i >> 5); };
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        int t = i * kScanBlock + threadIdx.x;
        size_t j = base + t;
        tile[pad(t)] = j < n ? widen(in[j], static_cast<T*>(nullptr)) : zero<T>();
    }
    __syncthreads();
    T local[kScanItems];
    T sum = zero<T>();
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        local[i] = tile[pad(threadIdx.x * kScanItems + i)];
        sum += local[i];
    }
    T block_total;
    T prefix = block_exclusive(sum, warp_sums, &block_total);
    const T offset = offsets ? offsets[blockIdx.x] : zero<T>();
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
    if (threadIdx.x == 0 && base + kScanTile >= n) out[n] = offset + block_total;
}

// Each level keeps its block sums and their scan (blocks + 1 entries each).
inline size_t scan_scratch_elems(size_t n) {
    size_t total = 0;
    while (n > kScanTile) {
        n = (n + kScanTile - 1) / kScanTile;
        total += 2 * (n + 1);
    }
    return total + 1;
}

// Number of kernel launches of exclusive_scan for n inputs.
inline int scan_launch_count(size_t n) {
    if (n == 0) return 0;
    if (n <= kScanTile) return 1;
    return 2 + scan_launch_count((n + kScanTile - 1) / kScanTile);
}

// out has n + 1 elements; out[n] receives the total. in and out may not alias.
template <typename In, typename T>
void exclusive_scan(const In* in, T* out, size_t n, T* scratch, cudaStream_t stream) {
    if (n == 0) {
        cudaMemsetAsync(out, 0, sizeof(T), stream);
        return;
    }
    const size_t blocks = (n + kScanTile - 1) / kScanTile;
    if (blocks == 1) {
        scan_apply_kernel<In, T><<<1, kScanBlock, 0, stream>>>(in, n, nullptr, out);
        return;
    }
    T* sums = scratch;              // blocks + 1 entries
    T* rest = scratch + blocks + 1;
    scan_reduce_kernel<In, T><<<static_cast<unsigned>(blocks), kScanBlock, 0, stream>>>(in, n, sums);
    exclusive_scan<T, T>(sums, rest, blocks, rest + blocks + 1, stream);
    scan_apply_kernel<In, T><<<static_cast<unsigned>(blocks), kScanBlock, 0, stream>>>(in, n, rest, out);
}

}  // namespace bt
