// scan.cuh — device-wide exclusive prefix sum (reduce-then-scan).
//
// Deterministic replacement for the reference's atomic reservations
// (resampling.wgsl:151,157 and spatial_grid.wgsl:110,119): offsets come out in
// index order. Three launches per level; levels recurse on the block sums.
// Sums are integers, so any association order gives the same result.
//
// A scan reads through a Source (read(j) gives element j; consume(j) runs
// after the last read of j, e.g. to clear an accumulator for its next use)
// and writes through a Sink (store(j, prefix)); plain arrays are the default.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"

namespace bt {

constexpr int kScanBlock = 256;

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

// Items per thread: tiles of 2048 elements up to 8 bytes, 1024 above (16-byte
// sums: fewer registers per thread, more resident blocks).
template <typename T>
__host__ __device__ constexpr int scan_items() {
    return sizeof(T) <= 8 ? 8 : 4;
}
template <typename T>
__host__ __device__ constexpr size_t scan_tile() {
    return static_cast<size_t>(kScanBlock) * scan_items<T>();
}

template <typename T>
struct ArraySource {
    const T* p;
    __device__ __forceinline__ T read(size_t j) const { return p[j]; }
    __device__ __forceinline__ void consume(size_t) const {}
};

template <typename T>
struct ArraySink {
    T* p;
    __device__ __forceinline__ void store(size_t j, T v) const { p[j] = v; }
};

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

// Shared-memory index of tile element i: one element of padding per 128
// bytes, so that both the striped stores (thread t, element k * 256 + t) and
// the blocked loads (thread t, elements t * items ..) are free of bank
// conflicts for 4- to 16-byte elements.
template <typename T>
__host__ __device__ constexpr int scan_pad(int i) {
    return i + i / static_cast<int>(128 / sizeof(T));
}

// Shared memory of one tile pass.
template <typename T>
struct ScanShared {
    T tile[scan_pad<T>(static_cast<int>(scan_tile<T>()))];
    T warp_sums[kScanBlock / 32 + 1];
};

// Sum of in[base .. min(base + tile, n)) over the block (all threads get it).
template <typename T, typename Source>
__device__ __forceinline__ T tile_reduce(const Source& in, size_t base, size_t n, ScanShared<T>& sh) {
    constexpr int kItems = scan_items<T>();
    T acc = zero<T>();
#pragma unroll
    for (int i = 0; i < kItems; ++i) {
        size_t j = base + static_cast<size_t>(i) * kScanBlock + threadIdx.x;
        if (j < n) acc += in.read(j);
    }
    return block_sum(acc, sh.warp_sums);
}

// out[j] = offset + sum(in[base .. j)) for the tile at base; the tile that
// reaches n also stores the total at n. Returns offset + the tile's sum (to
// every thread). Synchronises internally.
template <typename T, typename Source, typename Sink>
__device__ __forceinline__ T tile_apply(const Source& in, const Sink& out, size_t base, size_t n, T offset,
                                        ScanShared<T>& sh) {
    constexpr int kItems = scan_items<T>();
    constexpr int kTile = kScanBlock * kItems;
    auto pad = [](int i) { return scan_pad<T>(i); };
#pragma unroll
    for (int i = 0; i < kItems; ++i) {
        int t = i * kScanBlock + threadIdx.x;
        size_t j = base + t;
        if (j < n) {
            sh.tile[pad(t)] = in.read(j);
            in.consume(j);
        } else {
            sh.tile[pad(t)] = zero<T>();
        }
    }
    __syncthreads();
    T local[kItems];
    T sum = zero<T>();
#pragma unroll
    for (int i = 0; i < kItems; ++i) {
        local[i] = sh.tile[pad(threadIdx.x * kItems + i)];
        sum += local[i];
    }
    T block_total;
    T prefix = block_exclusive(sum, sh.warp_sums, &block_total);
    prefix += offset;
#pragma unroll
    for (int i = 0; i < kItems; ++i) {
        sh.tile[pad(threadIdx.x * kItems + i)] = prefix;
        prefix += local[i];
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < kItems; ++i) {
        int t = i * kScanBlock + threadIdx.x;
        size_t j = base + t;
        if (j < n) out.store(j, sh.tile[pad(t)]);
    }
    if (threadIdx.x == 0 && base + kTile >= n) out.store(n, offset + block_total);
    __syncthreads();
    return offset + block_total;
}

// Exclusive scan of in[0 .. n) by one block, tile after tile (out may alias
// in: each tile is staged in shared memory before it is written).
template <typename T, typename Source, typename Sink>
__device__ __forceinline__ void block_scan_all(const Source& in, const Sink& out, size_t n, ScanShared<T>& sh) {
    T carry = zero<T>();
    size_t base = 0;
    do {
        carry = tile_apply<T>(in, out, base, n, carry, sh);
        base += scan_tile<T>();
    } while (base < n);
}

template <typename T, typename Source>
__global__ void __launch_bounds__(kScanBlock) scan_reduce_kernel(Source in, size_t n, T* sums) {
    __shared__ ScanShared<T> sh;
    const T total = tile_reduce<T>(in, static_cast<size_t>(blockIdx.x) * scan_tile<T>(), n, sh);
    if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

// out[j] = offsets[block] + sum(in[tile start .. j)); out[n] = total.
template <typename T, typename Source, typename Sink>
__global__ void __launch_bounds__(kScanBlock) scan_apply_kernel(Source in, size_t n, const T* offsets, Sink out) {
    __shared__ ScanShared<T> sh;
    const T offset = offsets ? offsets[blockIdx.x] : zero<T>();
    tile_apply<T>(in, out, static_cast<size_t>(blockIdx.x) * scan_tile<T>(), n, offset, sh);
}

// Each level keeps its block sums and their scan (blocks + 1 entries each).
template <typename T>
inline size_t scan_scratch_elems(size_t n) {
    size_t total = 0;
    while (n > scan_tile<T>()) {
        n = (n + scan_tile<T>() - 1) / scan_tile<T>();
        total += 2 * (n + 1);
    }
    return total + 1;
}

// Number of kernel launches of a scan of n elements of T.
template <typename T>
inline int scan_launch_count(size_t n) {
    if (n == 0) return 0;
    if (n <= scan_tile<T>()) return 1;
    return 2 + scan_launch_count<T>((n + scan_tile<T>() - 1) / scan_tile<T>());
}

// Exclusive scan of n elements; the sink receives n + 1 values (the last is
// the total). Source and sink must not alias.
template <typename T, typename Source, typename Sink>
void exclusive_scan_with(Source in, Sink out, size_t n, T* scratch, cudaStream_t stream) {
    const size_t blocks = (n + scan_tile<T>() - 1) / scan_tile<T>();
    if (blocks <= 1) {
        scan_apply_kernel<T, Source, Sink><<<1, kScanBlock, 0, stream>>>(in, n, nullptr, out);
        return;
    }
    T* sums = scratch;              // blocks + 1 entries
    T* rest = scratch + blocks + 1;
    scan_reduce_kernel<T, Source><<<static_cast<unsigned>(blocks), kScanBlock, 0, stream>>>(in, n, sums);
    exclusive_scan_with<T>(ArraySource<T>{sums}, ArraySink<T>{rest}, blocks, rest + blocks + 1, stream);
    scan_apply_kernel<T, Source, Sink><<<static_cast<unsigned>(blocks), kScanBlock, 0, stream>>>(in, n, rest, out);
}

// Plain arrays: out has n + 1 elements.
template <typename T>
void exclusive_scan(const T* in, T* out, size_t n, T* scratch, cudaStream_t stream) {
    exclusive_scan_with<T>(ArraySource<T>{in}, ArraySink<T>{out}, n, scratch, stream);
}

// ---- Scans whose producer accumulated the tile sums ----
//
// A kernel that writes the scan's input can add each element to the sum of its
// tile (scan_tile<T>() elements) as it goes; the scan is then one block over
// the tile sums and one pass over the tiles, reading the data once.

template <typename T>
inline size_t scan_tiles(size_t n) {
    const size_t t = (n + scan_tile<T>() - 1) / scan_tile<T>();
    return t ? t : 1;
}

// Exclusive scan of the tile sums in place by one block (sums[count] = total).
template <typename T>
__global__ void __launch_bounds__(kScanBlock) tile_sums_scan_kernel(T* sums, size_t count) {
    __shared__ ScanShared<T> sh;
    block_scan_all<T>(ArraySource<T>{sums}, ArraySink<T>{sums}, count, sh);
}

// The same scan in one pass of a 1,024-thread block, each thread owning a
// contiguous run of at most kWideScanRun sums (read twice from L2: once for
// the run's total, once to write its prefixes). The tile sums are the single
// CTA on the binning chain's critical path; five passes of the 256-thread
// form over ~4.8K 16-byte sums took ~12 us cold (one pass: 0.3% off a
// steady-state iteration of the large workload).
constexpr int kWideScanBlock = 1024;
constexpr size_t kWideScanRun = 16;

template <typename T>
__global__ void __launch_bounds__(kWideScanBlock) tile_sums_scan_wide_kernel(T* sums, size_t count) {
    __shared__ T warp_sums[kWideScanBlock / 32 + 1];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const size_t per = (count + kWideScanBlock - 1) / kWideScanBlock;
    const size_t b = min(static_cast<size_t>(threadIdx.x) * per, count);
    const size_t e = min(b + per, count);
    T v = zero<T>();
    for (size_t j = b; j < e; ++j) v += sums[j];
    // Exclusive scan of the runs' totals across the block.
    T x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const T y = shfl_up(x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[warp] = x;
    __syncthreads();
    if (warp == 0) {
        const T w = warp_sums[lane];
        T t = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const T y = shfl_up(t, o);
            if (lane >= o) t += y;
        }
        warp_sums[lane] = t - w;
        if (lane == 31) warp_sums[32] = t;
    }
    __syncthreads();
    T run = warp_sums[warp] + (x - v);
    for (size_t j = b; j < e; ++j) {
        const T s = sums[j];
        sums[j] = run;
        run += s;
    }
    if (threadIdx.x == kWideScanBlock - 1) sums[count] = warp_sums[32];
}

// Exclusive scan of n elements given the sums of their tiles (scan_tiles(n)
// + 1 entries, scanned in place); the sink receives n + 1 values.
template <typename T, typename Source, typename Sink>
void exclusive_scan_presummed(Source in, Sink out, size_t n, T* tile_sums, cudaStream_t stream) {
    const size_t tiles = scan_tiles<T>(n);
    if (tiles <= kWideScanBlock * kWideScanRun)
        tile_sums_scan_wide_kernel<T><<<1, kWideScanBlock, 0, stream>>>(tile_sums, tiles);
    else
        tile_sums_scan_kernel<T><<<1, kScanBlock, 0, stream>>>(tile_sums, tiles);
    scan_apply_kernel<T, Source, Sink><<<static_cast<unsigned>(tiles), kScanBlock, 0, stream>>>(in, n, tile_sums, out);
}

// The tile sums of n elements, for a producer that did not accumulate them.
template <typename T, typename Source>
void reduce_tiles(Source in, size_t n, T* tile_sums, cudaStream_t stream) {
    scan_reduce_kernel<T, Source><<<static_cast<unsigned>(scan_tiles<T>(n)), kScanBlock, 0, stream>>>(in, n, tile_sums);
}

}  // namespace bt
