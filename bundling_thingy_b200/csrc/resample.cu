// resample.cu — evenly spaced samples along the polylines.
//
// Restates count_paths / emit_paths (src/shaders/resampling.wgsl:82-183).
// B200 layout: the count pass is one thread per path (a short closed-form walk
// over its control points); offsets come from a device scan in path order (no
// atomics); the emit pass is one warp per path, with lanes producing the
// samples of a segment in parallel and a warp ballot applying the reference's
// per-sample duplicate rule, so the output equals the serial walk exactly.
// The emit pass also splats the density and bins the samples for the first
// neighbour-mean iteration.
#include "kernels.cuh"

namespace bt {
namespace {

// push_sample in count mode (resampling.wgsl:50-58, 77-78).
__device__ __forceinline__ void push_count(uint32_t& count, float2& last, float2 p, uint32_t capacity) {
    if (count > 0u && p.x == last.x && p.y == last.y) return;
    if (count >= capacity) {
        count = capacity + 1u;
        return;
    }
    last = p;
    count += 1u;
}

// resample(path, write = false) (resampling.wgsl:82-136).
__device__ uint32_t count_path(const ResampleCountArgs& a, uint32_t p, float4* edge) {
    const uint32_t start = a.starts[p], end = a.starts[p + 1];
    const float2 first = normalized(a.norm, a.cp[start]);
    uint32_t count = 0u;
    float2 last = first;
    push_count(count, last, first, a.capacity);
    float2 prev = first;
    float remaining = 1.0f;
    for (uint32_t i = start + 1u; i < end; ++i) {
        const float2 cur = normalized(a.norm, a.cp[i]);
        const float dx = cur.x - prev.x, dy = cur.y - prev.y;
        const float ex = dx * a.sx, ey = dy * a.sy;
        const float distance = sqrtf(ex * ex + ey * ey);
        if (distance > 0.0f) {
            const uint32_t steps = u32_sat(fmaxf(floorf(distance - remaining) + 1.0f, 0.0f));
            if (steps > 0u) {
                const float t0 = remaining / distance;
                const float t1 = (remaining + static_cast<float>(steps - 1u)) / distance;
                const float ax = prev.x + dx * t0, ay = prev.y + dy * t0;
                const float bx = prev.x + dx * t1, by = prev.y + dy * t1;
                // Samples are a texel apart; only the first can repeat the prior one.
                count += steps - ((ax == last.x && ay == last.y) ? 1u : 0u);
                last = make_float2(bx, by);
                if (count > a.capacity) return a.capacity + 1u;
            }
            remaining = remaining + static_cast<float>(steps) - distance;
        }
        prev = cur;
    }
    *edge = make_float4(first.x, first.y, prev.x, prev.y);
    push_count(count, last, prev, a.capacity);
    // A short closed path keeps its excursion and returning endpoint.
    if (count == 1u) {
        for (uint32_t i = start + 1u; i < end; ++i) {
            const float2 next = normalized(a.norm, a.cp[i]);
            if (next.x != first.x || next.y != first.y) {
                push_count(count, last, next, a.capacity);
                push_count(count, last, prev, a.capacity);
                break;
            }
        }
    }
    return count;
}

__global__ void __launch_bounds__(128) resample_count_kernel(ResampleCountArgs a) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    unsigned long long samples = 0, drawn = 0;
    if (p < a.paths) {
        float4 edge = make_float4(0.f, 0.f, 0.f, 0.f);
        const uint32_t c = count_path(a, p, &edge);
        a.edges[p] = edge;
        const bool keep = c >= 2u;   // count_paths skips paths below two samples
        a.packed[p] = keep ? ((static_cast<unsigned long long>(c) << 32) | 1ull) : 0ull;
        samples = keep ? c : 0u;
        drawn = keep ? 1u : 0u;
    }
    // Warp-aggregated totals (u64: per-path counts saturate at capacity + 1).
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        samples += __shfl_down_sync(0xFFFFFFFFu, samples, o);
        drawn += __shfl_down_sync(0xFFFFFFFFu, drawn, o);
    }
    if ((threadIdx.x & 31) == 0 && (samples | drawn)) {
        atomicAdd(&a.totals[0], samples);
        atomicAdd(&a.totals[1], drawn);
    }
}

__global__ void paths_from_scan_kernel(const unsigned long long* packed, const unsigned long long* scan, uint32_t n,
                                       PathRec* out) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const uint32_t c = static_cast<uint32_t>(packed[p] >> 32);
    const unsigned long long v = scan[p];
    const uint32_t point_offset = static_cast<uint32_t>(v >> 32);
    const uint32_t drawn_before = static_cast<uint32_t>(v & 0xFFFFFFFFull);
    // Skipped paths keep a zeroed reservation (buffers start cleared).
    out[p] = c >= 2u ? PathRec{point_offset, point_offset - drawn_before, c} : PathRec{0u, 0u, 0u};
}

// Kernel arguments with the grid by value.
struct EmitKernelArgs {
    ResampleEmitArgs a;
    Grid g;
    int binning;
};

// One sample write of push_sample in emit mode (resampling.wgsl:58-76) plus
// the sample's first search cell.
__device__ __forceinline__ void write_sample(const EmitKernelArgs& k, const PathRec& rec, uint32_t p, uint32_t pos,
                                             float2 s) {
    const ResampleEmitArgs& a = k.a;
    const uint32_t index = rec.point_offset + pos;
    a.xy[index] = s;
    a.edge_ids[index] = p;
    if (pos > 0u) a.segments[rec.segment_offset + pos - 1u] = index - 1u;
    if (a.counts) {
        uint32_t d;
        if (splat_index(s.x, s.y, a.map, &d)) atomicAdd(&a.counts[d], 1u);
    }
    if (k.binning) {
        const bool movable = pos != 0u && pos != rec.count - 1u;   // neighbor_mean.wgsl:61-64
        const uint32_t c = search_cell(s, k.g);
        a.tag[index] = index | (movable ? kMovableBit : 0u);
        a.cell[index] = c;
        atomicAdd(&a.hist[c], 1u);
    }
}

struct WarpCursor {
    uint32_t count;
    float2 last;
    bool failed;
};

// push_sample in emit mode for one warp-uniform sample; lane 0 writes.
__device__ __forceinline__ void push_emit(const EmitKernelArgs& k, const PathRec& rec, uint32_t p, WarpCursor& c,
                                          float2 s, int lane) {
    if (c.failed) return;
    if (c.count > 0u && s.x == c.last.x && s.y == c.last.y) return;
    if (c.count >= rec.count) {
        c.failed = true;
        return;
    }
    if (lane == 0) write_sample(k, rec, p, c.count, s);
    c.last = s;
    c.count += 1u;
}

__global__ void __launch_bounds__(256) resample_emit_kernel(EmitKernelArgs k) {
    const ResampleEmitArgs& a = k.a;
    const int lane = threadIdx.x & 31;
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    const unsigned lt_mask = (1u << lane) - 1u;
    for (uint32_t p = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; p < a.n_paths; p += warps) {
        const PathRec rec = a.paths[p];
        if (rec.count < 2u) continue;
        const uint32_t start = a.starts[p], end = a.starts[p + 1];
        const float2 first = normalized(a.norm, a.cp[start]);
        WarpCursor c{0u, first, false};
        push_emit(k, rec, p, c, first, lane);
        float2 prev = first;
        float remaining = 1.0f;
        for (uint32_t i = start + 1u; i < end && !c.failed; ++i) {
            const float2 cur = normalized(a.norm, a.cp[i]);
            const float dx = cur.x - prev.x, dy = cur.y - prev.y;
            const float ex = dx * a.sx, ey = dy * a.sy;
            const float distance = sqrtf(ex * ex + ey * ey);
            if (distance > 0.0f) {
                const uint32_t steps = u32_sat(fmaxf(floorf(distance - remaining) + 1.0f, 0.0f));
                for (uint32_t base = 0; base < steps && !c.failed; base += 32u) {
                    const uint32_t j = base + lane;
                    const bool valid = j < steps;
                    float2 s = c.last;
                    bool keep = false;
                    if (valid) {
                        const float t = (remaining + static_cast<float>(j)) / distance;
                        s = make_float2(prev.x + dx * t, prev.y + dy * t);
                        // The prior sample: the cursor for the first, else this
                        // segment's previous sample (a skipped sample equals
                        // the last written one, so this is the emit-mode rule).
                        float2 before = c.last;
                        if (j > 0u) {
                            const float tb = (remaining + static_cast<float>(j - 1u)) / distance;
                            before = make_float2(prev.x + dx * tb, prev.y + dy * tb);
                        }
                        keep = !(s.x == before.x && s.y == before.y);
                    }
                    const unsigned mask = __ballot_sync(0xFFFFFFFFu, keep);
                    const uint32_t kept = __popc(mask);
                    if (c.count + kept > rec.count) {
                        c.failed = true;
                        break;
                    }
                    if (keep) write_sample(k, rec, p, c.count + __popc(mask & lt_mask), s);
                    c.count += kept;
                    const uint32_t active = steps - base < 32u ? steps - base : 32u;
                    c.last.x = __shfl_sync(0xFFFFFFFFu, s.x, active - 1u);
                    c.last.y = __shfl_sync(0xFFFFFFFFu, s.y, active - 1u);
                }
                remaining = remaining + static_cast<float>(steps) - distance;
            }
            prev = cur;
        }
        push_emit(k, rec, p, c, prev, lane);
        if (c.count == 1u && !c.failed) {
            for (uint32_t i = start + 1u; i < end; ++i) {
                const float2 next = normalized(a.norm, a.cp[i]);
                if (next.x != first.x || next.y != first.y) {
                    push_emit(k, rec, p, c, next, lane);
                    push_emit(k, rec, p, c, prev, lane);
                    break;
                }
            }
        }
        if ((c.failed || c.count != rec.count) && lane == 0) atomicOr(a.status, 2u);
    }
}

}  // namespace

void launch_resample_count(const ResampleCountArgs& a, cudaStream_t s) {
    if (a.paths == 0) return;
    resample_count_kernel<<<div_up(a.paths, 128), 128, 0, s>>>(a);
}

void launch_paths_from_scan(const unsigned long long* packed, const unsigned long long* scan, uint32_t paths,
                            PathRec* out, cudaStream_t s) {
    if (paths == 0) return;
    paths_from_scan_kernel<<<div_up(paths, 256), 256, 0, s>>>(packed, scan, paths, out);
}

void launch_resample_emit(const ResampleEmitArgs& a, cudaStream_t s) {
    if (a.n_paths == 0) return;
    EmitKernelArgs k{};
    k.a = a;
    k.binning = a.grid_host != nullptr;
    if (a.grid_host) k.g = *a.grid_host;
    // One warp per path, grid sized to a few waves of 148 SMs.
    const unsigned warps_needed = a.n_paths;
    unsigned blocks = div_up(warps_needed, 8);
    const unsigned cap = 148u * 16u;
    if (blocks > cap) blocks = cap;
    resample_emit_kernel<<<blocks, 256, 0, s>>>(k);
}

}  // namespace bt
